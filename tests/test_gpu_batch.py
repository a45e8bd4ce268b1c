"""Batched form: many independent graphs decomposed by ONE rtr_decompose on
their disjoint union.  Every graph's results must equal its standalone
decomposition (oracle), including cluster member order, which depends on the
graph-local ids the extraction hashes."""
import numpy as np
import pytest

import oracle
import rtrex_cuda_b200 as rtr
from rtrex_cuda_b200 import graphgen
from tests import helpers

pytestmark = pytest.mark.gpu


def _graphs():
    gs = graphgen.sbm_batch(10, seed0=4000, m_lo=1e3, m_hi=2e4)
    gs.append(helpers.case_graph("sbm_3000_4002"))  # order-sensitive at eps=0.1
    gs.append(helpers.case_graph("small_test"))
    gs.append(helpers.case_graph("isolated"))
    return gs


@pytest.mark.parametrize("eps", [0.1, 0.3])
def test_batch_equals_each_graph_alone(eps):
    gs = _graphs()
    with rtr.Graph.batch(gs) as g:
        g.decompose(eps)
        cl = g.clusters()
        st = g.status()
        pe, pv, sup, _ = g.weights()
        off, nb = g.csr()
        counts = g.batch_cluster_counts()
        bases = g.vertex_bases
    graph_of = np.searchsorted(bases, cl.seed, side="right") - 1
    for k, (n, u, v) in enumerate(gs):
        c = oracle.build_csr(n, u, v)
        s0 = oracle.count(c)
        s1 = oracle.initial_clean(c, s0, eps)
        ocl, s2 = oracle.extract(c, s1, eps)
        b = int(bases[k])
        idx = np.nonzero(graph_of == k)[0]
        assert counts[k] == len(ocl) == idx.size
        for j, ci in enumerate(idx):
            got = cl.vert[cl.off[ci]:cl.off[ci + 1]] - b
            assert (got == ocl.members(j)).all(), (k, j)
            assert cl.ne[ci] == ocl.ne[j] and cl.cut[ci] == ocl.cut[j]
        s_lo, s_hi = int(off[b]), int(off[b + n])
        assert (st[s_lo:s_hi] == s2.status).all()
        assert (helpers.bits(pe[s_lo:s_hi]) == helpers.bits(s2.perEdge)).all()
        assert (helpers.bits(pv[b:b + n]) == helpers.bits(s2.perVertex)).all()
