"""Extraction through the thread-block kernel (k_extract_big in
rtrex_cuda_b200/csrc/extract.cu): every component of at least the split size
replays its seed loop in one block, the two-hop scan's pairs worked out ahead
by seven warps and applied in the reference's order by the eighth.  With the
split at 2 every non-singleton component goes that way; clusters (creation
order, members in set-iteration order, statistics) and the final weights must
equal the oracle's bit for bit on every case, and equal the warp kernel's."""
import numpy as np
import pytest

import rtrex_cuda_b200 as rtr
from tests import helpers

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,eps", helpers.all_cases())
def test_block_extraction_bit_exact(name, eps):
    n, u, v = helpers.case_graph(name)
    (_, _, _), c, s0, s1, cl, s2 = helpers.oracle_run(name, eps)
    for split in (2, 64):
        with rtr.Graph.from_edges(n, u, v) as g:
            g.set_extract_split(split)
            assert g.decompose(eps) == len(cl), (name, eps, split)
            got = g.clusters()
            assert (got.seed == cl.seed).all() and (got.off == cl.off).all(), (name, eps, split)
            assert (got.vert == cl.vert).all(), (name, eps, split)
            assert (got.ne == cl.ne).all() and (got.cut == cl.cut).all(), (name, eps, split)
            pe, pv, sup, t = g.weights()
            assert (helpers.bits(pe) == helpers.bits(s2.perEdge)).all(), (name, eps, split)
            assert (helpers.bits(pv) == helpers.bits(s2.perVertex)).all(), (name, eps, split)
            assert t == s2.total, (name, eps, split)


def test_block_extraction_in_a_batch():
    gs = [helpers.case_graph(x) for x in ("sbm_3000_4002", "small_test", "gnp_cliques")]
    with rtr.Graph.batch(gs) as b:
        b.set_extract_split(2)
        b.decompose(0.1)
        counts = b.batch_cluster_counts()
    for (n, u, v), k in zip(gs, counts):
        with rtr.Graph.from_edges(n, u, v) as g:
            assert g.decompose(0.1) == k
