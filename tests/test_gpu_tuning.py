"""The counting work split (gallop ratio, heavy-vertex degree) and its
autotuner change the time, never a bit of the result."""
import numpy as np
import pytest

import rtrex_cuda_b200 as rtr
from tests import helpers

pytestmark = pytest.mark.gpu


def _count(n, u, v, tuning=None):
    with rtr.Graph.from_edges(n, u, v) as g:
        if tuning:
            g.set_tuning(*tuning)
        g.count()
        pe, pv, sup, t = g.weights()
        return helpers.bits(pe).copy(), helpers.bits(pv).copy(), sup.copy(), t


@pytest.mark.parametrize("name", ["sbm_3000_4002", "rmat14", "chung_lu", "small_test", "isolated"])
def test_every_work_split_gives_the_same_bits(name):
    n, u, v = helpers.case_graph(name)
    ref = _count(n, u, v)
    for tuning in [(1, 1, 1), (4, 8, 2), (64, 128, 64), (1 << 20, 1 << 30, 1 << 30), (2, 2, 16), (16, 32, 4)]:
        got = _count(n, u, v, tuning)
        for a, b in zip(got, ref):
            assert np.array_equal(a, b), (name, tuning)


def test_autotune_then_decompose_matches_reference():
    (n, u, v), c, s0, s1, cl, _ = helpers.oracle_run("gnp_cliques", 0.3)
    with rtr.Graph.from_edges(n, u, v) as g:
        gal, heavy, edge = g.autotune()
        assert gal in (4, 8, 16, 32, 64) and heavy in (8, 16, 32, 64, 128)
        assert edge in (128, 256, 512, 1024, 4096, 1 << 30)
        assert g.tuning() == (gal, heavy, edge)
        pe, pv, sup, t = g.weights()  # autotune leaves the graph counted
        assert t == s0.total and (helpers.bits(pe) == helpers.bits(s0.perEdge)).all()
        assert g.decompose(0.3) == len(cl)
        assert (g.clusters().vert == cl.vert).all()
