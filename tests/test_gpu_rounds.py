"""The clean's two replays -- one warp per unit, and parallel rounds for large
units (pops with disjoint cells together, perVertex folded afterwards in the
reference's pop order) -- against the oracle bit for bit, on the same graphs,
with the split forced each way and at its default."""
import numpy as np
import pytest

import oracle
import rtrex_cuda_b200 as rtr
from rtrex_cuda_b200 import graphgen
from tests import helpers

pytestmark = pytest.mark.gpu

ALL_ROUNDS = (1, 1e30)      # every unit replays in rounds
NO_ROUNDS = (1 << 62, 0.0)  # every unit replays one warp per unit


def _check_clean(n, u, v, eps, split):
    c = oracle.build_csr(n, u, v)
    s0 = oracle.count(c)
    s1 = oracle.initial_clean(c, s0, eps)
    with rtr.Graph.from_edges(n, u, v) as g:
        if split is not None:
            g.set_clean_split(*split)
            assert g.clean_split() == split
        g.count()
        left = g.clean(eps)
        pe, pv, sup, t = g.weights()
        assert left == s1.total == t
        assert (g.status() == s1.status).all()
        assert (helpers.bits(pe) == helpers.bits(s1.perEdge)).all()
        assert (helpers.bits(pv) == helpers.bits(s1.perVertex)).all()
        assert (sup == s1.support).all()
        return g.stats()


def _random(seed):
    rng = np.random.default_rng(7000 + seed)
    kind = seed % 3
    if kind == 0:  # sparse with planted cliques
        n = int(rng.integers(50, 600))
        m = int(rng.integers(n, 6 * n))
        u, v = rng.integers(0, n, m), rng.integers(0, n, m)
        for _ in range(int(rng.integers(1, 6))):
            cq = rng.choice(n, size=int(rng.integers(4, 14)), replace=False)
            a, b = np.triu_indices(cq.size, 1)
            u, v = np.concatenate([u, cq[a]]), np.concatenate([v, cq[b]])
    elif kind == 1:  # dense: long lists, the solo path
        n = int(rng.integers(30, 90))
        a, b = np.triu_indices(n, 1)
        keep = rng.random(a.size) < rng.uniform(0.3, 0.9)
        u, v = a[keep], b[keep]
    else:
        n, u, v = graphgen.rmat(scale=int(rng.integers(7, 11)), edge_factor=int(rng.integers(4, 16)), seed=int(seed))
        return n, u, v
    su, sv = graphgen.simplify(n, u, v)
    return n, su, sv


@pytest.mark.parametrize("seed", range(48))
@pytest.mark.parametrize("split", [ALL_ROUNDS, NO_ROUNDS])
def test_random_graphs_both_replays(seed, split):
    n, u, v = _random(seed)
    _check_clean(n, u, v, [0.3, 0.1, 0.5, 0.05][seed % 4], split)


@pytest.mark.parametrize("name,eps", helpers.all_cases())
def test_reference_cases_all_rounds(name, eps):
    n, u, v = helpers.case_graph(name)
    _check_clean(n, u, v, eps, ALL_ROUNDS)


@pytest.mark.parametrize("split", [None, ALL_ROUNDS])
def test_bench_graph_rounds(split):
    """The Chung-Lu bench graph: its giant unit takes the round replay by default."""
    n, u, v = graphgen.config_graph("chung_lu")
    _check_clean(n, u, v, 0.3, split)


@pytest.mark.parametrize("eps", [0.3, 0.1])
def test_rmat_rounds(eps):
    """R-MAT: a full cascade with long lists (solo pops between rounds)."""
    n, u, v = graphgen.rmat(scale=14, edge_factor=16, seed=14)
    _check_clean(n, u, v, eps, ALL_ROUNDS)


def test_split_is_validated():
    n, u, v = _random(0)
    with rtr.Graph.from_edges(n, u, v) as g:
        with pytest.raises(rtr.RtrError):
            g.set_clean_split(0)
        with pytest.raises(rtr.RtrError):
            g.set_clean_split(5, -1.0)
        assert g.clean_split() == (2048, 8.0)


def test_full_decomposition_with_rounds():
    """Extraction after a round-replayed clean: clusters identical to the oracle."""
    n, u, v = _random(3)
    c = oracle.build_csr(n, u, v)
    s1 = oracle.initial_clean(c, oracle.count(c), 0.3)
    cl, s2 = oracle.extract(c, s1, 0.3)
    with rtr.Graph.from_edges(n, u, v) as g:
        g.set_clean_split(*ALL_ROUNDS)
        g.count()
        g.clean(0.3)
        assert g.extract() == len(cl)
        got = g.clusters()
        for f in ("nv", "ne", "cut", "off", "vert"):
            assert (getattr(got, f) == getattr(cl, f)).all(), f
        _, pv, _, t2 = g.weights()
        assert t2 == s2.total and (helpers.bits(pv) == helpers.bits(s2.perVertex)).all()
