"""The oracle's per-cell restatement of commonNbr (oracle/rtr_cells.cpp), used to
check large graphs cell by cell, pinned on CPU:

* every perEdge / support / perVertex cell of the fixture cases equals the
  whole-graph restatement orc_count, and its digests equal the reference's own
  (tests/golden/golden.json, written by the reference built from its sources);
* the degree-oriented triangle total equals commonNbr's total;
* the hashed R-MAT generator (the definition the device generator follows) is
  deterministic, in range and simple, and at scale 16 / edge factor 16 / seed 3
  keeps 909,359 edges -- the count an independent C++ implementation of the same
  definition gave.
"""
import numpy as np
import pytest

import oracle
from rtrex_cuda_b200 import graphgen
from tests import helpers
from tests.golden.cases import SMALL


@pytest.mark.parametrize("name", SMALL + ["gnp_cliques", "clean_email", "random_graph_rtr"])
def test_cells_equal_whole_graph_restatement(name):
    (_, _, _), c, s0, _, _, _ = helpers.oracle_run(name, helpers.all_cases([name])[0][1])
    pe, sup = oracle.cells_edge(c.offsets, c.nbors, np.arange(c.m2))
    pv = oracle.cells_vertex(c.offsets, c.nbors, np.arange(c.n))
    assert (helpers.bits(pe) == helpers.bits(s0.perEdge)).all()
    assert (sup == s0.support).all()
    assert (helpers.bits(pv) == helpers.bits(s0.perVertex)).all()
    assert oracle.count_total(c.offsets, c.nbors) == s0.total
    gold = next(iter(helpers.golden()["cases"][name].values()))["count"]
    assert helpers.sha(helpers.bits(pe).tobytes()) == gold["perEdge"]
    assert helpers.sha(helpers.bits(pv).tobytes()) == gold["perVertex"]
    assert s0.total == gold["total"]


def test_cells_of_a_sample_match_in_any_order():
    (_, _, _), c, s0, _, _, _ = helpers.oracle_run("sbm_3000_4002", 0.1)
    rng = np.random.Generator(np.random.PCG64(5))
    slots = rng.integers(0, c.m2, 500)
    verts = rng.integers(0, c.n, 200)
    pe, sup = oracle.cells_edge(c.offsets, c.nbors, slots)
    pv = oracle.cells_vertex(c.offsets, c.nbors, verts)
    assert (helpers.bits(pe) == helpers.bits(s0.perEdge[slots])).all()
    assert (sup == s0.support[slots]).all()
    assert (helpers.bits(pv) == helpers.bits(s0.perVertex[verts])).all()


def test_hashed_rmat_definition():
    n, u, v = graphgen.rmat_hashed(16, 16, seed=3)
    assert n == 1 << 16 and u.size == 909_359
    assert (u < v).all() and u.min() >= 0 and v.max() < n
    key = u * n + v
    assert (np.diff(key) > 0).all()  # sorted, no repeats
    n2, u2, v2 = graphgen.rmat_hashed(16, 16, seed=3)
    assert (u2 == u).all() and (v2 == v).all()
    _, u3, _ = graphgen.rmat_hashed(16, 16, seed=4)
    assert u3.size != u.size or (u3 != u).any()
    deg = np.bincount(np.concatenate([u, v]), minlength=n)
    assert deg[0] == deg.max()  # the (a, a, ...) corner: vertex 0 is the largest hub
