"""Counting in the rows layout (no triangle lists): perEdge from the edge pass,
perVertex folded from 4-byte per-slot lists of its z > y terms
(rtrex_cuda_b200/csrc/count_rows.cu).

* Every fixture case, with work splits that send every vertex through each of
  the two perVertex folds (thread, warp) and every edge through the heavy-edge
  (warp) fill, bit for bit against the oracle's commonNbr restatement.
* The device R-MAT generator against its numpy definition.
* R-MAT scale 22 (2.1 G triangles: its lists would need ~200 GB, so the
  default count mode picks the rows layout by itself): the exact total against
  an independent CPU count, and seeded samples of perEdge / support / perVertex
  cells -- every edge and the perVertex of the highest-degree vertices among
  them -- recomputed from the CSR by the oracle's per-cell fold.
"""
import numpy as np
import pytest

import oracle
import rtrex_cuda_b200 as rtr
from rtrex_cuda_b200 import graphgen
from tests import helpers

pytestmark = pytest.mark.gpu

# (gallop, light degree, heavy-edge degree sum, perVertex terms from which a
# warp folds): the default split, then splits that push every vertex to one
# fold and every edge to the warp path
SPLITS = [
    (16, 32, 1024, 1024),
    (16, 1 << 30, 1 << 30, 1 << 30),  # every edge a thread, every vertex a thread
    (4, 1, 1, 1 << 30),               # every edge a warp, every vertex a thread
    (16, 1, 1, 1),                    # every edge a warp, every vertex with terms a warp
    (64, 4, 8, 16),                   # a mix
]


def _rows_count(n, u, v, split):
    gal, light, edge, hub = split
    with rtr.Graph.from_edges(n, u, v) as g:
        g.set_tuning(gal, light, edge)
        g.set_count_mode(2, hub)
        total = g.count()
        assert g.count_mode() == (2, hub, False)
        pe, pv, sup, _ = g.weights()
        with pytest.raises(rtr.RtrError) as ei:
            g.clean(0.3)
        assert ei.value.code == 4 and "rows layout" in str(ei.value)
    return total, pe, pv, sup


@pytest.mark.parametrize("name", sorted({c for c, _ in helpers.all_cases()}))
def test_rows_layout_bit_exact(name):
    (_, _, _), c, s0, _, _, _ = helpers.oracle_run(name, helpers.all_cases([name])[0][1])
    n, u, v = helpers.case_graph(name)
    for split in SPLITS:
        total, pe, pv, sup = _rows_count(n, u, v, split)
        assert total == s0.total, (name, split)
        assert (helpers.bits(pe) == helpers.bits(s0.perEdge)).all(), (name, split)
        assert (helpers.bits(pv) == helpers.bits(s0.perVertex)).all(), (name, split)
        assert (sup == s0.support).all(), (name, split)


@pytest.mark.parametrize("name", ["chung_lu", "rmat14", "clean_astro"])
def test_rows_layout_in_windows_bit_exact(name):
    """Per-slot lists taken in several windows of whole rows (as at R-MAT scale 24,
    where they do not fit in one): the same bits as the oracle."""
    (_, _, _), c, s0, _, _, _ = helpers.oracle_run(name, 0.3)
    n, u, v = helpers.case_graph(name)
    with rtr.Graph.from_edges(n, u, v) as g:
        g.set_count_mode(2)
        assert g.count() == s0.total
        windows, entries = g.count_windows()
        assert windows == 1 and entries == 3 * s0.total
        g.set_count_window(max(entries // 5, 1))  # a window must hold the largest vertex's terms
        try:
            total = g.count()
        except rtr.RtrError as e:  # one vertex alone above the window: pick a larger one
            assert e.code == 4 and "alone has" in str(e)
            g.set_count_window(entries // 2)
            total = g.count()
        assert total == s0.total
        windows, _ = g.count_windows()
        assert windows > 1, (name, windows)
        pe, pv, sup, _ = g.weights()
        assert (helpers.bits(pe) == helpers.bits(s0.perEdge)).all()
        assert (helpers.bits(pv) == helpers.bits(s0.perVertex)).all()
        assert (sup == s0.support).all()


def test_rows_layout_then_lists_again():
    n, u, v = helpers.case_graph("sbm_3000_4002")
    (_, _, _), c, s0, s1, _, _ = helpers.oracle_run("sbm_3000_4002", 0.1)
    with rtr.Graph.from_edges(n, u, v) as g:
        g.set_count_mode(2)
        assert g.count() == s0.total
        g.set_count_mode(0)
        assert g.count() == s0.total
        assert g.count_mode()[2] is True
        assert g.clean(0.1) == s1.total
        assert (g.status() == s1.status).all()


@pytest.mark.parametrize("scale,ef,abc,seed", [(8, 8, (0.57, 0.19, 0.19), 3), (12, 16, (0.57, 0.19, 0.19), 7),
                                               (11, 4, (0.45, 0.25, 0.15), 11)])
def test_device_rmat_matches_numpy_definition(scale, ef, abc, seed):
    n, u, v = graphgen.rmat_hashed(scale, ef, *abc, seed=seed)
    c = oracle.build_csr(n, u, v)
    with rtr.Graph.from_rmat(scale, ef, *abc, seed=seed) as g:
        off, nb = g.csr()
    assert (off == c.offsets).all() and (nb == c.nbors).all()


def test_rmat22_rows_layout_sampled_cells():
    with rtr.Graph.from_rmat(22, 16, seed=3) as g:
        total = g.count()
        mode, _, lists = g.count_mode()
        assert mode == 0 and lists is False  # ~200 GB of lists: the rows layout was chosen
        off, nb = g.csr()
        pe, pv, sup, _ = g.weights()
    n = off.size - 1
    deg = np.diff(off)
    assert total == oracle.count_total(off, nb)
    rng = np.random.Generator(np.random.PCG64(22))
    top = np.argsort(-deg, kind="stable")[:100]
    # perEdge / support: every edge of the 3 highest-degree vertices, the heaviest
    # row pairs among the top 100, and a uniform sample
    hub_slots = np.concatenate([np.arange(off[x], off[x + 1]) for x in top[:3]])
    top_set = np.zeros(n, bool)
    top_set[top] = True
    src = np.repeat(np.arange(n), deg)
    among_top = np.flatnonzero(top_set[src] & top_set[nb])
    slots = np.unique(np.concatenate([hub_slots, among_top, rng.integers(0, nb.size, 100_000)]))
    assert slots.size >= 100_000
    cpe, csup = oracle.cells_edge(off, nb, slots)
    assert (helpers.bits(pe[slots]) == helpers.bits(cpe)).all()
    assert (sup[slots] == csup).all()
    # perVertex: the 10 highest-degree vertices and a uniform sample
    verts = np.unique(np.concatenate([top[:10], rng.integers(0, n, 10_000)]))
    cpv = oracle.cells_vertex(off, nb, verts)
    assert (helpers.bits(pv[verts]) == helpers.bits(cpv)).all()
