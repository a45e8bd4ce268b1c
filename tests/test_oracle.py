"""Pin the restated CPU oracle against the reference (CPU only).

The digests in tests/golden/golden.json were produced by the reference's own
code (oracle/_ref/rtr_ref_dump, built from RTRex_Sequential's sources); the
restated oracle must reproduce every stage of every case bit for bit.
"""
import os
import subprocess
import tempfile

import numpy as np
import pytest

import oracle
from tests import helpers
from tests.golden.cases import SMALL

FAST = helpers.all_cases(SMALL + ["gnp_cliques", "random_graph_rtr", "clean_email"])
SLOW = [c for c in helpers.all_cases() if c not in FAST]


def _check(name, eps):
    (_, _, _), c, s0, s1, cl, _ = helpers.oracle_run(name, eps)
    got = helpers.digests(s0, s1, cl)
    want = helpers.expected(name, eps)
    for stage in ("count", "clean", "extract"):
        assert got[stage] == want[stage], f"{name} eps={eps}: {stage} differs from the reference"


@pytest.mark.parametrize("name,eps", FAST)
def test_oracle_matches_reference(name, eps):
    _check(name, eps)


@pytest.mark.slow
@pytest.mark.parametrize("name,eps", SLOW)
def test_oracle_matches_reference_large(name, eps):
    _check(name, eps)


@pytest.mark.parametrize("name,eps,thr", helpers.expand_cases(SMALL + ["gnp_cliques", "clean_email"]))
def test_oracle_expand_matches_reference(name, eps, thr):
    """expandClusters (mode e): clusters, statistics, member order and scores."""
    got = helpers.expand_digests(*helpers.oracle_expand(name, eps, thr))
    assert got == {k: v for k, v in helpers.expected(name, eps)["expand"][str(thr)].items() if k != "files"}


@pytest.mark.slow
@pytest.mark.parametrize("name,eps,thr", [c for c in helpers.expand_cases()
                                          if c[0] not in SMALL + ["gnp_cliques", "clean_email"]])
def test_oracle_expand_matches_reference_large(name, eps, thr):
    got = helpers.expand_digests(*helpers.oracle_expand(name, eps, thr))
    assert got == {k: v for k, v in helpers.expected(name, eps)["expand"][str(thr)].items() if k != "files"}


def test_small_test_full_arrays():
    """Every array of the reference's Example graph, not only digests."""
    ref = np.load(os.path.join(helpers.ROOT, "tests", "golden", "small_test.npz"))
    (_, _, _), c, s0, s1, cl, _ = helpers.oracle_run("small_test", 0.3)
    assert (c.offsets == ref["offsets"]).all() and (c.nbors == ref["nbors"]).all()
    assert (helpers.bits(s0.perEdge) == helpers.bits(ref["count_perEdge"])).all()
    assert (helpers.bits(s0.perVertex) == helpers.bits(ref["count_perVertex"])).all()
    assert (s1.status == ref["clean_status"][:c.m2]).all()
    assert (helpers.bits(s1.perEdge) == helpers.bits(ref["clean_perEdge"])).all()
    lines = helpers.cluster_lines(cl.nv, cl.ne, cl.cut, cl.off, cl.vert)
    assert lines == list(ref["clusters"])
    # the known answer: one non-trivial cluster {1,3,4,6}
    big = [set(cl.members(k).tolist()) for k in range(len(cl)) if cl.nv[k] > 1]
    assert big == [{1, 3, 4, 6}]


def test_partner_copies_identical():
    """Both directed copies of an edge always hold the same weight bits, which
    lets the device keep one cell per undirected edge."""
    (_, _, _), c, s0, s1, cl, s2 = helpers.oracle_run("gnp_cliques", 0.3)
    for s in (s0, s1, s2):
        assert (helpers.bits(s.perEdge) == helpers.bits(s.perEdge[c.partner])).all()
    assert (s1.status == s1.status[c.partner]).all()


def test_fold_order_restatement():
    """perEdge is the ascending-z fold of 1/(du dv dz); perVertex the (y, z>y) fold."""
    (_, _, _), c, s0, _, _, _ = helpers.oracle_run("sbm_3000_4002", 0.1)
    off, nb, deg = c.offsets, c.nbors, c.deg
    src = np.repeat(np.arange(c.n), deg)
    rng = np.random.default_rng(5)
    for i in rng.choice(c.m2, 300, replace=False):
        a, b = src[i], nb[i]
        acc = 0.0
        for z in np.intersect1d(nb[off[a]:off[a + 1]], nb[off[b]:off[b + 1]]):
            acc += 1.0 / float(int(deg[a]) * int(deg[b]) * int(deg[z]))
        assert acc == s0.perEdge[i]
    for x in rng.choice(c.n, 100, replace=False):
        acc = 0.0
        nx = nb[off[x]:off[x + 1]]
        for y in nx:
            zs = np.intersect1d(nx, nb[off[y]:off[y + 1]])
            for z in zs[zs > y]:
                acc += 1.0 / float(int(deg[x]) * int(deg[y]) * int(deg[z]))
        assert acc == s0.perVertex[x]


def test_support_is_live_triangle_count():
    (_, _, _), c, s0, s1, _, s2 = helpers.oracle_run("sbm_3000_4003", 0.1)
    assert int(s0.support.sum()) == 6 * s0.total
    alive = s1.status == ord("Y")
    assert int(s1.support[alive].sum()) == 6 * s1.total
    assert s2.total == 0 and int(s2.support.sum()) == 0


def test_order_sensitivity_is_exercised():
    """On this SBM case a FIFO replay of the same seeds leaves a different
    survivor set; the reference's LIFO order is what the product must follow."""
    from rtrex_cuda_b200 import graphgen
    name, eps = "sbm_3000_4002", 0.1
    (n, u, v), c, s0, s1, _, _ = helpers.oracle_run(name, eps)
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "g.txt")
        graphgen.write_escape(path, n, u, v)
        exe = os.path.join(helpers.ROOT, "tests", "_bin_bsp")
        src = os.path.join(helpers.ROOT, "tests", "bsp_peel.cpp")
        if not os.path.exists(exe) or os.path.getmtime(exe) < os.path.getmtime(src):
            subprocess.run(["g++", "-O2", "-std=c++17", "-o", exe, src], check=True)
        out = subprocess.run([exe, path, repr(eps)], check=True, capture_output=True, text=True).stdout
    bsp_alive = np.array([int(x) for x in out.split()], dtype=np.uint8)
    lifo_alive = (s1.status == ord("Y")).astype(np.uint8)
    assert (bsp_alive != lifo_alive).sum() > 0
