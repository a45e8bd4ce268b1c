"""Parity of the CUDA path (through the C ABI) with the restated oracle and the
reference's golden digests, stage by stage, bit for bit.

Checked per case: the CSR; after counting the triangle total and every
perEdge / perVertex bit and support count; after the clean the status bytes,
every weight bit and the triangles left; after extraction the clusters in
creation order with their members in set-iteration order and statistics,
plus the final weights; and the four output files of the drop-in writer
byte for byte against the reference CLI's.
"""
import ctypes
import hashlib
import os

import numpy as np
import pytest

import rtrex_cuda_b200 as rtr
from rtrex_cuda_b200 import graphgen
from tests import helpers

pytestmark = pytest.mark.gpu

CASES = helpers.all_cases()


def _gpu_stages(n, u, v, eps):
    g = rtr.Graph.from_edges(n, u, v)
    off, nb = g.csr()
    total = g.count()
    w0 = g.weights()
    left = g.clean(eps)
    w1 = g.weights()
    st = g.status()
    k = g.extract()
    cl = g.clusters()
    w2 = g.weights()
    stats = g.stats()
    g.close()
    return dict(off=off, nb=nb, total=total, w0=w0, left=left, w1=w1, st=st, k=k, cl=cl, w2=w2, stats=stats)


@pytest.mark.parametrize("name,eps", CASES)
def test_stages_bit_exact(name, eps):
    (n, u, v), c, s0, s1, cl, s2 = helpers.oracle_run(name, eps)
    r = _gpu_stages(n, u, v, eps)
    assert (r["off"] == c.offsets).all() and (r["nb"] == c.nbors).all()
    pe, pv, sup, t = r["w0"]
    assert r["total"] == s0.total == t
    assert (helpers.bits(pe) == helpers.bits(s0.perEdge)).all()
    assert (helpers.bits(pv) == helpers.bits(s0.perVertex)).all()
    assert (sup == s0.support).all()
    pe, pv, sup, t = r["w1"]
    assert r["left"] == s1.total == t
    assert (r["st"] == s1.status).all()
    assert (helpers.bits(pe) == helpers.bits(s1.perEdge)).all()
    assert (helpers.bits(pv) == helpers.bits(s1.perVertex)).all()
    assert (sup == s1.support).all()
    g = r["cl"]
    assert r["k"] == len(cl) == len(g)
    for f in ("seed", "nv", "ne", "cut", "off", "vert"):
        assert (getattr(g, f) == getattr(cl, f)).all(), f
    pe, pv, sup, t = r["w2"]
    assert (helpers.bits(pe) == helpers.bits(s2.perEdge)).all()
    assert (helpers.bits(pv) == helpers.bits(s2.perVertex)).all()
    assert t == s2.total
    # and against the reference's own digests
    want = helpers.expected(name, eps)
    got = helpers.digests(
        type("S", (), dict(total=r["total"], perEdge=r["w0"][0], perVertex=r["w0"][1]))(),
        type("S", (), dict(total=r["left"], status=r["st"], perEdge=r["w1"][0], perVertex=r["w1"][1]))(), g)
    for stage in ("count", "clean", "extract"):
        assert got[stage] == want[stage], stage


@pytest.mark.parametrize("name,eps", helpers.all_cases(["small_test", "k20", "tie_threshold", "gnp_cliques",
                                                        "sbm_3000_4002", "sbm_20000_4000", "chung_lu"]))
def test_dropin_output_files_byte_identical(name, eps, tmp_path):
    """rtr_run_file writes the same four files as the reference CLI."""
    n, u, v = helpers.case_graph(name)
    path = str(tmp_path / "g.txt")
    graphgen.write_escape(path, n, u, v)
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        rtr.run_file(path, "g", eps, prefix="RTRex-")
    finally:
        os.chdir(cwd)
    want = helpers.expected(name, eps)["files"]
    for kind in ("decomposition", "stats", "freq", "cut"):
        got = hashlib.sha256(open(tmp_path / f"RTRex-g-{kind}.txt", "rb").read()).hexdigest()
        assert got == want[kind], kind


@pytest.mark.parametrize("name,eps", helpers.all_cases(["small_test", "isolated", "two_k5_bridge", "gnp_cliques",
                                                        "sbm_20000_4000", "chung_lu"]))
def test_rtrex_mode_outputs_byte_identical(name, eps, tmp_path):
    """With the RTRex driver's prefix the CLI path also writes the connected
    components files and the survivor dump, byte-identical to the reference's."""
    n, u, v = helpers.case_graph(name)
    path = str(tmp_path / "g.txt")
    graphgen.write_escape(path, n, u, v)
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        rc = rtr.lib().rtr_run_file(path.encode(), b"g", eps, 0, b"RTRex-", 2)
        assert rc == 0, rtr.lib().rtr_last_error()
    finally:
        os.chdir(cwd)
    want = helpers.expected(name, eps)["files"]
    for kind in ("decomposition", "stats", "freq", "cut"):
        got = hashlib.sha256(open(tmp_path / f"connected-components-g-{kind}.txt", "rb").read()).hexdigest()
        assert got == want["cc_" + kind], kind
    got = hashlib.sha256(open(tmp_path / "amazon_cleaned_edges.txt", "rb").read()).hexdigest()
    assert got == want["cleaned_edges"]


def test_components_discovery_order_matches_bfs():
    """rtr_get_components: creation order and BFS discovery order of connectedComp."""
    from collections import deque
    n, u, v = helpers.case_graph("sbm_3000_4002")
    with rtr.Graph.from_edges(n, u, v) as g:
        k = ctypes.c_int64()
        assert rtr.lib().rtr_connected_components(g._h, ctypes.byref(k)) == 0
        off = np.zeros(k.value + 1, np.int64)
        vert = np.zeros(n, np.int64)
        assert rtr.lib().rtr_get_components(g._h, off.ctypes.data, vert.ctypes.data) == 0
        o, nb = g.csr()
    seen = np.zeros(n, bool)
    comps = []
    for s0 in range(n):
        if seen[s0]:
            continue
        order, q = [s0], deque([s0])
        seen[s0] = True
        while q:
            x = q.popleft()
            for y in nb[o[x]:o[x + 1]]:
                if not seen[y]:
                    seen[y] = True
                    q.append(y)
                    order.append(int(y))
        comps.append(order)
    assert k.value == len(comps)
    for c, order in enumerate(comps):
        assert vert[off[c]:off[c + 1]].tolist() == order


def test_from_host_csr_matches_edges():
    (n, u, v), c, s0, s1, cl, _ = helpers.oracle_run("sbm_3000_4002", 0.1)
    g = rtr.Graph.from_csr(c.offsets, c.nbors)
    assert g.decompose(0.1) == len(cl)
    got = g.clusters()
    assert (got.vert == cl.vert).all() and (got.off == cl.off).all()
    assert (g.status() == ord("N")).all()  # extraction deletes every edge
    g.close()


def test_repeat_runs_identical():
    """Run-to-run identity: no floating-point atomics anywhere."""
    n, u, v = helpers.case_graph("sbm_20000_4004")
    outs = []
    for _ in range(3):
        with rtr.Graph.from_edges(n, u, v) as g:
            g.count()
            g.clean(0.1)
            w = g.weights()
            g.extract()
            outs.append((helpers.bits(w[0]).copy(), helpers.bits(w[1]).copy(), g.clusters().vert.copy()))
    for o in outs[1:]:
        for a, b in zip(o, outs[0]):
            assert (a == b).all()


def test_recount_resets_state():
    (n, u, v), c, s0, s1, cl, _ = helpers.oracle_run("gnp_cliques", 0.3)
    with rtr.Graph.from_edges(n, u, v) as g:
        g.decompose(0.3)
        assert g.decompose(0.3) == len(cl)
        assert (g.clusters().vert == cl.vert).all()


def test_rejects_non_simple_input():
    with pytest.raises(rtr.RtrError) as e:
        rtr.Graph.from_edges(4, np.array([0, 1, 1]), np.array([1, 2, 1]))
    assert e.value.code == 3 and "self-loop" in str(e.value)
    with pytest.raises(rtr.RtrError) as e:
        rtr.Graph.from_edges(4, np.array([0, 1, 1]), np.array([1, 2, 0]))
    assert e.value.code == 3 and "duplicate" in str(e.value)


def test_rejects_out_of_range_ids():
    with pytest.raises(rtr.RtrError) as e:
        rtr.Graph.from_edges(3, np.array([0, 1]), np.array([1, 3]))
    assert e.value.code == 3


def test_simplify_flag_matches_oracle_on_simplified_graph():
    import oracle
    rng = np.random.default_rng(11)
    n = 300
    u = rng.integers(0, n, 4000)
    v = rng.integers(0, n, 4000)
    su, sv = graphgen.simplify(n, u, v)
    c = oracle.build_csr(n, su, sv)
    s0 = oracle.count(c)
    s1 = oracle.initial_clean(c, s0, 0.1)
    cl, _ = oracle.extract(c, s1, 0.1)
    with rtr.Graph.from_edges(n, u, v, simplify=True) as g:
        assert g.m == su.size
        assert g.decompose(0.1) == len(cl)
        assert (g.clusters().vert == cl.vert).all()


def test_stage_order_enforced():
    with rtr.Graph.from_edges(4, np.array([0, 1, 2]), np.array([1, 2, 0])) as g:
        with pytest.raises(rtr.RtrError) as e:
            g.extract()
        assert e.value.code == 5
        with pytest.raises(rtr.RtrError):
            g.clean(0.3)


@pytest.mark.parametrize("scale", [16])
def test_rmat_scale_parity(scale):
    """A larger power-law case, full bit parity against the oracle."""
    import oracle
    n, u, v = graphgen.rmat(scale=scale, edge_factor=16, seed=scale)
    c = oracle.build_csr(n, u, v)
    s0 = oracle.count(c)
    s1 = oracle.initial_clean(c, s0, 0.1)
    cl, _ = oracle.extract(c, s1, 0.1)
    r = _gpu_stages(n, u, v, 0.1)
    assert r["total"] == s0.total
    assert (helpers.bits(r["w0"][0]) == helpers.bits(s0.perEdge)).all()
    assert (r["st"] == s1.status).all()
    assert (helpers.bits(r["w1"][1]) == helpers.bits(s1.perVertex)).all()
    assert (r["cl"].vert == cl.vert).all() and (r["cl"].off == cl.off).all()
