"""Randomised parity: seeded random graphs of varied shape and density, every
stage of the CUDA path against the oracle bit for bit (count, clean, extraction,
expansion), and random Escape texts through the device parser against the host
loader.  Seeds are fixed, so a failure reproduces."""
import numpy as np
import pytest

import oracle
import rtrex_cuda_b200 as rtr
from rtrex_cuda_b200 import graphgen
from tests import helpers

pytestmark = pytest.mark.gpu


def _random_graph(seed):
    rng = np.random.default_rng(seed)
    kind = seed % 4
    if kind == 0:  # sparse G(n, m) with a few planted cliques
        n = int(rng.integers(20, 400))
        m = int(rng.integers(n, 6 * n))
        u, v = rng.integers(0, n, m), rng.integers(0, n, m)
        for _ in range(int(rng.integers(0, 4))):
            c = rng.choice(n, size=int(rng.integers(4, min(12, n))), replace=False)
            a, b = np.triu_indices(c.size, 1)
            u, v = np.concatenate([u, c[a]]), np.concatenate([v, c[b]])
    elif kind == 1:  # dense small graph: many ties and long triangle lists
        n = int(rng.integers(8, 60))
        p = rng.uniform(0.2, 0.8)
        a, b = np.triu_indices(n, 1)
        keep = rng.random(a.size) < p
        u, v = a[keep], b[keep]
    elif kind == 2:  # star-like hubs: skewed degrees
        n = int(rng.integers(50, 500))
        hubs = rng.choice(n, size=int(rng.integers(1, 6)), replace=False)
        m = int(rng.integers(n, 4 * n))
        u = rng.choice(hubs, m)
        v = rng.integers(0, n, m)
        u = np.concatenate([u, rng.integers(0, n, m // 2)])
        v = np.concatenate([v, rng.integers(0, n, m // 2)])
    else:  # small R-MAT
        n, u, v = graphgen.rmat(scale=int(rng.integers(6, 10)), edge_factor=int(rng.integers(2, 12)),
                                seed=int(seed))
        return n, u, v
    su, sv = graphgen.simplify(n, u, v)
    return n, su, sv


@pytest.mark.parametrize("seed", range(96))
def test_random_graph_all_stages(seed):
    n, u, v = _random_graph(seed)
    eps = [0.3, 0.1, 0.5, 0.05][seed % 4]
    c = oracle.build_csr(n, u, v)
    s0 = oracle.count(c)
    s1 = oracle.initial_clean(c, s0, eps)
    cl, s2 = oracle.extract(c, s1, eps)
    thr = [1, 2, 0][seed % 3]
    xcl, xv, xs = oracle.expand(c, thr)
    with rtr.Graph.from_edges(n, u, v) as g:
        if seed % 2:  # an unusual work split must not change a bit
            g.set_tuning(2, 2, 8)
        t = g.count()
        pe, pv, sup, _ = g.weights()
        assert t == s0.total
        assert (helpers.bits(pe) == helpers.bits(s0.perEdge)).all() and (sup == s0.support).all()
        assert (helpers.bits(pv) == helpers.bits(s0.perVertex)).all()
        left = g.clean(eps)
        pe, pv, sup, _ = g.weights()
        assert left == s1.total and (g.status() == s1.status).all()
        assert (helpers.bits(pe) == helpers.bits(s1.perEdge)).all()
        assert (helpers.bits(pv) == helpers.bits(s1.perVertex)).all()
        assert g.extract() == len(cl)
        got = g.clusters()
        for f in ("nv", "ne", "cut", "off", "vert"):
            assert (getattr(got, f) == getattr(cl, f)).all(), f
        pe, pv, _, t2 = g.weights()
        assert t2 == s2.total and (helpers.bits(pv) == helpers.bits(s2.perVertex)).all()
        g.expand(thr)
        gx, _ = g.expanded()
        gv, gs = g.scores()
        assert helpers.expand_digests(gx, gv, gs) == helpers.expand_digests(xcl, xv, xs)


@pytest.mark.parametrize("seed", range(32))
def test_random_escape_text_device_equals_host(seed, tmp_path):
    rng = np.random.default_rng(1000 + seed)
    n = int(rng.integers(1, 300))
    m = int(rng.integers(0, 800))
    pairs = [(int(rng.integers(0, n)), int(rng.integers(0, n))) for _ in range(m)]
    lines = []
    if rng.random() < 0.5:
        lines.append("# header comment")
    lines.append(f"{n}{' ' * int(rng.integers(1, 3))}{m}")
    for a, b in pairs:
        r = rng.random()
        if r < 0.05:
            lines.append("")
        elif r < 0.08:
            lines.append("# c")
        lines.append(f"{a}{rng.choice([' ', '\t', '  '])}{b}{rng.choice(['', ' 9', '\r'])}")
    extra = int(rng.integers(0, 3))
    lines += [f"{int(rng.integers(0, n))} {int(rng.integers(0, n))}" for _ in range(extra)]
    if seed % 5 == 4:  # short file
        lines = lines[:-max(1, extra + 1)]
    text = "\n".join(lines) + ("\n" if seed % 2 else "")
    path = str(tmp_path / "g.txt")
    open(path, "w").write(text)
    try:
        hn, hu, hv = rtr.load_escape(path)
        host = None
    except rtr.RtrError as e:
        host = (e.code, str(e))
    try:
        with rtr.Graph.from_escape_file(path, simplify=True) as g:
            dev = None
            off, nb = g.csr()
    except rtr.RtrError as e:
        dev = (e.code, str(e))
    assert host == dev
    if host is None:
        with rtr.Graph.from_edges(hn, hu, hv, simplify=True) as h:
            ho, hb = h.csr()
        assert (off == ho).all() and (nb == hb).all()
