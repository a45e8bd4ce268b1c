"""Shared helpers for the parity tests: fixture graphs, oracle runs, digests.

The digests are computed exactly as tests/golden/make_golden.py computes them
from the reference's own outputs, so a match proves bit-equality with the
reference on that stage.
"""
from __future__ import annotations

import functools
import hashlib
import json
import os

import numpy as np

import oracle
from tests.golden.cases import load_case

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden", "golden.json")


def sha(b: bytes) -> str:
    return hashlib.sha256(b).hexdigest()


@functools.lru_cache(maxsize=None)
def golden():
    with open(GOLDEN) as f:
        return json.load(f)


def case_graph(name: str):
    """(n, src, dst) for a fixture case (the bundled reference files are committed copies)."""
    return load_case(name)


@functools.lru_cache(maxsize=8)
def _oracle_cached(name: str, eps: float):
    n, u, v = case_graph(name)
    c = oracle.build_csr(n, u, v)
    s0 = oracle.count(c)
    s1 = oracle.initial_clean(c, s0, eps)
    cl, s2 = oracle.extract(c, s1, eps)
    return (n, u, v), c, s0, s1, cl, s2


def oracle_run(name: str, eps: float):
    return _oracle_cached(name, float(eps))


def bits(a: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


def cluster_lines(nv, ne, cut, off, vert):
    return [f"{nv[k]} {ne[k]} {cut[k]} :" + "".join(f" {x}" for x in vert[off[k]:off[k + 1]])
            for k in range(len(nv))]


def digests(s0, s1, clusters) -> dict:
    """Per-stage digests in the format of golden.json."""
    lines = cluster_lines(clusters.nv, clusters.ne, clusters.cut, clusters.off, clusters.vert)
    return {
        "count": {"total": int(s0.total), "perEdge": sha(bits(s0.perEdge).tobytes()),
                  "perVertex": sha(bits(s0.perVertex).tobytes())},
        "clean": {"total": int(s1.total), "status": sha(np.ascontiguousarray(s1.status, np.uint8).tobytes()),
                  "perEdge": sha(bits(s1.perEdge).tobytes()), "perVertex": sha(bits(s1.perVertex).tobytes())},
        "extract": {"clusters": len(lines), "digest": sha(("\n".join(lines) + "\n").encode())},
    }


def c_hexfloat(x: float) -> str:
    """printf("%a") of a positive normal double, as glibc writes it."""
    h = float(x).hex()  # '0x1.8000000000000p-1'
    mant, exp = h[2:].split("p")
    head, _, frac = mant.partition(".")
    frac = frac.rstrip("0")
    return "0x" + head + ("." + frac if frac else "") + "p" + exp


def expand_digests(cl, score_v, score_x) -> dict:
    """Digests of an expandClusters result in the format of golden.json."""
    lines = cluster_lines(cl.nv, cl.ne, cl.cut, cl.off, cl.vert)
    sc = "".join(f"{v} {c_hexfloat(x)}\n" for v, x in zip(score_v.tolist(), score_x.tolist()))
    return {"clusters": len(lines), "digest": sha(("\n".join(lines) + "\n").encode()),
            "scores": sha(sc.encode()), "nscores": len(score_v)}


def oracle_expand(name: str, eps: float, threshold: int):
    """The oracle's expandClusters on a fresh extraction of the case."""
    (_, _, _), c, s0, s1, _, _ = oracle_run(name, eps)
    oracle.extract(c, s1, eps)  # sets the member sets orc_expand continues from
    return oracle.expand(c, threshold)


def expand_cases(names=None):
    from tests.golden.cases import EXPAND
    return [(name, eps, t) for (name, eps), ts in EXPAND.items() for t in ts
            if names is None or name in names]


def expected(name: str, eps: float) -> dict:
    return golden()["cases"][name][repr(float(eps))]


def all_cases(names=None):
    from tests.golden.cases import CASES
    out = []
    for name, eps_list in CASES.items():
        if names is not None and name not in names:
            continue
        for eps in eps_list:
            out.append((name, eps))
    return out
