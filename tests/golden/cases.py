"""Fixture graphs for the parity suite.

Every case is either regenerated from a seed by rtrex_cuda_b200.graphgen, built
by hand below (edge cases), or one of the reference's bundled data files
(BUNDLED: RTRex_Sequential/clustering/{random_graph_rtr,clean_email,clean_astro}.txt,
kept byte for byte, gzip-compressed, under tests/golden/data/ so they run
wherever the tests run; tests/golden/make_golden.py --copy-bundled refreshes them
from a reference checkout).  CASES maps a case name to the thresholds it is checked at; 0.3 is
the reference's documented setting (RTRex_CUDA/README.md) and 0.1 the paper's.

The SBM cases at eps=0.1 are order-sensitive: a bulk-synchronous peel leaves a
different survivor set than the reference's LIFO cascade on them (10-300
directed edges differ), so they exercise the order-faithful replay.
"""
from __future__ import annotations

import numpy as np

from rtrex_cuda_b200 import graphgen

import os

# bundled case -> its file inside the reference project
BUNDLED = {
    "random_graph_rtr": "RTRex_Sequential/clustering/random_graph_rtr.txt",
    "clean_email": "RTRex_Sequential/clustering/clean_email.txt",
    "clean_astro": "RTRex_Sequential/clustering/clean_astro.txt",
}

DATA_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")


def bundled_path(name: str) -> str:
    """The committed (gzip) copy of a bundled case's data file."""
    return os.path.join(DATA_DIR, os.path.basename(BUNDLED[name]) + ".gz")

CASES = {
    # edge cases
    "isolated": [0.3],
    "no_edges_but_one": [0.3],
    "triangle_free_star": [0.3],
    "k4": [0.3, 0.1],
    "k20": [0.3],
    "two_k5_bridge": [0.3, 0.1],
    "tie_threshold": [0.3],
    "eps_zero": [0.0],
    "eps_one": [1.0],
    # the reference's example and seeded workloads
    "small_test": [0.3, 0.1],
    "gnp_cliques": [0.3, 0.1],
    "chung_lu": [0.3, 0.1],
    "sbm_3000_4002": [0.1, 0.3],
    "sbm_3000_4003": [0.1],
    "sbm_20000_4000": [0.1],
    "sbm_20000_4004": [0.1],
    "sbm_20000_4010": [0.1],
    "rmat12": [0.3, 0.1],
    "rmat14": [0.1],
    # bundled reference data
    "random_graph_rtr": [0.3],
    "clean_email": [0.3, 0.1],
    "clean_astro": [0.3, 0.1],
}

# expandClusters (the RTRex driver's mode e) thresholds checked per (case, eps).
# Thresholds below 1 let singletons join singleton clusters; they pin the
# oracle's container handling of that case.
EXPAND = {
    ("isolated", 0.3): [1],
    ("k20", 0.3): [1],
    ("two_k5_bridge", 0.3): [1, 0],
    ("small_test", 0.3): [1, 2, 0, -1],
    ("small_test", 0.1): [1],
    ("sbm_3000_4002", 0.1): [1, 2, 0],
    ("sbm_3000_4003", 0.1): [2],
    ("rmat12", 0.3): [1, 3, 0],
    ("gnp_cliques", 0.3): [1, 2, 3],
    ("sbm_20000_4000", 0.1): [1, 2],
    ("chung_lu", 0.3): [1, 2, 0],
    ("clean_email", 0.3): [2],
}

# Cases small enough for the fast CPU suite (the rest run in the GPU suite).
SMALL = ["isolated", "no_edges_but_one", "triangle_free_star", "k4", "k20", "two_k5_bridge", "tie_threshold",
         "eps_zero", "eps_one", "small_test", "sbm_3000_4002", "sbm_3000_4003", "rmat12"]


def _pairs(n, pairs):
    u = np.array([p[0] for p in pairs], dtype=np.int64)
    v = np.array([p[1] for p in pairs], dtype=np.int64)
    return n, u, v


def _clique(vs):
    return [(a, b) for i, a in enumerate(vs) for b in vs[i + 1:]]


def load_case(name: str):
    """(n, src, dst) for a fixture case (bundled files in file-line order)."""
    if name in BUNDLED:
        return graphgen.read_escape(bundled_path(name))
    if name == "isolated":
        return _pairs(5, [])
    if name == "no_edges_but_one":
        return _pairs(4, [(1, 2)])
    if name == "triangle_free_star":
        return _pairs(40, [(0, i) for i in range(1, 40)] + [(i, i + 1) for i in range(1, 39, 2)][:0])
    if name == "k4":
        return _pairs(4, _clique([0, 1, 2, 3]))
    if name == "k20":
        return _pairs(25, _clique(list(range(3, 23))))
    if name == "two_k5_bridge":
        return _pairs(12, _clique([0, 1, 2, 3, 4]) + _clique([6, 7, 8, 9, 10]) + [(4, 5), (5, 6), (4, 6), (11, 0)])
    if name == "tie_threshold":
        # edge (0,1) sits in three triangles whose third vertices have degree 10:
        # sum of 1/d_w = 3/10 equals eps = 0.3 exactly in rationals.
        pairs = [(0, 1)]
        nxt = 5
        for w in (2, 3, 4):
            pairs += [(0, w), (1, w)]
            for _ in range(8):
                pairs.append((w, nxt))
                nxt += 1
        return _pairs(nxt, pairs)
    if name == "eps_zero" or name == "eps_one":
        return graphgen.gnp_cliques(n=600, p=0.01, n_cliques=4, clique_size=8, seed=7)
    if name == "small_test":
        return graphgen.small_test()
    if name in ("gnp_cliques", "chung_lu"):
        return graphgen.config_graph(name)
    if name.startswith("sbm_"):
        _, m, seed = name.split("_")
        return graphgen.sbm(int(m), int(seed))
    if name.startswith("rmat"):
        sc = int(name[4:])
        return graphgen.rmat(scale=sc, edge_factor=16, seed=sc)
    raise KeyError(name)
