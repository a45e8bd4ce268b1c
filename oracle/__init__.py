"""ctypes front end for the restated CPU oracle (librtr_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, never by the product package.  The library is
built from oracle/rtr_oracle.cpp by oracle/Makefile (``make -C oracle``).

Every stage keeps the reference's arrays: int64 CSR ``offsets``/``nbors``,
``partner`` (getPartnerMap), float64 ``perEdge``/``perVertex``, the
``'Y'/'S'/'N'`` status bytes, plus the integer ``support`` companion.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "librtr_oracle.so")
_lib = None

_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
_i64 = ctypes.c_int64


def build() -> str:
    """Compile librtr_oracle.so (plain g++, no GPU)."""
    subprocess.run(["make", "-s", "-C", _HERE, "librtr_oracle.so"], check=True)
    return _LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = ctypes.CDLL(_LIB)
        L.orc_build_csr.argtypes = [_i64, _i64, _i64p, _i64p, _i64p, _i64p]
        L.orc_build_csr.restype = ctypes.c_int
        L.orc_partner.argtypes = [_i64, _i64p, _i64p, _i64p]
        L.orc_partner.restype = _i64
        L.orc_count.argtypes = [_i64, _i64p, _i64p, _i64p, _f64p, _f64p, _u32p,
                                ctypes.POINTER(_i64)]
        L.orc_count.restype = None
        L.orc_initial_clean.argtypes = [_i64, _i64p, _i64p, _i64p, ctypes.c_double, _f64p, _f64p,
                                        _u32p, ctypes.POINTER(_i64), _u8p, ctypes.c_void_p,
                                        ctypes.POINTER(_i64)]
        L.orc_initial_clean.restype = None
        L.orc_extract.argtypes = [_i64, _i64p, _i64p, _i64p, ctypes.c_double, _f64p, _f64p, _u32p,
                                  ctypes.POINTER(_i64), _u8p, _i64p, _i64p, _i64p, _i64p, _i64p, _i64p]
        L.orc_extract.restype = _i64
        L.orc_expand.argtypes = [_i64, _i64p, _i64p, _i64, _i64p, _i64p, _i64p, _i64p, _i64p,
                                 ctypes.POINTER(_i64), _i64p, _f64p]
        L.orc_expand.restype = _i64
        L.orc_cells_edge.argtypes = [_i64, _i64p, _i64p, _i64, _i64p, _f64p, _u32p]
        L.orc_cells_edge.restype = None
        L.orc_cells_vertex.argtypes = [_i64, _i64p, _i64p, _i64, _i64p, _f64p]
        L.orc_cells_vertex.restype = None
        L.orc_count_total.argtypes = [_i64, _i64p, _i64p]
        L.orc_count_total.restype = _i64
        L.orc_nucleus.argtypes = [_i64, _i64p, _i64p]
        L.orc_nucleus.restype = _i64
        L.orc_nucleus_sizes.argtypes = [ctypes.POINTER(_i64)] * 3
        L.orc_nucleus_sizes.restype = None
        L.orc_nucleus_get.argtypes = [ctypes.c_void_p] * 11
        L.orc_nucleus_get.restype = None
        L.orc_selfcheck_counts.argtypes = [ctypes.POINTER(_i64)] * 3
        L.orc_selfcheck_reset.argtypes = []
        _lib = L
    return _lib


@dataclass
class Csr:
    n: int
    offsets: np.ndarray
    nbors: np.ndarray
    partner: np.ndarray

    @property
    def m2(self) -> int:
        return int(self.offsets[-1])

    @property
    def deg(self) -> np.ndarray:
        return np.diff(self.offsets)


@dataclass
class State:
    perEdge: np.ndarray
    perVertex: np.ndarray
    support: np.ndarray
    total: int
    status: np.ndarray | None = None

    def copy(self) -> "State":
        return State(self.perEdge.copy(), self.perVertex.copy(), self.support.copy(), self.total,
                     None if self.status is None else self.status.copy())


@dataclass
class Clusters:
    seed: np.ndarray
    nv: np.ndarray
    ne: np.ndarray
    cut: np.ndarray
    off: np.ndarray
    vert: np.ndarray

    def __len__(self):
        return int(self.seed.size)

    def members(self, k: int) -> np.ndarray:
        return self.vert[self.off[k]:self.off[k + 1]]


def build_csr(n: int, u: np.ndarray, v: np.ndarray) -> Csr:
    u = np.ascontiguousarray(u, dtype=np.int64)
    v = np.ascontiguousarray(v, dtype=np.int64)
    m = u.size
    off = np.zeros(n + 1, dtype=np.int64)
    nb = np.zeros(max(1, 2 * m), dtype=np.int64)
    if lib().orc_build_csr(n, m, u, v, off, nb) != 0:
        raise ValueError("vertex id out of range")
    nb = nb[:2 * m].copy()
    partner = np.zeros(max(1, 2 * m), dtype=np.int64)
    bad = lib().orc_partner(n, off, nb if nb.size else np.zeros(1, np.int64), partner)
    if bad:
        raise ValueError(f"{bad} directed edges have no reverse copy")
    return Csr(n, off, nb, partner[:2 * m].copy())


def _nb(c: Csr):
    return c.nbors if c.nbors.size else np.zeros(1, np.int64)


def _pt(c: Csr):
    return c.partner if c.partner.size else np.zeros(1, np.int64)


def count(c: Csr) -> State:
    m2 = max(1, c.m2)
    pe = np.zeros(m2, dtype=np.float64)
    pv = np.zeros(max(1, c.n), dtype=np.float64)
    sup = np.zeros(m2, dtype=np.uint32)
    tot = _i64(0)
    lib().orc_count(c.n, c.offsets, _nb(c), _pt(c), pe, pv, sup, ctypes.byref(tot))
    return State(pe[:c.m2], pv[:c.n], sup[:c.m2], int(tot.value))


def _pad(a, size, dtype):
    out = np.zeros(max(1, size), dtype=dtype)
    out[:a.size] = a
    return out


def initial_clean(c: Csr, s: State, eps: float, trace: bool = False):
    """Run initialClean on a copy of ``s``; returns the new State (and the pop trace)."""
    pe = _pad(s.perEdge, c.m2, np.float64)
    pv = _pad(s.perVertex, c.n, np.float64)
    sup = _pad(s.support, c.m2, np.uint32)
    st = np.zeros(max(1, c.m2), dtype=np.uint8)
    tot = _i64(s.total)
    tr = np.zeros(max(1, c.m2), dtype=np.int64) if trace else None
    tl = _i64(0)
    lib().orc_initial_clean(c.n, c.offsets, _nb(c), _pt(c), float(eps), pe, pv, sup, ctypes.byref(tot), st,
                            tr.ctypes.data if trace else None, ctypes.byref(tl))
    out = State(pe[:c.m2], pv[:c.n], sup[:c.m2], int(tot.value), st[:c.m2])
    if trace:
        return out, tr[:tl.value].copy()
    return out


def extract(c: Csr, s: State, eps: float):
    """Run the extraction loop on a copy of the cleaned state ``s``."""
    pe = _pad(s.perEdge, c.m2, np.float64)
    pv = _pad(s.perVertex, c.n, np.float64)
    sup = _pad(s.support, c.m2, np.uint32)
    st = _pad(s.status, c.m2, np.uint8)
    tot = _i64(s.total)
    n1 = max(1, c.n)
    seed, nv, ne, cut = (np.zeros(n1, np.int64) for _ in range(4))
    off = np.zeros(n1 + 1, np.int64)
    vert = np.zeros(n1, np.int64)
    k = lib().orc_extract(c.n, c.offsets, _nb(c), _pt(c), float(eps), pe, pv, sup, ctypes.byref(tot), st,
                          seed, nv, ne, cut, off, vert)
    cl = Clusters(seed[:k].copy(), nv[:k].copy(), ne[:k].copy(), cut[:k].copy(), off[:k + 1].copy(),
                  vert[:c.n].copy())
    return cl, State(pe[:c.m2], pv[:c.n], sup[:c.m2], int(tot.value), st[:c.m2])


def expand(c: Csr, threshold: int):
    """expandClusters on the clusters of the last :func:`extract` call.

    Returns ``(clusters, score_vertices, score_values)``; the clusters keep the
    extraction's count and order (emptied singletons have no members) and the
    ``seed`` field holds -1 (expandClusters does not track seeds)."""
    n1 = max(1, c.n)
    nv, ne, cut = (np.zeros(n1, np.int64) for _ in range(3))
    off = np.zeros(n1 + 1, np.int64)
    vert = np.zeros(n1, np.int64)
    sv = np.zeros(n1, np.int64)
    sx = np.zeros(n1, np.float64)
    ns = _i64(0)
    k = lib().orc_expand(c.n, c.offsets, _nb(c), int(threshold), nv, ne, cut, off, vert,
                         ctypes.byref(ns), sv, sx)
    cl = Clusters(np.full(k, -1, np.int64), nv[:k].copy(), ne[:k].copy(), cut[:k].copy(),
                  off[:k + 1].copy(), vert[:off[k]].copy())
    return cl, sv[:ns.value].copy(), sx[:ns.value].copy()


def selfcheck_counts():
    a, b, c = _i64(0), _i64(0), _i64(0)
    lib().orc_selfcheck_counts(ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
    return int(a.value), int(b.value), int(c.value)


def run(n: int, u: np.ndarray, v: np.ndarray, eps: float):
    """Whole path: CSR, count, clean, extract.  Returns (csr, count, clean, clusters, final)."""
    c = build_csr(n, u, v)
    s0 = count(c)
    s1 = initial_clean(c, s0, eps)
    cl, s2 = extract(c, s1, eps)
    return c, s0, s1, cl, s2


def cells_edge(offsets: np.ndarray, nbors: np.ndarray, slots) -> tuple[np.ndarray, np.ndarray]:
    """perEdge and support of the sampled directed slots, recomputed from the CSR
    alone (commonNbr's left fold over the common neighbours in ascending order)."""
    offsets = np.ascontiguousarray(offsets, np.int64)
    nbors = np.ascontiguousarray(nbors, np.int64) if len(nbors) else np.zeros(1, np.int64)
    slots = np.ascontiguousarray(slots, np.int64)
    pe = np.zeros(max(1, slots.size), np.float64)
    sup = np.zeros(max(1, slots.size), np.uint32)
    if slots.size:
        lib().orc_cells_edge(offsets.size - 1, offsets, nbors, slots.size, slots, pe, sup)
    return pe[:slots.size], sup[:slots.size]


def cells_vertex(offsets: np.ndarray, nbors: np.ndarray, verts) -> np.ndarray:
    """perVertex of the sampled vertices, recomputed from the CSR alone."""
    offsets = np.ascontiguousarray(offsets, np.int64)
    nbors = np.ascontiguousarray(nbors, np.int64) if len(nbors) else np.zeros(1, np.int64)
    verts = np.ascontiguousarray(verts, np.int64)
    pv = np.zeros(max(1, verts.size), np.float64)
    if verts.size:
        lib().orc_cells_vertex(offsets.size - 1, offsets, nbors, verts.size, verts, pv)
    return pv[:verts.size]


def count_total(offsets: np.ndarray, nbors: np.ndarray) -> int:
    """Number of triangles of the CSR (degree-oriented count, independent of the folds)."""
    offsets = np.ascontiguousarray(offsets, np.int64)
    nbors = np.ascontiguousarray(nbors, np.int64) if len(nbors) else np.zeros(1, np.int64)
    return int(lib().orc_count_total(offsets.size - 1, offsets, nbors))


@dataclass
class Nuclei:
    """Truss-hierarchy clusters in the order nucleus.cpp writes them."""
    id: np.ndarray
    c: np.ndarray
    nv: np.ndarray
    ne: np.ndarray
    parent: np.ndarray
    off: np.ndarray
    vert: np.ndarray       # original labels
    kappa: np.ndarray      # per slot of the relabelled CSR (-1 on backward slots)
    rel_off: np.ndarray
    rel_nb: np.ndarray
    inverse: np.ndarray    # relabelled -> original
    reference_overflow: int  # nonzero: the reference overruns a fixed array on this input (undefined output)

    def text(self) -> str:
        """The cluster file nucleus.cpp writes (nucleus.cpp:62-76)."""
        out = []
        for k in range(self.id.size):
            out.append(f"Cluster id: {self.id[k]}, C: {self.c[k]}, n_vertices: {self.nv[k]}, "
                       f"n_edges: {self.ne[k]}, parent: {self.parent[k]}\n")
            out.append("".join(f"{x} " for x in self.vert[self.off[k]:self.off[k + 1]].tolist()) + "\n")
        return "".join(out)


def nucleus(c: "Csr") -> Nuclei:
    """The nucleus path on the CSR (makeCSR + sortById) of a graph."""
    L = lib()
    k = int(L.orc_nucleus(c.n, c.offsets, _nb(c)))
    nm, m2, ovf = _i64(), _i64(), _i64()
    L.orc_nucleus_sizes(ctypes.byref(nm), ctypes.byref(m2), ctypes.byref(ovf))
    a = {x: np.zeros(max(1, k), np.int64) for x in ("id", "c", "nv", "ne", "parent")}
    off = np.zeros(k + 1, np.int64)
    vert = np.zeros(max(1, nm.value), np.int64)
    kappa = np.zeros(max(1, m2.value), np.int64)
    rel_off = np.zeros(c.n + 1, np.int64)
    rel_nb = np.zeros(max(1, m2.value), np.int64)
    inverse = np.zeros(max(1, c.n), np.int64)
    ptr = lambda x: x.ctypes.data
    L.orc_nucleus_get(ptr(a["id"]), ptr(a["c"]), ptr(a["nv"]), ptr(a["ne"]), ptr(a["parent"]), ptr(off),
                      ptr(vert), ptr(kappa), ptr(rel_off), ptr(rel_nb), ptr(inverse))
    return Nuclei(a["id"][:k], a["c"][:k], a["nv"][:k], a["ne"][:k], a["parent"][:k], off, vert[:nm.value],
                  kappa[:m2.value], rel_off, rel_nb[:m2.value], inverse[:c.n], int(ovf.value))
