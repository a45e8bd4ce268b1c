"""B200-native RTRExtractor decomposition path.

Python front end over the C ABI of ``librtr.so`` (declared in
``include/rtr.h``).  The CUDA library is the only compute path: importing
works without a GPU, but every graph operation goes through librtr.so and
fails with :class:`RtrError` when no CUDA device is present; there is no CPU
fallback.

Typical use::

    import rtrex_cuda_b200 as rtr
    g = rtr.Graph.from_edges(n, src, dst)          # device CSR build
    total = g.count()                               # commonNbr
    left = g.clean(0.3)                             # initialClean
    k = g.extract()                                 # disjointExtract loop
    clusters = g.clusters()
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

__all__ = ["RtrError", "Graph", "Clusters", "lib", "lib_path", "run_file", "load_escape", "build"]

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "librtr.so")
_lib = None

RTR_FLAG_SIMPLIFY = 1
RTR_FLAG_RTREX_OUTPUTS = 2
RTR_FLAG_EXPAND = 4

_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
_vp = ctypes.c_void_p
_i64 = ctypes.c_int64


class RtrError(RuntimeError):
    """A librtr call returned a non-zero rtr_status."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"rtr error {code}: {msg}")
        self.code = code


def lib_path() -> str:
    return _LIB_PATH


def build(verbose: bool = False) -> str:
    from . import buildlib as _b
    return _b.build(verbose)


def lib():
    """Load librtr.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        raise RtrError(-1, f"{_LIB_PATH} is missing; run python -m rtrex_cuda_b200.buildlib")
    L = ctypes.CDLL(_LIB_PATH)
    P = ctypes.POINTER
    L.rtr_version.restype = ctypes.c_char_p
    L.rtr_last_error.restype = ctypes.c_char_p
    L.rtr_graph_create_from_edges.argtypes = [_vp, _vp, _i64, _i64, ctypes.c_int, ctypes.c_int, P(_vp)]
    L.rtr_graph_create_from_csr.argtypes = [_vp, _vp, _i64, ctypes.c_int, P(_vp)]
    L.rtr_graph_destroy.argtypes = [_vp]
    L.rtr_graph_info.argtypes = [_vp, P(_i64), P(_i64)]
    L.rtr_count.argtypes = [_vp, P(_i64)]
    L.rtr_clean.argtypes = [_vp, ctypes.c_double, P(_i64)]
    L.rtr_extract.argtypes = [_vp, P(_i64)]
    L.rtr_decompose.argtypes = [_vp, ctypes.c_double, P(_i64)]
    L.rtr_get_csr.argtypes = [_vp, _vp, _vp]
    L.rtr_get_weights.argtypes = [_vp, _vp, _vp, _vp, P(_i64)]
    L.rtr_get_status.argtypes = [_vp, _vp]
    L.rtr_get_clusters.argtypes = [_vp, _vp, _vp, _vp, _vp, _vp, _vp]
    L.rtr_get_cluster_of.argtypes = [_vp, _vp]
    L.rtr_num_clusters.argtypes = [_vp, P(_i64)]
    L.rtr_batch_create.argtypes = [_vp, _vp, _vp, _vp, _i64, ctypes.c_int, ctypes.c_int, P(_vp)]
    L.rtr_batch_cluster_counts.argtypes = [_vp, _vp]
    L.rtr_connected_components.argtypes = [_vp, P(_i64)]
    L.rtr_get_components.argtypes = [_vp, _vp, _vp]
    L.rtr_write_components.argtypes = [_vp, ctypes.c_char_p]
    L.rtr_get_stats.argtypes = [_vp, _vp, P(_i64), P(_i64)]
    L.rtr_get_kernel_ms.argtypes = [_vp, _vp, ctypes.c_int]
    L.rtr_write_decomposition.argtypes = [_vp, ctypes.c_char_p]
    L.rtr_load_escape.argtypes = [ctypes.c_char_p, P(_i64), P(_i64), P(_vp), P(_vp)]
    L.rtr_free.argtypes = [_vp]
    L.rtr_free.restype = None
    L.rtr_run_file.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_double, ctypes.c_int, ctypes.c_char_p,
                               ctypes.c_int]
    L.rtr_run_file_ex.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_double, ctypes.c_int, ctypes.c_char_p,
                                  ctypes.c_int, _i64]
    L.rtr_graph_create_from_escape_text.argtypes = [ctypes.c_char_p, _i64, ctypes.c_int, ctypes.c_int, P(_vp)]
    L.rtr_graph_create_from_escape_file.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, P(_vp)]
    L.rtr_get_memory.argtypes = [_vp, P(_i64), P(_i64)]
    L.rtr_set_tuning.argtypes = [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    L.rtr_get_tuning.argtypes = [_vp, P(ctypes.c_int), P(ctypes.c_int), P(ctypes.c_int)]
    L.rtr_autotune.argtypes = [_vp, P(ctypes.c_int), P(ctypes.c_int), P(ctypes.c_int)]
    L.rtr_set_count_mode.argtypes = [_vp, ctypes.c_int, ctypes.c_int]
    L.rtr_get_count_mode.argtypes = [_vp, P(ctypes.c_int), P(ctypes.c_int), P(ctypes.c_int)]
    L.rtr_get_count_windows.argtypes = [_vp, P(ctypes.c_int64), P(ctypes.c_int64)]
    L.rtr_set_count_window.argtypes = [_vp, ctypes.c_int64]
    L.rtr_graph_create_rmat.argtypes = [ctypes.c_int, _i64, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_uint64, ctypes.c_int, P(_vp)]
    L.rtr_set_clean_split.argtypes = [_vp, _i64, ctypes.c_double]
    L.rtr_set_clean_checks.argtypes = [_vp, _i64, _i64]
    L.rtr_set_extract_split.argtypes = [_vp, _i64]
    L.rtr_nucleus.argtypes = [_vp, P(_i64)]
    L.rtr_get_nuclei.argtypes = [_vp, P(_i64), P(_i64)] + [_vp] * 6
    L.rtr_write_nuclei.argtypes = [_vp, ctypes.c_char_p]
    L.rtr_get_clean_split.argtypes = [_vp, P(_i64), P(ctypes.c_double)]
    L.rtr_server_create.argtypes = [ctypes.c_int, _i64, ctypes.c_int, _i64, ctypes.c_int, P(_vp)]
    L.rtr_server_add_graph.argtypes = [_vp, _vp, _vp, _i64, _i64, ctypes.c_int, P(_i64)]
    L.rtr_server_submit.argtypes = [_vp, _i64, ctypes.c_double, _vp, P(_i64)]
    L.rtr_server_wait.argtypes = [_vp, _i64, _vp]
    L.rtr_server_stats.argtypes = [_vp, _vp, ctypes.c_int]
    L.rtr_server_destroy.argtypes = [_vp]
    L.rtr_expand.argtypes = [_vp, _i64, P(_i64)]
    L.rtr_get_expanded.argtypes = [_vp, _vp, _vp, _vp, _vp, _vp, _vp]
    L.rtr_get_scores.argtypes = [_vp, P(_i64), _vp, _vp]
    L.rtr_write_expanded.argtypes = [_vp, ctypes.c_char_p]
    _lib = L
    return L


def _check(rc: int):
    if rc != 0:
        msg = lib().rtr_last_error()
        raise RtrError(rc, msg.decode() if msg else "")


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data


@dataclass
class Clusters:
    """Clusters in creation order (the reference's vector<Cluster>)."""
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


class Graph:
    """One graph resident in HBM; stages run on the graph's own CUDA stream."""

    def __init__(self, handle: int):
        self._h = ctypes.c_void_p(handle)

    # -- construction -------------------------------------------------
    @classmethod
    def from_edges(cls, n: int, src, dst, device: int = 0, simplify: bool = False) -> "Graph":
        src = np.ascontiguousarray(src, dtype=np.int64)
        dst = np.ascontiguousarray(dst, dtype=np.int64)
        if src.shape != dst.shape:
            raise ValueError("src and dst differ in length")
        h = ctypes.c_void_p()
        _check(lib().rtr_graph_create_from_edges(_ptr(src), _ptr(dst), src.size, int(n), int(device),
                                                 RTR_FLAG_SIMPLIFY if simplify else 0, ctypes.byref(h)))
        return cls(h.value)

    @classmethod
    def batch(cls, graphs, device: int = 0, simplify: bool = False) -> "Graph":
        """One device graph holding independent graphs [(n, src, dst), ...] (disjoint union)."""
        nverts = np.array([int(g[0]) for g in graphs], dtype=np.int64)
        eoff = np.zeros(len(graphs) + 1, dtype=np.int64)
        eoff[1:] = np.cumsum([len(g[1]) for g in graphs])
        src = np.ascontiguousarray(np.concatenate([np.asarray(g[1], np.int64) for g in graphs]))
        dst = np.ascontiguousarray(np.concatenate([np.asarray(g[2], np.int64) for g in graphs]))
        h = ctypes.c_void_p()
        _check(lib().rtr_batch_create(_ptr(src), _ptr(dst), _ptr(eoff), _ptr(nverts), len(graphs), int(device),
                                      RTR_FLAG_SIMPLIFY if simplify else 0, ctypes.byref(h)))
        out = cls(h.value)
        out.vertex_bases = np.concatenate([[0], np.cumsum(nverts)])
        return out

    def batch_cluster_counts(self) -> np.ndarray:
        k = len(self.vertex_bases) - 1
        out = np.zeros(k, np.int64)
        _check(lib().rtr_batch_cluster_counts(self._h, _ptr(out)))
        return out

    @classmethod
    def from_escape_text(cls, text: bytes, device: int = 0, simplify: bool = False) -> "Graph":
        """Parse Escape edge-list text on the device and build the CSR there."""
        h = _vp()
        _check(lib().rtr_graph_create_from_escape_text(text, len(text), int(device),
                                                        RTR_FLAG_SIMPLIFY if simplify else 0, ctypes.byref(h)))
        return cls(h.value)

    @classmethod
    def from_escape_file(cls, path: str, device: int = 0, simplify: bool = False) -> "Graph":
        h = _vp()
        _check(lib().rtr_graph_create_from_escape_file(path.encode(), int(device),
                                                        RTR_FLAG_SIMPLIFY if simplify else 0, ctypes.byref(h)))
        return cls(h.value)

    @classmethod
    def from_rmat(cls, scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19,
                  seed: int = 3, device: int = 0) -> "Graph":
        """R-MAT graph generated on the device (graphgen.rmat_hashed is the same graph in numpy)."""
        h = _vp()
        _check(lib().rtr_graph_create_rmat(int(scale), int(edge_factor), float(a), float(b), float(c),
                                           int(seed) & ((1 << 64) - 1), int(device), ctypes.byref(h)))
        return cls(h.value)

    @classmethod
    def from_csr(cls, offsets, nbors, device: int = 0) -> "Graph":
        offsets = np.ascontiguousarray(offsets, dtype=np.int64)
        nbors = np.ascontiguousarray(nbors, dtype=np.int64)
        h = ctypes.c_void_p()
        _check(lib().rtr_graph_create_from_csr(_ptr(offsets), _ptr(nbors), offsets.size - 1, int(device),
                                               ctypes.byref(h)))
        return cls(h.value)

    def close(self):
        if self._h and self._h.value:
            lib().rtr_graph_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- info ------------------------------------------------------------
    @property
    def n(self) -> int:
        a, b = _i64(), _i64()
        _check(lib().rtr_graph_info(self._h, ctypes.byref(a), ctypes.byref(b)))
        return int(a.value)

    @property
    def m(self) -> int:
        a, b = _i64(), _i64()
        _check(lib().rtr_graph_info(self._h, ctypes.byref(a), ctypes.byref(b)))
        return int(b.value)

    # -- stages ----------------------------------------------------------
    def count(self) -> int:
        t = _i64()
        _check(lib().rtr_count(self._h, ctypes.byref(t)))
        return int(t.value)

    def clean(self, eps: float) -> int:
        t = _i64()
        _check(lib().rtr_clean(self._h, float(eps), ctypes.byref(t)))
        return int(t.value)

    def extract(self) -> int:
        t = _i64()
        _check(lib().rtr_extract(self._h, ctypes.byref(t)))
        return int(t.value)

    def decompose(self, eps: float) -> int:
        t = _i64()
        _check(lib().rtr_decompose(self._h, float(eps), ctypes.byref(t)))
        return int(t.value)

    # -- results -----------------------------------------------------------
    def csr(self):
        n, m = self.n, self.m
        off = np.zeros(n + 1, np.int64)
        nb = np.zeros(max(1, 2 * m), np.int64)
        _check(lib().rtr_get_csr(self._h, _ptr(off), _ptr(nb)))
        return off, nb[:2 * m]

    def weights(self, per_edge: bool = True, support: bool = True):
        """(perEdge[2m], perVertex[n], support[2m], total); per_edge / support
        False skips reading those arrays back (None in their place)."""
        n, m = self.n, self.m
        pe = np.zeros(max(1, 2 * m), np.float64) if per_edge else None
        pv = np.zeros(max(1, n), np.float64)
        sup = np.zeros(max(1, 2 * m), np.uint32) if support else None
        t = _i64()
        _check(lib().rtr_get_weights(self._h, _ptr(pe), _ptr(pv), _ptr(sup), ctypes.byref(t)))
        return (pe[:2 * m] if per_edge else None), pv[:n], (sup[:2 * m] if support else None), int(t.value)

    def status(self) -> np.ndarray:
        m = self.m
        st = np.zeros(max(1, 2 * m), np.uint8)
        _check(lib().rtr_get_status(self._h, _ptr(st)))
        return st[:2 * m]

    def num_clusters(self) -> int:
        t = _i64()
        _check(lib().rtr_num_clusters(self._h, ctypes.byref(t)))
        return int(t.value)

    def clusters(self) -> Clusters:
        n = self.n
        k = self.num_clusters()
        seed, nv, ne, cut = (np.zeros(max(1, k), np.int64) for _ in range(4))
        off = np.zeros(k + 1, np.int64)
        vert = np.zeros(max(1, n), np.int64)
        _check(lib().rtr_get_clusters(self._h, _ptr(seed), _ptr(nv), _ptr(ne), _ptr(cut), _ptr(off), _ptr(vert)))
        return Clusters(seed[:k], nv[:k], ne[:k], cut[:k], off, vert[:n])

    def cluster_of(self) -> np.ndarray:
        out = np.zeros(max(1, self.n), np.int64)
        _check(lib().rtr_get_cluster_of(self._h, _ptr(out)))
        return out[:self.n]

    def stats(self) -> dict:
        ms = np.zeros(4, np.float64)
        launches, resid = _i64(), _i64()
        _check(lib().rtr_get_stats(self._h, _ptr(ms), ctypes.byref(launches), ctypes.byref(resid)))
        return {"ms_build": ms[0], "ms_count": ms[1], "ms_clean": ms[2], "ms_extract": ms[3],
                "launches": int(launches.value), "residual_warnings": int(resid.value)}

    KERNELS = ("k_edge_fold", "k_tri_fill", "k_vertex_fold", "k_clean_units", "k_extract_components", "decompose",
               "k_edge_fold_light", "k_edge_count_heavy", "k_vfold_warp", "k_fill_light", "k_fill_heavy",
               "k_vfold_block")

    def kernel_ms(self) -> dict:
        """Device times (ms) of the last run's main kernels and of the whole decompose."""
        ms = np.zeros(len(self.KERNELS), np.float64)
        _check(lib().rtr_get_kernel_ms(self._h, _ptr(ms), len(self.KERNELS)))
        return {k: float(ms[i]) for i, k in enumerate(self.KERNELS)}

    def write_decomposition(self, name: str):
        _check(lib().rtr_write_decomposition(self._h, name.encode()))

    def set_tuning(self, gallop_ratio: int, heavy_degree: int, heavy_edge: int = 1024):
        """Counting work split (results are identical for every setting)."""
        _check(lib().rtr_set_tuning(self._h, int(gallop_ratio), int(heavy_degree), int(heavy_edge)))

    def set_count_mode(self, mode: int, hub_degree: int = 1024):
        """Counting layout: 0 keep triangle lists when they fit (default), 1 always,
        2 never (rows layout: 4-byte per-slot lists of z instead of the 32-byte
        triangle entries; same bits, but the clean needs the lists).  In the rows
        layout a vertex of at least hub_degree perVertex terms is folded by a warp,
        the others by a thread."""
        _check(lib().rtr_set_count_mode(self._h, int(mode), int(hub_degree)))

    def count_mode(self):
        """(mode, hub_degree, lists kept by the last count)."""
        a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(lib().rtr_get_count_mode(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return int(a.value), int(b.value), bool(c.value)

    def set_count_window(self, max_entries: int):
        """Rows layout: at most max_entries list entries per window (0: as many as fit)."""
        _check(lib().rtr_set_count_window(self._h, int(max_entries)))

    def count_windows(self):
        """(windows, list entries) of the last count's rows layout; (0, 0) with lists kept."""
        w, e = ctypes.c_int64(), ctypes.c_int64()
        _check(lib().rtr_get_count_windows(self._h, ctypes.byref(w), ctypes.byref(e)))
        return int(w.value), int(e.value)

    def set_clean_split(self, min_seeds: int, max_mean_list: float = 8.0):
        """Clean units with at least `min_seeds` seeds and triangle lists of at
        most `max_mean_list` entries on average replay in parallel rounds (one
        thread block each), the others one warp per unit (same bits)."""
        _check(lib().rtr_set_clean_split(self._h, int(min_seeds), float(max_mean_list)))

    def nucleus(self) -> int:
        """The nucleus (truss-hierarchy) path; returns the number of clusters."""
        k = _i64()
        _check(lib().rtr_nucleus(self._h, ctypes.byref(k)))
        return int(k.value)

    def nuclei(self):
        """(c, nv, ne, parent, off, vert) of the last nucleus run, in output order."""
        k, nm = _i64(), _i64()
        _check(lib().rtr_get_nuclei(self._h, ctypes.byref(k), ctypes.byref(nm), None, None, None, None, None,
                                    None))
        c, nv, ne, par = (np.zeros(max(1, k.value), np.int64) for _ in range(4))
        off = np.zeros(k.value + 1, np.int64)
        vert = np.zeros(max(1, nm.value), np.int64)
        _check(lib().rtr_get_nuclei(self._h, ctypes.byref(k), ctypes.byref(nm), _ptr(c), _ptr(nv), _ptr(ne),
                                    _ptr(par), _ptr(off), _ptr(vert)))
        kk = k.value
        return c[:kk], nv[:kk], ne[:kk], par[:kk], off, vert[:nm.value]

    def write_nuclei(self, path: str):
        _check(lib().rtr_write_nuclei(self._h, path.encode()))

    def set_extract_split(self, min_vertices: int = 512):
        """Components of at least min_vertices vertices are extracted by a thread
        block each, the others by a warp each (same bits)."""
        _check(lib().rtr_set_extract_split(self._h, int(min_vertices)))

    def set_clean_checks(self, first_wait_rounds: int = 0, stack_entries: int = -1):
        """Lower the clean's device-side check bounds (to test their error reports)."""
        _check(lib().rtr_set_clean_checks(self._h, int(first_wait_rounds), int(stack_entries)))

    def clean_split(self):
        v, x = _i64(), ctypes.c_double()
        _check(lib().rtr_get_clean_split(self._h, ctypes.byref(v), ctypes.byref(x)))
        return int(v.value), float(x.value)

    def tuning(self):
        a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(lib().rtr_get_tuning(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return int(a.value), int(b.value), int(c.value)

    def autotune(self):
        """Time the counting pass for candidate work splits; keep and return the fastest."""
        a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(lib().rtr_autotune(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return int(a.value), int(b.value), int(c.value)

    def expand(self, threshold: int) -> int:
        """expandClusters (the RTRex driver's mode e); returns the number of moved vertices."""
        t = _i64()
        _check(lib().rtr_expand(self._h, int(threshold), ctypes.byref(t)))
        return int(t.value)

    def expanded(self):
        """(clusters, cluster_of) after :meth:`expand`; ``seed`` holds -1 and
        ``cluster_of`` is -1 for a vertex in no cluster."""
        n, k = self.n, self.num_clusters()
        nv, ne, cut = (np.zeros(max(1, k), np.int64) for _ in range(3))
        off = np.zeros(k + 1, np.int64)
        vert = np.zeros(max(1, n), np.int64)
        cof = np.zeros(max(1, n), np.int64)
        _check(lib().rtr_get_expanded(self._h, _ptr(nv), _ptr(ne), _ptr(cut), _ptr(off), _ptr(vert), _ptr(cof)))
        cl = Clusters(np.full(k, -1, np.int64), nv[:k], ne[:k], cut[:k], off, vert[:off[k]])
        return cl, cof[:n]

    def scores(self):
        """(vertices, scores) of the moved vertices, ascending vertex order."""
        t = _i64()
        _check(lib().rtr_get_scores(self._h, ctypes.byref(t), None, None))
        k = int(t.value)
        v = np.zeros(max(1, k), np.int64)
        x = np.zeros(max(1, k), np.float64)
        _check(lib().rtr_get_scores(self._h, ctypes.byref(t), _ptr(v), _ptr(x)))
        return v[:k], x[:k]

    def write_expanded(self, name: str):
        _check(lib().rtr_write_expanded(self._h, name.encode()))


class RequestInfo(ctypes.Structure):
    """rtr_request_info."""
    _fields_ = [("status", ctypes.c_int), ("batched", ctypes.c_int), ("n_clusters", ctypes.c_int64),
                ("triangles", ctypes.c_int64), ("triangles_left", ctypes.c_int64), ("t_submit_ms", ctypes.c_double),
                ("t_start_ms", ctypes.c_double), ("t_end_ms", ctypes.c_double), ("error", ctypes.c_char * 160)]


class Server:
    """The request server (rtr_server_*): registered graphs resident in HBM under
    a budget, requests admitted continuously, small graphs batched."""

    STATS = ("resident_graphs", "bytes_in_use", "peak_bytes", "peak_inflight", "evictions", "batches",
             "batched_requests", "queued")

    def __init__(self, device: int = 0, hbm_budget: int = 120 << 30, workers: int = 8,
                 batch_max_edges: int = 20000, batch_max_graphs: int = 64):
        h = _vp()
        _check(lib().rtr_server_create(int(device), int(hbm_budget), int(workers), int(batch_max_edges),
                                       int(batch_max_graphs), ctypes.byref(h)))
        self._h = h.value
        self._n = []
        self._bufs = {}

    def add_graph(self, n: int, src, dst, simplify: bool = False) -> int:
        src = np.ascontiguousarray(src, dtype=np.int64)
        dst = np.ascontiguousarray(dst, dtype=np.int64)
        gid = _i64()
        _check(lib().rtr_server_add_graph(self._h, _ptr(src), _ptr(dst), src.size, int(n),
                                          RTR_FLAG_SIMPLIFY if simplify else 0, ctypes.byref(gid)))
        self._n.append(int(n))
        return int(gid.value)

    def submit(self, graph_id: int, eps: float, cluster_of: bool = True) -> int:
        n = self._n[graph_id] if 0 <= graph_id < len(self._n) else 0  # unknown ids: the library reports them
        buf = np.zeros(max(1, n), np.int64) if cluster_of else None
        rid = _i64()
        _check(lib().rtr_server_submit(self._h, int(graph_id), float(eps), _ptr(buf), ctypes.byref(rid)))
        self._bufs[int(rid.value)] = (buf, n)
        return int(rid.value)

    def wait(self, request_id: int) -> dict:
        info = RequestInfo()
        _check(lib().rtr_server_wait(self._h, int(request_id), ctypes.byref(info)))
        buf, n = self._bufs.pop(int(request_id))
        out = {f: getattr(info, f) for f, _ in RequestInfo._fields_ if f != "error"}
        out["error"] = info.error.decode(errors="replace")
        out["cluster_of"] = None if buf is None else buf[:n]
        return out

    def stats(self) -> dict:
        v = np.zeros(8, np.int64)
        _check(lib().rtr_server_stats(self._h, _ptr(v), 8))
        return {k: int(x) for k, x in zip(self.STATS, v)}

    def close(self):
        if getattr(self, "_h", None):
            lib().rtr_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def load_escape(path: str):
    """Parse an Escape edge list with the library's loader: (n, src, dst)."""
    n, m = _i64(), _i64()
    ps, pd = ctypes.c_void_p(), ctypes.c_void_p()
    _check(lib().rtr_load_escape(path.encode(), ctypes.byref(n), ctypes.byref(m), ctypes.byref(ps), ctypes.byref(pd)))
    try:
        k = int(m.value)
        src = np.ctypeslib.as_array(ctypes.cast(ps, ctypes.POINTER(ctypes.c_int64)), shape=(max(1, k),))[:k].copy()
        dst = np.ctypeslib.as_array(ctypes.cast(pd, ctypes.POINTER(ctypes.c_int64)), shape=(max(1, k),))[:k].copy()
    finally:
        lib().rtr_free(ps)
        lib().rtr_free(pd)
    return int(n.value), src, dst


def run_file(path: str, name: str, eps: float, device: int = 0, prefix: str = "RTRex-CUDA-", simplify=False,
             rtrex_outputs: bool = False, expand: int | None = None):
    """The drop-in driver.  rtrex_outputs adds the RTRex CLI's components files
    and survivor dump; expand=T adds its mode e outputs at threshold T."""
    flags = (RTR_FLAG_SIMPLIFY if simplify else 0) | (RTR_FLAG_RTREX_OUTPUTS if rtrex_outputs else 0)
    if expand is not None:
        flags |= RTR_FLAG_EXPAND
    _check(lib().rtr_run_file_ex(path.encode(), name.encode(), float(eps), int(device), prefix.encode(), flags,
                                 int(expand or 0)))
