"""Seeded synthetic graph generators for the decomposition workloads.

Every generator returns an undirected simple graph as ``(n, u, v)`` with
``u < v`` row-sorted int64 arrays (no self-loops, no duplicates), the form the
Escape loader expects after symmetrisation (RTRex_Sequential/GraphIO.cpp:19-74
reads ``n m`` then ``m`` lines ``u v`` and stores both directions).  The
reference reads no per-edge weights, so none are produced.

Workloads (all seeded, numpy PCG64):

* ``gnp_cliques``   G(n,p) background plus planted cliques
  (10,000 vertices, p=0.0016, 20 cliques of 20 random vertices, seed 1).
* ``chung_lu``      Chung-Lu power law (335,000 vertices, ~926k edges,
  exponent 2.3, expected degree capped at 550) plus 2,000 planted
  communities of 5-12 vertices at p=0.8 (seed 2); the shape of the
  com-amazon co-purchase network.
* ``rmat``          R-MAT (a,b,c,d)=(.57,.19,.19,.05), symmetrised,
  self-loops and duplicates removed.
* ``sbm``           stochastic block model with 4-64 blocks, intra-block
  mean degree 12, inter-block mean degree 2.
"""
from __future__ import annotations

import os
import numpy as np

__all__ = [
    "simplify", "gnp_cliques", "chung_lu", "rmat", "rmat_hashed", "rmat_hashed_pairs", "sbm", "small_test",
    "write_escape", "read_escape", "parse_escape", "config_graph",
]


def simplify(n: int, u: np.ndarray, v: np.ndarray):
    """Drop self-loops and duplicate pairs; return row-sorted ``u < v`` arrays."""
    u = np.asarray(u, dtype=np.int64)
    v = np.asarray(v, dtype=np.int64)
    keep = u != v
    u, v = u[keep], v[keep]
    a = np.minimum(u, v)
    b = np.maximum(u, v)
    key = np.unique(a * np.int64(n) + b)
    return key // n, key % n


def gnp_cliques(n=10_000, p=0.0016, n_cliques=20, clique_size=20, seed=1):
    rng = np.random.Generator(np.random.PCG64(seed))
    # G(n,p) by geometric skipping over the n(n-1)/2 upper-triangle slots.
    total = n * (n - 1) // 2
    m_exp = int(total * p)
    draws = []
    pos = -1
    while True:
        gaps = rng.geometric(p, size=max(1024, int(m_exp * 1.2) + 1024)).astype(np.int64)
        idx = pos + np.cumsum(gaps)
        draws.append(idx[idx < total])
        if idx[-1] >= total:
            break
        pos = idx[-1]
    slots = np.concatenate(draws)
    # slot -> (a, b), a < b, row-major over the upper triangle.
    # row a starts at s(a) = a*(2n-a-1)/2
    a = np.floor(((2 * n - 1) - np.sqrt((2.0 * n - 1) ** 2 - 8.0 * slots)) / 2).astype(np.int64)
    start = a * (2 * n - a - 1) // 2
    fix = slots < start
    a[fix] -= 1
    start = a * (2 * n - a - 1) // 2
    nxt = (a + 1) * (2 * n - a - 2) // 2
    fix = slots >= nxt
    a[fix] += 1
    start = a * (2 * n - a - 1) // 2
    b = a + 1 + (slots - start)
    us, vs = [a], [b]
    for _ in range(n_cliques):
        mem = rng.choice(n, size=clique_size, replace=False)
        i, j = np.triu_indices(clique_size, 1)
        us.append(mem[i])
        vs.append(mem[j])
    u, v = simplify(n, np.concatenate(us), np.concatenate(vs))
    return n, u, v


def chung_lu(n=335_000, target_edges=926_000, gamma=2.3, max_deg=550.0,
             n_comm=2_000, comm_min=5, comm_max=12, comm_p=0.8, seed=2,
             scale=None):
    """Chung-Lu power law + planted communities.

    Expected degrees follow ``w_i ~ (i+i0)^(-1/(gamma-1))`` capped at
    ``max_deg``; ``m' = sum(w)/2`` endpoint pairs are drawn proportionally to
    ``w`` (the fast Chung-Lu sampler), then communities are planted and the
    union is simplified.  ``scale`` multiplies the background size; by default
    it is the value calibrated so the simplified graph lands near
    ``target_edges`` for the default parameters.
    """
    rng = np.random.Generator(np.random.PCG64(seed))
    i = np.arange(n, dtype=np.float64)
    w = (i + 10.0) ** (-1.0 / (gamma - 1.0))
    w = w / w.mean() * 5.0
    w = np.minimum(w, max_deg)
    if scale is None:
        scale = _CHUNG_LU_SCALE
    m_bg = int(round(target_edges * scale))
    cdf = np.cumsum(w)
    cdf /= cdf[-1]
    eu = np.searchsorted(cdf, rng.random(m_bg), side="right")
    ev = np.searchsorted(cdf, rng.random(m_bg), side="right")
    perm = rng.permutation(n)  # decorrelate id from expected degree
    us, vs = [perm[eu]], [perm[ev]]
    sizes = rng.integers(comm_min, comm_max + 1, size=n_comm)
    for s in sizes:
        mem = rng.choice(n, size=int(s), replace=False)
        ii, jj = np.triu_indices(int(s), 1)
        keep = rng.random(ii.size) < comm_p
        us.append(mem[ii[keep]])
        vs.append(mem[jj[keep]])
    u, v = simplify(n, np.concatenate(us), np.concatenate(vs))
    return n, u, v


# Background-size factor for chung_lu() calibrated so the default call yields
# ~926k undirected edges after simplification (duplicates at the capped hubs
# are removed, so more than target_edges pairs must be drawn).
_CHUNG_LU_SCALE = 0.942


def rmat(scale=24, edge_factor=16, a=0.57, b=0.19, c=0.19, seed=3, chunk=1 << 24):
    """R-MAT generator (Chakrabarti et al.), symmetrised and simplified."""
    rng = np.random.Generator(np.random.PCG64(seed))
    n = 1 << scale
    m = edge_factor * n
    ab = a + b
    c_norm = c / (1.0 - ab)
    a_norm = a / ab
    keys = []
    done = 0
    while done < m:
        k = min(chunk, m - done)
        src = np.zeros(k, dtype=np.int64)
        dst = np.zeros(k, dtype=np.int64)
        for lvl in range(scale):
            bit = np.int64(1) << np.int64(scale - 1 - lvl)
            ii = rng.random(k) > ab
            jj = rng.random(k) > np.where(ii, c_norm, a_norm)
            src += ii * bit
            dst += jj * bit
        keep = src != dst
        s, d = src[keep], dst[keep]
        lo = np.minimum(s, d)
        hi = np.maximum(s, d)
        keys.append(np.unique(lo * np.int64(n) + hi))
        done += k
    key = np.unique(np.concatenate(keys))
    return n, key // n, key % n


_MIX_GOLDEN = np.uint64(0x9E3779B97F4A7C15)


def _mix64(z: np.ndarray) -> np.ndarray:
    """splitmix64 output function (Steele, Lea, Flood 2014) on uint64 arrays."""
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def _threshold32(p: float) -> int:
    if not p > 0.0:
        return 0
    if p >= 1.0:
        return 1 << 32
    return int(np.floor(p * 4294967296.0))


def rmat_hashed_pairs(scale=24, edge_factor=16, a=0.57, b=0.19, c=0.19, seed=3, chunk=1 << 22):
    """The raw generated pairs of rtr_graph_create_rmat (before symmetrising):
    pair k's bit at level l comes from mix64(seed * golden ^ (k << 6 | l)); the
    high 32 bits decide the source half, the low 32 bits the destination half."""
    M = edge_factor << scale
    t_ab, t_a, t_c = (np.uint64(_threshold32(p)) for p in (a + b, a / (a + b), c / (1.0 - a - b)))
    smix = np.uint64((int(seed) * 0x9E3779B97F4A7C15) & ((1 << 64) - 1))
    src = np.empty(M, np.int64)
    dst = np.empty(M, np.int64)
    with np.errstate(over="ignore"):
        for k0 in range(0, M, chunk):
            k = np.arange(k0, min(M, k0 + chunk), dtype=np.uint64)
            s = np.zeros(k.size, np.uint64)
            t = np.zeros(k.size, np.uint64)
            for lvl in range(scale):
                h = _mix64(smix ^ ((k << np.uint64(6)) | np.uint64(lvl)))
                hi = h >> np.uint64(32)
                lo = h & np.uint64(0xFFFFFFFF)
                ii = hi >= t_ab
                jj = lo >= np.where(ii, t_c, t_a)
                bit = np.uint64(scale - 1 - lvl)
                s |= ii.astype(np.uint64) << bit
                t |= jj.astype(np.uint64) << bit
            src[k0:k0 + k.size] = s.astype(np.int64)
            dst[k0:k0 + k.size] = t.astype(np.int64)
    return 1 << scale, src, dst


def rmat_hashed(scale=24, edge_factor=16, a=0.57, b=0.19, c=0.19, seed=3):
    """R-MAT graph of rtr_graph_create_rmat (device generator), simplified."""
    n, src, dst = rmat_hashed_pairs(scale, edge_factor, a, b, c, seed)
    u, v = simplify(n, src, dst)
    return n, u, v


def sbm(m_target: int, seed: int, mean_intra=12.0, mean_inter=2.0,
        min_blocks=4, max_blocks=64):
    """SBM sized so the edge count lands near ``m_target``."""
    rng = np.random.Generator(np.random.PCG64(seed))
    n = max(8, int(round(2.0 * m_target / (mean_intra + mean_inter))))
    k = int(rng.integers(min_blocks, max_blocks + 1))
    k = max(1, min(k, n // 2))
    block = np.sort(rng.integers(0, k, size=n))
    sizes = np.bincount(block, minlength=k)
    starts = np.concatenate([[0], np.cumsum(sizes)[:-1]])
    us, vs = [], []
    for bi in range(k):
        s = int(sizes[bi])
        if s < 2:
            continue
        p = min(1.0, mean_intra / max(1, s - 1))
        cnt = rng.binomial(s * (s - 1) // 2, p)
        x = rng.integers(0, s, size=cnt) + starts[bi]
        y = rng.integers(0, s, size=cnt) + starts[bi]
        us.append(x)
        vs.append(y)
    n_inter = int(n * mean_inter / 2)
    us.append(rng.integers(0, n, size=n_inter))
    vs.append(rng.integers(0, n, size=n_inter))
    perm = rng.permutation(n)
    u, v = simplify(n, perm[np.concatenate(us)], perm[np.concatenate(vs)])
    return n, u, v


def served_pool(count: int, seed0: int = 5000, m_lo: float = 1e3, m_hi: float = 1e7):
    """Graphs for the served form: edge targets log-uniform in [m_lo, m_hi],
    alternating the G(n,p)+planted-cliques shape (mean degree ~16.7 as at
    n=10,000, p=0.0016; one 20-clique per 500 vertices) and R-MAT (a,b,c =
    .57,.19,.19; scale and edge factor chosen for the target), seeds seed0+i.
    Edge counts land near the targets (R-MAT loses duplicates)."""
    out = []
    for i in range(count):
        rng = np.random.Generator(np.random.PCG64(seed0 + i))
        m = float(np.exp(rng.uniform(np.log(m_lo), np.log(m_hi))))
        if i % 2 == 0:
            n = max(64, int(round(m / 8.35)))
            out.append(gnp_cliques(n=n, p=16.7 / (n - 1), n_cliques=max(1, n // 500),
                                   clique_size=min(20, n // 4), seed=seed0 + i))
        else:
            scale = max(6, int(round(np.log2(m / 10.0))))
            ef = max(1, int(round(1.25 * m / (1 << scale))))
            out.append(rmat(scale=scale, edge_factor=ef, seed=seed0 + i))
    return out


def small_test():
    """A 10-vertex, 19-edge graph with one dense 4-vertex core."""
    pairs = [(1, 7), (3, 6), (1, 2), (0, 1), (1, 3), (1, 6), (1, 4), (3, 4), (2, 0), (2, 9),
             (9, 3), (5, 9), (2, 5), (5, 6), (6, 8), (5, 7), (7, 8), (4, 6), (2, 3)]
    u = np.array([p[0] for p in pairs], dtype=np.int64)
    v = np.array([p[1] for p in pairs], dtype=np.int64)
    return 10, u, v


def config_graph(name: str):
    """The named benchmark graphs (``"gnp_cliques"``, ``"chung_lu"``, ``"rmat24"``...)."""
    if name == "gnp_cliques":
        return gnp_cliques()
    if name == "chung_lu":
        return chung_lu()
    if name.startswith("rmat"):
        return rmat(scale=int(name[4:]))
    if name == "small_test":
        return small_test()
    raise KeyError(name)


def write_escape(path: str, n: int, u: np.ndarray, v: np.ndarray) -> None:
    """Write the Escape text format: ``n m`` then one ``u v`` line per edge."""
    u = np.asarray(u, dtype=np.int64)
    v = np.asarray(v, dtype=np.int64)
    with open(path, "w") as f:
        f.write(f"{n} {u.size}\n")
        if u.size:
            body = np.char.add(np.char.add(u.astype(str), " "), v.astype(str))
            f.write("\n".join(body.tolist()))
            f.write("\n")


def read_escape(path: str):
    """Parse an Escape file (plain or gzip-compressed, ``.gz``) into ``(n, u, v)``
    (lines in file order, no simplification)."""
    if path.endswith(".gz"):
        import gzip
        with gzip.open(path, "rb") as f:
            data = f.read()
    else:
        with open(path, "rb") as f:
            data = f.read()
    return parse_escape(data)


def parse_escape(data: bytes):
    """Parse Escape edge-list bytes into ``(n, u, v)`` (lines in order, no simplification)."""
    lines = [ln for ln in data.split(b"\n") if ln.strip() and not ln.startswith(b"#")]
    head = lines[0].split()
    n, m = int(head[0]), int(head[1])
    body = np.array(b" ".join(ln.split()[0] + b" " + ln.split()[1] for ln in lines[1:m + 1]).split(),
                    dtype=np.int64)
    return n, body[0::2].copy(), body[1::2].copy()


if __name__ == "__main__":  # pragma: no cover - manual use
    import sys
    name, out = sys.argv[1], sys.argv[2]
    g = config_graph(name)
    write_escape(out, *g)
    print(name, g[0], g[1].size, os.path.getsize(out))


def sbm_batch(count: int, seed0: int = 4000, m_lo: float = 1e3, m_hi: float = 2e5):
    """The batched workload: graph i is an SBM (4-64 blocks, intra-block mean
    degree 12, inter-block mean degree 2) whose edge target is log-uniform in
    [m_lo, m_hi], seeded with seed0 + i."""
    out = []
    for i in range(count):
        rng = np.random.Generator(np.random.PCG64(seed0 + i))
        m_target = int(np.exp(rng.uniform(np.log(m_lo), np.log(m_hi))))
        out.append(sbm(m_target, seed0 + i))
    return out
