"""The round replay's commit policy, restated in Python and checked bit for bit
against the oracle on CPU.

This mirrors the decisions of k_clean_rounds (rtrex_cuda_b200/csrc/clean_rounds.cu)
without its data structures: a window of W pending pops claims the edge cells
each would touch (its own edge and the two other edges of every live
triangle); a pop that owns all its cells is a winner; winners commit in one
round unless an earlier item is a winner that pushes (its pushes are spliced in
right after it) or a loser that might push (some live-triangle edge could fall
below threshold after every claim of the window); an item whose list is longer
than the kernel's 32 entries is popped alone at the front of the window and
elsewhere ends the commits before it; seeds whose support is already 0 when
they are loaded into the pending list are retired without a pop.
perVertex is not touched during the rounds: each pop's subtractions are logged
and replayed afterwards in the reference's pop order, recovered from a linked
sequence list.  If the policy were unsound, some perEdge / perVertex bit or
status would differ from the oracle's sequential replay.
"""
import numpy as np
import pytest

import oracle
from rtrex_cuda_b200 import graphgen


def _graph(seed):
    rng = np.random.default_rng(9100 + seed)
    if seed % 3 == 2:
        n, u, v = graphgen.rmat(scale=int(rng.integers(7, 10)), edge_factor=int(rng.integers(4, 12)), seed=seed)
        return n, u, v
    n = int(rng.integers(40, 300))
    m = int(rng.integers(n, 6 * n))
    u, v = rng.integers(0, n, m), rng.integers(0, n, m)
    for _ in range(int(rng.integers(1, 8))):
        cq = rng.choice(n, size=int(rng.integers(4, 12)), replace=False)
        a, b = np.triu_indices(cq.size, 1)
        u, v = np.concatenate([u, cq[a]]), np.concatenate([v, cq[b]])
    su, sv = graphgen.simplify(n, u, v)
    return n, su, sv


def _round_replay(n, u, v, eps, W, refill, loser_cut=True, long_list=32):
    c = oracle.build_csr(n, u, v)
    s0 = oracle.count(c)
    off, nb = c.offsets, c.nbors
    src = np.repeat(np.arange(n), np.diff(off))
    deg = np.diff(off)
    fwd = src < nb

    def fslot(a, b):
        a, b = min(a, b), max(a, b)
        return int(off[a] + np.searchsorted(nb[off[a]:off[a + 1]], b))

    tri = {}

    def tris(e):
        if e not in tri:
            a, b = int(src[e]), int(nb[e])
            zs = np.intersect1d(nb[off[a]:off[a + 1]], nb[off[b]:off[b + 1]], assume_unique=True)
            tri[e] = [(int(z), fslot(a, z), fslot(b, z)) for z in zs.tolist()]
        return tri[e]

    thr = eps * (1 / (deg[src].astype(np.float64) * deg[nb]))
    P = s0.perEdge.copy()
    S = s0.support.astype(np.int64).copy()
    T = np.full(nb.size, ord('Y'), np.uint8)
    seedmask = fwd & (P < thr)
    T[seedmask & (S > 0)] = ord('S')
    T[seedmask & (S == 0)] = ord('N')
    seeds = [int(e) for e in np.nonzero(seedmask & (S > 0))[0]]

    def live(e, pr):
        """Live triangles of pop e (pair pr) as (lower-edge, higher-edge, z, weight)."""
        u_, v_ = pr
        du, dv = int(deg[u_]), int(deg[v_])
        lower = u_ if du < dv else v_
        out = []
        if S[e] > 0:
            for (z, az, bz) in tris(e):
                lw, hw = (az, bz) if lower == min(u_, v_) else (bz, az)
                if T[lw] != ord('N') and T[hw] != ord('N'):
                    out.append((lw, hw, z, 1 / float(du * dv * int(deg[z]))))
        return out

    # sequence list: seeds chained in pop order (highest slot first)
    order = seeds[::-1]
    nxt = {a: b for a, b in zip(order, order[1:])}
    head = order[0] if order else None
    log = []  # (vertex, pop, weights in triangle order)
    seedq = [(e, (int(src[e]), int(nb[e]))) for e in seeds]  # popped from the end
    pend = []  # top at the end
    while True:
        while len(pend) < W and seedq:  # refill, retiring seeds already at support 0
            k = min(refill, len(seedq))
            chunk = seedq[-k:]
            del seedq[-k:]
            kept = []
            for it in chunk:
                if S[it[0]] == 0:
                    T[it[0]] = ord('N')
                else:
                    kept.append(it)
            pend = kept + pend
        if not pend:
            break
        # an item with a list longer than long_list is popped alone at the front;
        # elsewhere it claims no cell and nothing after it commits
        width = 1 if len(tris(pend[-1][0])) > long_list else W
        win = [pend.pop() for _ in range(min(width, len(pend)))]
        lng = [i > 0 and len(tris(e)) > long_list for i, (e, _) in enumerate(win)]
        owner, acc, claims = {}, {}, []
        for i, (e, pr) in enumerate(win):
            cl = [] if lng[i] else [(e, 0.0)] + [(x, w) for (lw, hw, z, w) in live(e, pr) for x in (lw, hw)]
            claims.append(cl)
            for x, w in cl:
                owner.setdefault(x, i)
                acc[x] = acc.get(x, 0.0) + w
        cut, p1, pushes, results = len(win), None, [], {}
        for i, (e, pr) in enumerate(win):
            if lng[i]:
                cut = min(cut, i)
                continue
            if all(owner[x] == i for x, _ in claims[i]):  # winner: exact on round-start values
                u_, v_ = pr
                du, dv = int(deg[u_]), int(deg[v_])
                lower, higher = (u_, v_) if du < dv else (v_, u_)
                dl, dh = min(du, dv), max(du, dv)
                pu = []
                for (lw, hw, z, w) in live(e, pr):
                    if T[lw] != ord('S') and P[lw] - w < eps * (1 / float(dl * int(deg[z]))):
                        pu.append((lw, (lower, z)))
                    if T[hw] != ord('S') and P[hw] - w < eps * (1 / float(dh * int(deg[z]))):
                        pu.append((hw, (higher, z)))
                results[i] = pu
                if pu and p1 is None:
                    p1, pushes = i, pu
            else:  # loser: might it push when it pops?
                for x, w in claims[i][1:]:
                    if T[x] != ord('S') and (P[x] - acc[x]) - thr[x] < 1e-9 * (abs(P[x]) + acc[x]):
                        cut = min(cut, i) if loser_cut else cut
        cutoff = min(cut, p1 + 1 if p1 is not None else len(win))
        done = [False] * len(win)
        for i, (e, pr) in enumerate(win):
            if i not in results or i >= cutoff:
                continue
            u_, v_ = pr
            du, dv = int(deg[u_]), int(deg[v_])
            dl, dh = min(du, dv), max(du, dv)
            tl = live(e, pr)
            for (lw, hw, z, w) in tl:
                P[e] -= w
                P[lw] -= w
                P[hw] -= w
                S[e] -= 1
                S[lw] -= 1
                S[hw] -= 1
                if T[lw] != ord('S') and P[lw] < eps * (1 / float(dl * int(deg[z]))):
                    T[lw] = ord('S')
                if T[hw] != ord('S') and P[hw] < eps * (1 / float(dh * int(deg[z]))):
                    T[hw] = ord('S')
            if tl:
                ws = [w for (_, _, _, w) in tl]
                log += [(u_, e, ws), (v_, e, ws)] + [(z, e, [w]) for (_, _, z, w) in tl]
            T[e] = ord('N')
            done[i] = True
        if p1 is not None and p1 < cutoff:  # splice the pushes in after the pusher
            e1 = win[p1][0]
            old = nxt.get(e1)
            prev = e1
            for x, _ in reversed(pushes):
                nxt[prev] = x
                prev = x
            if old is not None:
                nxt[prev] = old
            else:
                nxt.pop(prev, None)
        rest = []
        for i in range(len(win)):
            if not done[i]:
                rest.append(win[i])
            if p1 is not None and i == p1 and p1 < cutoff:
                rest += list(reversed(pushes))
        pend += list(reversed(rest))
    rank, x, r = {}, head, 0
    while x is not None:
        rank[x] = r
        r += 1
        x = nxt.get(x)
    PV = s0.perVertex.copy()
    for (vx, e, ws) in sorted(log, key=lambda t: (t[0], rank[t[1]])):
        for w in ws:
            PV[vx] -= w
    return c, s0, P, S, T, PV


@pytest.mark.parametrize("seed", range(12))
@pytest.mark.parametrize("W,refill,long_list", [(16, 512, 32), (4, 3, 32), (16, 64, 2)])
def test_round_policy_matches_sequential_replay(seed, W, refill, long_list):
    """long_list=2 makes most items "long": popped alone at the front, ending the
    commits elsewhere (the kernel's path for lists over 32 entries)."""
    n, u, v = _graph(seed)
    eps = [0.3, 0.1, 0.5][seed % 3]
    c, s0, P, S, T, PV = _round_replay(n, u, v, eps, W, refill, long_list=long_list)
    s1 = oracle.initial_clean(c, s0, eps)
    fwd = np.repeat(np.arange(n), np.diff(c.offsets)) < c.nbors
    assert (T[fwd] == s1.status[fwd]).all()
    assert (P[fwd].view(np.int64) == s1.perEdge[fwd].view(np.int64)).all()
    assert (S[fwd] == s1.support[fwd].astype(np.int64)).all()
    assert (PV.view(np.int64) == s1.perVertex.view(np.int64)).all()


def _matches(n, u, v, eps, **kw):
    c, s0, P, S, T, PV = _round_replay(n, u, v, eps, 16, 512, **kw)
    s1 = oracle.initial_clean(c, s0, eps)
    fwd = np.repeat(np.arange(n), np.diff(c.offsets)) < c.nbors
    return bool((T[fwd] == s1.status[fwd]).all() and (P[fwd].view(np.int64) == s1.perEdge[fwd].view(np.int64)).all()
                and (PV.view(np.int64) == s1.perVertex.view(np.int64)).all())


def test_dropping_the_loser_cut_is_caught():
    """A planted mistake: let winners pass losers that might push.  A loser's
    later pop can then push an edge whose cascade touches a passed winner's
    cells out of order, and some graph here must show it."""
    bad = [seed for seed in range(24) if not _matches(*_graph(seed), [0.3, 0.1, 0.5][seed % 3], loser_cut=False)]
    assert bad, "the unsound policy matched the oracle on every graph: the test has no teeth"
