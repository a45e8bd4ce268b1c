"""The request server: every result served in a mix of concurrent, batched and
evicted-and-rebuilt requests equals the same graph's decomposition run alone
(bit-identical cluster assignment in creation order, same triangle counts)."""
import numpy as np
import pytest

import rtrex_cuda_b200 as rtr
from rtrex_cuda_b200 import graphgen
from tests import helpers

pytestmark = pytest.mark.gpu


def _pool():
    gs = graphgen.sbm_batch(14, seed0=4100, m_lo=1e3, m_hi=6e4)
    gs += [helpers.case_graph(c) for c in ("sbm_3000_4002", "sbm_20000_4000", "gnp_cliques", "rmat12", "rmat14",
                                          "small_test", "isolated", "k20")]
    return gs


def _alone(n, u, v, eps):
    with rtr.Graph.from_edges(n, u, v) as g:
        t = g.count()
        left = g.clean(eps)
        k = g.extract()
        return dict(triangles=t, triangles_left=left, n_clusters=k, cluster_of=g.cluster_of().copy())


@pytest.mark.parametrize("budget_mb,batch", [(4096, 32), (96, 16), (4096, 1)])
def test_served_results_equal_alone(budget_mb, batch):
    pool = _pool()
    rng = np.random.default_rng(budget_mb + batch)
    want = {}
    jobs = [(int(rng.integers(0, len(pool))), float(rng.choice([0.1, 0.3]))) for _ in range(160)]
    for gid, eps in set(jobs):
        want[(gid, eps)] = _alone(*pool[gid], eps)
    with rtr.Server(hbm_budget=budget_mb << 20, workers=6, batch_max_edges=20000, batch_max_graphs=batch) as srv:
        ids = [srv.add_graph(*g) for g in pool]
        assert ids == list(range(len(pool)))
        rids = [(srv.submit(gid, eps), gid, eps) for gid, eps in jobs]
        got = [(srv.wait(r), gid, eps) for r, gid, eps in rids]
        st = srv.stats()
    for res, gid, eps in got:
        assert res["status"] == 0, res["error"]
        w = want[(gid, eps)]
        for k in ("triangles", "triangles_left", "n_clusters"):
            assert res[k] == w[k], (gid, eps, k)
        assert (res["cluster_of"] == w["cluster_of"]).all(), (gid, eps)
        assert res["t_submit_ms"] <= res["t_start_ms"] <= res["t_end_ms"]
    assert st["peak_inflight"] > 1  # requests overlapped
    if batch > 1:
        assert st["batches"] > 0 and st["batched_requests"] > st["batches"]
    if budget_mb < 1024:
        assert st["evictions"] > 0  # graphs were evicted and rebuilt


def test_served_results_match_oracle():
    """A served result against the CPU oracle directly (cluster membership)."""
    import oracle
    n, u, v = helpers.case_graph("sbm_3000_4002")
    c = oracle.build_csr(n, u, v)
    s0 = oracle.count(c)
    s1 = oracle.initial_clean(c, s0, 0.1)
    cl, _ = oracle.extract(c, s1, 0.1)
    cof = np.empty(n, np.int64)
    for k in range(len(cl)):
        cof[cl.members(k)] = k
    with rtr.Server(workers=2, batch_max_edges=0, batch_max_graphs=1) as srv:
        gid = srv.add_graph(n, u, v)
        res = srv.wait(srv.submit(gid, 0.1))
    assert res["n_clusters"] == len(cl) and res["triangles"] == s0.total and res["triangles_left"] == s1.total
    assert (res["cluster_of"] == cof).all()


def test_server_reports_request_errors():
    with rtr.Server(workers=1) as srv:
        gid = srv.add_graph(3, np.array([0, 1]), np.array([1, 1]))  # self-loop: rejected when built
        res = srv.wait(srv.submit(gid, 0.3))
        assert res["status"] == 3 and "self-loop" in res["error"]
        ok = srv.add_graph(3, np.array([0, 1, 2]), np.array([1, 2, 0]))
        assert srv.wait(srv.submit(ok, 0.3))["status"] == 0
        with pytest.raises(rtr.RtrError):
            srv.submit(99, 0.3)
