// Request server for the decomposition path: graphs registered once, kept
// resident in HBM while the budget allows, and decomposition requests admitted
// continuously.
//
//   * Admission.  Workers (host threads) take the oldest queued request whose
//     graph is idle and whose device memory fits the budget: the graph's
//     measured working set (plus its resident size when it must be rebuilt);
//     an estimate from m and n before its first run.  Idle resident graphs are
//     evicted least-recently-used first to make room.  A request that does not
//     fit waits while later ones that fit go ahead; one that exceeds the whole
//     budget runs alone.
//   * Overlap.  Every graph has its own CUDA stream, so admitted requests run
//     concurrently on the device: a request that arrives while others are on
//     the GPU starts as soon as a worker and memory are free.
//   * Batching.  Requests for small graphs (m <= batch_max_edges) that are
//     waiting together, at the same eps and flags, are decomposed in one
//     launch sequence on the disjoint union of their graphs (rtr_batch_create);
//     results are split per graph and equal the graphs' own decompositions.
//     If a batched launch fails, its requests are re-run one by one so each
//     reports its own status.
//   * Results.  Per request: status, clusters, triangles before and after the
//     clean, optional cluster_of[n] (cluster index in creation order), and the
//     submit / start / end times on the server clock.
#include "../../include/rtr.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <vector>

namespace rtr {
void set_error(const char* fmt, ...);
}

namespace {

using Clock = std::chrono::steady_clock;

struct GraphEntry {
    std::vector<int64_t> src, dst;
    int64_t n = 0, m = 0;
    int flags = 0;
    rtr_graph* g = nullptr;      // resident on the device, or null
    bool busy = false;
    int64_t resident_bytes = 0;  // measured while resident
    int64_t scratch_bytes = 0;   // measured peak working set (0 = not run yet)
    uint64_t last_use = 0;
};

struct Request {
    int64_t id = 0, gid = 0;
    double eps = 0;
    int64_t* cluster_of = nullptr;
    int attempts = 0;
    bool solo = false;  // run alone (after its batch failed)
    bool done = false;
    rtr_request_info info{};
};

// Working set and resident size before a graph's first run: CSR and state are
// about 80 B per edge and 64 B per vertex; the triangle lists (96 B per
// triangle) are unknown, so allow 96 B per edge for them.
int64_t estimate_resident(const GraphEntry& G) { return 176 * G.m + 64 * G.n + (1 << 20); }
int64_t estimate_scratch(const GraphEntry& G) { return 96 * G.m + 96 * G.n + (1 << 20); }

}  // namespace

struct rtr_server {
    int device = 0;
    int64_t budget = 0;
    int64_t batch_max_edges = 0;
    int batch_max_graphs = 1;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<GraphEntry> graphs;  // stable addresses
    std::deque<Request*> queue;
    std::unordered_map<int64_t, Request*> reqs;
    int64_t next_id = 1;
    int64_t used = 0;  // reserved working sets + resident graphs
    int running = 0;
    bool stop = false;
    uint64_t tick = 0;
    Clock::time_point t0 = Clock::now();
    int64_t peak_used = 0, peak_running = 0, evictions = 0, batches = 0, batched_requests = 0;
    std::vector<std::thread> workers;

    double now_ms() const { return std::chrono::duration<double, std::milli>(Clock::now() - t0).count(); }

    // Evict idle resident graphs (LRU) outside `keep` until `need` fits.
    void make_room(int64_t need, const std::unordered_set<int64_t>& keep)
    {
        while (used + need > budget) {
            int64_t victim = -1;
            for (size_t i = 0; i < graphs.size(); ++i) {
                const GraphEntry& G = graphs[i];
                if (!G.g || G.busy || keep.count((int64_t)i)) continue;
                if (victim < 0 || G.last_use < graphs[victim].last_use) victim = (int64_t)i;
            }
            if (victim < 0) return;
            GraphEntry& V = graphs[victim];
            rtr_graph_destroy(V.g);
            V.g = nullptr;
            used -= V.resident_bytes;
            V.resident_bytes = 0;
            ++evictions;
        }
    }

    // Under the lock: take the next admissible work item.
    bool pick(std::vector<Request*>& out, int64_t& reserve, bool& batched)
    {
        for (auto it = queue.begin(); it != queue.end(); ++it) {
            Request* r = *it;
            GraphEntry& G = graphs[r->gid];
            if (G.busy) continue;
            std::vector<Request*> chosen{r};
            std::unordered_set<int64_t> gids{r->gid};
            int64_t need = 0;
            const bool small = batch_max_graphs > 1 && G.m <= batch_max_edges && !r->solo;
            if (small) {
                need = estimate_resident(G) + estimate_scratch(G);
                for (auto jt = std::next(it); jt != queue.end() && (int)chosen.size() < batch_max_graphs; ++jt) {
                    Request* q = *jt;
                    GraphEntry& H = graphs[q->gid];
                    if (H.busy || H.m > batch_max_edges || q->solo || q->eps != r->eps || H.flags != G.flags ||
                        gids.count(q->gid))
                        continue;
                    chosen.push_back(q);
                    gids.insert(q->gid);
                    need += estimate_resident(H) + estimate_scratch(H);
                }
            } else {
                const int64_t scratch = G.scratch_bytes ? G.scratch_bytes : estimate_scratch(G);
                need = G.g ? scratch : estimate_resident(G) + scratch;
                need += need / 8 * r->attempts;  // grow after an allocation failure
            }
            if (used + need > budget) make_room(need, gids);
            if (used + need > budget && running > 0) continue;  // wait for memory; later requests may fit
            for (Request* q : chosen) {
                graphs[q->gid].busy = true;
                queue.erase(std::find(queue.begin(), queue.end(), q));
            }
            used += need;
            ++running;
            peak_used = std::max(peak_used, used);
            peak_running = std::max<int64_t>(peak_running, running);
            out = std::move(chosen);
            reserve = need;
            batched = small;
            return true;
        }
        return false;
    }

    void run_single(Request* r, int64_t reserve);
    void run_batch(std::vector<Request*>& rs, int64_t reserve);
    void worker();
};

void rtr_server::run_single(Request* r, int64_t reserve)
{
    GraphEntry& G = graphs[r->gid];
    const int64_t was_resident = G.g ? G.resident_bytes : 0;
    bool built = false;
    int rc = RTR_OK;
    r->info.t_start_ms = now_ms();
    if (!G.g) {
        rc = rtr_graph_create_from_edges(G.src.data(), G.dst.data(), G.m, G.n, device, G.flags, &G.g);
        built = rc == RTR_OK;
    }
    int64_t tri = 0, left = 0, ncl = 0;
    if (!rc) rc = rtr_count(G.g, &tri);
    if (!rc) rc = rtr_clean(G.g, r->eps, &left);
    if (!rc) rc = rtr_extract(G.g, &ncl);
    if (!rc && r->cluster_of) rc = rtr_get_cluster_of(G.g, r->cluster_of);
    const std::string err = rc ? rtr_last_error() : "";
    int64_t res = 0, peak = 0;
    if (G.g) rtr_get_memory(G.g, &res, &peak);
    std::lock_guard<std::mutex> lk(mu);
    used -= reserve + was_resident;
    --running;
    if (rc && G.g && built) {  // a failed first build leaves nothing resident
        rtr_graph_destroy(G.g);
        G.g = nullptr;
        res = 0;
    }
    G.resident_bytes = G.g ? res : 0;
    used += G.resident_bytes;
    if (peak > G.scratch_bytes) G.scratch_bytes = peak;
    G.busy = false;
    G.last_use = ++tick;
    if (rc == RTR_ERR_CUDA && running > 0 && r->attempts < 3) {
        // most likely device memory taken by the requests in flight: retry
        ++r->attempts;
        queue.push_front(r);
    } else {
        r->info.status = rc;
        r->info.n_clusters = ncl;
        r->info.triangles = tri;
        r->info.triangles_left = left;
        r->info.batched = 1;
        r->info.t_end_ms = now_ms();
        snprintf(r->info.error, sizeof r->info.error, "%s", err.c_str());
        r->done = true;
    }
    cv_done.notify_all();
    cv_work.notify_all();
}

void rtr_server::run_batch(std::vector<Request*>& rs, int64_t reserve)
{
    const int64_t K = (int64_t)rs.size();
    std::vector<int64_t> eoff(K + 1, 0), nv(K), base(K + 1, 0);
    for (int64_t k = 0; k < K; ++k) {
        const GraphEntry& G = graphs[rs[k]->gid];
        eoff[k + 1] = eoff[k] + G.m;
        nv[k] = G.n;
        base[k + 1] = base[k] + G.n;
    }
    std::vector<int64_t> src(eoff[K] + 1), dst(eoff[K] + 1);
    for (int64_t k = 0; k < K; ++k) {
        const GraphEntry& G = graphs[rs[k]->gid];
        std::copy(G.src.begin(), G.src.end(), src.begin() + eoff[k]);
        std::copy(G.dst.begin(), G.dst.end(), dst.begin() + eoff[k]);
    }
    const double t_start = now_ms();
    rtr_graph* bg = nullptr;
    int rc = rtr_batch_create(src.data(), dst.data(), eoff.data(), nv.data(), K, device,
                              graphs[rs[0]->gid].flags, &bg);
    const int64_t N = base[K];
    int64_t total = 0, left = 0, ncl = 0, n_all = 0, m_all = 0;
    std::vector<int64_t> tri(K, 0), tri_left(K, 0), off;
    std::vector<uint32_t> sup;
    auto per_graph = [&](std::vector<int64_t>& out) -> int {
        int r2 = rtr_get_weights(bg, nullptr, nullptr, sup.data(), nullptr);
        if (r2) return r2;
        for (int64_t k = 0; k < K; ++k) {
            int64_t s = 0;
            for (int64_t j = off[base[k]]; j < off[base[k + 1]]; ++j) s += sup[j];
            out[k] = s / 6;  // each triangle: three edges, both directions
        }
        return RTR_OK;
    };
    if (!rc) {
        rtr_graph_info(bg, &n_all, &m_all);
        off.resize(n_all + 1);
        sup.resize(2 * m_all + 1);
        rc = rtr_get_csr(bg, off.data(), nullptr);
    }
    if (!rc) rc = rtr_count(bg, &total);
    if (!rc) rc = per_graph(tri);
    if (!rc) rc = rtr_clean(bg, rs[0]->eps, &left);
    if (!rc) rc = per_graph(tri_left);
    if (!rc) rc = rtr_extract(bg, &ncl);
    std::vector<int64_t> seed(ncl + 1), cof(N + 1), local(ncl + 1), cnt(K, 0);
    if (!rc) rc = rtr_get_clusters(bg, seed.data(), nullptr, nullptr, nullptr, nullptr, nullptr);
    if (!rc) rc = rtr_get_cluster_of(bg, cof.data());
    if (!rc) {
        // clusters are in global seed order; restricted to one graph that is
        // the graph's own creation order
        for (int64_t c = 0; c < ncl; ++c) {
            const int64_t k = std::upper_bound(base.begin(), base.end(), seed[c]) - base.begin() - 1;
            local[c] = cnt[k]++;
        }
        for (int64_t k = 0; k < K; ++k)
            if (rs[k]->cluster_of)
                for (int64_t v = 0; v < nv[k]; ++v) rs[k]->cluster_of[v] = local[cof[base[k] + v]];
    }
    const std::string err = rc ? rtr_last_error() : "";
    if (bg) rtr_graph_destroy(bg);
    std::lock_guard<std::mutex> lk(mu);
    used -= reserve;
    --running;
    ++batches;
    batched_requests += K;
    const double t_end = now_ms();
    for (int64_t k = 0; k < K; ++k) {
        Request* r = rs[k];
        GraphEntry& G = graphs[r->gid];
        G.busy = false;
        G.last_use = ++tick;
        if (rc) {  // one bad graph fails the whole launch: run each request alone
            r->solo = true;
            queue.push_front(r);
            continue;
        }
        r->info.status = rc;
        r->info.n_clusters = rc ? 0 : cnt[k];
        r->info.triangles = tri[k];
        r->info.triangles_left = tri_left[k];
        r->info.batched = (int)K;
        r->info.t_start_ms = t_start;
        r->info.t_end_ms = t_end;
        snprintf(r->info.error, sizeof r->info.error, "%s", err.c_str());
        r->done = true;
    }
    cv_done.notify_all();
    cv_work.notify_all();
}

void rtr_server::worker()
{
    for (;;) {
        std::vector<Request*> work;
        int64_t reserve = 0;
        bool batched = false;
        {
            std::unique_lock<std::mutex> lk(mu);
            cv_work.wait(lk, [&] { return stop || pick(work, reserve, batched); });
            if (work.empty()) return;  // stopping
        }
        if (batched)
            run_batch(work, reserve);
        else
            run_single(work[0], reserve);
    }
}

extern "C" {

int rtr_server_create(int device, int64_t hbm_budget_bytes, int workers, int64_t batch_max_edges,
                      int batch_max_graphs, rtr_server** out)
{
    if (!out || workers < 1 || hbm_budget_bytes <= 0 || batch_max_graphs < 1) {
        rtr::set_error("rtr_server_create: bad arguments");
        return RTR_ERR_ARG;
    }
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0 || device < 0 || device >= ndev) {
        rtr::set_error("no CUDA device %d is visible (librtr has no CPU path)", device);
        return RTR_ERR_CUDA;
    }
    rtr_server* S = new rtr_server();
    S->device = device;
    S->budget = hbm_budget_bytes;
    S->batch_max_edges = batch_max_edges;
    S->batch_max_graphs = batch_max_graphs;
    for (int i = 0; i < workers; ++i) S->workers.emplace_back([S] { S->worker(); });
    *out = S;
    return RTR_OK;
}

int rtr_server_add_graph(rtr_server* S, const int64_t* src, const int64_t* dst, int64_t m, int64_t n, int flags,
                         int64_t* graph_id)
{
    if (!S || !graph_id || m < 0 || n < 0 || ((!src || !dst) && m > 0)) {
        rtr::set_error("rtr_server_add_graph: bad arguments");
        return RTR_ERR_ARG;
    }
    GraphEntry G;
    G.src.assign(src, src + m);
    G.dst.assign(dst, dst + m);
    G.n = n;
    G.m = m;
    G.flags = flags;
    std::lock_guard<std::mutex> lk(S->mu);
    S->graphs.push_back(std::move(G));
    *graph_id = (int64_t)S->graphs.size() - 1;
    return RTR_OK;
}

int rtr_server_submit(rtr_server* S, int64_t graph_id, double eps, int64_t* cluster_of, int64_t* request_id)
{
    if (!S || !request_id) {
        rtr::set_error("rtr_server_submit: null argument");
        return RTR_ERR_ARG;
    }
    std::lock_guard<std::mutex> lk(S->mu);
    if (graph_id < 0 || graph_id >= (int64_t)S->graphs.size() || S->stop) {
        rtr::set_error("rtr_server_submit: unknown graph %lld", (long long)graph_id);
        return RTR_ERR_ARG;
    }
    Request* r = new Request();
    r->id = S->next_id++;
    r->gid = graph_id;
    r->eps = eps;
    r->cluster_of = cluster_of;
    r->info.t_submit_ms = S->now_ms();
    S->reqs[r->id] = r;
    S->queue.push_back(r);
    *request_id = r->id;
    S->cv_work.notify_one();
    return RTR_OK;
}

int rtr_server_wait(rtr_server* S, int64_t request_id, rtr_request_info* info)
{
    if (!S) {
        rtr::set_error("null server");
        return RTR_ERR_ARG;
    }
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->reqs.find(request_id);
    if (it == S->reqs.end()) {
        rtr::set_error("rtr_server_wait: unknown request %lld", (long long)request_id);
        return RTR_ERR_ARG;
    }
    Request* r = it->second;
    S->cv_done.wait(lk, [&] { return r->done; });
    if (info) *info = r->info;
    S->reqs.erase(it);
    delete r;
    return RTR_OK;
}

int rtr_server_stats(rtr_server* S, int64_t* stats, int n)
{
    if (!S || !stats) {
        rtr::set_error("null argument");
        return RTR_ERR_ARG;
    }
    std::lock_guard<std::mutex> lk(S->mu);
    int64_t resident = 0;
    for (const GraphEntry& G : S->graphs) resident += G.g ? 1 : 0;
    const int64_t v[8] = {resident, S->used, S->peak_used, S->peak_running,
                          S->evictions, S->batches, S->batched_requests, (int64_t)S->queue.size()};
    for (int i = 0; i < n && i < 8; ++i) stats[i] = v[i];
    return RTR_OK;
}

int rtr_server_destroy(rtr_server* S)
{
    if (!S) return RTR_OK;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
        for (Request* r : S->queue) {  // queued requests are cancelled
            r->info.status = RTR_ERR_STATE;
            r->done = true;
        }
        S->queue.clear();
        S->cv_work.notify_all();
        S->cv_done.notify_all();
    }
    for (std::thread& t : S->workers) t.join();
    for (GraphEntry& G : S->graphs)
        if (G.g) rtr_graph_destroy(G.g);
    for (auto& kv : S->reqs) delete kv.second;
    delete S;
    return RTR_OK;
}

}  // extern "C"
