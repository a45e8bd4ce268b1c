#!/usr/bin/env python3
"""Benchmark of the RTRExtractor decomposition path on B200.

One step = one full decomposition (count + clean + extract) of the
335,000-vertex Chung-Lu power-law graph with 2,000 planted communities
(~926k undirected edges, seed 2; the co-purchase-network shape), at
eps = 0.3, through librtr.so.

Prints ONE JSON line (rank 0):
  value      decomposed edges/s, whole job (all ranks), graph resident in HBM,
             device-timed (CUDA events on the library's stream) per step,
             L2 flushed (256 MiB write) before every step
  e2e        the same metric through the public C ABI with host buffers:
             pinned host edge arrays -> rtr_graph_create_from_edges (H2D +
             device CSR build) -> rtr_decompose -> cluster_of read back (D2H)
  roofline   the dominant kernel's algorithmic bytes / its event-timed duration
             against the measured HBM copy bandwidth
  cpu_baseline  the reference's own sequential RTRex (oracle/_ref/RTRex, mode s,
             1 thread) on the same graph, or the restated oracle when that
             binary is absent
Multi-GPU (torchrun): replicas only -- each rank decomposes its own copy, the
step time is the max over ranks, value counts every rank's edges.

``--impl reference`` times the reference's CPU implementation instead (mode p,
all host threads) on the same workload and metric.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import shutil
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "decomposed edges/s (count+clean+extract)"
UNIT = "edges/s"
EPS = 0.3
WORKLOAD = "chung_lu"
WORKLOAD_DESC = ("Chung-Lu power law n=335,000, ~926k edges, exponent 2.3, expected degree cap 550, "
                 "+2,000 planted communities of 5-12 vertices at p=0.8, seed 2; eps=0.3")
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "RTRex")


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--eps", type=float, default=EPS)
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--no-clocks", action="store_true")
    ap.add_argument("--skip-extras", action="store_true",
                    help="leave out the R-MAT scale-24 count, batched and reference-GPU legs of the default run")
    ap.add_argument("--serve-requests", type=int, default=240)
    ap.add_argument("--serve-rate", type=float, default=2000.0, help="Poisson arrival rate (requests/s)")
    ap.add_argument("--serve-pool", type=int, default=32)
    ap.add_argument("--serve-max-edges", type=float, default=2e6)
    ap.add_argument("--serve-workers", type=int, default=8)
    ap.add_argument("--serve-budget-gb", type=float, default=120.0)
    ap.add_argument("--rmat-scale", type=int, default=24)
    ap.add_argument("--count-mode", type=int, default=0, help="rtr_set_count_mode for --workload rmat_count")
    ap.add_argument("--workload", default=WORKLOAD, choices=[WORKLOAD, "batch", "serve", "rmat_count", "bundled"],
                    help="batch: the 4,096-graph SBM batch, batched vs per-graph plain decompositions")
    ap.add_argument("--batch-graphs", type=int, default=4096)
    return ap.parse_args()


def workload():
    from rtrex_cuda_b200 import graphgen
    return graphgen.config_graph(WORKLOAD)


# ------------------------------------------------------------------ CPU legs

def _phase_seconds(stdout: str) -> float:
    """count + clean + extract from the reference's phase timers (Decomposition.h:556,563,926)."""
    keys = ["Time for getting the weights", "Time for the initial clean", "Time for getting the clusters"]
    tot = 0.0
    for k in keys:
        m = re.search(re.escape(k) + r":\s*([0-9.eE+-]+)s", stdout)
        if not m:
            raise RuntimeError(f"reference output lacks '{k}'")
        tot += float(m.group(1))
    return tot


def run_reference_binary(path: str, mode: str, threads: int) -> float:
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    with tempfile.TemporaryDirectory() as td:
        out = subprocess.run([REF_BIN, path, "bench", repr(EPS), mode], cwd=td, env=env, capture_output=True,
                             text=True, timeout=900)
    if out.returncode != 0:
        raise RuntimeError(f"reference run failed: {out.stderr[-300:]}")
    return _phase_seconds(out.stdout)


def run_oracle_port(n, u, v) -> float:
    import oracle  # the restated sequential oracle, used only as a timed baseline
    c = oracle.build_csr(n, u, v)
    t0 = time.perf_counter()
    s0 = oracle.count(c)
    s1 = oracle.initial_clean(c, s0, EPS)
    oracle.extract(c, s1, EPS)
    return time.perf_counter() - t0


def cpu_times(n, u, v, runs: int, mode: str, threads: int):
    """[(seconds, kind)] for `runs` timed runs of the CPU implementation."""
    from rtrex_cuda_b200 import graphgen
    if os.path.exists(REF_BIN):
        with tempfile.TemporaryDirectory() as td:
            path = os.path.join(td, "g.txt")
            graphgen.write_escape(path, n, u, v)
            return [run_reference_binary(path, mode, threads) for _ in range(runs)], "reference"
    return [run_oracle_port(n, u, v) for _ in range(runs)], "port"


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    n, u, v = workload()
    m = int(u.size)
    threads = os.cpu_count() or 1
    mode = "p"
    cpu_times(n, u, v, args.warmup, mode, threads) if args.warmup > 0 else None
    times, kind = cpu_times(n, u, v, args.steps, mode, threads)
    if kind == "port":
        threads = 1
    sec = float(np.mean(times))
    value = m / sec
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "desc": WORKLOAD_DESC, "n": n, "m": m, "eps": EPS},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                         "sample": f"full decomposition of the workload graph per step, mode {mode}"
                                   if kind == "reference" else "full decomposition, restated oracle, 1 thread"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ replicas

def replica_max(x: float, world: int, device) -> float:
    """Max of a per-rank time over all ranks (the slowest replica bounds the step)."""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def shard(items, rank: int, world: int):
    """Rank `rank`'s share of independent work items (graphs, requests): every
    world-th item, so sizes drawn from one distribution spread evenly."""
    return list(items)[rank::world] if world > 1 else list(items)


def gather_values(vals, world: int):
    """Concatenate every rank's list of values (all ranks receive the result)."""
    if world <= 1:
        return list(vals)
    import torch.distributed as dist
    parts = [None] * world
    dist.all_gather_object(parts, list(vals))
    return [x for part in parts for x in part]


def dist_init():
    """(world, rank, local device) under torchrun; NCCL only for barriers and
    the max / gather of timings -- no collective is on the data path."""
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))
    return world, rank, local


def replica_value(edges_per_rank: int, world: int, ms_step: float) -> float:
    """Whole-job edges/s: every rank decomposes its own copy in ms_step (max over ranks)."""
    return world * edges_per_rank / (ms_step / 1e3)


# ------------------------------------------------------------------ GPU leg

class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int, enabled: bool):
        self.device = device
        self.proc = None
        self.lines = []
        self.enabled = enabled and shutil.which("nvidia-smi") is not None

    def __enter__(self):
        if self.enabled:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.th.join(timeout=2)

    def summary(self):
        if not self.enabled or not self.lines:
            return None
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def count_bytes(n, off, nb):
    """Algorithmic bytes of the counting stage: 8(n+1) + 4*sum over the degree-
    oriented edges (u->v) of (d+(u) + d+(v)) + 2m*12 + 8n."""
    deg = np.diff(off)
    src = np.repeat(np.arange(n), deg)
    key_s = deg[src] * np.int64(n) + src
    key_d = deg[nb] * np.int64(n) + nb
    out = key_s < key_d  # orient from lower (deg, id) to higher
    dplus = np.bincount(src[out], minlength=n)
    s = int((dplus[src[out]] + dplus[nb[out]]).sum())
    m2 = int(nb.size)
    return 8 * (n + 1) + 4 * s + m2 * 12 + 8 * n, s


def clean_bytes(n, off, nb, status, tri_removed):
    """Algorithmic bytes of the clean: per removed undirected edge 4*(d(u)+d(v)),
    one status byte per directed slot, 48 bytes per removed triangle."""
    deg = np.diff(off)
    src = np.repeat(np.arange(n), deg)
    fwd = (src < nb) & (status == ord("N"))
    return int(4 * (deg[src[fwd]] + deg[nb[fwd]]).sum() + nb.size + 48 * tri_removed)


def oriented_sum_chunked(off, nb, chunk=1 << 24):
    """Sum over the degree-oriented edges u->v of d+(u) + d+(v), which equals the
    sum over undirected edges of min(deg u, deg v); vertex chunks keep the host
    memory bounded on graphs of hundreds of millions of edges."""
    n = off.size - 1
    deg = np.diff(off)
    total = 0
    a = 0
    while a < n:
        b = int(np.searchsorted(off, off[a] + chunk, side="right"))
        b = max(b, a + 1)
        b = min(b, n)
        s0, s1 = int(off[a]), int(off[b])
        src = np.repeat(np.arange(a, b, dtype=np.int64), deg[a:b])
        dst = nb[s0:s1]
        fwd = src < dst
        total += int(np.minimum(deg[src[fwd]], deg[dst[fwd]]).sum())
        a = b
    return total


def rmat24_leg(args, dev, flush_l2, peak, peak_kind, scale=24, steps=None, mode=0, e2e_runs=2):
    """R-MAT scale 24 (edge factor 16, a,b,c = .57,.19,.19, seed 3) counted on
    the device: its triangle lists would need ~1 TB, so rtr_count folds
    straight from the CSR rows.  Device-timed count steps (CUDA events; the
    graph is resident and 4 GB of rows exceed L2), then end to end from pinned
    host edges (H2D + CSR build + count + perVertex read back).  Other scales
    (and a forced count mode) serve profiling."""
    import torch
    import rtrex_cuda_b200 as rtr
    steps = max(1, min(args.steps, 3)) if steps is None else steps
    g = rtr.Graph.from_rmat(scale, 16, seed=3, device=dev)
    g.set_count_mode(mode)
    gen_ms = g.stats()["ms_build"]
    n, m = g.n, g.m
    g.count()  # warm-up
    ms, launches0 = [], g.stats()["launches"]
    for k in range(steps):
        flush_l2(k)
        total = g.count()
        ms.append(g.stats()["ms_count"])
    launches = (g.stats()["launches"] - launches0) // steps
    layout = "rows (no triangle lists)" if not g.count_mode()[2] else "triangle lists"
    windows, list_entries = g.count_windows()
    kms = g.kernel_ms()
    off, nb = g.csr()
    g.close()
    osum = oriented_sum_chunked(off, nb)
    b_count = 8 * (n + 1) + 4 * osum + 24 * m + 8 * n
    t = float(np.mean(ms)) / 1e3
    out = {"workload": f"rmat{scale}", "desc": f"R-MAT scale {scale}, edge factor 16, a,b,c,d = .57,.19,.19,.05, "
                                                "seed 3, symmetrised, self-loops and repeats dropped (device generator)",
           "n": n, "m": m, "triangles": total, "layout": layout, "list_windows": windows,
           "list_entries": list_entries, "steps": steps,
           "ms_per_count": t * 1e3, "edges_per_s": m / t, "triangles_per_s": total / t,
           "generation_and_csr_build_ms": gen_ms,
           "kernel_ms": {"edge_fold_and_heavy_count": kms["k_edge_fold"],
                         "edge_fold_light_edges": kms["k_edge_fold_light"],
                         "edge_count_heavy_edges": kms["k_edge_count_heavy"], "list_fill": kms["k_tri_fill"],
                         "list_fill_light": kms["k_fill_light"], "list_fill_heavy": kms["k_fill_heavy"],
                         "vertex_fold": kms["k_vertex_fold"], "vertex_fold_warps": kms["k_vfold_warp"],
                         "vertex_fold_blocks": kms["k_vfold_block"]},
           "gpu_launches_per_count": launches,
           "roofline_count": {"bound": "hbm", "algorithmic_bytes": b_count, "oriented_sum": osum,
                              "achieved": b_count / t / 1e9, "peak": peak, "unit": "GB/s",
                              "frac": b_count / t / 1e9 / peak, "peak_kind": peak_kind}}
    if not args.skip_e2e:
        src = np.repeat(np.arange(n, dtype=np.int64), np.diff(off))
        fwd = src < nb
        hu = torch.from_numpy(src[fwd]).pin_memory()
        hv = torch.from_numpy(nb[fwd]).pin_memory()
        del src, fwd
        times = []
        for k in range(e2e_runs):
            flush_l2(k)
            t0 = time.perf_counter()
            g2 = rtr.Graph.from_edges(n, hu.numpy(), hv.numpy(), device=dev)
            g2.count()
            _, pv, _, _ = g2.weights(per_edge=False, support=False)
            g2.close()
            times.append(time.perf_counter() - t0)
        sec = float(np.min(times))
        out["e2e"] = {"value": m / sec, "unit": "edges/s", "h2d_bytes_per_step": 16 * m,
                      "d2h_bytes_per_step": int(pv.nbytes) + 8, "ms_per_step": sec * 1e3}
    return out


def rmat_count_arm(args):
    """--workload rmat_count: the config-3 counting line on its own (R-MAT at
    --rmat-scale, rows layout unless --count-mode says otherwise)."""
    import torch
    torch.cuda.set_device(0)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.int32, device="cuda:0")

    def flush_l2(k):
        flush.fill_(k)
        torch.cuda.synchronize(0)

    peak, peak_kind = measured_peaks()
    r = rmat24_leg(args, 0, flush_l2, peak, peak_kind, scale=args.rmat_scale, steps=args.steps, mode=args.count_mode)
    line = {"metric": "counted edges/s (weighted triangle counting)", "value": r["edges_per_s"], "unit": "edges/s",
            "n_gpus": 1, "steps": r["steps"], "warmup": 1, "ms_per_step": r["ms_per_count"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": r["workload"], "desc": r["desc"], "n": r["n"], "m": r["m"],
                       "layout": r["layout"], "list_windows": r["list_windows"],
                       "l2": "flushed (256 MiB write) before every step"},
            "triangles": r["triangles"], "triangles_per_s": r["triangles_per_s"], "e2e": r.get("e2e"),
            "roofline": r["roofline_count"], "gpu_launches": r["gpu_launches_per_count"] * r["steps"],
            "kernel_ms": r["kernel_ms"], "generation_and_csr_build_ms": r["generation_and_csr_build_ms"]}
    print(json.dumps(line), flush=True)


def bundled_arm(args):
    """--workload bundled: the reference's own bundled graphs (clean_email,
    clean_astro, random_graph_rtr; committed copies under tests/golden/data/)
    decomposed at eps, device stage times (CUDA events, mean of --steps after
    --warmup) beside the reference's phase timers (oracle/_ref/RTRex, mode s,
    one core) on the same box."""
    import torch
    import rtrex_cuda_b200 as rtr
    from rtrex_cuda_b200 import graphgen
    torch.cuda.set_device(0)
    out = {}
    for name in ("clean_email", "clean_astro", "random_graph_rtr"):
        path = os.path.join(ROOT, "tests", "golden", "data", name + ".txt.gz")
        n, u, v = graphgen.read_escape(path)
        ms = {"count": [], "clean": [], "extract": [], "decompose": []}
        with rtr.Graph.from_edges(n, u, v) as g:
            for k in range(args.warmup + args.steps):
                ncl = g.decompose(args.eps)
                st, km = g.stats(), g.kernel_ms()
                if k >= args.warmup:
                    ms["count"].append(st["ms_count"])
                    ms["clean"].append(st["ms_clean"])
                    ms["extract"].append(st["ms_extract"])
                    ms["decompose"].append(km["decompose"])
        res = {"n": n, "m": int(u.size), "clusters": ncl,
               "device_ms": {k: float(np.mean(x)) for k, x in ms.items()}}
        if os.path.exists(REF_BIN):
            with tempfile.TemporaryDirectory() as td:
                p2 = os.path.join(td, "g.txt")
                graphgen.write_escape(p2, n, u, v)
                r = subprocess.run([REF_BIN, p2, "bench", repr(args.eps), "s"], cwd=td, capture_output=True,
                                   text=True, timeout=900, env=dict(os.environ, OMP_NUM_THREADS="1"))
            grab = lambda k: float(re.search(re.escape(k) + r":\s*([0-9.eE+-]+)s", r.stdout).group(1)) * 1e3
            res["reference_ms_1core"] = {"count": grab("Time for getting the weights"),
                                         "clean": grab("Time for the initial clean"),
                                         "extract": grab("Time for getting the clusters")}
        out[name] = res
    line = {"metric": "decomposed edges/s (count+clean+extract)", "unit": "edges/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "dtype": "f64",
            "data": "the reference's bundled graphs", "config": {"workload": "bundled", "eps": args.eps},
            "value": sum(r["m"] for r in out.values()) / sum(r["device_ms"]["decompose"] / 1e3 for r in out.values()),
            "graphs": out}
    print(json.dumps(line), flush=True)


def batched_leg(args, dev):
    """The batched form's driver-measured ratio: the 4,096-graph SBM batch
    (edge targets log-uniform in [1K, 200K], seeds 4000+i) as one decomposition
    of the disjoint union against one plain decomposition per graph, both end
    to end through the C ABI from host arrays."""
    import rtrex_cuda_b200 as rtr
    from rtrex_cuda_b200 import graphgen
    t0 = time.perf_counter()
    graphs = graphgen.sbm_batch(4096)
    gen_s = time.perf_counter() - t0
    K = len(graphs)
    with rtr.Graph.batch(graphs, device=dev) as g:
        tuning = g.autotune()
    times, dev_ms = [], []
    for k in range(3):  # one warm-up, two timed
        t0 = time.perf_counter()
        with rtr.Graph.batch(graphs, device=dev) as g:
            g.set_tuning(*tuning)
            g.decompose(args.eps)
            counts = g.batch_cluster_counts()
            dev_ms.append(g.kernel_ms()["decompose"])
        if k:
            times.append(time.perf_counter() - t0)
    batched_s = float(np.mean(times))
    t0 = time.perf_counter()
    plain_counts = []
    for (n, u, v) in graphs:
        with rtr.Graph.from_edges(n, u, v, device=dev) as g1:
            plain_counts.append(g1.decompose(args.eps))
    plain_s = time.perf_counter() - t0
    return {"workload": "sbm_batch", "graphs": K, "edges": int(sum(x[1].size for x in graphs)),
            "batched_graphs_per_s": K / batched_s, "batched_device_graphs_per_s": K / (np.mean(dev_ms[1:]) / 1e3),
            "plain_graphs_per_s": K / plain_s, "batched_vs_plain": plain_s / batched_s,
            "per_graph_cluster_counts_equal": bool((np.asarray(plain_counts) == counts).all()),
            "autotune": {"gallop_ratio": tuning[0], "heavy_degree": tuning[1], "heavy_edge": tuning[2]},
            "generation_s": gen_s, "timing": "end to end through the C ABI from host arrays, mean of 2"}


REF_CUDA_BIN = os.path.join(ROOT, "oracle", "_ref", "RTRex_CUDA")


def gpu_baseline_leg(dev, timeout_s=120):
    """The reference's CUDA port (RTRex_CUDA, built from its sources for sm_100a
    by oracle/Makefile ref-cuda) on configs 1 and 2: its own phase timers, and how
    its results diverge from the reference's sequential code (its outputs are not
    a parity target: it skips triangles, breaks ties differently and defers
    singletons)."""
    from rtrex_cuda_b200 import graphgen
    if not os.path.exists(REF_CUDA_BIN):
        return {"unavailable": "oracle/_ref/RTRex_CUDA was not built (needs the reference sources)"}
    import hashlib
    gold_path = os.path.join(ROOT, "tests", "golden", "golden.json")
    with open(gold_path) as f:
        gold = json.load(f)["cases"]
    out = {}
    for name in ("gnp_cliques", "chung_lu"):
        n, u, v = graphgen.config_graph(name)
        res = {"n": n, "m": int(u.size)}
        with tempfile.TemporaryDirectory() as td:
            path = os.path.join(td, "g.txt")
            graphgen.write_escape(path, n, u, v)
            t0 = time.perf_counter()
            try:
                r = subprocess.run([REF_CUDA_BIN, path, "g", repr(EPS), str(dev)], cwd=td, capture_output=True,
                                   text=True, timeout=timeout_s)
                stdout, rc = r.stdout, r.returncode
            except subprocess.TimeoutExpired as e:
                stdout = e.stdout.decode() if isinstance(e.stdout, bytes) else (e.stdout or "")
                rc = None
                res["timed_out_after_s"] = timeout_s
            res["wall_s"] = time.perf_counter() - t0
            res["rc"] = rc
            grab = lambda pat: (lambda mm: float(mm.group(1)) if mm else None)(re.search(pat, stdout))
            res["count_s"] = grab(r"\[GPU Triangle Count\] Found \d+ triangles in ([0-9.]+) s")
            res["clean_s"] = grab(r"\[GPU Clean\] Done in ([0-9.]+) s")
            res["extract_s"] = grab(r"\[Extraction\] \d+ clusters in ([0-9.]+) s")
            tri = re.search(r"\[GPU Triangle Count\] Found (\d+) triangles", stdout)
            ncl = re.search(r"\[Extraction\] (\d+) clusters", stdout)
            res["triangles"] = int(tri.group(1)) if tri else None
            res["clusters"] = int(ncl.group(1)) if ncl else None
            want = gold[name]["0.3"]
            res["triangles_reference_cpu"] = want["count"]["total"]
            res["clusters_reference_cpu"] = want["extract"]["clusters"]
            if rc == 0:
                sec = sum(x for x in (res["count_s"], res["clean_s"], res["extract_s"]) if x)
                res["edges_per_s"] = u.size / sec if sec else None
                files = {}
                for kind in ("decomposition", "stats", "freq", "cut"):
                    fp = os.path.join(td, f"RTRex-CUDA-g-{kind}.txt")
                    files[kind] = (os.path.exists(fp) and
                                   hashlib.sha256(open(fp, "rb").read()).hexdigest() == want["files"][kind])
                res["output_files_equal_reference_cpu"] = files
        out[name] = res
    return out


def ours_arm(args):
    import torch
    import torch.distributed as dist
    import rtrex_cuda_b200 as rtr

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))
    dev = local
    torch.cuda.set_device(dev)

    def barrier():
        if world > 1:
            dist.barrier()

    def allmax(x: float) -> float:
        return replica_max(x, world, torch.device("cuda", dev))

    n, u, v = workload()
    m = int(u.size)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.int32, device=f"cuda:{dev}")  # 256 MiB > 126 MB L2

    def flush_l2(k):
        flush.fill_(k)
        torch.cuda.synchronize(dev)

    g = rtr.Graph.from_edges(n, u, v, device=dev)
    for k in range(args.warmup):
        flush_l2(k)
        g.decompose(args.eps)
    launches0 = g.stats()["launches"]
    step_ms, kms = [], []
    barrier()
    torch.cuda.synchronize(dev)
    with ClockSampler(dev, not args.no_clocks) as clocks:
        wall0 = time.perf_counter()
        count_ms = []
        for k in range(args.steps):
            flush_l2(k + 1)
            ncl = g.decompose(args.eps)
            km = g.kernel_ms()
            step_ms.append(km["decompose"])
            kms.append(km)
            count_ms.append(g.stats()["ms_count"])
        torch.cuda.synchronize(dev)
        wall = time.perf_counter() - wall0
    barrier()
    launches = g.stats()["launches"] - launches0
    ms_step = allmax(float(np.mean(step_ms)))
    value = replica_value(m, world, ms_step)

    # roofline of the dominant kernel (per-launch averages over the timed steps)
    names = ["k_edge_fold", "k_tri_fill", "k_vertex_fold", "k_clean_units", "k_extract_components"]
    avg = {k: float(np.mean([x[k] for x in kms])) for k in names}
    dominant = max(names, key=lambda k: avg[k])
    off, nb = g.csr()
    total = g.count()
    left = g.clean(args.eps)
    status = g.status()
    b_count, orient_sum = count_bytes(n, off, nb)
    b_clean = clean_bytes(n, off, nb, status, total - left)
    peak, peak_kind = measured_peaks()
    traffic, traffic_source = None, None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            tj = json.load(f)
        traffic = tj.get(dominant)
        traffic_source = "profiles/traffic.json: " + tj.get("_captured", "ncu capture of an earlier build")
    if dominant == "k_clean_units":
        # the clean-replay stage timer: k_clean_rounds (large units, side stream)
        # with k_clean_units (small units) and the perVertex fold of the rounds
        alg, t_ms = b_clean, avg[dominant]
    elif dominant in ("k_edge_fold", "k_tri_fill", "k_vertex_fold"):
        alg, t_ms = b_count, avg["k_edge_fold"] + avg["k_tri_fill"] + avg["k_vertex_fold"]
    else:
        alg, t_ms = None, avg[dominant]
    achieved = (alg / (t_ms / 1e3) / 1e9) if alg else None
    label = {"k_clean_units": "clean replay stage (k_clean_rounds + k_clean_units + perVertex fold)"}
    roofline = {"kernel": label.get(dominant, dominant), "bound": "hbm", "achieved": achieved, "peak": peak,
                "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                "traffic_source": traffic_source,
                "algorithmic_bytes": alg, "ms_per_launch": t_ms, "peak_kind": peak_kind}
    t_count = avg["k_edge_fold"] + avg["k_tri_fill"] + avg["k_vertex_fold"]
    roofline_count = {"kernels": "k_edge_fold+k_tri_fill+k_vertex_fold", "bound": "hbm",
                      "achieved": b_count / (t_count / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                      "frac": b_count / (t_count / 1e3) / 1e9 / peak, "algorithmic_bytes": b_count,
                      "oriented_sum": orient_sum, "ms": t_count}

    # end to end through the C ABI with host buffers
    e2e = None
    if not args.skip_e2e:
        hu = torch.from_numpy(u).pin_memory().numpy()
        hv = torch.from_numpy(v).pin_memory().numpy()
        times = []
        for k in range(args.warmup + args.steps):
            flush_l2(k)
            t0 = time.perf_counter()
            g2 = rtr.Graph.from_edges(n, hu, hv, device=dev)
            g2.decompose(args.eps)
            cof = g2.cluster_of()
            g2.close()
            t1 = time.perf_counter()
            if k >= args.warmup:
                times.append(t1 - t0)
        sec = allmax(float(np.mean(times)))
        e2e = {"value": world * m / sec, "unit": UNIT, "h2d_bytes_per_step": 16 * m,
               "d2h_bytes_per_step": int(cof.nbytes), "ms_per_step": sec * 1e3}

    cpu = None
    if rank == 0 and world == 1 and not args.skip_cpu:
        times, kind = cpu_times(n, u, v, 2, "s", 1)
        sec = float(np.mean(times))
        cpu = {"value": m / sec, "unit": UNIT, "cores": 1, "kind": kind,
               "sample": "full decomposition of the workload graph (2 runs, mode s)" if kind == "reference"
               else "full decomposition with the restated oracle (2 runs)",
               "seconds_per_run": sec}

    g.close()
    t_count_stage = float(np.mean(count_ms)) / 1e3
    extras = {}
    if rank == 0 and world == 1 and not args.skip_extras:
        for key, fn in (("config3_rmat24_count",
                         lambda: rmat24_leg(args, dev, flush_l2, peak, peak_kind, steps=1, e2e_runs=1)),
                        ("batched", lambda: batched_leg(args, dev)),
                        ("served", lambda: served_leg(args, dev)),
                        ("gpu_baseline", lambda: gpu_baseline_leg(dev))):
            try:
                extras[key] = fn()
            except Exception as e:  # a leg that cannot run is reported, not fatal
                extras[key] = {"unavailable": f"{type(e).__name__}: {e}"[:300]}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "desc": WORKLOAD_DESC, "n": n, "m": m, "eps": args.eps,
                       "clusters": ncl, "l2": "flushed (256 MiB write) before every step",
                       "parallelism": f"replicas x{world}"},
            "e2e": e2e, "roofline": roofline, "roofline_count": roofline_count, "cpu_baseline": cpu,
            "gpu_launches": launches, "kernel_ms": avg, "wall_s_timed": wall,
            "triangles": total, "triangles_per_s": total / t_count_stage, "count_stage_ms": t_count_stage * 1e3,
            "clocks": clocks.summary(),
        }
        line.update(extras)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def batch_arm(args):
    """Batched form: K independent SBM graphs (edge targets log-uniform in
    [1K, 200K], seeds 4000+i) decomposed by one rtr_decompose on their disjoint
    union, against one plain decomposition per graph on the same GPU.  Both legs
    go through the C ABI from host arrays (H2D + CSR build + decomposition +
    cluster counts read back); graphs/s is the headline."""
    import torch
    import rtrex_cuda_b200 as rtr
    from rtrex_cuda_b200 import graphgen
    world, rank, dev = dist_init()
    allmax = lambda x: replica_max(x, world, torch.device("cuda", dev))
    t0 = time.perf_counter()
    all_graphs = graphgen.sbm_batch(args.batch_graphs)
    gen_s = time.perf_counter() - t0
    K = len(all_graphs)
    edges = int(sum(g[1].size for g in all_graphs))
    graphs = shard(all_graphs, rank, world)  # independent graphs: every rank its own share
    # the counting work split is chosen by the autotuner on the first batch
    # (untimed) and reused for every later batch
    with rtr.Graph.batch(graphs, device=dev) as g:
        tuning = g.autotune()
    # batched leg
    times, dev_ms = [], []
    for k in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        with rtr.Graph.batch(graphs, device=dev) as g:
            g.set_tuning(*tuning)
            g.decompose(args.eps)
            counts = g.batch_cluster_counts()
            dev_ms.append(g.kernel_ms()["decompose"])
        t1 = time.perf_counter()
        if k >= args.warmup:
            times.append(t1 - t0)
    batched_s = allmax(float(np.mean(times)))
    dev_s = allmax(float(np.mean(dev_ms[args.warmup:])) / 1e3)
    # plain leg: one graph at a time, one pass (warmed by the batched leg)
    t0 = time.perf_counter()
    plain_counts = []
    for (n, u, v) in graphs:
        with rtr.Graph.from_edges(n, u, v, device=dev) as g1:
            plain_counts.append(g1.decompose(args.eps))
    plain_s = allmax(time.perf_counter() - t0)
    same = bool(all(gather_values([bool((np.asarray(plain_counts) == counts).all())], world)))
    if rank != 0:
        return
    line = {
        "metric": "batched graphs/s (count+clean+extract)", "value": K / dev_s, "unit": "graphs/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_s * 1e3,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "sbm_batch", "graphs": K, "edges": edges, "eps": args.eps,
                   "parallelism": f"graphs sharded over {world} GPU(s), every {world}th graph per rank",
                   "desc": "SBM graphs, 4-64 blocks, intra mean degree 12, inter 2, edge targets log-uniform "
                           "in [1K, 200K], seeds 4000+i; disjoint union decomposed in one call",
                   "autotune": {"gallop_ratio": tuning[0], "heavy_degree": tuning[1], "heavy_edge": tuning[2]}},
        "e2e": {"value": K / batched_s, "unit": "graphs/s", "h2d_bytes_per_step": 16 * edges,
                "d2h_bytes_per_step": 8 * K},
        "plain_per_graph": {"value": K / plain_s, "unit": "graphs/s", "seconds": plain_s},
        "batched_vs_plain": (K / batched_s) / (K / plain_s),
        "per_graph_cluster_counts_equal": same, "generation_s": gen_s,
    }
    print(json.dumps(line), flush=True)


def serve_arm(args):
    """Served form: a Poisson stream of decomposition requests over a pool of
    resident graphs (G(n,p)+cliques and R-MAT shapes, edge targets log-uniform
    in [1K, --serve-max-edges]) through the request server (continuous
    admission, per-graph streams, small-graph batching, HBM budget), against the
    plain form on the same request list: one graph at a time, built from host
    arrays and decomposed, no overlap.  Every served result is compared with the
    plain one (clusters, triangle counts, cluster of every vertex)."""
    world, rank, dev = dist_init()
    line = serve_run(args, world, rank, dev)
    if rank == 0:
        print(json.dumps(line), flush=True)


def served_leg(args, dev):
    """A short served run for the default line (one GPU): 80 requests at 2,000/s
    over 16 resident graphs of 1K-200K edges, against the plain form."""
    import copy
    a = copy.copy(args)
    a.serve_requests, a.serve_pool, a.serve_max_edges = 80, 16, 2e5
    line = serve_run(a, 1, 0, dev)
    keep = ("p50_ms", "p99_ms", "service_p50_ms", "service_p99_ms", "throughput_req_s", "plain",
            "served_vs_plain_throughput", "results_differing_from_plain")
    out = {k: line[k] for k in keep}
    out["config"] = {k: line["config"][k] for k in ("requests", "arrival_rate_per_s", "pool_graphs", "edge_range")}
    return out


def serve_run(args, world, rank, dev):
    """The served and plain legs of serve_arm; the result line on rank 0 (None elsewhere)."""
    import hashlib
    import torch
    import rtrex_cuda_b200 as rtr
    from rtrex_cuda_b200 import graphgen
    allmax = lambda x: replica_max(x, world, torch.device("cuda", dev))
    t0 = time.perf_counter()
    pool = graphgen.served_pool(args.serve_pool, m_hi=args.serve_max_edges)
    gen_s = time.perf_counter() - t0
    rng = np.random.default_rng(6000)
    N = args.serve_requests
    all_graph = rng.integers(0, len(pool), size=N)
    all_arrivals = np.cumsum(rng.exponential(1.0 / args.serve_rate, size=N))
    # independent requests: rank r serves every world-th request of the stream,
    # at that request's own arrival time
    mine = shard(range(N), rank, world)
    req_graph = all_graph[mine]
    arrivals = all_arrivals[mine]
    eps = args.eps
    digest = lambda a: hashlib.sha256(np.ascontiguousarray(a, np.int64).tobytes()).hexdigest()
    # plain leg (also the reference results): each request alone, in order
    for (n, u, v) in pool[:2]:  # warm the library
        with rtr.Graph.from_edges(n, u, v, device=dev) as g:
            g.decompose(eps)
    plain = {}
    plain_lat = []
    t0 = time.perf_counter()
    for gid in req_graph.tolist():
        n, u, v = pool[gid]
        t1 = time.perf_counter()
        with rtr.Graph.from_edges(n, u, v, device=dev) as g:
            tri = g.count()
            left = g.clean(eps)
            k = g.extract()
            cof = g.cluster_of()
        plain_lat.append(time.perf_counter() - t1)
        plain.setdefault(gid, (tri, left, k, digest(cof)))
    plain_s = allmax(time.perf_counter() - t0)
    # served leg
    with rtr.Server(device=dev, hbm_budget=int(args.serve_budget_gb * (1 << 30)), workers=args.serve_workers,
                    batch_max_edges=20000, batch_max_graphs=64) as srv:
        for (n, u, v) in pool:
            srv.add_graph(n, u, v)
        rids = []
        start = time.perf_counter()
        for i, gid in enumerate(req_graph.tolist()):
            delay = start + arrivals[i] - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            rids.append(srv.submit(gid, eps))
        res = [srv.wait(r) for r in rids]
        st = srv.stats()
    # every rank's latencies pooled; the job's span is the slowest rank's
    lat = np.array(gather_values([r["t_end_ms"] - r["t_submit_ms"] for r in res], world))
    service = np.array(gather_values([r["t_end_ms"] - r["t_start_ms"] for r in res], world))
    span_ms = allmax(max(r["t_end_ms"] for r in res) - min(r["t_submit_ms"] for r in res) if res else 0.0)
    plain_lat = gather_values(plain_lat, world)
    bad = sum(gather_values([sum(1 for r, gid in zip(res, req_graph.tolist())
                                 if r["status"] != 0 or (r["triangles"], r["triangles_left"], r["n_clusters"],
                                                         digest(r["cluster_of"])) != plain[gid])], world))
    every_st = gather_values([st], world)
    st = {k: sum(d[k] for d in every_st) for k in st}
    edges = int(sum(pool[g][1].size for g in all_graph.tolist()))
    if rank != 0:
        return None
    line = {
        "metric": "served p99 latency (ms)", "value": float(np.percentile(lat, 99)), "unit": "ms",
        "n_gpus": world, "steps": N, "warmup": 2, "ms_per_step": float(span_ms / N), "higher_is_better": False,
        "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "served", "requests": N, "arrival_rate_per_s": args.serve_rate,
                   "parallelism": f"requests sharded over {world} GPU(s), every {world}th request per rank",
                   "pool_graphs": len(pool), "edge_range": [1000, args.serve_max_edges], "eps": eps,
                   "workers": args.serve_workers, "hbm_budget_gb": args.serve_budget_gb,
                   "batch_max_edges": 20000, "batch_max_graphs": 64,
                   "desc": "Poisson arrivals over a pool alternating G(n,p)+planted cliques and R-MAT graphs, "
                           "edge targets log-uniform, seeds 5000+i"},
        "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
        "service_p50_ms": float(np.percentile(service, 50)), "service_p99_ms": float(np.percentile(service, 99)),
        "throughput_req_s": N / (span_ms / 1e3), "throughput_edges_s": edges / (span_ms / 1e3),
        "plain": {"req_s": N / plain_s, "edges_s": edges / plain_s, "p50_ms": 1e3 * float(np.percentile(plain_lat, 50)),
                  "p99_ms": 1e3 * float(np.percentile(plain_lat, 99)), "seconds": plain_s},
        "served_vs_plain_throughput": (N / (span_ms / 1e3)) / (N / plain_s),
        "results_differing_from_plain": bad, "server_stats": st, "generation_s": gen_s,
        "edges_requested": edges,
    }
    return line


def main():
    args = parse_args()
    if args.workload in ("batch", "serve"):
        (batch_arm if args.workload == "batch" else serve_arm)(args)
        import torch.distributed as dist
        if dist.is_available() and dist.is_initialized():
            dist.destroy_process_group()
        return
    if args.workload == "bundled":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the bundled workload reports the reference's "
                              "phase timers beside the device times in its own line"}), flush=True)
            return
        bundled_arm(args)
        return
    if args.workload == "rmat_count":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no counting-only entry point; "
                              "its commonNbr at this scale runs for hours on the host"}), flush=True)
            return
        rmat_count_arm(args)
        return
    if args.impl == "reference":
        reference_arm(args)
    else:
        ours_arm(args)


if __name__ == "__main__":
    main()
