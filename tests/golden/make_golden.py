"""Regenerate tests/golden/golden.json from the reference itself.

Runs the reference's own sequential code (oracle/_ref/rtr_ref_dump, compiled
from RTRex_Sequential's sources by ``make -C oracle ref``) on every fixture
graph and records, per stage, the reference's results:

* count:   total triangles, sha256 of perEdge bits and of perVertex bits
* clean:   triangles left, sha256 of the status bytes, perEdge bits, perVertex bits
* extract: number of clusters and sha256 of the cluster list (creation order,
           "nv ne cut : members" in set-iteration order, one line per cluster)
* files:   sha256 of RTRex-<name>-{decomposition,stats,freq,cut}.txt, of
           connected-components-<name>-*.txt (cc_*) and of amazon_cleaned_edges.txt
           written by the reference CLI (oracle/_ref/RTRex <graph> <name> <eps> s)
* expand:  per threshold of cases.EXPAND, expandClusters' clusters (same line
           format as extract), its scores ("<v> <score %a>" lines) and the five
           RTRex-expanded-<name>-* files of ``RTRex <graph> <name> <eps> e <t>``

small_test (the reference's RTRex_Sequential/Example/small-test.txt graph)
additionally stores full arrays in small_test.npz.  Graph inputs are either
regenerated from seeds (rtrex_cuda_b200.graphgen) or, for the bundled data
files, the committed copies under tests/golden/data/ (``--copy-bundled``
refreshes those copies, byte for byte, from the reference checkout first).

* nonsimple: the four files of ``RTRex <graph> g 0.3 s`` on a file with a repeated
           and a reversed line, and on the same edges with the repeats dropped
* nucleus: sha256 of the cluster file of the reference's ``nucleus <graph> <out>``
           (clustering/nucleus.cpp) on every fixture graph

Usage: python tests/golden/make_golden.py [--reference DIR] [--copy-bundled] [--expand-only] [--nonsimple-only] [--nucleus-only]
(DIR defaults to $RTR_REFERENCE_DIR, else /root/reference; --expand-only
recomputes only the expand entries of an existing golden.json)
"""
from __future__ import annotations

import argparse
import gzip
import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from rtrex_cuda_b200 import graphgen  # noqa: E402
from tests.golden.cases import CASES, BUNDLED, EXPAND, bundled_path, load_case  # noqa: E402


def sha(b: bytes) -> str:
    return hashlib.sha256(b).hexdigest()


def cluster_text_from_lines(lines):
    return ("\n".join(lines) + "\n").encode()


def run_reference(dump_bin: str, path: str, eps: float):
    with tempfile.TemporaryDirectory() as td:
        subprocess.run([dump_bin, path, repr(eps), td], check=True, stdout=subprocess.DEVNULL,
                       stderr=subprocess.DEVNULL)
        rd = lambda f, dt: np.fromfile(os.path.join(td, f), dtype=dt)
        out = {
            "count": {
                "total": int(rd("count_total.i64", np.int64)[0]),
                "perEdge": sha(rd("count_perEdge.f64", np.uint64).tobytes()),
                "perVertex": sha(rd("count_perVertex.f64", np.uint64).tobytes()),
            },
            "clean": {
                "total": int(rd("clean_total.i64", np.int64)[0]),
                "status": sha(rd("clean_status.u8", np.uint8).tobytes()),
                "perEdge": sha(rd("clean_perEdge.f64", np.uint64).tobytes()),
                "perVertex": sha(rd("clean_perVertex.f64", np.uint64).tobytes()),
            },
        }
        lines = open(os.path.join(td, "clusters.txt")).read().splitlines()
        out["extract"] = {"clusters": len(lines), "digest": sha(cluster_text_from_lines(lines))}
        arrays = {k: rd(f, dt) for k, f, dt in [
            ("offsets", "csr_offsets.i64", np.int64), ("nbors", "csr_nbors.i64", np.int64),
            ("count_perEdge", "count_perEdge.f64", np.float64), ("count_perVertex", "count_perVertex.f64", np.float64),
            ("clean_status", "clean_status.u8", np.uint8), ("clean_perEdge", "clean_perEdge.f64", np.float64),
            ("clean_perVertex", "clean_perVertex.f64", np.float64)]}
        arrays["clusters"] = np.array(lines)
        return out, arrays


def run_reference_cli(cli_bin: str, path: str, eps: float):
    """sha256 of the four files RTRex <graph> <name> <eps> s writes (RTRex.cpp:194)."""
    with tempfile.TemporaryDirectory() as td:
        subprocess.run([cli_bin, path, "g", repr(eps), "s"], check=True, cwd=td, stdout=subprocess.DEVNULL,
                       stderr=subprocess.DEVNULL)
        out = {kind: sha(open(os.path.join(td, f"RTRex-g-{kind}.txt"), "rb").read())
               for kind in ("decomposition", "stats", "freq", "cut")}
        for kind in ("decomposition", "stats", "freq", "cut"):
            out["cc_" + kind] = sha(open(os.path.join(td, f"connected-components-g-{kind}.txt"), "rb").read())
        out["cleaned_edges"] = sha(open(os.path.join(td, "amazon_cleaned_edges.txt"), "rb").read())
        return out


def run_reference_expand(dump_bin: str, cli_bin: str, path: str, eps: float, thresholds):
    out = {}
    with tempfile.TemporaryDirectory() as td:
        subprocess.run([dump_bin, path, repr(eps), td] + [str(t) for t in thresholds], check=True,
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        for t in thresholds:
            lines = open(os.path.join(td, f"expanded_{t}.txt")).read().splitlines()
            sc = open(os.path.join(td, f"scores_{t}.txt"), "rb").read()
            out[str(t)] = {"clusters": len(lines), "digest": sha(cluster_text_from_lines(lines)),
                           "scores": sha(sc), "nscores": sc.count(b"\n")}
    for t in thresholds:
        with tempfile.TemporaryDirectory() as td:
            subprocess.run([cli_bin, path, "g", repr(eps), "e", str(t)], check=True, cwd=td,
                           stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
            out[str(t)]["files"] = {kind: sha(open(os.path.join(td, f"RTRex-expanded-g-{kind}.txt"), "rb").read())
                                    for kind in ("decomposition", "stats", "freq", "cut", "scores")}
    return out


def bundled_text(name, td):
    """Decompress the committed copy of a bundled file to td (the reference reads plain text)."""
    path = os.path.join(td, os.path.basename(BUNDLED[name]))
    with gzip.open(bundled_path(name), "rb") as f, open(path, "wb") as g:
        g.write(f.read())
    return path


def copy_bundled(reference):
    """Refresh tests/golden/data/ from the reference's own data files (gzip -9, no name/time stamp)."""
    os.makedirs(os.path.dirname(bundled_path(next(iter(BUNDLED)))), exist_ok=True)
    for name, rel in BUNDLED.items():
        with open(os.path.join(reference, rel), "rb") as f:
            data = f.read()
        with open(bundled_path(name), "wb") as raw:
            with gzip.GzipFile(filename="", mode="wb", compresslevel=9, fileobj=raw, mtime=0) as g:
                g.write(data)
        print("copied", rel, len(data), "bytes")


def case_path(name, td, reference):
    if name in BUNDLED:
        return bundled_text(name, td)
    n, u, v = load_case(name)
    path = os.path.join(td, name + ".txt")
    graphgen.write_escape(path, n, u, v)
    return path


def add_expand(golden, dump_bin, cli_bin, reference):
    with tempfile.TemporaryDirectory() as td:
        for (name, eps), thresholds in EXPAND.items():
            entry = golden["cases"].get(name, {}).get(repr(eps))
            path = case_path(name, td, reference)
            if entry is None or path is None:
                print("skip expand", name, eps)
                continue
            entry["expand"] = run_reference_expand(dump_bin, cli_bin, path, eps, thresholds)
            print("expand", name, eps, {t: e["nscores"] for t, e in entry["expand"].items()}, flush=True)


# A file with a repeated line ("2 3" twice) and a reversed repeat ("1 0" after
# "0 1"): loadGraph_Escape stores every line in both directions
# (RTRex_Sequential/GraphIO.cpp:42-63) and makeCSR keeps repeated pairs
# (Graph.cpp:344-384), so the reference decomposes a multigraph CSR.
NONSIMPLE_TEXT = "5 8\n0 1\n1 2\n0 2\n2 3\n3 4\n2 4\n1 0\n2 3\n"


def add_nonsimple(golden, cli_bin):
    """The reference CLI's four files on NONSIMPLE_TEXT and on the same edge set
    with the repeats dropped (what --simplify decomposes)."""
    out = {"text": NONSIMPLE_TEXT, "eps": 0.3}
    lines = NONSIMPLE_TEXT.strip().split("\n")
    n = int(lines[0].split()[0])
    pairs = sorted({tuple(sorted(map(int, ln.split()))) for ln in lines[1:]})
    simple = f"{n} {len(pairs)}\n" + "".join(f"{a} {b}\n" for a, b in pairs)
    for key, text in (("files", NONSIMPLE_TEXT), ("simplified_files", simple)):
        with tempfile.TemporaryDirectory() as td:
            path = os.path.join(td, "g.txt")
            with open(path, "w") as f:
                f.write(text)
            subprocess.run([cli_bin, path, "g", "0.3", "s"], check=True, cwd=td, stdout=subprocess.DEVNULL,
                           stderr=subprocess.DEVNULL)
            out[key] = {kind: sha(open(os.path.join(td, f"RTRex-g-{kind}.txt"), "rb").read())
                        for kind in ("decomposition", "stats", "freq", "cut")}
            if key == "files":
                out["decomposition_text"] = open(os.path.join(td, "RTRex-g-decomposition.txt")).read()
    golden["nonsimple"] = out


def add_nucleus(golden, nucleus_bin):
    """The reference nucleus driver (clustering/nucleus.cpp) on every fixture
    graph: sha256 and line count of the cluster file it writes."""
    out = {}
    with tempfile.TemporaryDirectory() as td:
        for name in CASES:
            path = case_path(name, td, None)
            res = os.path.join(td, name + ".nuclei")
            subprocess.run([nucleus_bin, path, res], check=True, stdout=subprocess.DEVNULL,
                           stderr=subprocess.DEVNULL, timeout=600)
            data = open(res, "rb").read()
            out[name] = {"sha": sha(data), "clusters": data.count(b"Cluster id:")}
            print("nucleus", name, out[name]["clusters"], flush=True)
    golden["nucleus"] = out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("RTR_REFERENCE_DIR", "/root/reference"))
    ap.add_argument("--copy-bundled", action="store_true")
    ap.add_argument("--expand-only", action="store_true")
    ap.add_argument("--nonsimple-only", action="store_true")
    ap.add_argument("--nucleus-only", action="store_true")
    args = ap.parse_args()
    if args.copy_bundled:
        copy_bundled(args.reference)
    dump_bin = os.path.join(ROOT, "oracle", "_ref", "rtr_ref_dump")
    cli_bin = os.path.join(ROOT, "oracle", "_ref", "RTRex")
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref", f"REF={args.reference}"], check=True)
    nucleus_bin = os.path.join(ROOT, "oracle", "_ref", "nucleus")
    if args.nucleus_only:
        with open(os.path.join(HERE, "golden.json")) as f:
            golden = json.load(f)
        add_nucleus(golden, nucleus_bin)
        with open(os.path.join(HERE, "golden.json"), "w") as f:
            json.dump(golden, f, indent=1, sort_keys=True)
        return
    if args.nonsimple_only:
        with open(os.path.join(HERE, "golden.json")) as f:
            golden = json.load(f)
        add_nonsimple(golden, cli_bin)
        with open(os.path.join(HERE, "golden.json"), "w") as f:
            json.dump(golden, f, indent=1, sort_keys=True)
        return
    if args.expand_only:
        with open(os.path.join(HERE, "golden.json")) as f:
            golden = json.load(f)
        add_expand(golden, dump_bin, cli_bin, args.reference)
        with open(os.path.join(HERE, "golden.json"), "w") as f:
            json.dump(golden, f, indent=1, sort_keys=True)
        return
    golden = {"eps": {}, "cases": {}}
    with tempfile.TemporaryDirectory() as td:
        for name, eps_list in CASES.items():
            if name in BUNDLED:
                path = bundled_text(name, td)
            else:
                n, u, v = load_case(name)
                path = os.path.join(td, name + ".txt")
                graphgen.write_escape(path, n, u, v)
            entry = {}
            for eps in eps_list:
                res, arrays = run_reference(dump_bin, path, eps)
                res["files"] = run_reference_cli(os.path.join(ROOT, "oracle", "_ref", "RTRex"), path, eps)
                entry[repr(eps)] = res
                if name == "small_test" and eps == 0.3:
                    np.savez_compressed(os.path.join(HERE, "small_test.npz"), **arrays)
                print(name, eps, res["count"]["total"], res["clean"]["total"], res["extract"]["clusters"], flush=True)
            golden["cases"][name] = entry
    add_expand(golden, dump_bin, cli_bin, args.reference)
    add_nonsimple(golden, cli_bin)
    add_nucleus(golden, nucleus_bin)
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(golden, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
