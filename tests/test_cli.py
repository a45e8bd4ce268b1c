"""The drop-in command line, rtrex_b200 (rtrex_cuda_b200/csrc/cli.cpp), run as a
process: the argument surface of RTRex_CUDA (RTRex_CUDA/main.cu:343-391) --
<graph_file> <output_name> <eps> [gpu_device] -- with its default
"RTRex-CUDA-" output prefix and exit code 1 when the graph cannot be loaded
(main.cu:362-365), plus the RTRex driver's outputs (--prefix RTRex-) and mode e
(--expand T).  Output files are compared with the digests of the files the
reference CLI wrote on the same graphs (tests/golden/golden.json).
"""
import hashlib
import os
import subprocess

import pytest

from rtrex_cuda_b200 import graphgen
from tests import helpers

CLI = os.path.join(helpers.ROOT, "rtrex_cuda_b200", "rtrex_b200")

pytestmark = pytest.mark.skipif(not os.path.exists(CLI), reason="rtrex_b200 is not built")


def _run(args, cwd):
    return subprocess.run([CLI, *args], cwd=cwd, capture_output=True, text=True, timeout=300)


def _sha(path):
    with open(path, "rb") as f:
        return hashlib.sha256(f.read()).hexdigest()


def test_usage_exits_1(tmp_path):
    r = _run(["only_a_graph.txt", "name"], tmp_path)
    assert r.returncode == 1
    assert "Usage" in r.stdout


def test_missing_graph_exits_1(tmp_path):
    r = _run([str(tmp_path / "no_such_graph.txt"), "g", "0.3"], tmp_path)
    assert r.returncode == 1
    assert "could not open file" in r.stderr
    assert not list(tmp_path.glob("RTRex-CUDA-*"))


@pytest.mark.gpu
@pytest.mark.parametrize("name,eps", [("small_test", 0.3), ("gnp_cliques", 0.1), ("two_k5_bridge", 0.3)])
def test_default_prefix_and_device_argument(name, eps, tmp_path):
    n, u, v = helpers.case_graph(name)
    path = str(tmp_path / "g.txt")
    graphgen.write_escape(path, n, u, v)
    r = _run([path, "g", repr(eps), "0"], tmp_path)
    assert r.returncode == 0, r.stderr
    assert "[Main] Done." in r.stdout
    want = helpers.expected(name, eps)["files"]
    for kind in ("decomposition", "stats", "freq", "cut"):
        assert _sha(tmp_path / f"RTRex-CUDA-g-{kind}.txt") == want[kind], kind


@pytest.mark.gpu
def test_rtrex_prefix_and_expand(tmp_path):
    name, eps, t = "small_test", 0.3, 1
    n, u, v = helpers.case_graph(name)
    path = str(tmp_path / "g.txt")
    graphgen.write_escape(path, n, u, v)
    r = _run([path, "g", repr(eps), "--prefix", "RTRex-", "--expand", str(t)], tmp_path)
    assert r.returncode == 0, r.stderr
    want = helpers.expected(name, eps)
    for kind in ("decomposition", "stats", "freq", "cut"):
        assert _sha(tmp_path / f"RTRex-g-{kind}.txt") == want["files"][kind], kind
        assert _sha(tmp_path / f"connected-components-g-{kind}.txt") == want["files"]["cc_" + kind], kind
    assert _sha(tmp_path / "amazon_cleaned_edges.txt") == want["files"]["cleaned_edges"]
    for kind in ("decomposition", "stats", "freq", "cut", "scores"):
        assert _sha(tmp_path / f"RTRex-expanded-g-{kind}.txt") == want["expand"][str(t)]["files"][kind], kind


@pytest.mark.gpu
def test_device_out_of_range_exits_1(tmp_path):
    n, u, v = helpers.case_graph("small_test")
    path = str(tmp_path / "g.txt")
    graphgen.write_escape(path, n, u, v)
    r = _run([path, "g", "0.3", "97"], tmp_path)
    assert r.returncode == 1
    assert "out of range" in r.stderr
