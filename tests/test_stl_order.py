"""The device restatements of std::sort's permutation and std::unordered_set's
iteration order (rtrex_cuda_b200/csrc/stl_order.cuh) match the host C++
library they restate, on tie-heavy, adversarial and random inputs (CPU only)."""
import os
import subprocess
import tempfile

from tests import helpers


def test_stl_order_restatement_matches_libstdcxx():
    src = os.path.join(helpers.ROOT, "tests", "stl_order_check.cpp")
    with tempfile.TemporaryDirectory() as td:
        exe = os.path.join(td, "chk")
        subprocess.run(["g++", "-std=c++17", "-O2", "-o", exe, src], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.startswith("OK"), out.stdout
