"""The C-ABI library without a GPU: it loads, exports every symbol rtr.h
declares, parses Escape files with the reference loader's rules, and fails
loudly (no CPU fallback) when no CUDA device is present."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

import rtrex_cuda_b200 as rtr
from tests import helpers


def _declared_functions():
    text = open(os.path.join(helpers.ROOT, "include", "rtr.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(rtr_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    names = _declared_functions()
    assert len(names) >= 18
    L = rtr.lib()
    for nm in names:
        assert hasattr(L, nm), f"librtr.so does not export {nm}"
    out = subprocess.run(["nm", "-D", "--defined-only", rtr.lib_path()], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (rtr_[a-z0-9_]+)", out))
    assert set(names) <= exported


def test_version():
    assert b"sm_100a" in rtr.lib().rtr_version()


def _write(tmp_path, text):
    p = tmp_path / "g.txt"
    p.write_text(text)
    return str(p)


def test_escape_parser_rules(tmp_path):
    # comments and blank lines are skipped; the first data line is "n m"
    p = _write(tmp_path, "# header comment\n\n4 3\n0 1\n# mid comment\n1 2\n   \n2 3\n")
    n, u, v = rtr.load_escape(p)
    assert n == 4 and u.tolist() == [0, 1, 2] and v.tolist() == [1, 2, 3]


def test_escape_parser_short_file(tmp_path):
    # fewer edges than declared -> the reference's ecIOError (GraphIO.cpp:67-71)
    p = _write(tmp_path, "5 4\n0 1\n1 2\n")
    with pytest.raises(rtr.RtrError) as e:
        rtr.load_escape(p)
    assert e.value.code == 7 and "expected 8 edges, only got 4" in str(e.value)


def test_escape_parser_missing_file(tmp_path):
    with pytest.raises(rtr.RtrError) as e:
        rtr.load_escape(str(tmp_path / "nope.txt"))
    assert e.value.code == 7


def test_escape_parser_malformed(tmp_path):
    p = _write(tmp_path, "3 2\n0 1\nx y\n")
    with pytest.raises(rtr.RtrError):
        rtr.load_escape(p)


def test_escape_parser_matches_graphgen_writer(tmp_path):
    from rtrex_cuda_b200 import graphgen
    n, u, v = graphgen.sbm(2000, 4001)
    p = str(tmp_path / "s.txt")
    graphgen.write_escape(p, n, u, v)
    n2, u2, v2 = rtr.load_escape(p)
    assert n2 == n and (u2 == u).all() and (v2 == v).all()


def test_no_cpu_fallback_without_gpu():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(rtr.RtrError) as e:
        rtr.Graph.from_edges(3, np.array([0, 1]), np.array([1, 2]))
    assert e.value.code == 2 and "no CUDA device" in str(e.value)


def test_null_arguments_rejected():
    L = rtr.lib()
    assert L.rtr_count(None, None) == 1
    assert L.rtr_graph_destroy(None) == 0
    h = ctypes.c_void_p()
    assert L.rtr_graph_create_from_edges(None, None, 5, 3, 0, 0, ctypes.byref(h)) == 1


def test_expand_entry_points_reject_null_graph():
    L = rtr.lib()
    n = ctypes.c_int64()
    assert L.rtr_expand(None, 1, ctypes.byref(n)) == 1
    assert L.rtr_get_expanded(None, None, None, None, None, None, None) == 5
    assert L.rtr_get_scores(None, ctypes.byref(n), None, None) == 5
    assert L.rtr_write_expanded(None, b"x") == 1


def test_escape_device_entry_points_argument_errors(tmp_path):
    L = rtr.lib()
    h = ctypes.c_void_p()
    assert L.rtr_graph_create_from_escape_text(None, 5, 0, 0, ctypes.byref(h)) == 1
    assert L.rtr_graph_create_from_escape_text(b"1 0\n", -1, 0, 0, ctypes.byref(h)) == 1
    assert L.rtr_graph_create_from_escape_file(None, 0, 0, ctypes.byref(h)) == 1
    missing = str(tmp_path / "missing.txt").encode()
    assert L.rtr_graph_create_from_escape_file(missing, 0, 0, ctypes.byref(h)) == 7
    assert b"could not open file" in L.rtr_last_error()


def test_server_entry_points_without_gpu():
    L = rtr.lib()
    h = ctypes.c_void_p()
    assert L.rtr_server_create(0, 1 << 30, 0, 0, 1, ctypes.byref(h)) == 1  # no workers
    assert L.rtr_server_create(0, 0, 2, 0, 1, ctypes.byref(h)) == 1        # no budget
    assert L.rtr_server_destroy(None) == 0
    assert L.rtr_server_wait(None, 1, None) == 1
    if not torch_cuda_available():
        assert L.rtr_server_create(0, 1 << 30, 2, 0, 1, ctypes.byref(h)) == 2
        assert b"no CUDA device" in L.rtr_last_error()


def torch_cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def test_tuning_entry_points_argument_errors():
    L = rtr.lib()
    a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    assert L.rtr_set_tuning(None, 16, 32, 1024) == 1
    assert L.rtr_get_tuning(None, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)) == 1
    assert L.rtr_autotune(None, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)) == 1


def test_clean_split_entry_points_argument_errors():
    L = rtr.lib()
    k, x = ctypes.c_int64(), ctypes.c_double()
    assert L.rtr_set_clean_split(None, 2048, 8.0) == 1
    assert L.rtr_get_clean_split(None, ctypes.byref(k), ctypes.byref(x)) == 1


def test_count_layout_entry_points_argument_errors():
    L = rtr.lib()
    a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    w, e = ctypes.c_int64(), ctypes.c_int64()
    assert L.rtr_set_count_mode(None, 2, 1024) == 1
    assert L.rtr_get_count_mode(None, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)) == 1
    assert L.rtr_set_count_window(None, 1000) == 1
    assert L.rtr_get_count_windows(None, ctypes.byref(w), ctypes.byref(e)) == 1
