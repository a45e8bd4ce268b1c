"""rtr_count_noalloc: weighted triangle counting for callers that cannot let
the library allocate device memory (they own every buffer, e.g. a server that
pre-reserves its HBM and hands out memory only from its own arena).

The test owns all device buffers (torch tensors), calls the entry point through
the C ABI, and checks its outputs bit for bit against the allocating path
(rtr_count + rtr_get_weights) and against the reference's own commonNbr
digests (tests/golden/golden.json) on consecutive calls with different graphs,
so stale contents of the shared static scratch cannot leak between calls; a
power-law graph sends its hubs through the warp-per-vertex kernel.  The file is
named to be collected last.
"""
import ctypes

import numpy as np
import pytest

import rtrex_cuda_b200 as rtr
from tests import helpers

pytestmark = pytest.mark.gpu


def _entry():
    f = rtr.lib().rtr_count_noalloc
    f.argtypes = [ctypes.c_void_p] * 2 + [ctypes.c_int64] + [ctypes.c_void_p] * 5
    f.restype = ctypes.c_int
    return f


def _reference_outputs(n, u, v):
    with rtr.Graph.from_edges(n, u, v) as g:
        off, nb = g.csr()
        g.count()
        pe, pv, sup, total = g.weights()
    return off, nb, pe, pv, sup, total


def _call_noalloc(off, nb, n):
    import torch
    dev = torch.device("cuda", 0)
    m2 = int(nb.size)
    d_off = torch.from_numpy(np.ascontiguousarray(off, np.int64)).to(dev)
    d_nb = torch.from_numpy(np.ascontiguousarray(nb, np.int32)).to(dev)
    d_pe = torch.full((max(1, m2),), float("nan"), dtype=torch.float64, device=dev)
    d_pv = torch.full((max(1, n),), float("nan"), dtype=torch.float64, device=dev)
    d_sup = torch.full((max(1, m2),), -1, dtype=torch.int32, device=dev)
    d_tot = torch.full((1,), -1, dtype=torch.int64, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    rc = _entry()(d_off.data_ptr(), d_nb.data_ptr(), n, d_pe.data_ptr(), d_pv.data_ptr(), d_sup.data_ptr(),
                  d_tot.data_ptr(), stream)
    assert rc == 0, rtr.lib().rtr_last_error()
    torch.cuda.synchronize(dev)
    return (d_pe.cpu().numpy()[:m2], d_pv.cpu().numpy()[:n], d_sup.cpu().numpy().view(np.uint32)[:m2],
            int(d_tot.cpu().item()))


def _golden_count(name):
    """The reference's own commonNbr digests for the case (any threshold entry)."""
    entry = helpers.golden()["cases"][name]
    return next(iter(entry.values()))["count"]


@pytest.mark.parametrize("sequence", [("gnp_cliques", "chung_lu", "sbm_3000_4002", "gnp_cliques")])
def test_noalloc_matches_allocating_path_on_consecutive_calls(sequence):
    for name in sequence:
        n, u, v = helpers.case_graph(name)
        off, nb, pe, pv, sup, total = _reference_outputs(n, u, v)
        got_pe, got_pv, got_sup, got_total = _call_noalloc(off, nb, n)
        assert got_total == total, name
        assert (helpers.bits(got_pe) == helpers.bits(pe)).all(), name
        assert (helpers.bits(got_pv) == helpers.bits(pv)).all(), name
        assert (got_sup == sup).all(), name
        # and directly against the reference's digests (chung_lu's hubs go to the warp kernel)
        gold = _golden_count(name)
        assert got_total == gold["total"], name
        assert helpers.sha(helpers.bits(got_pe).tobytes()) == gold["perEdge"], name
        assert helpers.sha(helpers.bits(got_pv).tobytes()) == gold["perVertex"], name


def test_noalloc_rejects_graphs_beyond_its_fixed_scratch():
    import torch
    dummy = torch.zeros(4, dtype=torch.int64, device="cuda")
    p = dummy.data_ptr()
    rc = _entry()(p, p, (1 << 20) + 1, p, p, p, p, None)
    assert rc == 4
    assert b"exceeds the fixed scratch limit" in rtr.lib().rtr_last_error()


def test_noalloc_rejects_null_buffers():
    import torch
    dummy = torch.zeros(4, dtype=torch.int64, device="cuda")
    p = dummy.data_ptr()
    for k in (1, 3, 5):  # d_nbors, d_perEdge, d_support
        args = [p, p, 3, p, p, p, p, None]
        args[k] = None
        assert _entry()(*args) == 1
        assert b"null buffer" in rtr.lib().rtr_last_error()


def test_noalloc_reports_out_of_range_neighbours():
    # a triangle 0-1-2 whose row 2 also names vertex 7 of a 3-vertex graph: the
    # id is skipped (never dereferenced) and the total comes back as -1
    off = np.array([0, 2, 4, 7], np.int64)
    nb = np.array([1, 2, 0, 2, 0, 1, 7], np.int32)
    _, _, _, total = _call_noalloc(off, nb, 3)
    assert total == -1
    off = np.array([0, 2, 4, 6], np.int64)
    nb = np.array([1, 2, 0, 2, 0, 1], np.int32)
    _, _, sup, total = _call_noalloc(off, nb, 3)
    assert total == 1 and (sup == 1).all()  # the error word does not outlive its call
