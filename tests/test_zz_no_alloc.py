"""rtr_count_noalloc: weighted triangle counting for callers that cannot let
the library allocate device memory (they own every buffer, e.g. a server that
pre-reserves its HBM and hands out memory only from its own arena).

The test owns all device buffers (torch tensors), calls the entry point through
the C ABI, and checks its outputs bit for bit against the allocating path
(rtr_count + rtr_get_weights) on consecutive calls with different graphs, so
stale contents of the shared static scratch cannot leak between calls.  The
file is named to be collected last.
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


@pytest.mark.parametrize("sequence", [("gnp_cliques", "sbm_3000_4002", "gnp_cliques")])
def test_noalloc_matches_allocating_path_on_consecutive_calls(sequence):
    for name in sequence:
        n, u, v = helpers.case_graph(name)
        off, nb, pe, pv, sup, total = _reference_outputs(n, u, v)
        got_pe, got_pv, got_sup, got_total = _call_noalloc(off, nb, n)
        assert got_total == total, name
        assert (helpers.bits(got_pe) == helpers.bits(pe)).all(), name
        assert (helpers.bits(got_pv) == helpers.bits(pv)).all(), name
        assert (got_sup == sup).all(), name


def test_noalloc_rejects_graphs_beyond_its_fixed_scratch():
    import torch
    dummy = torch.zeros(4, dtype=torch.int64, device="cuda")
    p = dummy.data_ptr()
    rc = _entry()(p, p, (1 << 20) + 1, p, p, p, p, None)
    assert rc == 4
    assert b"exceeds the fixed scratch limit" in rtr.lib().rtr_last_error()
