"""The clean's device-side self-checks report, and the device stays usable.

The warp-per-unit replay (rtrex_cuda_b200/csrc/clean.cu) bounds every wait on
its asynchronous window copies and every cascade stack; when a bound is hit
the warp sets a bit of the graph's device error word and stops, and rtr_clean
turns the word into RTR_ERR_DEVICE.  rtr_set_clean_checks lowers the bounds so
that they are hit on ordinary input -- nothing is made to fault or hang: the
first wait is cut to one try (the copies themselves complete, and are drained
under the full bound before the warp stops), and the stack regions to zero
entries (a unit that needs to spill reports instead).  Each test then checks
the error, destroys the graph, and decomposes a fresh graph bit for bit.
"""
import pytest

import rtrex_cuda_b200 as rtr
from tests import helpers

pytestmark = pytest.mark.gpu


def _fresh_decomposition_still_exact():
    name, eps = "small_test", 0.3
    n, u, v = helpers.case_graph(name)
    (_, _, _), c, s0, s1, cl, s2 = helpers.oracle_run(name, eps)
    with rtr.Graph.from_edges(n, u, v) as g:
        assert g.count() == s0.total
        assert g.clean(eps) == s1.total
        assert (g.status() == s1.status).all()
        assert g.extract() == len(cl)
        got = g.clusters()
        assert (got.vert == cl.vert).all() and (got.off == cl.off).all()


@pytest.mark.parametrize("name,eps", [("gnp_cliques", 0.3), ("sbm_20000_4000", 0.1)])
def test_first_wait_running_out_is_reported(name, eps):
    n, u, v = helpers.case_graph(name)
    g = rtr.Graph.from_edges(n, u, v)
    g.set_clean_split(1 << 62, 0.0)  # every unit through the warp-per-unit replay
    g.set_clean_checks(first_wait_rounds=1)
    g.count()
    with pytest.raises(rtr.RtrError) as ei:
        g.clean(eps)
    assert ei.value.code == 6
    assert "a bounded wait on an asynchronous copy ran out" in str(ei.value)
    g.close()
    _fresh_decomposition_still_exact()


@pytest.mark.parametrize("name,eps", [("rmat12", 0.3), ("rmat14", 0.1)])
def test_stack_overflow_is_reported(name, eps):
    n, u, v = helpers.case_graph(name)
    g = rtr.Graph.from_edges(n, u, v)
    g.set_clean_split(1 << 62, 0.0)
    g.set_clean_checks(stack_entries=0)
    g.count()
    with pytest.raises(rtr.RtrError) as ei:
        g.clean(eps)
    assert ei.value.code == 6
    assert "cascade stack overflowed" in str(ei.value)
    g.close()
    _fresh_decomposition_still_exact()


def test_checks_at_their_defaults_leave_results_exact():
    name, eps = "rmat12", 0.3
    n, u, v = helpers.case_graph(name)
    (_, _, _), c, s0, s1, _, _ = helpers.oracle_run(name, eps)
    with rtr.Graph.from_edges(n, u, v) as g:
        g.set_clean_split(1 << 62, 0.0)
        g.set_clean_checks(1, 0)
        g.set_clean_checks(0, -1)  # back to the full bounds
        g.count()
        assert g.clean(eps) == s1.total
        assert (g.status() == s1.status).all()
