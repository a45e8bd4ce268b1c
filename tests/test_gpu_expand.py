"""expandClusters (the RTRex driver's mode e) on the device, through the C ABI:
clusters (same count and order), recomputed statistics, member iteration order
after the moves, the scores, and the five RTRex-expanded-* files, against the
reference's own digests.  Thresholds >= 1 take the parallel path, thresholds
<= 0 the replay in which singleton clusters can absorb singletons."""
import hashlib
import os

import numpy as np
import pytest

import rtrex_cuda_b200 as rtr
from rtrex_cuda_b200 import graphgen
from tests import helpers

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,eps,thr", helpers.expand_cases())
def test_expand_matches_reference(name, eps, thr):
    n, u, v = helpers.case_graph(name)
    with rtr.Graph.from_edges(n, u, v) as g:
        g.decompose(eps)
        moved = g.expand(thr)
        cl, cof = g.expanded()
        sv, sx = g.scores()
    assert moved == len(sv)
    got = helpers.expand_digests(cl, sv, sx)
    want = helpers.expected(name, eps)["expand"][str(thr)]
    assert got == {k: x for k, x in want.items() if k != "files"}
    # cluster_of agrees with the member lists
    for k in range(len(cl)):
        assert (cof[cl.members(k)] == k).all()
    assert (cof >= 0).sum() == cl.off[-1]


@pytest.mark.parametrize("name,eps,thr", helpers.expand_cases(["small_test", "two_k5_bridge", "sbm_3000_4002",
                                                               "gnp_cliques", "chung_lu"]))
def test_expand_output_files_byte_identical(name, eps, thr, tmp_path):
    n, u, v = helpers.case_graph(name)
    path = str(tmp_path / "g.txt")
    graphgen.write_escape(path, n, u, v)
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        rtr.run_file(path, "g", eps, prefix="RTRex-", rtrex_outputs=True, expand=thr)
    finally:
        os.chdir(cwd)
    want = helpers.expected(name, eps)["expand"][str(thr)]["files"]
    for kind in ("decomposition", "stats", "freq", "cut", "scores"):
        got = hashlib.sha256(open(tmp_path / f"RTRex-expanded-g-{kind}.txt", "rb").read()).hexdigest()
        assert got == want[kind], kind
    # the plain outputs are unchanged by the expansion
    base = helpers.expected(name, eps)["files"]
    for kind in ("decomposition", "stats", "freq", "cut"):
        got = hashlib.sha256(open(tmp_path / f"RTRex-g-{kind}.txt", "rb").read()).hexdigest()
        assert got == base[kind], kind


def test_expand_repeatable_and_after_reextract():
    """Expanding twice at different thresholds reads the same extraction."""
    n, u, v = helpers.case_graph("sbm_3000_4002")
    with rtr.Graph.from_edges(n, u, v) as g:
        g.decompose(0.1)
        a = helpers.expand_digests(*_drop_cof(g, 2))
        b = helpers.expand_digests(*_drop_cof(g, 1))
        c = helpers.expand_digests(*_drop_cof(g, 2))
        g.decompose(0.1)
        d = helpers.expand_digests(*_drop_cof(g, 1))
    assert a == c and b == d
    want = helpers.expected("sbm_3000_4002", 0.1)["expand"]
    assert a["digest"] == want["2"]["digest"] and b["digest"] == want["1"]["digest"]


def _drop_cof(g, thr):
    g.expand(thr)
    cl, _ = g.expanded()
    sv, sx = g.scores()
    return cl, sv, sx


def test_expand_stage_order():
    with rtr.Graph.from_edges(4, np.array([0, 1, 2]), np.array([1, 2, 0])) as g:
        g.count()
        with pytest.raises(rtr.RtrError) as e:
            g.expand(1)
        assert e.value.code == 5
        g.clean(0.3)
        g.extract()
        g.expand(1)
        g.count()  # a new count invalidates the expansion
        with pytest.raises(rtr.RtrError):
            g.expanded()


def test_expand_rejects_batch():
    gs = [helpers.case_graph("small_test"), helpers.case_graph("k4")]
    with rtr.Graph.batch(gs) as g:
        g.decompose(0.3)
        with pytest.raises(rtr.RtrError) as e:
            g.expand(1)
        assert e.value.code == 1
