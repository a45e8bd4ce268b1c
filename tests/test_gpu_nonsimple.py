"""Input with repeated or reversed lines: where this library and the reference
part ways, pinned.

The reference stores every Escape line in both directions with no
deduplication (RTRex_Sequential/GraphIO.cpp:42-63) and makeCSR keeps repeated
pairs (Graph.cpp:344-384), so a file that lists "u v" twice, or "u v" and
"v u", is decomposed as a multigraph: degrees count the repeats, commonNbr
meets a triangle once per copy of its edges, and the output changes (on the
5-vertex file below the reference returns the clusters {2,3,4} and {0,1}; on
the same edges listed once, all singletons).  This library accepts simple
graphs only: by default such input is rejected with RTR_ERR_INPUT, and with
the simplify flag the repeats are dropped first -- which equals the
reference run on the deduplicated file, not on the original one.  The golden
digests come from the reference built from its sources
(tests/golden/make_golden.py, add_nonsimple).
"""
import hashlib
import os

import pytest

import rtrex_cuda_b200 as rtr
from tests import helpers

pytestmark = pytest.mark.gpu


def _files(tmp_path, prefix="RTRex-"):
    return {kind: hashlib.sha256(open(tmp_path / f"{prefix}g-{kind}.txt", "rb").read()).hexdigest()
            for kind in ("decomposition", "stats", "freq", "cut")}


def test_repeated_and_reversed_lines_are_rejected_by_default():
    gold = helpers.golden()["nonsimple"]
    with pytest.raises(rtr.RtrError) as ei:
        rtr.Graph.from_escape_text(gold["text"].encode())
    assert ei.value.code == 3
    assert "not a simple graph" in str(ei.value) and "duplicate" in str(ei.value)


def test_simplify_equals_the_reference_on_the_deduplicated_file(tmp_path):
    gold = helpers.golden()["nonsimple"]
    path = tmp_path / "g.txt"
    path.write_text(gold["text"])
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        rtr.run_file(str(path), "g", gold["eps"], prefix="RTRex-", simplify=True)
    finally:
        os.chdir(cwd)
    got = _files(tmp_path)
    assert got == gold["simplified_files"]
    # the reference's own output on the file as written differs: that is the divergence
    assert gold["files"] != gold["simplified_files"]
    assert got["decomposition"] != gold["files"]["decomposition"]
