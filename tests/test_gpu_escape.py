"""Escape text parsed on the device (rtr_graph_create_from_escape_text / _file):
the CSR equals the one built from the host loader's edge arrays, and every
malformed input fails with the host loader's status and message."""
import os

import numpy as np
import pytest

import rtrex_cuda_b200 as rtr
from rtrex_cuda_b200 import graphgen
from tests import helpers

pytestmark = pytest.mark.gpu


def _host_csr(path):
    n, u, v = rtr.load_escape(path)
    with rtr.Graph.from_edges(n, u, v) as g:
        return g.csr()


def _escape_bytes(n, u, v):
    body = "".join(f"{a} {b}\n" for a, b in zip(u.tolist(), v.tolist()))
    return f"{n} {len(u)}\n{body}".encode()


@pytest.mark.parametrize("name", ["small_test", "k20", "isolated", "gnp_cliques", "sbm_3000_4002", "chung_lu"])
def test_device_parse_equals_host_loader(name, tmp_path):
    n, u, v = helpers.case_graph(name)
    path = str(tmp_path / "g.txt")
    graphgen.write_escape(path, n, u, v)
    want = _host_csr(path)
    with rtr.Graph.from_escape_file(path) as g:
        assert (g.n, g.m) == (n, len(u))
        off, nb = g.csr()
    assert (off == want[0]).all() and (nb == want[1]).all()
    with rtr.Graph.from_escape_text(open(path, "rb").read()) as g:
        off2, nb2 = g.csr()
    assert (off2 == off).all() and (nb2 == nb).all()


def test_device_parse_format_variants(tmp_path):
    """Comments, blank and whitespace-only lines, CRLF, tabs, signs, extra
    columns, lines past the m-th pair, no final newline."""
    n, u, v = helpers.case_graph("sbm_3000_4002")
    rng = np.random.default_rng(3)
    lines = ["# a comment line", "", "   \t", f"  {n}\t{len(u)}  trailing words"]
    for a, b in zip(u.tolist(), v.tolist()):
        r = rng.integers(0, 8)
        if r == 0:
            lines.append("#" + "x" * int(rng.integers(0, 3000)))
        if r == 1:
            lines.append(" \r")
        sep = [" ", "\t", "  ", " \t "][int(rng.integers(0, 4))]
        tail = ["", " 17", "\r", " extra", "\t1.5"][int(rng.integers(0, 5))]
        pre = ["", " ", "+"][int(rng.integers(0, 3))]
        lines.append(f"{pre}{a}{sep}{b}{tail}")
    lines += ["1 2", "this line is past the edges and ignored? no: it is a data line after m"]
    text_bad = ("\n".join(lines)).encode()
    # the last line is malformed data: both loaders reject it at the same line
    path = str(tmp_path / "bad.txt")
    open(path, "wb").write(text_bad)
    with pytest.raises(rtr.RtrError) as host:
        rtr.load_escape(path)
    with pytest.raises(rtr.RtrError) as dev:
        rtr.Graph.from_escape_file(path)
    assert host.value.code == dev.value.code == 7
    assert str(host.value) == str(dev.value)
    # without it: extra well-formed lines past m are ignored, no final newline
    text = ("\n".join(lines[:-1])).encode()
    path = str(tmp_path / "ok.txt")
    open(path, "wb").write(text)
    want = _host_csr(path)
    with rtr.Graph.from_escape_text(text) as g:
        off, nb = g.csr()
    assert (off == want[0]).all() and (nb == want[1]).all()
    c = helpers.oracle_run("sbm_3000_4002", 0.1)[1]
    assert (off == c.offsets).all() and (nb == c.nbors).all()


@pytest.mark.parametrize("text", [
    b"",                               # no header
    b"# only a comment\n\n",           # no header
    b"x 3\n0 1\n",                     # malformed header
    b"4\n0 1\n",                       # header with one value
    b"-4 2\n0 1\n1 2\n",               # negative header
    b"4 3\n0 1\n1 2\n",                # short edge count
    b"4 3\n0 1\n1 z\n2 3\n",           # malformed data line
    b"4 2\n0 1\n\n# c\n1 2\n3\n",      # malformed line after the m-th edge
    b"4 0\n",                          # zero edges: valid
    b"4 1\n0 1",                       # no final newline: valid
])
def test_device_parse_errors_match_host(text, tmp_path):
    path = str(tmp_path / "g.txt")
    open(path, "wb").write(text)
    host_err = dev_err = None
    try:
        rtr.load_escape(path)
    except rtr.RtrError as e:
        host_err = (e.code, str(e))
    try:
        rtr.Graph.from_escape_file(path).close()
    except rtr.RtrError as e:
        dev_err = (e.code, str(e))
    assert host_err == dev_err


def test_device_parse_chunked_large_file(tmp_path):
    """A file larger than the direct-copy size goes through the pinned chunk ring."""
    n, u, v = graphgen.rmat(scale=18, edge_factor=16, seed=18)
    path = str(tmp_path / "big.txt")
    graphgen.write_escape(path, n, u, v)
    assert os.path.getsize(path) > 40 << 20
    want = _host_csr(path)
    with rtr.Graph.from_escape_file(path) as g:
        off, nb = g.csr()
    assert (off == want[0]).all() and (nb == want[1]).all()


def test_run_file_uses_device_parse(tmp_path):
    """The drop-in driver (device parse) still writes the reference's files."""
    import hashlib
    n, u, v = helpers.case_graph("gnp_cliques")
    path = str(tmp_path / "g.txt")
    graphgen.write_escape(path, n, u, v)
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        rtr.run_file(path, "g", 0.3, prefix="RTRex-")
    finally:
        os.chdir(cwd)
    want = helpers.expected("gnp_cliques", 0.3)["files"]
    for kind in ("decomposition", "stats", "freq", "cut"):
        assert hashlib.sha256(open(tmp_path / f"RTRex-g-{kind}.txt", "rb").read()).hexdigest() == want[kind]
