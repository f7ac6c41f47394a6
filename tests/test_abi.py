"""CPU-side checks of the C ABI library: it loads without a GPU, exports every
function include/*.h declares, and its host helpers (generators, adjacency-list
I/O) behave as documented."""
import os
import re
import subprocess

import numpy as np
import pytest

import cds_b200 as cds
from conftest import ROOT


def declared_functions():
    names = set()
    for h in ("cds.h", "cds_gen.h"):
        with open(os.path.join(ROOT, "include", h)) as f:
            src = f.read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"\b(cds_[a-z0-9_]+)\s*\(", src):
            names.add(m.group(1))
    return sorted(names)


def test_library_loads_and_exports_every_declared_symbol():
    L = cds.lib()
    out = subprocess.run(["nm", "-D", "--defined-only", cds.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, missing
    for n in declared_functions():
        assert hasattr(L, n)
    # the Python binding covers the whole ABI
    assert set(declared_functions()) <= set(cds.exported_symbols())


def test_version_and_status_strings():
    assert b"sm_100a" in cds.lib().cds_version()
    assert cds.lib().cds_status_string(0) == b"ok"
    assert cds.lib().cds_status_string(3) == b"device iteration budget exhausted"


def test_generators_are_deterministic_and_canonical():
    a = cds.gen_rmat(10, 8.0, 5)
    b = cds.gen_rmat(10, 8.0, 5)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    c = cds.gen_rmat(10, 8.0, 6)
    assert not np.array_equal(a[1], c[1])
    for off, adj in (a, cds.gen_er(500, 0.02, 1)):
        n = len(off) - 1
        src = np.repeat(np.arange(n), np.diff(off).astype(np.int64))
        assert np.all(src != adj)  # no self-loops
        for v in range(n):  # rows strictly ascending
            row = adj[off[v]:off[v + 1]]
            assert np.all(np.diff(row.astype(np.int64)) > 0)
        fwd = set(zip(src.tolist(), adj.tolist()))
        assert all((w, u) in fwd for u, w in fwd)  # symmetric


def test_rmat_size_matches_edge_factor():
    off, adj = cds.gen_rmat(14, 8.0, 1)
    m = len(adj) // 2
    assert len(off) - 1 == 16384
    assert 100_000 < m < 131_072


def test_planted_community_is_dense():
    off, adj = cds.gen_er(2000, 0.004, 0)
    o2, a2, members = cds.gen_plant(off, adj, 40, 0.6, 0)
    assert len(set(members.tolist())) == 40
    S = set(members.tolist())
    inside = sum(1 for v in S for w in a2[o2[v]:o2[v + 1]] if int(w) in S) // 2
    assert 0.45 * 780 < inside < 0.75 * 780


def test_adjlist_round_trip(tmp_path):
    off, adj = cds.gen_er(300, 0.03, 3)
    p = str(tmp_path / "g.txt")
    cds.write_adjlist(p, off, adj)
    o2, a2 = cds.read_adjlist(p)
    assert np.array_equal(off, o2) and np.array_equal(adj, a2)
    with open(p) as f:
        head = f.readline().split()
    assert int(head[0]) == 300 and int(head[1]) == len(adj) // 2


def test_reader_accepts_unordered_duplicate_and_one_sided_lines(tmp_path):
    p = tmp_path / "g.txt"
    # lines out of order, a missing vertex line, a self-loop, a duplicate and
    # an edge listed on one side only
    p.write_text("5 4\n3 1 2\n1 3 3 1\n0 1\n2 3\n")
    off, adj = cds.read_adjlist(str(p))
    rows = [adj[off[v]:off[v + 1]].tolist() for v in range(5)]
    assert rows == [[1], [0, 3], [3], [1, 2], []]


def test_reader_rejects_bad_input(tmp_path):
    p = tmp_path / "g.txt"
    p.write_text("3 1\n0 7\n")
    with pytest.raises(cds.CdsError):
        cds.read_adjlist(str(p))
    with pytest.raises(cds.CdsError):
        cds.read_adjlist(str(tmp_path / "missing.txt"))


def test_create_rejects_too_many_streams_before_touching_a_device():
    """The stream count is checked before any CUDA call, so this runs
    without a GPU."""
    with pytest.raises(cds.CdsError) as e:
        cds.Context(0, streams=65)
    assert e.value.status == 4  # CDS_ERR_INPUT


def test_binary_csr_cache_round_trip(tmp_path):
    """cds_write_csr_binary writes a 32-byte header and the arrays; the host
    reader recognises the file by its magic and returns the same CSR."""
    off, adj = cds.gen_rmat(11, 8.0, 9)
    p = str(tmp_path / "g.csrbin")
    cds.write_csr_binary(p, off, adj)
    raw = open(p, "rb").read()
    assert raw[:8] == b"CDSCSR\x01\n" and len(raw) == 32 + 8 * len(off) + 4 * len(adj)
    n, nnz = np.frombuffer(raw[16:32], np.uint64)
    assert (n, nnz) == (len(off) - 1, len(adj))
    o2, a2 = cds.read_adjlist(p)
    assert np.array_equal(o2, off) and np.array_equal(a2, adj)
    with open(p, "wb") as f:
        f.write(raw[:-4])
    with pytest.raises(cds.CdsError):
        cds.read_adjlist(p)
