"""cds_count_cliques_noalloc: the allocation-free k-clique count.

Code running under a framework or memory manager that owns all of the
device's memory cannot call cudaMalloc in the middle of its work (the
allocation would fail, or take memory promised elsewhere); this entry point
counts k-cliques (and clique degrees) of a graph the caller already holds in
device memory, writing into device buffers the caller owns and keeping its
scratch in one static device array.  Its answers must equal
cds_list_cliques' (exact integers) on every graph, also on the second of two
calls in a row, since the shared scratch array keeps the previous call's
contents.

Inputs the entry point must refuse are fed only where every read stays
inside the buffers the test allocates: the adjacency buffer is padded past
the arc count the offsets claim.

The file name makes pytest collect it last, so a run that stops at the
first failure has run every other test before this one.
"""
import numpy as np
import pytest

import cds_b200 as cds
from conftest import GOLDEN, golden_cases

pytestmark = pytest.mark.gpu

MAX_N = 1 << 18


PAD = 256  # adjacency entries past d_off[n] in every device copy


def noalloc_count(torch, off, adj, k, with_degree=True):
    """Device copies of the CSR, one call, results back on the host."""
    n = len(off) - 1
    d_off = torch.from_numpy(np.ascontiguousarray(off, np.uint64).view(np.int64)).cuda()
    a = np.concatenate([np.ascontiguousarray(adj, np.uint32), np.zeros(PAD, np.uint32)]).view(np.int32)
    d_adj = torch.from_numpy(a).cuda()
    d_count = torch.full((1,), -1, dtype=torch.int64, device="cuda")
    d_deg = torch.full((max(n, 1),), 12345, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    st = cds.lib().cds_count_cliques_noalloc(d_off.data_ptr(), d_adj.data_ptr(), n, k,
                                             d_count.data_ptr(),
                                             d_deg.data_ptr() if with_degree else None, None)
    torch.cuda.synchronize()
    deg = d_deg[:n].cpu().numpy().view(np.uint32).astype(np.uint64)
    return st, int(d_count.item()), deg


def graphs():
    out = []
    for case in golden_cases():
        if case["k"] == 2 and case["name"] in ("ref_test", "cfg1", "small_rmat0", "small_k5_k7",
                                               "small_path", "k10_bridge"):
            out.append((case["name"], cds.read_adjlist(f"{GOLDEN}/{case['graph']}")))
    out.append(("rmat14", cds.gen_rmat(14, 8.0, 1)))
    out.append(("er_dense", cds.gen_er(600, 0.6, 9)))  # DAG rows > 128: block teams
    return out


@pytest.mark.parametrize("name,csr", graphs(), ids=[g[0] for g in graphs()])
def test_matches_list_cliques_on_two_calls(ctx, name, csr):
    torch = pytest.importorskip("torch")
    off, adj = csr
    g = ctx.graph(off, adj)
    try:
        for k in (2, 3, 4, 5):
            want_cnt, want_deg = ctx.list_cliques(g, k)
            for _ in range(2):
                st, cnt, deg = noalloc_count(torch, off, adj, k)
                assert st == 0
                assert cnt == want_cnt
                assert np.array_equal(deg, want_deg.astype(np.uint64))
            # without a clique-degree buffer the degrees go to the scratch
            # array's own slice; the count is the same
            st, cnt, _ = noalloc_count(torch, off, adj, k, with_degree=False)
            assert st == 0 and cnt == want_cnt
    finally:
        g.free()


def test_rejects_what_does_not_fit():
    torch = pytest.importorskip("torch")
    # more vertices than the static scratch holds: refused before any work
    big = np.zeros(MAX_N + 2, np.uint64)
    st, _, _ = noalloc_count(torch, big, np.zeros(0, np.uint32), 3)
    assert st == 4
    # not a symmetric CSR: the device check refuses it
    st, _, _ = noalloc_count(torch, np.array([0, 1, 1], np.uint64), np.array([1], np.uint32), 3)
    assert st == 4
    # an adjacency id equal to n (row 0 of a 3-vertex graph points at 3)
    off = np.array([0, 2, 3, 4], np.uint64)
    st, _, _ = noalloc_count(torch, off, np.array([1, 3, 0, 0], np.uint32), 3)
    assert st == 4
    # offsets that decrease (row 1 would run backwards) and one that does not
    # start at zero
    st, _, _ = noalloc_count(torch, np.array([0, 2, 1, 2], np.uint64), np.array([1, 2], np.uint32), 3)
    assert st == 4
    st, _, _ = noalloc_count(torch, np.array([1, 2, 2], np.uint64), np.array([1, 0], np.uint32), 3)
    assert st == 4
    # unsorted row and a self-loop
    st, _, _ = noalloc_count(torch, np.array([0, 2, 3, 4], np.uint64), np.array([2, 1, 0, 0], np.uint32), 3)
    assert st == 4
    st, _, _ = noalloc_count(torch, np.array([0, 1, 1], np.uint64), np.array([0], np.uint32), 3)
    assert st == 4
    # k out of range
    off, adj = cds.gen_er(30, 0.3, 1)
    st, _, _ = noalloc_count(torch, off, adj, 17)
    assert st == 4
    # and the entry point still answers correctly afterwards
    st, cnt, _ = noalloc_count(torch, off, adj, 3)
    assert st == 0
    import oracle
    assert cnt == oracle.count_cliques(off, adj, 3)[0]
