"""Batched solves and the request server give every instance the answer it
gets alone (which the parity tests tie to the oracle), whatever the mix of
sizes and k in the batch, and in whatever order requests arrive."""
import hashlib
import json
import os
import threading
import time

import numpy as np
import pytest

import cds_b200 as cds
import oracle
from cds_b200 import workloads
from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def mixed_instances(count, seed):
    """Small instances of uneven size: ER and R-MAT with planted
    communities, k in {2, 3, 4}."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(np.exp(rng.uniform(np.log(60), np.log(3000))))
        if i % 2 == 0:
            off, adj = cds.gen_er(n, float(rng.uniform(4, 16)) / max(n - 1, 1), seed * 1000 + i)
        else:
            scale = int(np.ceil(np.log2(max(n, 2))))
            off, adj = cds.gen_rmat(scale, float(rng.uniform(2, 8)), seed * 1000 + i, n=n)
        size = int(rng.integers(6, min(40, n)))
        off, adj, _ = cds.gen_plant(off, adj, size, 0.5, seed * 1000 + i + 7)
        out.append((off, adj, int(rng.integers(2, 5))))
    return out


def key(sol):
    return (sol.num, sol.den, sol.vertices.tolist(), sol.total_cliques, sol.max_core,
            sol.core_threshold, sol.core_density, sol.core_size)


@pytest.fixture(scope="module")
def instances():
    return mixed_instances(24, 5)


def test_batch_equals_single_solves(ctx, instances):
    gs = [ctx.graph(o, a) for o, a, _ in instances]
    try:
        single = [key(ctx.solve(g, k)) for g, (_, _, k) in zip(gs, instances)]
        jobs = [(g, cds.make_params(k)) for g, (_, _, k) in zip(gs, instances)]
        batch = [key(s) for s in ctx.solve_batch(jobs)]
        assert batch == single
        # and a second batch in another order
        order = list(reversed(range(len(jobs))))
        again = ctx.solve_batch([jobs[i] for i in order])
        assert [key(s) for s in again] == [single[i] for i in order]
    finally:
        for g in gs:
            g.free()


def test_batch_against_oracle(ctx, instances):
    picks = instances[:8]
    gs = [ctx.graph(o, a) for o, a, _ in picks]
    try:
        sols = ctx.solve_batch([(g, cds.make_params(k)) for g, (_, _, k) in zip(gs, picks)])
        for s, (o, a, k) in zip(sols, picks):
            ora = oracle.solve(o, a, k)
            assert (s.num, s.den) == (ora["num"], ora["den"])
            assert s.vertices.tolist() == ora["vertices"].tolist()
    finally:
        for g in gs:
            g.free()


def _digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _matches(sol, want):
    if (sol.total_cliques, sol.num, sol.den, len(sol.vertices)) != (
            want["total_cliques"], want["num"], want["den"], want["size"]):
        return False
    if "vertices" in want:
        return sol.vertices.tolist() == want["vertices"]
    return _digest(sol.vertices.astype("<u4")) == want["vertices_sha256"]


def test_batch_mix_sample_against_oracle(ctx):
    """A seeded 32-instance sub-sample of the 256-instance batched
    configuration (tests/golden/make_batch_sample.py), solved in one batched
    call and one instance per call: both equal the oracle's committed
    answers (count, exact density, vertex set)."""
    with open(os.path.join(GOLDEN, "batch_mix_sample.json")) as f:
        fx = json.load(f)["instances"]
    idx = [r["index"] for r in fx]
    inst = workloads.batch_mix(256, 2, only=set(idx))
    for (o, a, k), r in zip(inst, fx):
        assert k == r["k"] and len(o) - 1 == r["n"]
        assert _digest(o.astype("<u8")) == r["off_sha256"] and _digest(a.astype("<u4")) == r["adj_sha256"]
    gs = [ctx.graph(o, a) for o, a, _ in inst]
    try:
        batch = ctx.solve_batch([(g, cds.make_params(k)) for g, (_, _, k) in zip(gs, inst)])
        bad = [r["index"] for s, r in zip(batch, fx) if not _matches(s, r)]
        assert not bad, f"batched answers differ from the oracle's on instances {bad}"
        plain = [ctx.solve(g, k) for g, (_, _, k) in zip(gs, inst)]
        bad = [r["index"] for s, r in zip(plain, fx) if not _matches(s, r)]
        assert not bad, f"plain answers differ from the oracle's on instances {bad}"
    finally:
        for g in gs:
            g.free()


def test_server_alone_and_in_the_mix(ctx, instances):
    gs = [ctx.graph(o, a) for o, a, _ in instances]
    try:
        single = [key(ctx.solve(g, k)) for g, (_, _, k) in zip(gs, instances)]
        srv = ctx.server(max_batch=8, max_inflight=3)
        try:
            # one at a time
            for i in (0, 5, 11):
                t = srv.submit(gs[i], cds.make_params(instances[i][2]))
                assert key(srv.wait(t)) == single[i]
            # everything at once, from two threads, polled out of order
            tickets = {}

            def submit(idx):
                for i in idx:
                    tickets[i] = srv.submit(gs[i], cds.make_params(instances[i][2]))
                    time.sleep(0.001)

            th = [threading.Thread(target=submit, args=(range(j, len(gs), 2),)) for j in (0, 1)]
            for t in th:
                t.start()
            for t in th:
                t.join()
            got = {}
            deadline = time.time() + 120
            while len(got) < len(gs) and time.time() < deadline:
                for i in reversed(range(len(gs))):
                    if i in got:
                        continue
                    s = srv.poll(tickets[i])
                    if s is not None:
                        got[i] = key(s)
                time.sleep(0.002)
            assert len(got) == len(gs)
            assert [got[i] for i in range(len(gs))] == single
            # a ticket is answered once
            with pytest.raises(cds.CdsError) as e:
                srv.poll(tickets[0])
            assert e.value.status == 6
        finally:
            srv.stop()
    finally:
        for g in gs:
            g.free()


def test_autotune_writes_and_reuses_its_cache(ctx, tmp_path):
    off, adj = cds.gen_rmat(11, 8.0, 3)
    g = ctx.graph(off, adj)
    try:
        path = str(tmp_path / "tune.txt")
        ctx.autotune([g], 3, path)
        lines = open(path).read().split("\n")
        for key in ("flow_rounds", "list_warp_dmax", "peel_chunk", "peel_order"):
            assert any(l.startswith(f"3 {key} ") for l in lines), key
        t0 = time.time()
        ctx.autotune([g], 3, path)  # read back, no timing
        assert time.time() - t0 < 1.0
        s = ctx.solve(g, 3)
        ora = oracle.solve(off, adj, 3)
        assert (s.num, s.den) == (ora["num"], ora["den"])
    finally:
        g.free()


@pytest.mark.parametrize("k", [3, 4])
def test_loaded_tuning_keeps_answers(k, tmp_path):
    """Non-default shapes from a cache file (small warp teams, short peel
    items, few rounds between global relabels, a balancing warm start before
    each max-flow, the other peel item order) give the same exact answers."""
    path = str(tmp_path / "tune.txt")
    with open(path, "w") as f:
        f.write(f"{k} list_warp_dmax 32\n{k} peel_chunk 128\n{k} flow_rounds 4\n{k} list_warp_block 128\n"
                f"{k} flow_warm 16\n{k} peel_order {0 if k <= 3 else 1}\n")
    off, adj = cds.gen_rmat(12, 8.0, 5)
    with cds.Context(0) as c:
        c.autotune([], k, path)
        g = c.graph(off, adj)
        s = c.solve(g, k)
        g.free()
    ora = oracle.solve(off, adj, k)
    assert (s.num, s.den) == (ora["num"], ora["den"])
    assert s.vertices.tolist() == ora["vertices"].tolist()


@pytest.mark.parametrize("warm", [1, 2, 5])
@pytest.mark.parametrize("k", [2, 3, 4, 5])
@pytest.mark.parametrize("wide", [False, True])
def test_warm_split_keeps_answers(warm, k, wide, tmp_path):
    """The balanced split of each clique's units before a max-flow (one
    split from clique degrees, or after weight updates), on 32-bit flow state
    in the clique records and on the separate 64-bit flow array, on a graph
    and on a batch of several networks: the same exact answers and sets."""
    path = str(tmp_path / "tune.txt")
    with open(path, "w") as f:
        f.write(f"{k} flow_warm {warm}\n")
    graphs = [cds.gen_rmat(12, 8.0, 5), cds.gen_er(3000, 0.004, 3)]
    graphs.append(cds.gen_plant(*graphs[1], 40, 0.6, 3)[:2])
    with cds.Context(0, flags=cds.CONFIG_WIDE_FLOW if wide else 0) as c:
        c.autotune([], k, path)
        gs = [c.graph(off, adj) for off, adj in graphs]
        try:
            sols = [c.solve(g, k) for g in gs]
            batch = c.solve_batch([(g, cds.make_params(k)) for g in gs])
        finally:
            for g in gs:
                g.free()
    for (off, adj), sol, bsol in zip(graphs, sols, batch):
        ora = oracle.solve(off, adj, k)
        assert (sol.num, sol.den) == (ora["num"], ora["den"])
        assert sol.vertices.tolist() == ora["vertices"].tolist()
        assert (bsol.num, bsol.den) == (ora["num"], ora["den"])
        assert bsol.vertices.tolist() == ora["vertices"].tolist()


@pytest.mark.parametrize("n,deg,k", [(6000, 30.0, 2), (3000, 60.0, 3)])
def test_warm_split_large_networks(n, deg, k, tmp_path):
    """The split on networks of thousands of vertices, past the 4,096 whose
    loads are summed per block in shared memory where the core is that
    large: the same exact answers as the oracle."""
    path = str(tmp_path / "tune.txt")
    with open(path, "w") as f:
        f.write(f"{k} flow_warm 3\n")
    off, adj = cds.gen_er(n, deg / (n - 1), 12)
    with cds.Context(0) as c:
        c.autotune([], k, path)
        g = c.graph(off, adj)
        try:
            sol = c.solve(g, k)
        finally:
            g.free()
    ora = oracle.solve(off, adj, k)
    assert (sol.num, sol.den) == (ora["num"], ora["den"])
    assert sol.vertices.tolist() == ora["vertices"].tolist()
    assert sol.core_size > 1024


def test_cache_lines_out_of_range_are_ignored(tmp_path):
    """Block sizes that are not whole warps or lie outside the kernels'
    ranges, and round counts below 1, are skipped when a cache is loaded
    (they never reach a launch); valid lines in the same file still apply."""
    path = str(tmp_path / "tune.txt")
    with open(path, "w") as f:
        f.write("3 list_warp_block 100\n3 list_team_block 2048\n3 flow_block 200\n"
                "3 flow_rounds 0\n3 list_warp_dmax 7\n3 peel_order 5\n3 peel_chunk 256\n")
    off, adj = cds.gen_rmat(12, 8.0, 6)
    with cds.Context(0) as c:
        c.autotune([], 3, path)
        g = c.graph(off, adj)
        s = c.solve(g, 3)
        g.free()
    ora = oracle.solve(off, adj, 3)
    assert (s.num, s.den) == (ora["num"], ora["den"])
    assert s.vertices.tolist() == ora["vertices"].tolist()


def test_server_rejects_too_many_workers(ctx):
    with pytest.raises(cds.CdsError) as e:
        ctx.server(max_batch=1, max_inflight=65)
    assert e.value.status == 4  # CDS_ERR_INPUT
    srv = ctx.server(max_batch=1, max_inflight=64)  # the cap itself is allowed
    srv.stop()


def _bipartite(a, b):
    """K_{a,b} as a canonical CSR: high DAG out-degrees, no triangles."""
    n = a + b
    rows = [np.arange(a, n, dtype=np.uint32)] * a + [np.arange(0, a, dtype=np.uint32)] * b
    off = np.zeros(n + 1, np.uint64)
    off[1:] = np.cumsum([len(r) for r in rows])
    return off, np.concatenate(rows)


def test_concurrent_requests_with_different_listing_footprints(ctx):
    """Server workers list graphs concurrently whose block teams need very
    different shared memory (K_800,800: ~90 KB per team; K_300,300: ~17 KB;
    a planted graph with real cliques); every request must succeed and match
    its single solve."""
    graphs = [_bipartite(800, 800), _bipartite(300, 300)]
    o, a = cds.gen_er(1500, 0.01, 4)
    o, a, _ = cds.gen_plant(o, a, 60, 0.6, 5)
    graphs.append((o, a))
    gs = [ctx.graph(o, a) for o, a in graphs]
    try:
        single = [key(ctx.solve(g, 3)) for g in gs]
        srv = ctx.server(max_batch=1, max_inflight=4)
        try:
            order = [i % len(gs) for i in range(24)]
            tickets = [srv.submit(gs[i], cds.make_params(3)) for i in order]
            got = [key(srv.wait(t)) for t in tickets]
        finally:
            srv.stop()
        assert got == [single[i] for i in order]
    finally:
        for g in gs:
            g.free()


def test_served_host_csr_requests_against_oracle(ctx):
    """Requests carrying their graph as a host CSR (cds_submit_csr, the way
    the served bench sends them): R-MAT graphs of the served configuration's
    shapes at small sizes, k = 3 and 4, each answer equal to the oracle's;
    a malformed CSR answers CDS_ERR_INPUT for its own ticket only, and the
    queue and service times are reported."""
    rng = np.random.default_rng(11)
    csrs, ks = [], []
    for i in range(8):
        n = int(np.exp(rng.uniform(np.log(1000), np.log(6000))))
        scale = int(np.ceil(np.log2(n)))
        csrs.append(cds.gen_rmat(scale, float(rng.uniform(4, 16)) * n / (1 << scale), 300 + i, n=n))
        ks.append(3 if i % 4 else 4)
    keep = [(np.ascontiguousarray(o, np.uint64), np.ascontiguousarray(a, np.uint32)) for o, a in csrs]
    bad_off = np.array([0, 1, 1], np.uint64)  # 0 -> 1 without 1 -> 0
    bad_adj = np.array([1], np.uint32)
    srv = ctx.server(max_batch=4, max_inflight=2)
    try:
        tickets = [srv.submit_csr(o.ctypes.data, a.ctypes.data, len(o) - 1, cds.make_params(k))
                   for (o, a), k in zip(keep, ks)]
        tbad = srv.submit_csr(bad_off.ctypes.data, bad_adj.ctypes.data, 2, cds.make_params(3))
        sols = [srv.wait(t) for t in tickets]
        with pytest.raises(cds.CdsError) as e:
            srv.wait(tbad)
        assert e.value.status == 4
    finally:
        srv.stop()
    for s, (o, a), k in zip(sols, keep, ks):
        ora = oracle.solve(o, a, k)
        assert (s.num, s.den) == (ora["num"], ora["den"])
        assert s.vertices.tolist() == ora["vertices"].tolist()
        assert s.queue_ms >= 0 and s.service_ms > 0


def test_server_batches_keep_their_k_when_large_requests_wait(ctx):
    """Two workers, two large requests (at least 2^20 arcs: run alone, and one
    worker always stays free for small ones) at the head of the queue, then
    small requests alternating k = 3 and 4: the free worker passes over the
    waiting large request, and every batch it forms must hold one k only --
    each answer equals its plain solve."""
    big = cds.gen_rmat(17, 8.0, 21)
    assert big[0][-1] >= 1 << 20
    smalls = [cds.gen_rmat(10, 6.0, 40 + i) for i in range(12)]
    gb = ctx.graph(*big)
    gs = [ctx.graph(o, a) for o, a in smalls]
    try:
        ks = [3 if i % 2 == 0 else 4 for i in range(len(gs))]
        want = [key(ctx.solve(g, k)) for g, k in zip(gs, ks)]
        want_big = key(ctx.solve(gb, 3))
        srv = ctx.server(max_batch=8, max_inflight=2)
        try:
            tb = [srv.submit(gb, cds.make_params(3)) for _ in range(2)]
            ts = [srv.submit(g, cds.make_params(k)) for g, k in zip(gs, ks)]
            got = [key(srv.wait(t)) for t in ts]
            got_big = [key(srv.wait(t)) for t in tb]
        finally:
            srv.stop()
        assert got == want
        assert got_big == [want_big, want_big]
    finally:
        gb.free()
        for g in gs:
            g.free()
