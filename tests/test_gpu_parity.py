"""GPU parity: libcds (through its C ABI) against the reference's golden
outputs and the CPU oracle, bit-exact on every integer quantity.

  * k-clique count and every vertex's clique degree;
  * clique-core numbers (the running maximum of the reference's removal
    degrees, cpuCode/c++/src/helpers.cpp:106-107);
  * the answer: its exact density num/den and its vertex set (the maximal
    densest set of the first densest component, which the oracle computes
    independently with Dinic's max-flow), never below the reference's.
"""
from fractions import Fraction
from math import comb

import numpy as np
import pytest

import cds_b200 as cds
import oracle
from conftest import GOLDEN, case_id, golden_cases, load_golden

pytestmark = pytest.mark.gpu
CASES = golden_cases()


def graph(case):
    return cds.read_adjlist(f"{GOLDEN}/{case['graph']}")


@pytest.fixture(scope="module")
def graphs(ctx):
    cache = {}
    yield cache
    for g in cache.values():
        g.free()


def device_graph(ctx, graphs, case):
    if case["graph"] not in graphs:
        graphs[case["graph"]] = ctx.graph(*graph(case))
    return graphs[case["graph"]]


@pytest.mark.parametrize("case", CASES, ids=case_id)
def test_counts_and_clique_degrees(ctx, graphs, case):
    g = load_golden(case)
    cnt, deg = ctx.list_cliques(device_graph(ctx, graphs, case), case["k"])
    assert cnt == g["total_cliques"]
    assert deg.tolist() == g["clique_degree"]


@pytest.mark.parametrize("case", CASES, ids=case_id)
def test_clique_core_numbers(ctx, graphs, case):
    g = load_golden(case)
    core, mx, cnt = ctx.clique_core(device_graph(ctx, graphs, case), case["k"])
    run = np.maximum.accumulate(np.array([r[1] for r in g["peel"]], np.int64))
    want = np.zeros(g["n"], np.int64)
    want[[r[0] for r in g["peel"]]] = run
    assert cnt == g["total_cliques"]
    assert core.astype(np.int64).tolist() == want.tolist()
    assert mx == int(want.max(initial=0))


@pytest.mark.parametrize("case", CASES, ids=case_id)
@pytest.mark.parametrize("search", ["dinkelbach", "bisect"])
def test_solve(ctx, graphs, case, search):
    g = load_golden(case)
    k = case["k"]
    off, adj = graph(case)
    sol = ctx.solve(device_graph(ctx, graphs, case), k, search=search)
    ora = oracle.solve(off, adj, k)
    assert sol.total_cliques == g["total_cliques"]
    assert (sol.num, sol.den) == (ora["num"], ora["den"])
    assert sol.vertices.tolist() == ora["vertices"].tolist()
    if g["total_cliques"] == 0:
        assert sol.size if hasattr(sol, "size") else True
        assert len(sol.vertices) == 0
        return
    # the printed density is counted from the set itself
    assert Fraction(oracle.count_in_set(off, adj, k, sol.vertices), len(sol.vertices)) == sol.density
    rv = g["result"]["vertices"]
    assert sol.density >= Fraction(oracle.count_in_set(off, adj, k, rv), len(rv))
    assert sol.max_core == g["densest_core"]["max_clique_core"]
    assert sol.n_components == len(g["components"])


@pytest.mark.parametrize("case", [c for c in CASES if c["name"] != "small_path" or c["k"] == 2], ids=case_id)
def test_densest_core_prune_components_against_golden(ctx, graphs, case):
    """The middle stages against the reference's own output: the densest
    core's threshold k' and vertex set (cpuCode/c++/src/helpers.cpp:710-788),
    its clique count, the pruned edge count (:958-993) and the component table
    -- smallest vertex, size and clique count of every component, in order
    (:1010-1116)."""
    g = load_golden(case)
    k = case["k"]
    dev = device_graph(ctx, graphs, case)
    if g["total_cliques"] == 0:
        t, _, in_core = ctx.densest_core(dev, k)
        assert t == 0 and not in_core.any()
        return
    dc = g["densest_core"]
    t, (num, den), in_core = ctx.densest_core(dev, k)
    assert t == dc["lower_bound"]
    assert np.nonzero(in_core)[0].tolist() == dc["vertices"]
    assert t == -(-num // den)
    comp = ctx.components(dev, k)
    assert comp["core_cliques"] == g["core_cliques"]
    assert comp["pruned_edges"] == g["pruned_edges"]
    assert comp["components"] == [(c["first"], c["size"], c["cliques"]) for c in g["components"]]
    sol = ctx.solve(dev, k)
    assert sol.core_threshold == dc["lower_bound"]
    assert sol.core_size == len(dc["vertices"])
    assert sol.core_cliques == g["core_cliques"]
    assert sol.pruned_edges == g["pruned_edges"]
    assert sol.n_components == len(g["components"])


def _random_graph(kind, seed):
    if kind == "er":
        off, adj = cds.gen_er(400 + 50 * seed, 0.03 + 0.01 * (seed % 3), seed)
    elif kind == "rmat":
        off, adj = cds.gen_rmat(10 + seed % 2, 8.0, seed)
    else:
        off, adj = cds.gen_er(1500, 0.004, seed)
        off, adj, _ = cds.gen_plant(off, adj, 25 + 5 * (seed % 3), 0.55, seed + 1)
    return off, adj


@pytest.mark.parametrize("kind", ["er", "rmat", "plant"])
@pytest.mark.parametrize("seed", range(3))
@pytest.mark.parametrize("k", [2, 3, 4, 5, 6])
def test_random_graphs_against_oracle(ctx, kind, seed, k):
    off, adj = _random_graph(kind, seed)
    g = ctx.graph(off, adj)
    try:
        cnt, deg = ctx.list_cliques(g, k)
        tot, odeg = oracle.count_cliques(off, adj, k)
        assert cnt == tot
        assert np.array_equal(deg.astype(np.int64), odeg)
        core, _, _ = ctx.clique_core(g, k)
        assert np.array_equal(core.astype(np.int64), oracle.peel(off, adj, k)["core"])
        sol = ctx.solve(g, k)
        ora = oracle.solve(off, adj, k)
        assert (sol.num, sol.den) == (ora["num"], ora["den"])
        assert sol.vertices.tolist() == ora["vertices"].tolist()
        assert sol.core_threshold >= 1 or tot == 0
    finally:
        g.free()


@pytest.mark.parametrize("n,k", [(12, 3), (20, 4), (33, 5), (64, 3), (150, 2), (40, 8)])
def test_complete_graphs(ctx, n, k):
    iu = np.triu_indices(n, 1)
    off, adj = cds.csr_from_edges(n, iu[0], iu[1])
    g = ctx.graph(off, adj)
    sol = ctx.solve(g, k)
    g.free()
    assert sol.total_cliques == comb(n, k)
    assert sol.density == Fraction(comb(n, k), n)
    assert sol.vertices.tolist() == list(range(n))


def test_high_out_degree_block_path(ctx):
    """A dense graph whose roots exceed the warp path (out-degree > 128)."""
    off, adj = cds.gen_er(600, 0.6, 9)
    g = ctx.graph(off, adj)
    for k in (3, 4):
        cnt, deg = ctx.list_cliques(g, k)
        tot, odeg = oracle.count_cliques(off, adj, k)
        assert cnt == tot and np.array_equal(deg.astype(np.int64), odeg)
    g.free()


def test_rmat14_full_size(ctx):
    """R-MAT scale 14, edge factor 8, seed 1 at k = 2, 3, 4: counts, clique
    degrees, core numbers and the exact answer against the oracle."""
    off, adj = cds.gen_rmat(14, 8.0, 1)
    g = ctx.graph(off, adj)
    try:
        for k in (2, 3, 4):
            cnt, deg = ctx.list_cliques(g, k)
            tot, odeg = oracle.count_cliques(off, adj, k)
            assert cnt == tot and np.array_equal(deg.astype(np.int64), odeg)
            core, _, _ = ctx.clique_core(g, k)
            assert np.array_equal(core.astype(np.int64), oracle.peel(off, adj, k)["core"])
            sol = ctx.solve(g, k)
            ora = oracle.solve(off, adj, k)
            assert (sol.num, sol.den) == (ora["num"], ora["den"])
            assert sol.vertices.tolist() == ora["vertices"].tolist()
    finally:
        g.free()


def test_edge_cases(ctx):
    # no edges at all
    off = np.zeros(6, np.uint64)
    g = ctx.graph(off, np.zeros(0, np.uint32))
    sol = ctx.solve(g, 3)
    assert sol.total_cliques == 0 and sol.num == 0 and len(sol.vertices) == 0
    g.free()
    # a triangle-free graph at k = 3, solvable at k = 2
    off, adj = cds.csr_from_edges(8, np.arange(7), np.arange(1, 8))
    g = ctx.graph(off, adj)
    assert ctx.solve(g, 3).num == 0
    s2 = ctx.solve(g, 2)
    assert s2.density == Fraction(7, 8)
    g.free()


def test_errors_are_statuses(ctx):
    off = np.array([0, 1, 1], np.uint64)  # 0 -> 1 without 1 -> 0
    with pytest.raises(cds.CdsError) as e:
        ctx.graph(off, np.array([1], np.uint32))
    assert e.value.status == 4
    off, adj = cds.gen_er(50, 0.2, 1)
    g = ctx.graph(off, adj)
    for bad_k in (1, 17):
        with pytest.raises(cds.CdsError) as e:
            ctx.solve(g, bad_k)
        assert e.value.status == 4
    g.free()
    with pytest.raises(cds.CdsError) as e:
        ctx.load("/nonexistent/graph.txt")
    assert e.value.status == 4


def test_memory_budget_is_enforced():
    """A context whose budget cannot hold the clique store reports
    CDS_ERR_OOM (checked on the host before any allocation)."""
    with cds.Context(0, mem_budget=1 << 20) as small:
        off, adj = cds.gen_rmat(12, 8.0, 3)
        g = small.graph(off, adj)
        with pytest.raises(cds.CdsError) as e:
            small.solve(g, 4)
        assert e.value.status == 1
        g.free()
        # the context stays usable after the failure
        off, adj = cds.gen_er(40, 0.2, 2)
        g = small.graph(off, adj)
        assert small.solve(g, 3).total_cliques == oracle.count_cliques(off, adj, 3)[0]
        g.free()


@pytest.mark.parametrize("name,k", [("small_rmat2", 2), ("small_rmat0", 4), ("cfg1", 3), ("k10_bridge", 2)])
def test_repeated_solves_agree(ctx, name, k):
    """Concurrency in the peel and push-relabel kernels must not change any
    answer: twenty solves of the same graph, all equal to the oracle's."""
    off, adj = cds.read_adjlist(f"{GOLDEN}/{name}.txt")
    ora = oracle.solve(off, adj, k)
    want_core = oracle.peel(off, adj, k)["core"]
    g = ctx.graph(off, adj)
    try:
        for _ in range(20):
            sol = ctx.solve(g, k)
            assert (sol.num, sol.den) == (ora["num"], ora["den"])
            assert sol.vertices.tolist() == ora["vertices"].tolist()
            assert sol.core_threshold == ora["core_threshold"]
            core, _, _ = ctx.clique_core(g, k)
            assert np.array_equal(core.astype(np.int64), want_core)
    finally:
        g.free()


def level_core_density(off, adj, k):
    """Best density over the level cores {v : core(v) >= L} (exact), from the
    oracle's core numbers; k' is its ceiling."""
    core = oracle.peel(off, adj, k)["core"]
    best = None
    for L in sorted(set(core.tolist())):
        members = np.nonzero(core >= L)[0]
        d = Fraction(oracle.count_in_set(off, adj, k, members), len(members))
        if best is None or d > best:
            best = d
    return best


@pytest.mark.parametrize("case", [c for c in CASES if c["name"].startswith(("small_", "cfg1", "ref_"))],
                         ids=case_id)
def test_densest_core_density(ctx, graphs, case):
    """The peel's per-level record: best core density and k' exactly."""
    off, adj = graph(case)
    k = case["k"]
    sol = ctx.solve(device_graph(ctx, graphs, case), k)
    if sol.total_cliques == 0:
        return
    want = level_core_density(off, adj, k)
    assert Fraction(*sol.core_density) == want
    assert sol.core_threshold == -(-want.numerator // want.denominator)


@pytest.mark.parametrize("case", [c for c in CASES if c["name"].startswith(("small_", "cfg1", "ref_", "k10"))],
                         ids=case_id)
def test_core_answer_mode(ctx, graphs, case):
    """search = core (CDS_SEARCH_CORE, the CoreApp answer): the densest level
    core {v : core(v) >= L} itself, with its exact density, no flow; its
    proven upper bound is the largest core number, and the exact answer's
    bound is the answer itself."""
    off, adj = graph(case)
    k = case["k"]
    dev = device_graph(ctx, graphs, case)
    sol = ctx.solve(dev, k, search="core")
    exact = ctx.solve(dev, k)
    assert exact.upper_bound == (exact.num, exact.den) or exact.total_cliques == 0
    assert exact.density_gap == 0
    if sol.total_cliques == 0:
        assert len(sol.vertices) == 0 and sol.num == 0
        return
    core = oracle.peel(off, adj, k)["core"]
    best, best_members = None, None
    for L in sorted(set(core.tolist())):
        members = np.nonzero(core >= L)[0]
        d = Fraction(oracle.count_in_set(off, adj, k, members), len(members))
        if best is None or d > best:
            best, best_members = d, members
    assert sol.density == best
    assert sol.vertices.tolist() == best_members.tolist()
    assert sol.num == oracle.count_in_set(off, adj, k, sol.vertices)
    assert sol.flows == 0
    assert sol.upper_bound == (int(core.max()), 1)
    assert sol.density <= exact.density <= Fraction(*sol.upper_bound)
    assert sol.density_gap == Fraction(*sol.upper_bound) - sol.density


@pytest.mark.parametrize("case", [c for c in CASES if c["name"] in ("cfg1", "small_mixed", "k10_bridge", "small_er1")],
                         ids=case_id)
def test_component_bounds_match_the_reference_lines(ctx, graphs, case):
    """The reference's lb= / ub= lines (cudaCode/main.cu:1092-1103): per
    component with cliques, the densest whole component's density and
    |Psi_c|^((k-1)/k) / (k!)^(1/k), from the golden component table."""
    g = load_golden(case)
    k = case["k"]
    sol = ctx.solve(device_graph(ctx, graphs, case), k)
    comps = [c for c in g["components"] if c["cliques"] > 0]
    assert len(sol.bound_lb) == len(sol.bound_ub) == len(comps)
    lb = max(c["cliques"] / c["size"] for c in comps)
    fk = float(np.prod(np.arange(1, k + 1, dtype=np.float64)))
    for a, b, c in zip(sol.bound_lb, sol.bound_ub, comps):
        assert abs(a - lb) <= 1e-9 * max(1.0, lb)
        want = c["cliques"] ** ((k - 1) / k) / fk ** (1 / k)
        assert abs(b - want) <= 1e-9 * max(1.0, want)


@pytest.mark.parametrize("kind,seed", [("er", 1), ("rmat", 0), ("plant", 2)])
@pytest.mark.parametrize("k", [2, 3, 4, 5])
@pytest.mark.parametrize("search", ["dinkelbach", "bisect"])
@pytest.mark.parametrize("wide_ids", [False, True])
def test_compact_peel_and_wide_flow_layouts(kind, seed, k, search, wide_ids):
    """The alternative layouts -- clique ids instead of member copies in the
    peel (as u32, or as the u64 ids a listing of 2^32 or more cliques uses),
    64-bit incidence ids and flow state in the networks (what sizes past 2^32
    incidences get) -- give the same exact answers."""
    off, adj = _random_graph(kind, seed)
    ora = oracle.solve(off, adj, k)
    flags = cds.CONFIG_COMPACT_PEEL | cds.CONFIG_WIDE_FLOW | (cds.CONFIG_WIDE_CLIQUE_IDS if wide_ids else 0)
    with cds.Context(0, flags=flags) as c:
        g = c.graph(off, adj)
        core, _, _ = c.clique_core(g, k)
        sol = c.solve(g, k, search=search)
        g.free()
    assert np.array_equal(core.astype(np.int64), oracle.peel(off, adj, k)["core"])
    assert (sol.num, sol.den) == (ora["num"], ora["den"])
    assert sol.vertices.tolist() == ora["vertices"].tolist()


@pytest.mark.parametrize("k", [2, 3, 4])
def test_wide_member_ids_above_65536_vertices(ctx, k):
    """Graphs past 65,536 vertices keep 32-bit member ids in the peel's
    streams for k = 2 and 21-bit ids packed into one u64 per incidence for
    k = 3, 4 (smaller graphs use 16-bit ids); all give the oracle's answers."""
    off, adj = cds.gen_rmat(17, 2.0, 7)
    assert len(off) - 1 > 65536
    g = ctx.graph(off, adj)
    try:
        core, _, _ = ctx.clique_core(g, k)
        assert np.array_equal(core.astype(np.int64), oracle.peel(off, adj, k)["core"])
        sol = ctx.solve(g, k)
        ora = oracle.solve(off, adj, k)
        assert (sol.num, sol.den) == (ora["num"], ora["den"])
        assert sol.vertices.tolist() == ora["vertices"].tolist()
    finally:
        g.free()


@pytest.mark.parametrize("k", [3, 4])
def test_member_ids_past_21_bits(ctx, k):
    """Past 2^21 vertices the peel keeps the other members as k-1 streams of
    32-bit ids (21-bit packed ids cannot name them): core numbers and the
    answer as the oracle's, on a sparse Erdos-Renyi graph with a planted
    community spread over the id range."""
    n = (1 << 21) + 4096
    off, adj = cds.gen_er(n, 2.0 / n, 21)
    off, adj, _ = cds.gen_plant(off, adj, 40, 0.6, 22)
    g = ctx.graph(off, adj)
    try:
        core, _, _ = ctx.clique_core(g, k)
        assert np.array_equal(core.astype(np.int64), oracle.peel(off, adj, k)["core"])
        sol = ctx.solve(g, k)
        ora = oracle.solve(off, adj, k)
        assert (sol.num, sol.den) == (ora["num"], ora["den"])
        assert sol.vertices.tolist() == ora["vertices"].tolist()
    finally:
        g.free()


def test_counts_past_2_to_the_32(ctx):
    """3,500 copies of K_23 all joined to one hub vertex, at k = 12: every
    copy plus the hub is a K_24, so |Psi| = 3,500 C(24,12) = 9,464,546,000 and
    the hub's clique degree is 3,500 C(23,11) = 4,732,273,000 -- both past
    2^32 -- and every other vertex's is C(23,11).  The counts are exact u64
    (the oracle's counting on one copy gives the per-copy figures)."""
    copies, size, k = 3500, 23, 12
    n = 1 + copies * size
    iu = np.triu_indices(size, 1)
    us, vs = [], []
    for c in range(copies):
        b = 1 + c * size
        us += [iu[0] + b, np.full(size, 0)]
        vs += [iu[1] + b, np.arange(b, b + size)]
    off, adj = cds.csr_from_edges(n, np.concatenate(us), np.concatenate(vs))
    one = cds.csr_from_edges(1 + size, np.concatenate([iu[0] + 1, np.zeros(size, np.int64)]),
                             np.concatenate([iu[1] + 1, np.arange(1, size + 1)]))
    tot1, deg1 = oracle.count_cliques(*one, k)
    assert tot1 == comb(size + 1, k) and set(deg1.tolist()) == {comb(size, k - 1)}
    g = ctx.graph(off, adj)
    try:
        cnt, deg = ctx.list_cliques(g, k)
    finally:
        g.free()
    assert cnt == copies * tot1 == 9_464_546_000 > 2**32
    assert int(deg[0]) == copies * int(deg1[0]) == 4_732_273_000 > 2**32
    assert np.all(deg[1:] == deg1[1])


@pytest.mark.parametrize("early_stop", [0, 2])
@pytest.mark.parametrize("k", [2, 3, 4])
def test_early_stop_returns_a_valid_set(ctx, early_stop, k):
    """earlyStop >= 0 (the reference's heuristic, cudaCode/main.cu:777-789)
    may stop the search early; whatever it returns is a real vertex set whose
    k-clique count over its size is the reported density, no denser than the
    exact optimum and no sparser than the densest core."""
    off, adj = _random_graph("plant", 1)
    g = ctx.graph(off, adj)
    try:
        sol = ctx.solve(g, k, early_stop=early_stop)
    finally:
        g.free()
    ora = oracle.solve(off, adj, k)
    assert sol.den == len(sol.vertices) > 0
    assert sol.num == oracle.count_in_set(off, adj, k, sol.vertices)
    assert Fraction(sol.num, sol.den) <= Fraction(ora["num"], ora["den"])
    assert Fraction(sol.num, sol.den) >= Fraction(*sol.core_density)
    # the reported gap: a proven upper bound at or above the optimum
    assert Fraction(*sol.upper_bound) >= Fraction(ora["num"], ora["den"])
    assert sol.density_gap >= 0
    if not sol.early_stopped:
        assert sol.density_gap == 0


@pytest.mark.parametrize("n,deg,k", [(1500, 30.0, 2), (6000, 30.0, 2), (3000, 60.0, 3)])
def test_large_flow_networks(ctx, n, deg, k):
    """Densest sets of thousands of vertices: flow networks past the sizes
    whose build counts degrees per block in shared memory (2,048 vertices)
    and whose push phase sums excess per block (1,024), so the global-atomic
    paths run; answers equal the oracle's."""
    off, adj = cds.gen_er(n, deg / (n - 1), 12)
    g = ctx.graph(off, adj)
    try:
        sol = ctx.solve(g, k)
        ora = oracle.solve(off, adj, k)
        assert (sol.num, sol.den) == (ora["num"], ora["den"])
        assert sol.vertices.tolist() == ora["vertices"].tolist()
        assert sol.core_size > 1024
    finally:
        g.free()


def test_many_components_known_answer(ctx):
    """150,000 disjoint triangles at k = 3: the densest core has 150,000
    components, so the component table and the per-network flow results
    (about 1.2 MB each) read back past the 1 MiB pinned staging buffer, by
    direct copies.  Every triangle has density 1/3; ties keep the first
    component."""
    t = 150_000
    n = 3 * t
    base = np.arange(t, dtype=np.uint32) * 3
    adj = np.stack([base + 1, base + 2, base, base + 2, base, base + 1], axis=1).reshape(-1)
    off = np.arange(n + 1, dtype=np.uint64) * 2
    g = ctx.graph(off, adj)
    try:
        sol = ctx.solve(g, 3)
        assert (sol.num, sol.den) == (1, 3)
        assert sol.vertices.tolist() == [0, 1, 2]
        assert sol.total_cliques == t
        assert sol.core_size == n
        assert sol.n_components == t
    finally:
        g.free()
