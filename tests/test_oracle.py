"""The CPU oracle (oracle/cds_oracle.c) pinned against the reference program.

tests/golden/ holds the output of the reference CPU pipeline compiled from its
own sources (oracle/_ref/ref_dump, generated by tests/golden/make_golden.py).
The oracle must reproduce it exactly on every integer quantity, and its exact
answer must be at least as dense as the reference's (the reference searches
in float with a 0.01 stopping gap, cpuCode/c++/src/helpers.cpp:1259-1286).
"""
from fractions import Fraction
from itertools import combinations

import numpy as np
import pytest

import cds_b200 as cds
import oracle
from conftest import GOLDEN, case_id, golden_cases, load_golden

CASES = golden_cases()

# Cases where the reference returns a set that is not densest: its float
# binary search stops 0.01 short, or its bound is carried across components.
REFERENCE_SUBOPTIMAL = {("k10_bridge", 2), ("small_er1", 2)}


def graph(case):
    return cds.read_adjlist(f"{GOLDEN}/{case['graph']}")


def test_reader_matches_reference_reader():
    """The product reader and the restated reference reader agree on a
    well-formed file (the product's CSR rows come out sorted)."""
    for case in CASES[:10]:
        off, adj = graph(case)
        roff, radj = oracle.read_adjlist(f"{GOLDEN}/{case['graph']}")
        assert np.array_equal(off, roff)
        for v in range(len(off) - 1):
            assert sorted(radj[roff[v]:roff[v + 1]]) == list(adj[off[v]:off[v + 1]])


@pytest.mark.parametrize("case", CASES, ids=case_id)
def test_counts_and_degrees(case):
    g = load_golden(case)
    off, adj = graph(case)
    tot, deg = oracle.count_cliques(off, adj, case["k"])
    assert tot == g["total_cliques"]
    assert deg.tolist() == g["clique_degree"]


@pytest.mark.parametrize("case", CASES, ids=case_id)
def test_peel_table(case):
    """Removal order, removal degree and cliques left, row for row
    (cpuCode/c++/src/helpers.cpp:92-134)."""
    g = load_golden(case)
    off, adj = graph(case)
    pe = oracle.peel(off, adj, case["k"])
    rows = np.stack([pe["order"].astype(np.int64), pe["removal_degree"], pe["cliques_left"]], 1)
    assert rows.tolist() == g["peel"]
    # clique-core numbers are the running maximum of the removal degree
    run = np.maximum.accumulate(np.array([r[1] for r in g["peel"]], np.int64))
    core = np.zeros(len(off) - 1, np.int64)
    core[[r[0] for r in g["peel"]]] = run
    assert np.array_equal(core, pe["core"])


@pytest.mark.parametrize("case", CASES, ids=case_id)
def test_pipeline_stages_and_answer(case):
    g = load_golden(case)
    off, adj = graph(case)
    k = case["k"]
    s = oracle.solve(off, adj, k)
    assert s["total_cliques"] == g["total_cliques"]
    if g["total_cliques"] == 0:
        # the reference answers a clique-free graph with {0} at density 0;
        # the oracle answers with the empty set
        assert s["num"] == 0 and len(s["vertices"]) == 0
        return
    dc = g["densest_core"]
    assert s["core_threshold"] == dc["lower_bound"]
    assert s["core_size"] == len(dc["vertices"])
    assert s["max_core"] == dc["max_clique_core"]
    assert s["core_cliques"] == g["core_cliques"]
    assert s["pruned_edges"] == g["pruned_edges"]
    assert s["n_components"] == len(g["components"])
    # exact density of the reference's answer, recounted
    rv = g["result"]["vertices"]
    ref = Fraction(oracle.count_in_set(off, adj, k, rv), len(rv))
    assert abs(float(ref) - g["result"]["density"]) < 1e-5 * max(1.0, float(ref))
    mine = s["density"]
    assert Fraction(oracle.count_in_set(off, adj, k, s["vertices"]), len(s["vertices"])) == mine
    if (case["name"], k) in REFERENCE_SUBOPTIMAL:
        assert mine > ref
    else:
        assert mine == ref


def _brute(n, edges, k):
    """Max density over all vertex subsets and the union of all optimal sets."""
    adj = [set() for _ in range(n)]
    for u, v in edges:
        adj[u].add(v)
        adj[v].add(u)
    cl = [c for c in combinations(range(n), k)
          if all(b in adj[a] for a, b in combinations(c, 2))]
    best, union = Fraction(0), set()
    for mask in range(1, 1 << n):
        S = {i for i in range(n) if mask >> i & 1}
        d = Fraction(sum(1 for c in cl if set(c) <= S), len(S))
        if d > best:
            best, union = d, set(S)
        elif d == best and d > 0:
            union |= S
    return best, union, len(cl)


@pytest.mark.parametrize("seed", range(12))
def test_oracle_vs_brute_force(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(6, 12))
    p = float(rng.uniform(0.3, 0.8))
    edges = [(u, v) for u in range(n) for v in range(u + 1, n) if rng.random() < p]
    if not edges:
        edges = [(0, 1)]
    u = np.array([e[0] for e in edges])
    v = np.array([e[1] for e in edges])
    off, adj = cds.csr_from_edges(n, u, v)
    for k in (2, 3, 4):
        best, union, ncl = _brute(n, edges, k)
        s = oracle.solve(off, adj, k)
        assert s["total_cliques"] == ncl
        if ncl == 0:
            assert s["num"] == 0
            continue
        assert s["density"] == best
        # within the answer's component, the answer is the maximal densest set
        assert set(s["vertices"].tolist()) <= union


@pytest.mark.parametrize("n,k", [(5, 2), (6, 3), (7, 4), (8, 5), (9, 3)])
def test_complete_graph(n, k):
    from math import comb
    iu = np.triu_indices(n, 1)
    off, adj = cds.csr_from_edges(n, iu[0], iu[1])
    s = oracle.solve(off, adj, k)
    assert s["density"] == Fraction(comb(n, k), n)
    assert s["vertices"].tolist() == list(range(n))


@pytest.mark.parametrize("k", [2, 3, 4])
def test_sampled_count_partitions_the_cliques(k):
    """The bench's CPU-baseline sample: the counts rooted at each residue
    class of vertex ids add up to the full count."""
    off, adj = cds.gen_rmat(11, 8.0, 5)
    total, _ = oracle.count_cliques(off, adj, k)
    assert sum(oracle.count_cliques_sampled(off, adj, k, 7, p) for p in range(7)) == total
    assert oracle.count_cliques_sampled(off, adj, k, 1, 0) == total
