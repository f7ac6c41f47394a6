"""The largest configuration on the GPU: R-MAT scale 18 (262,144 vertices),
edge factor 16, planted 300-vertex community (p = 0.5), seed 4, k = 4 --
2.29 G 4-cliques, a ~150 GB solve.

Pinned against the CPU oracle's committed counts (tests/golden/
rmat18_plant.json, made by tests/golden/make_large.py): the k-clique count
and every vertex's clique degree at k = 2, 3, 4, bit-exact.  The oracle
cannot run the rest of the pipeline at this size (its peel would hold the
clique store and incidence lists, ~74 GB, in host memory), so the later
stages are checked through properties that hold whatever the size:

  * the answer's density is recounted from its vertex set by the oracle
    (the k-cliques of the induced subgraph) and must equal num/den exactly;
  * the answer is at least as dense as the densest core, and k' is the
    ceiling of the best core density;
  * the clique-core numbers are the same from both peel layouts (member
    copies and clique ids), which share no sweep code.
"""
import hashlib
import json
import os
from fractions import Fraction

import numpy as np
import pytest

import cds_b200 as cds
import oracle
from cds_b200 import workloads
from conftest import GOLDEN

pytestmark = pytest.mark.gpu
K = 4


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def induced(off, adj, members):
    """CSR of the subgraph induced by `members` (ascending), relabelled 0.."""
    members = np.asarray(members, np.int64)
    n = len(off) - 1
    local = np.full(n, -1, np.int64)
    local[members] = np.arange(len(members))
    rows = []
    for v in members:
        nb = adj[off[v]:off[v + 1]].astype(np.int64)
        nb = local[nb]
        rows.append(np.sort(nb[nb >= 0]))
    sub_off = np.zeros(len(members) + 1, np.uint64)
    sub_off[1:] = np.cumsum([len(r) for r in rows])
    sub_adj = np.concatenate(rows).astype(np.uint32) if rows else np.zeros(0, np.uint32)
    return sub_off, sub_adj


@pytest.fixture(scope="module")
def large():
    with open(os.path.join(GOLDEN, "rmat18_plant.json")) as f:
        fx = json.load(f)
    off, adj = workloads.rmat18_plant()
    assert digest(off.astype("<u8")) == fx["off_sha256"], "generator produced a different graph"
    assert digest(adj.astype("<u4")) == fx["adj_sha256"], "generator produced a different graph"
    return fx, off, adj


def test_rmat18_counts_core_and_answer(large):
    fx, off, adj = large
    with cds.Context(0) as ctx:
        g = ctx.graph(off, adj)
        for k in (2, 3, 4):
            cnt, deg = ctx.list_cliques(g, k)
            want = fx["k"][str(k)]
            assert cnt == want["total_cliques"]
            assert digest(deg.astype("<u8")) == want["clique_degree_sha256"]
        sol = ctx.solve(g, K)
        core, max_core, count = ctx.clique_core(g, K)
        g.free()
    assert sol.total_cliques == fx["k"]["4"]["total_cliques"] == count
    assert sol.den == len(sol.vertices) > 0
    assert np.all(np.diff(sol.vertices.astype(np.int64)) > 0)
    sub_off, sub_adj = induced(off, adj, sol.vertices)
    inside, _ = oracle.count_cliques(sub_off, sub_adj, K)
    assert inside == sol.num
    best_core = Fraction(*sol.core_density)
    assert sol.density >= best_core
    assert sol.core_threshold == -(-best_core.numerator // best_core.denominator)
    assert sol.max_core == max_core == int(core.max())
    # the (k', Psi)-core: every member's core number is at least k'
    assert sol.core_size == int(np.count_nonzero(core >= sol.core_threshold))

    with cds.Context(0, flags=cds.CONFIG_COMPACT_PEEL) as c2:
        g2 = c2.graph(off, adj)
        core2, max2, _ = c2.clique_core(g2, K)
        g2.free()
    assert max2 == max_core
    assert np.array_equal(core2, core)
