"""A sequential model of the vertex-level push-relabel of
cds_b200/csrc/flow.cu (k_flow), checked against Edmonds-Karp on the explicit
clique-vertex network of the reference (cpuCode/c++/src/helpers.cpp:1302-1341).

Network for alpha = p/q, every capacity times q:
    s -> v  q * deg(v)      v -> t  k * p      v -> psi  q      psi -> v  q(k-1)
The model keeps the kernel's reformulation: clique nodes hold no excess and
carry no label, a push moves flow v -> psi -> w in one step (admissible when
d(w) = d(v) - 1 with residual on both arcs), labels live on vertices only, a
global relabel is a BFS from t over residual arcs, and rounds are prepare
(push to t from label 1, offer the excess), push (labels frozen, only the
offered excess moves) and relabel (a vertex left with part of its offer
takes 1 + the lowest residual neighbour).  Vertices and incidences run in a
fresh random order every round.  The max-flow value and the set of vertices
that cannot reach t afterwards (the answer set) must equal those of a plain
augmenting-path max-flow on the explicit network.
"""
import random
from collections import deque
from fractions import Fraction

import numpy as np
import pytest

import cds_b200 as cds
from test_peel_model import cliques_of

INF = 1 << 30


def warm_split(n, cl, k, p, q, passes):
    """The warm start of flow.cu (k_split_init / k_split_loads /
    k_split_update / k_split_apply) in the kernels' float32 arithmetic:
    weights 1 / clique degree, passes - 1 multiplicative updates towards the
    sink capacity k p / q, then each clique's k q units split as floors of
    k q w_j / sum with the rest to the (first) heaviest member.  Returns the
    flow words x and the units each vertex holds."""
    f32 = np.float32
    deg = [0] * n
    for c in cl:
        for v in c:
            deg[v] += 1
    w = [f32(1.0) / f32(d) if d else f32(1.0) for d in deg]
    cap = f32(k) * f32(p / q)
    for _ in range(passes - 1):
        load = [f32(0.0)] * n
        for c in cl:
            ws = [w[v] for v in c]
            tot = f32(0.0)
            for x_ in ws:
                tot = f32(tot + x_)
            fac = f32(f32(k) / tot)
            for v, x_ in zip(c, ws):
                load[v] = f32(load[v] + f32(x_ * fac))
        for v in range(n):
            if load[v] > 0:
                w[v] = f32(min(max(f32(w[v] * f32(cap / load[v])), f32(1e-30)), f32(1e30)))
    kq = k * q
    x, units = [], [0] * n
    for c in cl:
        ws = [w[v] for v in c]
        tot = f32(0.0)
        for x_ in ws:
            tot = f32(tot + x_)
        jm = max(range(k), key=lambda j: (ws[j], -j))
        a, acc = [0] * k, 0
        for j in range(k):
            if j == jm:
                continue
            aj = int(float(kq) * float(f32(ws[j] / tot)))
            aj = max(0, min(aj, kq - acc))
            acc += aj
            a[j] = aj
        a[jm] = kq - acc
        x.append([q - aj for aj in a])
        for v, aj in zip(c, a):
            units[v] += aj
    return x, units


def model_flow(n, cl, k, p, q, rounds, rng, warm=0):
    deg = [0] * n
    for c in cl:
        for v in c:
            deg[v] += 1
    inc = [[] for _ in range(n)]  # (clique index, slot)
    for ci, c in enumerate(cl):
        for j, v in enumerate(c):
            inc[v].append((ci, j))
    if warm:
        # a split of every clique's units is a valid flow state: member j
        # keeps a_j = q - x_j, the x of a clique sum to 0 and lie in
        # [-q(k-1), q]; each vertex's excess is the units it holds
        x, e = warm_split(n, cl, k, p, q, warm)
        for xs in x:
            assert sum(xs) == 0 and all(-q * (k - 1) <= xj <= q for xj in xs)
    else:
        x = [[0] * k for _ in cl]
        e = [q * deg[v] for v in range(n)]  # preflow: s -> v saturated
    rt = [k * p] * n
    qk1 = q * (k - 1)

    def residual_neighbours(v):
        for ci, j in inc[v]:
            if q - x[ci][j] <= 0:
                continue
            for jw, w in enumerate(cl[ci]):
                if jw != j and qk1 + x[ci][jw] > 0:
                    yield ci, j, jw, w

    def global_relabel():
        d = [1 if rt[v] > 0 else INF for v in range(n)]
        queue = deque(v for v in range(n) if d[v] == 1)
        while queue:
            v = queue.popleft()
            # w can push to v through psi: residual w -> psi and psi -> v
            for ci, j in inc[v]:
                if qk1 + x[ci][j] <= 0:
                    continue
                for jw, w in enumerate(cl[ci]):
                    if jw != j and q - x[ci][jw] > 0 and d[w] == INF:
                        d[w] = d[v] + 1
                        queue.append(w)
        return d

    for cycle in range(10_000):
        d = global_relabel()
        if not any(e[v] > 0 and d[v] < INF for v in range(n)):
            break
        for _ in range(rounds):
            # prepare
            offer = [0] * n
            for v in range(n):
                if e[v] <= 0 or d[v] >= INF:
                    continue
                if d[v] == 1 and rt[v] > 0:
                    dl = min(e[v], rt[v])
                    rt[v] -= dl
                    e[v] -= dl
                offer[v] = e[v]
            if not any(offer):
                break
            # push, labels frozen, only offered excess moves
            order = [v for v in range(n) if offer[v] > 0 and d[v] > 1]
            rng.shuffle(order)
            for v in order:
                incs = inc[v][:]
                rng.shuffle(incs)
                for ci, j in incs:
                    if offer[v] <= 0:
                        break
                    for jw, w in enumerate(cl[ci]):
                        if jw == j or d[w] != d[v] - 1:
                            continue
                        r1, r2 = q - x[ci][j], qk1 + x[ci][jw]
                        amt = min(offer[v], r1, r2)
                        if amt <= 0:
                            continue
                        x[ci][j] += amt
                        x[ci][jw] -= amt
                        offer[v] -= amt
                        e[v] -= amt
                        e[w] += amt
            # relabel vertices left with part of their offer
            newd = d[:]
            for v in range(n):
                if offer[v] <= 0:
                    continue
                m = 0 if rt[v] > 0 else INF
                for ci, j, jw, w in residual_neighbours(v):
                    m = min(m, d[w])
                newd[v] = INF if m >= INF - 1 else m + 1
            d = newd
    flow = sum(k * p - rt[v] for v in range(n))
    d = global_relabel()
    return flow, sorted(v for v in range(n) if d[v] >= INF)


def explicit_flow(n, cl, k, p, q):
    """Edmonds-Karp on s, t, vertices and clique nodes."""
    s, t = n + len(cl), n + len(cl) + 1
    N = t + 1
    cap = [dict() for _ in range(N)]

    def arc(a, b, c):
        cap[a][b] = cap[a].get(b, 0) + c
        cap[b].setdefault(a, 0)

    deg = [0] * n
    for c in cl:
        for v in c:
            deg[v] += 1
    for v in range(n):
        arc(s, v, q * deg[v])
        arc(v, t, k * p)
    for ci, c in enumerate(cl):
        for v in c:
            arc(v, n + ci, q)
            arc(n + ci, v, q * (k - 1))
    flow = 0
    while True:
        prev = {s: None}
        queue = deque([s])
        while queue and t not in prev:
            a = queue.popleft()
            for b, c in cap[a].items():
                if c > 0 and b not in prev:
                    prev[b] = a
                    queue.append(b)
        if t not in prev:
            break
        path, b = [], t
        while prev[b] is not None:
            path.append((prev[b], b))
            b = prev[b]
        amt = min(cap[a][b] for a, b in path)
        for a, b in path:
            cap[a][b] -= amt
            cap[b][a] += amt
        flow += amt
    # vertices that can reach t in the residual graph
    reach = {t}
    queue = deque([t])
    while queue:
        b = queue.popleft()
        for a in range(N):
            if a not in reach and cap[a].get(b, 0) > 0:
                reach.add(a)
                queue.append(a)
    return flow, sorted(v for v in range(n) if v not in reach)


@pytest.mark.parametrize("k", [2, 3, 4])
@pytest.mark.parametrize("seed", range(4))
def test_vertex_level_push_relabel_matches_the_explicit_network(k, seed):
    rng = random.Random(seed * 10 + k)
    off, adj = cds.gen_er(16, 0.45, seed + 31)
    if seed % 2:
        off, adj = cds.gen_plant(off, adj, 7, 0.9, seed + 40)[:2]
    n = len(off) - 1
    inc = cliques_of(off, adj, k)
    cl = sorted({c for lst in inc for c in lst})
    if not cl:
        pytest.skip("no cliques")
    rho = Fraction(len(cl), n)
    # densities around the answer: below, at and above the whole graph's
    for alpha in (rho / 2, rho, rho * 3 / 2, Fraction(len(cl), 3)):
        p, q = alpha.numerator, alpha.denominator
        want = explicit_flow(n, cl, k, p, q)
        for rounds in (1, 4, 32):
            got = model_flow(n, cl, k, p, q, rounds, rng)
            assert got == want, (k, seed, alpha, rounds)
        # started from the warm split (one split, or after weight updates)
        for warm in (1, 3):
            got = model_flow(n, cl, k, p, q, 4, rng, warm=warm)
            assert got == want, (k, seed, alpha, "warm", warm)


@pytest.mark.parametrize("k", [3, 4])
@pytest.mark.parametrize("seed", range(3))
def test_warm_split_balances_a_dense_network(k, seed):
    """On a dense network at its own density, where every vertex can be
    brought to its sink capacity, the split leaves less than half the excess
    of the plain start (each vertex keeping q of each of its cliques), and
    two weight updates before it leave less again."""
    off, adj = cds.gen_er(40, 0.5, seed + 3)
    n = len(off) - 1
    inc = cliques_of(off, adj, k)
    cl = sorted({c for lst in inc for c in lst})
    rho = Fraction(len(cl), n)
    p, q = rho.numerator, rho.denominator
    deg = [0] * n
    for c in cl:
        for v in c:
            deg[v] += 1

    def excess(units):
        return sum(max(0, u - k * p) for u in units)

    plain = excess([q * d for d in deg])
    one = excess(warm_split(n, cl, k, p, q, 1)[1])
    three = excess(warm_split(n, cl, k, p, q, 3)[1])
    assert one < plain / 2
    assert three < one
