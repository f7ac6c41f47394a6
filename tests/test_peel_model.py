"""A sequential model of the clique-core sweeps of cds_b200/csrc/peel.cu
(k_hindex), checked against the oracle's peel on small graphs.

The model keeps the kernel's rules and randomises what the GPU leaves to
scheduling:
  * items of at most `chunk` incidences; a vertex with one item gets its
    exact h-index from the values current when its item runs, a hub's items
    read values at their own times and the last one computes the new value
    from the exact window (32 values below tau) and the log-scale bins
    (sixteen per octave) -- an upper bound below the window;
  * values are stored at once (later items of the same sweep read them);
  * a hub item that starts once the hub's finished items hold t cliques
    with x >= t (t its value) counts nothing: the value stands;
  * a sweep skips every vertex whose value is below the smallest value
    changed in the previous sweep; the model asserts that such a vertex's
    exact h-index at that moment equals its value (the claim that makes the
    skip exact);
  * after a sweep without change one more sweep recounts everything.
Items run in a fresh random order every sweep.  The final values must equal
the reference peel's core numbers whatever the order and the chunk size.
"""
import random

import numpy as np
import pytest

import cds_b200 as cds
import oracle

WIN, SUB_BITS = 32, 4
SUB = 1 << SUB_BITS
NLOG = 32 * SUB


def log_bin(e):
    j = e.bit_length() - 1
    s = (e >> (j - SUB_BITS)) & (SUB - 1) if j >= SUB_BITS else (e << (SUB_BITS - j)) & (SUB - 1)
    return j * SUB + s


def log_bin_lo(b):
    return (((SUB + b % SUB) << (b // SUB)) + SUB - 1) >> SUB_BITS


def exact_h(xs, t):
    """Largest h <= t with at least h values >= h."""
    s = sorted((min(x, t) for x in xs), reverse=True)
    h = 0
    while h < len(s) and s[h] >= h + 1:
        h += 1
    return h


def hub_bound(xs, t):
    """New value of a hub from its counts, as the kernel's hub_tau."""
    ge = sum(1 for x in xs if x >= t)
    if ge >= t:
        return t
    win = [0] * WIN
    bins = [0] * NLOG
    for x in xs:
        if x >= t:
            continue
        d = t - 1 - x
        if d < WIN:
            win[d] += 1
        else:
            bins[log_bin(d + 1 - WIN)] += 1
    c = ge
    for d in range(WIN):
        c += win[d]
        h = t - 1 - d
        if h <= 0 or c >= h:
            return h
    for b in range(NLOG):
        c += bins[b]
        lo, hi = log_bin_lo(b), log_bin_lo(b + 1)
        xlo = t - WIN - hi + 1
        if hi > lo and (xlo <= 0 or c >= xlo):
            return max(0, t - WIN - lo)
    raise AssertionError("no bin qualified")


def cliques_of(off, adj, k):
    n = len(off) - 1
    nb = [set(adj[off[v]:off[v + 1]].tolist()) for v in range(n)]
    out = []

    def grow(clique, cand):
        if len(clique) == k:
            out.append(tuple(clique))
            return
        for u in sorted(cand):
            if u > clique[-1]:
                grow(clique + [u], cand & nb[u])

    for v in range(n):
        grow([v], nb[v])
    inc = [[] for _ in range(n)]
    for c in out:
        for v in c:
            inc[v].append(c)
    return inc


def run_model(inc, chunk, rng):
    n = len(inc)
    tau = [len(inc[v]) for v in range(n)]
    nitems = [1 if len(inc[v]) <= chunk else -(-len(inc[v]) // chunk) for v in range(n)]
    items = [(v, i) for v in range(n) if inc[v] for i in range(nitems[v])]
    sweep, verify, low, skipped = 0, False, 0, 0
    while True:
        rng.shuffle(items)
        got = {v: [] for v in range(n) if nitems[v] > 1}
        done = dict.fromkeys(got, 0)
        changes = []
        for v, i in items:
            t = tau[v]
            if t == 0:
                continue
            xs_now = lambda part: [min(tau[u] for u in c if u != v) for c in part]
            if sweep > 0 and not verify and t < low:
                assert exact_h(xs_now(inc[v]), t) == t, "a skipped vertex was not exact"
                skipped += 1
                continue
            if nitems[v] == 1:
                nt = exact_h(xs_now(inc[v]), t)
            else:
                # an item that starts after the hub's finished items found t
                # cliques with x >= t counts nothing (its value stands)
                if sum(1 for x in got[v] if x >= t) < t:
                    got[v] += xs_now(inc[v][i * chunk:(i + 1) * chunk])
                done[v] += 1
                if done[v] < nitems[v]:
                    continue
                nt = hub_bound(got[v], t)
            if nt < t:
                tau[v] = nt
                changes.append(nt)
        sweep += 1
        if not changes:
            if verify:
                return tau, sweep, skipped
            verify = True
        else:
            verify = False
        low = min(changes) if changes else 0
        assert sweep < 10_000


def graphs():
    out = []
    for seed in range(3):
        out.append(("er", cds.gen_er(60, 0.2, seed)))
        o, a = cds.gen_er(70, 0.08, seed + 10)
        out.append(("plant", cds.gen_plant(o, a, 18, 0.8, seed + 20)[:2]))
    return out


@pytest.mark.parametrize("k", [2, 3, 4])
@pytest.mark.parametrize("chunk", [4, 16, 1024])
def test_model_reaches_the_core_numbers(k, chunk):
    rng = random.Random(k * 100 + chunk)
    total_skipped = 0
    for name, (off, adj) in graphs():
        inc = cliques_of(off, adj, k)
        want = oracle.peel(off, adj, k)["core"].astype(np.int64).tolist()
        for _ in range(3):
            tau, sweeps, skipped = run_model(inc, chunk, rng)
            assert tau == want, (name, k, chunk)
            total_skipped += skipped
    assert total_skipped > 0  # the skip rule was exercised


def test_hub_bound_is_an_upper_bound_within_a_seventeenth():
    """Below the window the bound is >= the exact h-index and shrinks the
    gap to at most about a seventeenth of the distance below the window."""
    rng = random.Random(7)
    for _ in range(1500):
        t = rng.randrange(1, 4000)
        xs = [rng.randrange(0, 2 * t) for _ in range(rng.randrange(t // 2 + 1, 3 * t + 2))]
        h, u = exact_h(xs, t), hub_bound(xs, t)
        assert h <= u <= t
        if h < t - WIN:
            assert u - h <= (t - WIN - h) / SUB + 1
