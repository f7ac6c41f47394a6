"""Seeded synthetic inputs of the five benchmark configurations.

Host-side helpers (no GPU needed) built on the library's generators: the
same graphs feed the parity tests, the bench and the profiling driver.

  plain_small    Erdos-Renyi G(2000, 0.004) + planted 40-vertex community
                 (p = 0.6), seed 0; solved at k = 3
  rmat14         R-MAT scale 14, edge factor 8 (a=0.57, b=c=0.19), seed 1;
                 solved at k = 2, 3, 4
  batch_mix      256 instances: n log-uniform in [500, 50,000], half
                 Erdos-Renyi (average degree uniform 4-32), half R-MAT, each
                 with a planted community of 20-200 vertices (p = 0.5),
                 k uniform in {2, 3, 4}, seed 2
  served_stream  Poisson arrivals of DSD requests: graph sizes log-uniform in
                 [1,000, 200,000] (R-MAT, edge factor 4-16), k in {3, 4} at
                 3:1, seed 3
  rmat18_plant   R-MAT scale 18, edge factor 16, planted 300-vertex community
                 (p = 0.5), seed 4; solved at k = 4
"""
from __future__ import annotations

from typing import List, Tuple

import numpy as np

from . import gen_er, gen_plant, gen_rmat

PLAIN_SMALL_ARGS = dict(p_size=8000, cp_size=16000, gl_buffer_size=60000, partition_size=30000,
                        early_stop=-1)


def plain_small():
    """Erdos-Renyi G(2000, 0.004) with a planted 40-vertex community
    (p = 0.6) on random ids, seed 0."""
    off, adj = gen_er(2000, 0.004, 0)
    off, adj, _ = gen_plant(off, adj, 40, 0.6, 0)
    return off, adj


def rmat14():
    """R-MAT scale 14 (16,384 vertices), edge factor 8, seed 1."""
    return gen_rmat(14, 8.0, 1)


def rmat18_plant():
    """R-MAT scale 18 (262,144 vertices), edge factor 16, with a planted
    300-vertex community (p = 0.5), seed 4."""
    off, adj = gen_rmat(18, 16.0, 4)
    off, adj, _ = gen_plant(off, adj, 300, 0.5, 4)
    return off, adj


def batch_mix(count: int = 256, seed: int = 2, only=None) -> List[Tuple[np.ndarray, np.ndarray, int]]:
    """The batched configuration: `count` instances, n log-uniform in
    [500, 50,000], even indices Erdos-Renyi (average degree uniform 4-32), odd
    ones R-MAT (a=0.57, b=c=0.19), each with a planted community of 20-200
    vertices (p = 0.5), k uniform in {2, 3, 4}.  With `only` (a set of
    indices) the other instances are drawn but not generated, so a
    sub-sample has exactly the shapes it has in the full batch."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(round(np.exp(rng.uniform(np.log(500), np.log(50000)))))
        avg = float(rng.uniform(4, 32))
        gen = only is None or i in only
        if gen:
            if i % 2 == 0:
                off, adj = gen_er(n, avg / (n - 1), seed * 100003 + i)
            else:
                scale = int(np.ceil(np.log2(n)))
                off, adj = gen_rmat(scale, avg / 2 * n / (1 << scale), seed * 100003 + i, n=n)
        size = int(rng.integers(20, 201))
        k = int(rng.integers(2, 5))
        if gen:
            off, adj, _ = gen_plant(off, adj, min(size, n), 0.5, seed * 100003 + i + 17)
            out.append((off, adj, k))
    return out


def served_stream(requests: int, pool: int, seed: int = 3):
    """Graphs and requests of the served configuration: `pool` distinct R-MAT
    graphs (n log-uniform in [1,000, 200,000], edge factor uniform 4-16) and
    `requests` (graph index, k) pairs with k = 3 or 4 at 3:1."""
    rng = np.random.default_rng(seed)
    graphs = []
    for i in range(pool):
        n = int(round(np.exp(rng.uniform(np.log(1000), np.log(200000)))))
        scale = int(np.ceil(np.log2(n)))
        ef = float(rng.uniform(4, 16))
        graphs.append(gen_rmat(scale, ef * n / (1 << scale), seed * 7919 + i, n=n))
    reqs = [(int(rng.integers(0, pool)), 3 if rng.random() < 0.75 else 4) for _ in range(requests)]
    return graphs, reqs
