"""Regenerates tests/golden/batch_mix_sample.json: the CPU oracle's exact
answers on a seeded 32-instance sub-sample of the batched configuration
(256 instances, n log-uniform in [500, 50,000], half Erdos-Renyi, half
R-MAT, planted communities of 20-200 vertices at p = 0.5, k in {2, 3, 4},
seed 2; cds_b200.workloads.batch_mix), for tests/test_gpu_batch_serve.py.

    python tests/golden/make_batch_sample.py     # a few minutes of one core

The sample is numpy.random.default_rng(32).choice(256, 32, replace=False).
Per instance the file holds its index, size, k, the SHA-256 digests of its
CSR (the test first checks that its host generated the same graph) and the
oracle's answer (oracle.solve: oracle/cds_oracle.c, the reference pipeline
restated with exact arithmetic): the k-clique count, the exact density
num/den and the vertex set (its SHA-256 digest when it has more than 1,000
vertices).
"""
import hashlib
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from cds_b200 import workloads  # noqa: E402
import oracle  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "batch_mix_sample.json")


def sample_indices():
    return sorted(int(i) for i in np.random.default_rng(32).choice(256, 32, replace=False))


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main():
    idx = sample_indices()
    inst = workloads.batch_mix(256, 2, only=set(idx))
    rows = []
    for i, (off, adj, k) in zip(idx, inst):
        t0 = time.perf_counter()
        r = oracle.solve(off, adj, k)
        rows.append({"index": i, "n": int(len(off) - 1), "k": k, "off_sha256": digest(off.astype("<u8")),
                     "adj_sha256": digest(adj.astype("<u4")), "total_cliques": r["total_cliques"],
                     "num": r["num"], "den": r["den"], "size": int(len(r["vertices"])),
                     "oracle_s": round(time.perf_counter() - t0, 2)})
        # the vertex set itself when small, else its digest (u32 ids, ascending)
        if len(r["vertices"]) <= 1000:
            rows[-1]["vertices"] = [int(v) for v in r["vertices"]]
        else:
            rows[-1]["vertices_sha256"] = digest(np.asarray(r["vertices"], "<u4"))
        print(rows[-1]["index"], rows[-1]["n"], k, rows[-1]["total_cliques"], rows[-1]["oracle_s"], flush=True)
    with open(OUT, "w") as f:
        json.dump({"config": "batch_mix(256, seed 2), sample default_rng(32).choice(256, 32)", "instances": rows},
                  f, indent=1)


if __name__ == "__main__":
    main()
