"""Regenerates tests/golden/rmat18_plant.json: the CPU oracle's exact clique
counts on the largest configuration (R-MAT scale 18, edge factor 16,
a=0.57 b=c=0.19, planted 300-vertex community p=0.5, seed 4), for the GPU
tests in tests/test_gpu_large.py.

    python tests/golden/make_large.py        # about 75 s of one CPU core

The graph comes from the library's seeded generator (cds_b200.workloads),
so its SHA-256 digest is recorded too: a test first checks that the host it
runs on generated the same graph.  Per k the file holds the total k-clique
count and the SHA-256 digest of every vertex's clique degree (little-endian
u64, vertex order), from oracle.count_cliques (oracle/cds_oracle.c, the
reference's listing restated; pinned against the reference's golden
outputs by tests/test_oracle.py).  The clique-core numbers and the answer
are not pinned here: the oracle's peel needs the whole 2.29 G-clique store
and its incidence lists in host memory (~74 GB), and its max-flow a network
of that size.
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

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "rmat18_plant.json")


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main():
    off, adj = workloads.rmat18_plant()
    rec = {"graph": "R-MAT scale 18, edge factor 16, a=0.57 b=c=0.19, planted 300 @ 0.5, seed 4",
           "n": int(len(off) - 1), "arcs": int(off[-1]),
           "off_sha256": digest(off.astype("<u8")), "adj_sha256": digest(adj.astype("<u4")), "k": {}}
    for k in (2, 3, 4):
        t0 = time.perf_counter()
        tot, deg = oracle.count_cliques(off, adj, k)
        rec["k"][str(k)] = {"total_cliques": tot, "clique_degree_sha256": digest(deg.astype("<u8")),
                            "max_clique_degree": int(deg.max()), "oracle_s": round(time.perf_counter() - t0, 1)}
        print(k, rec["k"][str(k)], flush=True)
    with open(OUT, "w") as f:
        json.dump(rec, f, indent=1)


if __name__ == "__main__":
    main()
