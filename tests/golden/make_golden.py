"""Regenerates the golden fixtures in tests/golden/ from the reference program.

Each case is an adjacency-list graph (<name>.txt) and the reference CPU
pipeline's output on it (<name>.k<k>.json), produced by oracle/_ref/ref_dump,
which is the reference's cpuCode/c++ sources compiled unchanged (see
oracle/Makefile).  Run from the repository root where the reference sources
are available:

    CDS_REFERENCE=<reference checkout> make -C oracle ref
    CDS_REFERENCE=<reference checkout> python tests/golden/make_golden.py

Inputs:
  * ref_test       -- the reference's own fixture cudaCode/data/test.txt
  * ref_log        -- the 10-vertex graph the reference's debug trace prints
                      (cpuCode/c++/build/out.log:3-12), whose clique degrees
                      at k = 3 the same trace records (out.log, last line)
  * k10_bridge     -- a K10 joined by one edge to a random graph of average
                      degree 8 on 2000 vertices: the case where the
                      reference's UB2 bound discards the densest set
  * cfg1           -- Erdos-Renyi G(2000, 0.004) with a planted 40-vertex
                      community (p = 0.6), seed 0
  * small_*        -- seeded small ER / R-MAT / planted graphs and edge cases
"""
import json
import os
import re
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
import cds_b200 as cds  # noqa: E402
import oracle  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
# a checkout of the reference project (wajidmanzoor/CDS), from the environment
REF = os.environ.get("CDS_REFERENCE", "")
if not REF or not os.path.isdir(REF):
    sys.exit("set CDS_REFERENCE to a checkout of the reference project")


def save_graph(name, off, adj):
    path = os.path.join(OUT, f"{name}.txt")
    cds.write_adjlist(path, off, adj)
    return path


def union(*parts):
    """Disjoint union of CSR graphs."""
    us, vs, n = [], [], 0
    for off, adj in parts:
        m = len(off) - 1
        src = np.repeat(np.arange(m, dtype=np.uint32), np.diff(off).astype(np.int64))
        us.append(src + n)
        vs.append(adj.astype(np.uint32) + n)
        n += m
    return cds.csr_from_edges(n, np.concatenate(us), np.concatenate(vs))


def clique(n):
    iu = np.triu_indices(n, 1)
    return cds.csr_from_edges(n, iu[0], iu[1])


def add_edges(off, adj, pairs):
    n = len(off) - 1
    src = np.repeat(np.arange(n, dtype=np.uint32), np.diff(off).astype(np.int64))
    p = np.asarray(pairs, np.uint32).reshape(-1, 2)
    return cds.csr_from_edges(n, np.concatenate([src, p[:, 0]]), np.concatenate([adj, p[:, 1]]))


def cases():
    out = []
    # the reference's own fixture, read with the reference's own reader
    off, adj = oracle.read_adjlist(os.path.join(REF, "cudaCode/data/test.txt"))
    out.append(("ref_test", cds.csr_from_edges(len(off) - 1,
                                               np.repeat(np.arange(len(off) - 1), np.diff(off).astype(np.int64)),
                                               adj), (2, 3, 4)))
    # the graph printed by the reference's debug trace
    rows = []
    with open(os.path.join(REF, "cpuCode/c++/build/out.log")) as f:
        for line in f.readlines()[2:12]:
            m = re.match(r"(\d+): (.*)", line.strip())
            rows.append([int(x) for x in m.group(2).split()])
    us = [i for i, r in enumerate(rows) for _ in r]
    vs = [x for r in rows for x in r]
    out.append(("ref_log", cds.csr_from_edges(len(rows), us, vs), (2, 3, 4)))
    # K10 bridged to a sparse random graph
    o, a = cds.gen_er(2000, 8.0 / 1999, 11)
    g = union(clique(10), (o, a))
    g = add_edges(*g, [(9, 10)])
    out.append(("k10_bridge", g, (2, 3)))
    # cfg1
    o, a = cds.gen_er(2000, 0.004, 0)
    o, a, _ = cds.gen_plant(o, a, 40, 0.6, 0)
    out.append(("cfg1", (o, a), (2, 3, 4)))
    # small seeded graphs
    for seed in range(4):
        o, a = cds.gen_er(120, 0.08 + 0.02 * seed, 100 + seed)
        o, a, _ = cds.gen_plant(o, a, 12 + 2 * seed, 0.7, 200 + seed)
        out.append((f"small_er{seed}", (o, a), (2, 3, 4, 5)))
    for seed in range(3):
        o, a = cds.gen_rmat(9, 6.0, 300 + seed)
        out.append((f"small_rmat{seed}", (o, a), (2, 3, 4)))
    # two cliques: the larger one wins
    out.append(("small_k5_k7", union(clique(5), clique(7)), (2, 3, 4)))
    # two equal cliques: ties keep the first component
    out.append(("small_k6_k6", union(clique(6), clique(6)), (2, 3, 4)))
    # no triangles (a path) plus isolated vertices
    n = 30
    out.append(("small_path", cds.csr_from_edges(n + 5, np.arange(n - 1), np.arange(1, n)), (2, 3)))
    # several components of different density, with isolated vertices
    o, a = cds.gen_er(60, 0.15, 7)
    g = union(clique(4), (o, a), clique(5), cds.csr_from_edges(3, [0], [1]))
    out.append(("small_mixed", g, (2, 3, 4)))
    return out


def main():
    if not oracle.have_reference():
        sys.exit("oracle/_ref is not built; run `make -C oracle ref` first")
    manifest = []
    for name, (off, adj), ks in cases():
        path = save_graph(name, off, adj)
        for k in ks:
            d = oracle.reference_dump(path, k, "all", timeout=1800)
            # keep what the tests compare; the peel table as [vertex, degree, left]
            slim = {
                "n": d["n"], "k": k, "total_cliques": d["total_cliques"],
                "clique_degree": d["clique_degree"],
                "peel": [[int(r[0]), int(r[1]), int(r[3])] for r in d["peel"][1:]],
                "densest_core": d["densest_core"], "core_cliques": d["core_cliques"],
                "pruned_edges": d["pruned_edges"], "components": d["components"],
                "result": d["result"],
            }
            jpath = os.path.join(OUT, f"{name}.k{k}.json")
            with open(jpath, "w") as f:
                json.dump(slim, f, separators=(",", ":"))
            manifest.append({"name": name, "k": k, "graph": f"{name}.txt", "json": f"{name}.k{k}.json"})
            print(name, k, d["total_cliques"], d["result"]["size"], d["result"]["density"])
    with open(os.path.join(OUT, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1)


if __name__ == "__main__":
    main()
