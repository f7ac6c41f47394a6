"""One densest-subgraph solve of a seeded R-MAT graph, for profiling.

    python -m cds_b200.case --scale 14 --ef 8 --k 4 [--repeat 2] [--seed 1] [--profile] [--tune FILE]
                            [--plant SIZE [--plant-p 0.5]]

Generates the graph with the library's R-MAT generator (a=0.57, b=c=0.19),
optionally with a planted community of SIZE vertices (edge probability
--plant-p, same seed; the largest configuration is --scale 18 --ef 16
--plant 300 --seed 4 --k 4), solves it `--repeat` times on device 0 through
the C ABI and prints the answer and the stage times of the last solve; with
--profile also the device time of each main kernel over the last solve
(cds_profile).  The profile summaries name this command so that a capture
can be repeated on the same launches.
"""
import argparse

from . import Context, gen_plant, gen_rmat


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m cds_b200.case")
    ap.add_argument("--scale", type=int, default=14)
    ap.add_argument("--ef", type=float, default=8.0)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--k", type=int, default=4)
    ap.add_argument("--repeat", type=int, default=2)
    ap.add_argument("--search", default="dinkelbach", choices=["dinkelbach", "bisect"])
    ap.add_argument("--profile", action="store_true")
    ap.add_argument("--tune", default=None, help="autotune cache file (\"k key value\" lines) to load")
    ap.add_argument("--plant", type=int, default=0, help="planted community size (0: none)")
    ap.add_argument("--plant-p", type=float, default=0.5)
    a = ap.parse_args(argv)
    off, adj = gen_rmat(a.scale, a.ef, a.seed)
    if a.plant:
        off, adj, _ = gen_plant(off, adj, a.plant, a.plant_p, a.seed)
    with Context(0) as ctx:
        g = ctx.graph(off, adj)
        if a.tune:
            ctx.autotune([], a.k, a.tune)
        sol = None
        for i in range(max(1, a.repeat)):
            if a.profile and i == max(1, a.repeat) - 1:
                ctx.profile(True)
                ctx.profile_read()
            sol = ctx.solve(g, a.k, search=a.search)
        print(f"n={len(off) - 1} k={a.k} cliques={sol.total_cliques} density={sol.num}/{sol.den} "
              f"size={len(sol.vertices)} levels={sol.peel_levels} flows={sol.flows} "
              f"components={sol.n_components} core={sol.core_size}")
        print({s: round(t, 3) for s, t in sol.times_ms.items()})
        if a.profile:
            for name, (launches, ms) in sorted(ctx.profile_read().items(), key=lambda kv: -kv[1][1]):
                print(f"  {name:28s} {launches:6d} {ms:10.3f}")
        g.free()


if __name__ == "__main__":
    main()
