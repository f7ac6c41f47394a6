"""The command-line driver keeps the reference's surface: seven positional
arguments (cudaCode/main.cu:865-887), "Server wrong input parameters!" and
exit status 1 otherwise, and the reference's output keys."""
import re
import subprocess
from fractions import Fraction

import pytest

import cds_b200 as cds
import oracle
from conftest import GOLDEN


def run(*args, timeout=300):
    return subprocess.run([cds.CLI_PATH, *map(str, args)], capture_output=True, text=True,
                          timeout=timeout)


def test_wrong_argument_count_is_rejected_like_the_reference():
    for args in ([], ["g.txt"], ["g.txt", 3, 1, 2, 3, 4], ["g.txt", 3, 1, 2, 3, 4, -1, "extra"],
                 ["g.txt", 3, 1, 2, 3, 4, -1, "--search", "nonsense"]):
        r = run(*args)
        assert r.returncode == 1
        assert "Server wrong input parameters!" in r.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("name,k", [("ref_test", 3), ("cfg1", 3), ("small_rmat1", 4), ("k10_bridge", 2)])
def test_cli_answer(name, k):
    path = f"{GOLDEN}/{name}.txt"
    r = run(path, k, 8000, 16000, 60000, 30000, -1)
    assert r.returncode == 0, r.stderr
    out = r.stdout
    for key in ("Final Max Density", "Total Cliques=", "Densest Core Density=", "Total Components=",
                "Clique Listing Time =", "Core Decompose Time =", "Exact Time =", "Time taken=",
                "Mac Clique Core=", "K: ", "Density: ", "Size: ", "densest subgraph: "):
        assert key in out, key
    off, adj = cds.read_adjlist(path)
    ora = oracle.solve(off, adj, k)
    frac = re.search(r"Density_fraction: (\d+)/(\d+)", out)
    assert (int(frac.group(1)), int(frac.group(2))) == (ora["num"], ora["den"])
    verts = [int(x) for x in re.search(r"densest subgraph: (.*)", out).group(1).split()]
    assert verts == ora["vertices"].tolist()
    assert int(re.search(r"Total Cliques=(\d+)", out).group(1)) == ora["total_cliques"]
    dens = float(re.search(r"\nDensity: ([0-9.e+]+)", out).group(1))
    assert abs(dens - float(Fraction(ora["num"], ora["den"]))) < 1e-4 * max(1, dens)
    # the reference's per-component bound lines
    lbs = re.search(r"\nlb=(.*)", out).group(1).split()
    ubs = re.search(r"\nub=(.*)", out).group(1).split()
    assert len(lbs) == len(ubs) == ora["n_components"]
    assert "\neub=n/a" in out
    assert "Approximate:" not in out


@pytest.mark.gpu
def test_cli_core_mode_reports_its_gap():
    path = f"{GOLDEN}/cfg1.txt"
    r = run(path, 3, 8000, 16000, 60000, 30000, -1, "--search", "core")
    assert r.returncode == 0, r.stderr
    assert "Approximate: densest core" in r.stdout
    num, den = map(int, re.search(r"Density_fraction: (\d+)/(\d+)", r.stdout).groups())
    un, ud = map(int, re.search(r"Density_upper_bound: (\d+)/(\d+)", r.stdout).groups())
    assert Fraction(num, den) <= Fraction(un, ud)
    assert float(re.search(r"Density_gap: (\S+)", r.stdout).group(1)) >= 0


@pytest.mark.gpu
def test_cli_bisect_and_missing_file():
    path = f"{GOLDEN}/small_er2.txt"
    a = run(path, 3, 8000, 16000, 60000, 30000, -1)
    b = run(path, 3, 8000, 16000, 60000, 30000, -1, "--search", "bisect")
    fa = re.search(r"Density_fraction: (\S+)", a.stdout).group(1)
    fb = re.search(r"Density_fraction: (\S+)", b.stdout).group(1)
    assert a.returncode == 0 and b.returncode == 0 and fa == fb
    r = run("/nonexistent.txt", 3, 1, 1, 1, 1, -1)
    assert r.returncode == 2 and "Graph file Open Failed" in r.stdout
