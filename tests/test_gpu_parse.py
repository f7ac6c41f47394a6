"""Graph files parsed on the device (cds_graph_load_file) give exactly the
canonical CSR of the host reader (cds_read_adjlist, which the oracle tests
tie to the reference's reader, cudaCode/src/graph.cpp:7-40): symmetric,
ascending rows, duplicates merged, self-loops dropped, vertex lines in any
order or missing.  The binary CSR cache loads to the same graph, and
malformed files are refused with CDS_ERR_INPUT."""
import os

import numpy as np
import pytest

import cds_b200 as cds
from cds_b200 import workloads
from conftest import GOLDEN, golden_cases

pytestmark = pytest.mark.gpu


def loaded(ctx, path):
    g = ctx.load(path)
    try:
        return g.csr()
    finally:
        g.free()


@pytest.mark.parametrize("name", sorted({c["graph"] for c in golden_cases()}))
def test_golden_files(ctx, name):
    path = f"{GOLDEN}/{name}"
    off, adj = cds.read_adjlist(path)
    doff, dadj = loaded(ctx, path)
    assert np.array_equal(doff, off) and np.array_equal(dadj, adj)


def test_messy_text(ctx, tmp_path):
    """Lines out of order, repeated neighbours, one-sided entries, self-loops,
    blank lines, tabs and CRLF line ends, a vertex line missing."""
    text = ("7 9\r\n"
            "3 1 1 2\t5\r\n"
            "\n"
            "0 1 2 0 2\n"
            "5 6 3\n"
            "1 0 3\n"
            "  6   5 4   \n"
            "2 0\n")
    p = tmp_path / "messy.txt"
    p.write_bytes(text.encode())
    off, adj = cds.read_adjlist(str(p))
    doff, dadj = loaded(ctx, str(p))
    assert np.array_equal(doff, off) and np.array_equal(dadj, adj)
    assert len(off) == 8 and 4 in adj.tolist()  # vertex 4 only named as a neighbour


def test_large_rows_and_binary_cache(ctx, tmp_path):
    """R-MAT scale 18 with edge factor 16 and a planted community: hub rows of
    more than 8,192 entries take the block sort in global memory.  The text
    written by cds_write_adjlist and the binary cache both load back to the
    generated CSR."""
    off, adj = workloads.rmat18_plant()
    assert int(np.diff(off).max()) > 8192
    txt = str(tmp_path / "r18.txt")
    cds.write_adjlist(txt, off, adj)
    doff, dadj = loaded(ctx, txt)
    assert np.array_equal(doff, off) and np.array_equal(dadj, adj)
    binp = str(tmp_path / "r18.csrbin")
    cds.write_csr_binary(binp, off, adj)
    boff, badj = loaded(ctx, binp)
    assert np.array_equal(boff, off) and np.array_equal(badj, adj)


def test_shuffled_lines_with_duplicates(ctx, tmp_path):
    off, adj = cds.gen_rmat(13, 8.0, 3)
    n = len(off) - 1
    rng = np.random.default_rng(4)
    lines = []
    for v in rng.permutation(n):
        nb = adj[off[v]:off[v + 1]]
        half = nb[rng.random(len(nb)) < 0.6]  # the reverse arc supplies the rest
        dup = np.concatenate([half, half[: len(half) // 3]])
        rng.shuffle(dup)
        lines.append(" ".join(map(str, [v, *dup.tolist()])))
    p = tmp_path / "shuffled.txt"
    p.write_text(f"{n} {len(adj) // 2}\n" + "\n".join(lines) + "\n")
    hoff, hadj = cds.read_adjlist(str(p))
    doff, dadj = loaded(ctx, str(p))
    assert np.array_equal(doff, hoff) and np.array_equal(dadj, hadj)


@pytest.mark.parametrize("text", ["4 2\n0 1 x\n", "3 1\n0 5\n", "3 1\n0 99999999999\n", "",
                                  "5\n0 1\n"])
def test_malformed_text_is_refused(ctx, tmp_path, text):
    p = tmp_path / "bad.txt"
    p.write_text(text)
    with pytest.raises(cds.CdsError) as e:
        ctx.load(str(p))
    assert e.value.status == 4


def test_malformed_binary_is_refused(ctx, tmp_path):
    off, adj = cds.gen_er(50, 0.2, 1)
    p = str(tmp_path / "g.csrbin")
    cds.write_csr_binary(p, off, adj)
    raw = bytearray(open(p, "rb").read())
    with open(p, "wb") as f:
        f.write(raw[:-4])  # truncated
    with pytest.raises(cds.CdsError) as e:
        ctx.load(p)
    assert e.value.status == 4
    # one-sided arc: the upload's CSR check refuses it
    bad_adj = adj.copy()
    bad_adj[0] = (bad_adj[0] + 1) % 50 if bad_adj[0] + 1 != 0 else 2
    cds.write_csr_binary(p, off, np.sort(bad_adj))
    with pytest.raises(cds.CdsError) as e:
        ctx.load(p)
    assert e.value.status == 4
    # the context stays usable
    g = ctx.load(os.path.join(GOLDEN, "ref_test.txt"))
    assert g.n > 0
    g.free()
