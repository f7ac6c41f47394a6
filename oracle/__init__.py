"""oracle -- CPU checker for the k-clique densest-subgraph engine.

TEST INFRASTRUCTURE ONLY.  Imported by tests/, __graft_entry__.smoke() and
bench.py's cpu_baseline / reference legs, never by the product.  Wraps:

  * liboracle.so -- cds_oracle.c, a C restatement of the reference CPU
    pipeline (wajidmanzoor/CDS cpuCode/c++/src/helpers.cpp) with exact
    arithmetic; see the header of cds_oracle.c for where it departs from the
    reference and why;
  * _ref/dsd and _ref/ref_dump -- the reference CPU program compiled unchanged
    from its sources by oracle/Makefile (present only where the reference
    sources were available at build time).
"""
from __future__ import annotations

import ctypes
import json
import os
import subprocess
import tempfile
from fractions import Fraction

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_DSD = os.path.join(HERE, "_ref", "dsd")
REF_DUMP = os.path.join(HERE, "_ref", "ref_dump")

_u64p = ctypes.POINTER(ctypes.c_uint64)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_i64p = ctypes.POINTER(ctypes.c_int64)


class OracleResult(ctypes.Structure):
    _fields_ = [(name, ctypes.c_int64) for name in (
        "total_cliques", "core_threshold", "core_size", "core_cliques", "max_core",
        "pruned_edges", "n_components", "flows", "num", "den")]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            subprocess.run(["make", "-C", HERE, "liboracle.so"], check=True,
                           stdout=subprocess.DEVNULL)
        L = ctypes.CDLL(LIB)
        L.oracle_count_cliques.restype = ctypes.c_int64
        L.oracle_count_cliques.argtypes = [ctypes.c_uint32, _u64p, _u32p, ctypes.c_uint32, _i64p]
        L.oracle_count_cliques_sampled.restype = ctypes.c_int64
        L.oracle_count_cliques_sampled.argtypes = [ctypes.c_uint32, _u64p, _u32p, ctypes.c_uint32,
                                                   ctypes.c_uint32, ctypes.c_uint32]
        L.oracle_count_in_set.restype = ctypes.c_int64
        L.oracle_count_in_set.argtypes = [ctypes.c_uint32, _u64p, _u32p, ctypes.c_uint32,
                                          ctypes.POINTER(ctypes.c_uint8)]
        L.oracle_peel.restype = ctypes.c_int64
        L.oracle_peel.argtypes = [ctypes.c_uint32, _u64p, _u32p, ctypes.c_uint32, _u32p,
                                  _i64p, _i64p, _i64p]
        L.oracle_solve.restype = ctypes.c_int
        L.oracle_solve.argtypes = [ctypes.c_uint32, _u64p, _u32p, ctypes.c_uint32,
                                   ctypes.POINTER(OracleResult), ctypes.POINTER(ctypes.c_uint8)]
        L.oracle_read_adjlist.restype = ctypes.c_int
        L.oracle_read_adjlist.argtypes = [ctypes.c_char_p, _u32p, ctypes.POINTER(_u64p),
                                          ctypes.POINTER(_u32p)]
        L.oracle_free.argtypes = [ctypes.c_void_p]
        _lib = L
    return _lib


def _csr(off, adj):
    off = np.ascontiguousarray(off, np.uint64)
    adj = np.ascontiguousarray(adj, np.uint32)
    if adj.size == 0:
        adj = np.zeros(1, np.uint32)
    return len(off) - 1, off, adj


def read_adjlist(path):
    """CSR exactly as the reference reader builds it (rows in file order)."""
    n = ctypes.c_uint32()
    o, a = _u64p(), _u32p()
    if lib().oracle_read_adjlist(path.encode(), ctypes.byref(n), ctypes.byref(o), ctypes.byref(a)):
        raise ValueError(f"oracle cannot read {path}")
    off = np.ctypeslib.as_array(o, (n.value + 1,)).copy()
    adj = np.ctypeslib.as_array(a, (max(int(off[-1]), 1),))[: int(off[-1])].copy()
    lib().oracle_free(ctypes.cast(o, ctypes.c_void_p))
    lib().oracle_free(ctypes.cast(a, ctypes.c_void_p))
    return off, adj


def count_cliques(off, adj, k):
    n, off, adj = _csr(off, adj)
    deg = np.zeros(max(n, 1), np.int64)
    tot = lib().oracle_count_cliques(n, off.ctypes.data_as(_u64p), adj.ctypes.data_as(_u32p), k,
                                     deg.ctypes.data_as(_i64p))
    if tot < 0:
        raise RuntimeError("oracle_count_cliques failed")
    return int(tot), deg[:n]


def count_cliques_sampled(off, adj, k, stride, phase):
    """k-cliques rooted at the vertices u with u % stride == phase (the
    enumeration's first vertex): a bounded sample of the listing work."""
    n, off, adj = _csr(off, adj)
    tot = lib().oracle_count_cliques_sampled(n, off.ctypes.data_as(_u64p), adj.ctypes.data_as(_u32p),
                                             k, stride, phase)
    if tot < 0:
        raise RuntimeError("oracle_count_cliques_sampled failed")
    return int(tot)


def count_in_set(off, adj, k, members):
    n, off, adj = _csr(off, adj)
    flags = np.zeros(max(n, 1), np.uint8)
    flags[np.asarray(members, np.int64)] = 1
    return int(lib().oracle_count_in_set(n, off.ctypes.data_as(_u64p), adj.ctypes.data_as(_u32p),
                                         k, flags.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))))


def peel(off, adj, k):
    """Removal order, removal degree, cliques left and clique-core numbers."""
    n, off, adj = _csr(off, adj)
    order = np.zeros(max(n, 1), np.uint32)
    rdeg = np.zeros(max(n, 1), np.int64)
    left = np.zeros(max(n, 1), np.int64)
    core = np.zeros(max(n, 1), np.int64)
    tot = lib().oracle_peel(n, off.ctypes.data_as(_u64p), adj.ctypes.data_as(_u32p), k,
                            order.ctypes.data_as(_u32p), rdeg.ctypes.data_as(_i64p),
                            left.ctypes.data_as(_i64p), core.ctypes.data_as(_i64p))
    if tot < 0:
        raise RuntimeError("oracle_peel failed")
    return {"total": int(tot), "order": order[:n], "removal_degree": rdeg[:n],
            "cliques_left": left[:n], "core": core[:n]}


def solve(off, adj, k):
    n, off, adj = _csr(off, adj)
    res = OracleResult()
    in_set = np.zeros(max(n, 1), np.uint8)
    if lib().oracle_solve(n, off.ctypes.data_as(_u64p), adj.ctypes.data_as(_u32p), k,
                          ctypes.byref(res), in_set.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))):
        raise RuntimeError("oracle_solve failed")
    out = {f: int(getattr(res, f)) for f, _ in OracleResult._fields_}
    out["vertices"] = np.nonzero(in_set[:n])[0].astype(np.uint32)
    out["density"] = Fraction(out["num"], out["den"]) if out["den"] else Fraction(0)
    return out


# ---------------------------------------------------------------------------
# the reference program itself (oracle/_ref, built from the reference sources)
# ---------------------------------------------------------------------------
def have_reference() -> bool:
    return os.path.exists(REF_DSD) and os.path.exists(REF_DUMP)


def reference_dump(graph_path, k, stages="all", timeout=600):
    """JSON of every stage of the reference CPU pipeline (ub1 on, ub2 off)."""
    out = subprocess.run([REF_DUMP, graph_path, str(k), "1", "0", stages], check=True,
                         capture_output=True, text=True, timeout=timeout)
    return json.loads(out.stdout)


def reference_run(graph_path, k, timeout=600):
    """Runs `dsd <graph> <motif> 1 0` and parses its answer lines."""
    with tempfile.NamedTemporaryFile("w", suffix=".motif", delete=False) as f:
        f.write(f"{k} 1 1\n")
        motif = f.name
    try:
        out = subprocess.run([REF_DSD, graph_path, motif, "1", "0"], check=True,
                             capture_output=True, text=True, timeout=timeout).stdout
    finally:
        os.unlink(motif)
    res = {}
    for line in out.splitlines():
        if line.startswith("Total_cliques:"):
            res["total_cliques"] = int(line.split()[1])
        elif line.startswith("Size:"):
            res["size"] = int(line.split()[1])
        elif line.startswith("Density:"):
            res["density"] = float(line.split()[1])
        elif line.startswith("densest subgraph:"):
            res["vertices"] = [int(x) for x in line.split(":")[1].split()]
    return res
