"""cds_b200 -- Python binding of libcds, the B200 k-clique densest-subgraph engine.

A thin ctypes layer over the C ABI in include/cds.h (and the host-side graph
generators of include/cds_gen.h).  Every call goes to the compiled library;
there is no Python or CPU implementation of the solver behind it, and loading
fails loudly when cds_b200/lib/libcds.so has not been built.

The solver surface mirrors the reference driver (wajidmanzoor/CDS,
cudaCode/main.cu:865-1107): ``solve(graph, k, p_size, cp_size,
gl_buffer_size, partition_size, early_stop)`` takes the same positional
arguments as ``./main <graph> <k> <pSize> <cpSize> <glBufferSize>
<partitionSize> <earlyStop>``.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field
from fractions import Fraction
from typing import List, Optional, Sequence, Tuple

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libcds.so")
CLI_PATH = os.path.join(_HERE, "bin", "main")
MAX_K = 16

_u32p = ctypes.POINTER(ctypes.c_uint32)
_u64p = ctypes.POINTER(ctypes.c_uint64)

STATUS = {
    0: "CDS_OK",
    1: "CDS_ERR_OOM",
    2: "CDS_ERR_OVERFLOW",
    3: "CDS_ERR_TIMEOUT",
    4: "CDS_ERR_INPUT",
    5: "CDS_ERR_CUDA",
    6: "CDS_ERR_STATE",
    7: "CDS_ERR_NOT_READY",
}
CDS_ERR_NOT_READY = 7

T_DAG, T_LIST, T_PEEL, T_CORE, T_PRUNE, T_COMPONENTS, T_EXACT, T_TOTAL = range(8)
STAGES = ("dag", "listing", "peel", "densest_core", "prune", "components", "exact", "total")
# cds_params.search: the exact searches, and the densest core alone (approximate)
SEARCH = {"dinkelbach": 0, "bisect": 1, "core": 2}


class CdsError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status
        self.message = message


class Config(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("mem_budget", ctypes.c_uint64),
                ("streams", ctypes.c_uint32), ("flags", ctypes.c_uint32)]


class Params(ctypes.Structure):
    _fields_ = [("k", ctypes.c_uint32), ("p_size", ctypes.c_uint32),
                ("cp_size", ctypes.c_uint32), ("gl_buffer_size", ctypes.c_uint32),
                ("partition_size", ctypes.c_uint32), ("early_stop", ctypes.c_int32),
                ("search", ctypes.c_uint32)]


class Result(ctypes.Structure):
    _fields_ = [("num", ctypes.c_uint64), ("den", ctypes.c_uint64),
                ("total_cliques", ctypes.c_uint64), ("max_core", ctypes.c_uint64),
                ("core_threshold", ctypes.c_uint64), ("core_num", ctypes.c_uint64),
                ("core_den", ctypes.c_uint64), ("core_size", ctypes.c_uint64),
                ("core_cliques", ctypes.c_uint64), ("pruned_edges", ctypes.c_uint64),
                ("n_components", ctypes.c_uint32), ("flows", ctypes.c_uint32),
                ("early_stopped", ctypes.c_uint32), ("peel_levels", ctypes.c_uint32),
                ("t_ms", ctypes.c_double * 8), ("size", ctypes.c_uint64),
                ("vertices", _u32p), ("ub_num", ctypes.c_uint64), ("ub_den", ctypes.c_uint64),
                ("n_bounds", ctypes.c_uint32), ("bound_lb", ctypes.POINTER(ctypes.c_double)),
                ("bound_ub", ctypes.POINTER(ctypes.c_double)), ("t_queue_ms", ctypes.c_double),
                ("t_service_ms", ctypes.c_double)]


class Job(ctypes.Structure):
    _fields_ = [("graph", ctypes.c_void_p), ("params", Params)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("max_batch", ctypes.c_uint32), ("mem_budget", ctypes.c_uint64),
                ("max_inflight", ctypes.c_uint32), ("flags", ctypes.c_uint32)]


# Every function the C headers declare, with its ctypes signature.
_SIGNATURES = {
    "cds_version": (ctypes.c_char_p, []),
    "cds_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "cds_create": (ctypes.c_int, [ctypes.POINTER(Config), ctypes.POINTER(ctypes.c_void_p)]),
    "cds_destroy": (None, [ctypes.c_void_p]),
    "cds_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "cds_mem_usage": (ctypes.c_int, [ctypes.c_void_p, _u64p, _u64p]),
    "cds_graph_load_file": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p,
                                           ctypes.POINTER(ctypes.c_void_p)]),
    "cds_graph_from_csr": (ctypes.c_int, [ctypes.c_void_p, _u64p, _u32p, ctypes.c_uint32,
                                          ctypes.POINTER(ctypes.c_void_p)]),
    "cds_graph_info": (ctypes.c_int, [ctypes.c_void_p, _u32p, _u64p, _u32p]),
    "cds_graph_download": (ctypes.c_int, [ctypes.c_void_p, _u64p, _u32p]),
    "cds_graph_free": (None, [ctypes.c_void_p]),
    "cds_list_cliques": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32,
                                        ctypes.c_uint32, ctypes.c_uint32, _u64p, _u64p]),
    "cds_clique_core": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32,
                                       ctypes.c_uint32, _u64p, _u64p, _u64p]),
    "cds_densest_core": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32,
                                        _u64p, _u64p, _u64p, ctypes.POINTER(ctypes.c_uint8)]),
    "cds_components": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, _u64p,
                                      _u64p, _u32p, _u32p, _u64p, _u64p, ctypes.c_size_t]),
    "cds_solve": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(Params),
                                 ctypes.POINTER(Result)]),
    "cds_result_free": (None, [ctypes.POINTER(Result)]),
    "cds_solve_batch": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Job), ctypes.c_size_t,
                                       ctypes.POINTER(Result)]),
    "cds_server_start": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ServerConfig),
                                        ctypes.POINTER(ctypes.c_void_p)]),
    "cds_submit": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(Params),
                                  _u64p]),
    "cds_submit_csr": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32,
                                      ctypes.POINTER(Params), _u64p]),
    "cds_poll": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(Result)]),
    "cds_wait": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(Result)]),
    "cds_server_stop": (ctypes.c_int, [ctypes.c_void_p]),
    "cds_autotune": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p),
                                    ctypes.c_size_t, ctypes.c_uint32, ctypes.c_char_p]),
    "cds_kernel_launches": (ctypes.c_uint64, []),
    "cds_profile": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "cds_count_cliques_noalloc": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32,
                                                 ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p,
                                                 ctypes.c_void_p]),
    "cds_profile_read": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]),
    # cds_gen.h
    "cds_gen_er": (ctypes.c_int, [ctypes.c_uint32, ctypes.c_double, ctypes.c_uint64,
                                  ctypes.POINTER(_u64p), ctypes.POINTER(_u32p)]),
    "cds_gen_rmat": (ctypes.c_int, [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_double,
                                    ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                    ctypes.c_uint64, _u32p, ctypes.POINTER(_u64p),
                                    ctypes.POINTER(_u32p)]),
    "cds_gen_plant": (ctypes.c_int, [ctypes.c_uint32, _u64p, _u32p, ctypes.c_uint32,
                                     ctypes.c_double, ctypes.c_uint64, ctypes.POINTER(_u64p),
                                     ctypes.POINTER(_u32p), _u32p]),
    "cds_csr_from_edges": (ctypes.c_int, [ctypes.c_uint32, _u32p, _u32p, ctypes.c_uint64,
                                          ctypes.POINTER(_u64p), ctypes.POINTER(_u32p)]),
    "cds_read_adjlist": (ctypes.c_int, [ctypes.c_char_p, _u32p, ctypes.POINTER(_u64p),
                                        ctypes.POINTER(_u32p)]),
    "cds_write_adjlist": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_uint32, _u64p, _u32p]),
    "cds_write_csr_binary": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_uint32, _u64p, _u32p]),
    "cds_free": (None, [ctypes.c_void_p]),
}

_lib = None


def lib() -> ctypes.CDLL:
    """The loaded libcds; raises when the library has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"libcds is not built ({LIB_PATH} missing); "
                               "run `make -C cds_b200/csrc` or __graft_entry__.build()")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def exported_symbols() -> List[str]:
    return list(_SIGNATURES)


def kernel_launches() -> int:
    """Kernels this process has launched through libcds so far."""
    return int(lib().cds_kernel_launches())


# ---------------------------------------------------------------------------
# host-side graph helpers (no GPU needed)
# ---------------------------------------------------------------------------
def _take_csr(n: int, off_p, adj_p) -> Tuple[np.ndarray, np.ndarray]:
    off = np.ctypeslib.as_array(off_p, (n + 1,)).copy()
    nnz = int(off[-1])
    adj = np.ctypeslib.as_array(adj_p, (max(nnz, 1),))[:nnz].copy()
    lib().cds_free(ctypes.cast(off_p, ctypes.c_void_p))
    lib().cds_free(ctypes.cast(adj_p, ctypes.c_void_p))
    return off.astype(np.uint64), adj.astype(np.uint32)


def gen_er(n: int, p: float, seed: int):
    off, adj = _u64p(), _u32p()
    if lib().cds_gen_er(n, p, seed, ctypes.byref(off), ctypes.byref(adj)) != 0:
        raise CdsError(4, "cds_gen_er failed")
    return _take_csr(n, off, adj)


def gen_rmat(scale: int, edge_factor: float, seed: int, n: int = 0, a=0.57, b=0.19, c=0.19):
    off, adj = _u64p(), _u32p()
    nout = ctypes.c_uint32()
    if lib().cds_gen_rmat(scale, n, edge_factor, a, b, c, seed, ctypes.byref(nout),
                          ctypes.byref(off), ctypes.byref(adj)) != 0:
        raise CdsError(4, "cds_gen_rmat failed")
    return _take_csr(nout.value, off, adj)


def gen_plant(off: np.ndarray, adj: np.ndarray, size: int, p: float, seed: int):
    n = len(off) - 1
    off = np.ascontiguousarray(off, np.uint64)
    adj = np.ascontiguousarray(adj, np.uint32)
    o2, a2 = _u64p(), _u32p()
    members = np.zeros(max(size, 1), np.uint32)
    if lib().cds_gen_plant(n, off.ctypes.data_as(_u64p), adj.ctypes.data_as(_u32p), size, p,
                           seed, ctypes.byref(o2), ctypes.byref(a2),
                           members.ctypes.data_as(_u32p)) != 0:
        raise CdsError(4, "cds_gen_plant failed")
    o, a = _take_csr(n, o2, a2)
    return o, a, members[:size]


def csr_from_edges(n: int, u, v):
    u = np.ascontiguousarray(u, np.uint32)
    v = np.ascontiguousarray(v, np.uint32)
    off, adj = _u64p(), _u32p()
    if lib().cds_csr_from_edges(n, u.ctypes.data_as(_u32p), v.ctypes.data_as(_u32p), len(u),
                                ctypes.byref(off), ctypes.byref(adj)) != 0:
        raise CdsError(4, "cds_csr_from_edges failed")
    return _take_csr(n, off, adj)


def read_adjlist(path: str):
    off, adj = _u64p(), _u32p()
    n = ctypes.c_uint32()
    if lib().cds_read_adjlist(path.encode(), ctypes.byref(n), ctypes.byref(off),
                              ctypes.byref(adj)) != 0:
        raise CdsError(4, f"cannot read {path}")
    return _take_csr(n.value, off, adj)


def write_adjlist(path: str, off: np.ndarray, adj: np.ndarray) -> None:
    off = np.ascontiguousarray(off, np.uint64)
    adj = np.ascontiguousarray(adj, np.uint32)
    if lib().cds_write_adjlist(path.encode(), len(off) - 1, off.ctypes.data_as(_u64p),
                               adj.ctypes.data_as(_u32p)) != 0:
        raise CdsError(4, f"cannot write {path}")


def write_csr_binary(path: str, off: np.ndarray, adj: np.ndarray) -> None:
    """Writes a CSR as a binary cache file (cds_write_csr_binary)."""
    off = np.ascontiguousarray(off, np.uint64)
    adj = np.ascontiguousarray(adj, np.uint32)
    if lib().cds_write_csr_binary(path.encode(), len(off) - 1, off.ctypes.data_as(_u64p),
                                  adj.ctypes.data_as(_u32p)) != 0:
        raise CdsError(4, f"cannot write {path}")


# ---------------------------------------------------------------------------
# device-side engine
# ---------------------------------------------------------------------------
@dataclass
class Solution:
    """Answer of one solve; density is the exact fraction num/den."""
    num: int
    den: int
    vertices: np.ndarray
    total_cliques: int
    max_core: int
    core_threshold: int
    core_density: Tuple[int, int]
    core_size: int
    core_cliques: int
    pruned_edges: int
    n_components: int
    flows: int
    early_stopped: bool
    peel_levels: int
    times_ms: dict = field(default_factory=dict)
    queue_ms: float = 0.0    # server: submission to the start of its batch
    service_ms: float = 0.0  # server: start of its batch to its answer
    upper_bound: Tuple[int, int] = (0, 1)  # proven upper bound of the optimum (num, den)
    bound_lb: List[float] = field(default_factory=list)  # per component: lb= line
    bound_ub: List[float] = field(default_factory=list)  # per component: ub= line

    @property
    def density(self) -> Fraction:
        return Fraction(self.num, self.den) if self.den else Fraction(0)

    @property
    def density_gap(self) -> Fraction:
        """Proven upper bound of the optimum minus the answer's density
        (zero for an exact answer)."""
        ub = Fraction(*self.upper_bound) if self.upper_bound[1] else Fraction(0)
        return ub - self.density


def _solution(r: Result) -> Solution:
    verts = np.ctypeslib.as_array(r.vertices, (r.size,)).copy() if r.size else np.zeros(0, np.uint32)
    sol = Solution(int(r.num), int(r.den), verts.astype(np.uint32), int(r.total_cliques),
                   int(r.max_core), int(r.core_threshold), (int(r.core_num), int(r.core_den)),
                   int(r.core_size), int(r.core_cliques), int(r.pruned_edges),
                   int(r.n_components), int(r.flows), bool(r.early_stopped), int(r.peel_levels),
                   {STAGES[i]: float(r.t_ms[i]) for i in range(8)}, float(r.t_queue_ms),
                   float(r.t_service_ms), (int(r.ub_num), int(r.ub_den)),
                   [float(r.bound_lb[i]) for i in range(r.n_bounds)],
                   [float(r.bound_ub[i]) for i in range(r.n_bounds)])
    lib().cds_result_free(ctypes.byref(r))
    return sol


def make_params(k: int, p_size: int = 8000, cp_size: int = 16000, gl_buffer_size: int = 0,
                partition_size: int = 30000, early_stop: int = -1, search: str = "dinkelbach") -> Params:
    return Params(k, p_size, cp_size, gl_buffer_size, partition_size, early_stop, SEARCH[search])


class Graph:
    def __init__(self, ctx: "Context", handle: int):
        self.ctx = ctx
        self.handle = ctypes.c_void_p(handle)
        n, m, d = ctypes.c_uint32(), ctypes.c_uint64(), ctypes.c_uint32()
        lib().cds_graph_info(self.handle, ctypes.byref(n), ctypes.byref(m), ctypes.byref(d))
        self.n, self.m, self.max_degree = n.value, m.value, d.value

    def csr(self) -> Tuple[np.ndarray, np.ndarray]:
        """The graph's canonical CSR, copied back from the device."""
        off = np.zeros(self.n + 1, np.uint64)
        adj = np.zeros(max(2 * self.m, 1), np.uint32)
        self.ctx._check(lib().cds_graph_download(self.handle, off.ctypes.data_as(_u64p),
                                                 adj.ctypes.data_as(_u32p)), "cds_graph_download")
        return off, adj[:2 * self.m]

    def free(self) -> None:
        if self.handle:
            lib().cds_graph_free(self.handle)
            self.handle = ctypes.c_void_p(None)

    def __del__(self):
        try:
            if self.handle and self.ctx.handle:
                self.free()
        except Exception:
            pass


CONFIG_COMPACT_PEEL = 1  # cds.h CDS_CONFIG_COMPACT_PEEL
CONFIG_WIDE_FLOW = 2     # cds.h CDS_CONFIG_WIDE_FLOW
CONFIG_WIDE_CLIQUE_IDS = 4  # cds.h CDS_CONFIG_WIDE_CLIQUE_IDS


class Context:
    """A CUDA device with its streams and memory pool (cds_create)."""

    def __init__(self, device: int = 0, mem_budget: int = 0, streams: int = 0, flags: int = 0):
        h = ctypes.c_void_p()
        st = lib().cds_create(ctypes.byref(Config(device, mem_budget, streams, flags)), ctypes.byref(h))
        if st != 0:
            raise CdsError(st, "cds_create failed")
        self.handle = h

    def _check(self, st: int, what: str) -> None:
        if st != 0:
            raise CdsError(st, f"{what}: {lib().cds_last_error(self.handle).decode()}")

    def close(self) -> None:
        if self.handle:
            lib().cds_destroy(self.handle)
            self.handle = ctypes.c_void_p(None)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def profile(self, on: bool = True) -> None:
        """Bracket the main kernels with device events (cds_profile)."""
        self._check(lib().cds_profile(self.handle, 1 if on else 0), "cds_profile")

    def profile_read(self) -> dict:
        """{kernel: (launches, total_ms)} since the last read."""
        import json
        buf = ctypes.create_string_buffer(1 << 16)
        self._check(lib().cds_profile_read(self.handle, buf, len(buf)), "cds_profile_read")
        return {k: (int(v[0]), float(v[1])) for k, v in json.loads(buf.value.decode()).items()}

    def mem_usage(self) -> Tuple[int, int]:
        a, b = ctypes.c_uint64(), ctypes.c_uint64()
        lib().cds_mem_usage(self.handle, ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    def graph(self, off: np.ndarray, adj: np.ndarray) -> Graph:
        off = np.ascontiguousarray(off, np.uint64)
        adj = np.ascontiguousarray(adj, np.uint32)
        h = ctypes.c_void_p()
        self._check(lib().cds_graph_from_csr(self.handle, off.ctypes.data_as(_u64p),
                                             adj.ctypes.data_as(_u32p), len(off) - 1,
                                             ctypes.byref(h)), "cds_graph_from_csr")
        return Graph(self, h.value)

    def graph_ptr(self, off_ptr: int, adj_ptr: int, n: int) -> Graph:
        """Graph from host CSR buffers given by address (e.g. pinned tensors)."""
        h = ctypes.c_void_p()
        self._check(lib().cds_graph_from_csr(self.handle, ctypes.cast(off_ptr, _u64p),
                                             ctypes.cast(adj_ptr, _u32p), n, ctypes.byref(h)),
                    "cds_graph_from_csr")
        return Graph(self, h.value)

    def load(self, path: str) -> Graph:
        h = ctypes.c_void_p()
        self._check(lib().cds_graph_load_file(self.handle, path.encode(), ctypes.byref(h)),
                    "cds_graph_load_file")
        return Graph(self, h.value)

    def list_cliques(self, g: Graph, k: int, p_size: int = 0, cp_size: int = 0,
                     degrees: bool = True):
        cnt = ctypes.c_uint64()
        deg = np.zeros(max(g.n, 1), np.uint64)
        self._check(lib().cds_list_cliques(self.handle, g.handle, k, p_size, cp_size,
                                           ctypes.byref(cnt),
                                           deg.ctypes.data_as(_u64p) if degrees else None),
                    "cds_list_cliques")
        return cnt.value, deg[:g.n]

    def clique_core(self, g: Graph, k: int, gl_buffer_size: int = 0):
        core = np.zeros(max(g.n, 1), np.uint64)
        mx, cnt = ctypes.c_uint64(), ctypes.c_uint64()
        self._check(lib().cds_clique_core(self.handle, g.handle, k, gl_buffer_size,
                                          core.ctypes.data_as(_u64p), ctypes.byref(mx),
                                          ctypes.byref(cnt)), "cds_clique_core")
        return core[:g.n], mx.value, cnt.value

    def densest_core(self, g: Graph, k: int):
        t, a, b = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        inc = np.zeros(max(g.n, 1), np.uint8)
        self._check(lib().cds_densest_core(self.handle, g.handle, k, ctypes.byref(t),
                                           ctypes.byref(a), ctypes.byref(b),
                                           inc.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))),
                    "cds_densest_core")
        return t.value, (a.value, b.value), inc[:g.n].astype(bool)

    def components(self, g: Graph, k: int):
        """Core cliques, pruned edges and the component table
        [(first, size, cliques), ...] of the densest core."""
        cc, pe, cnt = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint32()
        self._check(lib().cds_components(self.handle, g.handle, k, ctypes.byref(cc), ctypes.byref(pe),
                                         ctypes.byref(cnt), None, None, None, 0), "cds_components")
        m = cnt.value
        first = np.zeros(max(m, 1), np.uint32)
        size = np.zeros(max(m, 1), np.uint64)
        cl = np.zeros(max(m, 1), np.uint64)
        self._check(lib().cds_components(self.handle, g.handle, k, ctypes.byref(cc), ctypes.byref(pe),
                                         ctypes.byref(cnt), first.ctypes.data_as(_u32p),
                                         size.ctypes.data_as(_u64p), cl.ctypes.data_as(_u64p), m),
                    "cds_components")
        return {"core_cliques": cc.value, "pruned_edges": pe.value,
                "components": [(int(first[i]), int(size[i]), int(cl[i])) for i in range(m)]}

    def solve(self, g: Graph, k: int, p_size: int = 8000, cp_size: int = 16000,
              gl_buffer_size: int = 0, partition_size: int = 30000, early_stop: int = -1,
              search: str = "dinkelbach") -> Solution:
        r = Result()
        p = make_params(k, p_size, cp_size, gl_buffer_size, partition_size, early_stop, search)
        self._check(lib().cds_solve(self.handle, g.handle, ctypes.byref(p), ctypes.byref(r)),
                    "cds_solve")
        return _solution(r)

    def solve_batch(self, jobs: Sequence[Tuple[Graph, Params]]) -> List[Solution]:
        arr = (Job * len(jobs))()
        for i, (g, p) in enumerate(jobs):
            arr[i].graph = g.handle
            arr[i].params = p
        res = (Result * len(jobs))()
        self._check(lib().cds_solve_batch(self.handle, arr, len(jobs), res), "cds_solve_batch")
        return [_solution(res[i]) for i in range(len(jobs))]

    def autotune(self, graphs: Sequence[Graph], k: int, cache_path: Optional[str] = None) -> None:
        """Time the launch shapes for clique size k on the sample graphs and
        keep the fastest in this context (cds_autotune); with cache_path the
        result is written as "k key value" lines, and when the file already
        holds lines for k they are loaded and nothing is timed.  Keys: list_warp_block,
        list_warp_dmax, list_team_block, flow_rounds, flow_block, peel_chunk,
        flow_warm (balancing passes before each max-flow; -1: by network
        size), peel_order, flow_inc_per_block, peel_static."""
        arr = (ctypes.c_void_p * len(graphs))(*[g.handle.value for g in graphs])
        self._check(lib().cds_autotune(self.handle, arr, len(graphs), k,
                                       cache_path.encode() if cache_path else None),
                    "cds_autotune")

    def server(self, max_batch: int = 64, mem_budget: int = 0, max_inflight: int = 0) -> "Server":
        """Start a request server (cds_server_start): up to max_batch
        same-k requests per batch, within mem_budget bytes (0: the
        context's), max_inflight worker batches at once (0: one per context
        stream), each cooperative kernel on that share of the device."""
        return Server(self, max_batch, mem_budget, max_inflight)


class Server:
    """Continuous-batching request loop (cds_server_*)."""

    def __init__(self, ctx: Context, max_batch: int, mem_budget: int, max_inflight: int):
        self.ctx = ctx
        h = ctypes.c_void_p()
        ctx._check(lib().cds_server_start(ctx.handle, ctypes.byref(
            ServerConfig(max_batch, mem_budget, max_inflight, 0)), ctypes.byref(h)),
            "cds_server_start")
        self.handle = h

    def submit(self, g: Graph, params: Params) -> int:
        t = ctypes.c_uint64()
        self.ctx._check(lib().cds_submit(self.handle, g.handle, ctypes.byref(params),
                                         ctypes.byref(t)), "cds_submit")
        return t.value

    def submit_csr(self, off_ptr: int, adj_ptr: int, n: int, params: Params) -> int:
        """A request on a host CSR given by address (e.g. pinned tensors);
        the buffers must stay alive until the request is answered."""
        t = ctypes.c_uint64()
        self.ctx._check(lib().cds_submit_csr(self.handle, ctypes.c_void_p(off_ptr), ctypes.c_void_p(adj_ptr),
                                             n, ctypes.byref(params), ctypes.byref(t)), "cds_submit_csr")
        return t.value

    def poll(self, ticket: int) -> Optional[Solution]:
        r = Result()
        st = lib().cds_poll(self.handle, ticket, ctypes.byref(r))
        if st == CDS_ERR_NOT_READY:
            return None
        self.ctx._check(st, "cds_poll")
        return _solution(r)

    def wait(self, ticket: int) -> Solution:
        r = Result()
        self.ctx._check(lib().cds_wait(self.handle, ticket, ctypes.byref(r)), "cds_wait")
        return _solution(r)

    def stop(self) -> None:
        if self.handle:
            lib().cds_server_stop(self.handle)
            self.handle = ctypes.c_void_p(None)
