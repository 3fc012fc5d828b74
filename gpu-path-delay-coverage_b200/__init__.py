"""Python binding of the B200 path-delay-fault grader (ctypes over include/pdf.h).

The product is the C ABI in libpdf_b200.so (CUDA kernels for sm_100a and a
C++ host layer).  This module only declares that ABI for Python callers
(tests, bench.py, the serving loop) and adds numpy/torch conveniences.  It
never computes a grading result itself: if the library is missing it raises.

Reference interface mirrored (lordofhyphens/gpu-path-delay-coverage):
``Circuit`` = GPU_Circuit after ``copy()`` (main.cu:137), ``State`` = the
persistent first-detect list and totals (main.cu:141,169,224), ``grade`` = one
pass of the chunk loop (main.cu:171-231), ``Circuit.sim/mark/merge/cover`` =
gpuRunSimulation / gpuMarkPaths / gpuMergeSegments<1> / gpuCountPaths<1>.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpdf_b200.so")
# the seeded workload generator alone (no CUDA): gen_netlist / gen_pairs
GEN_LIB_PATH = os.path.join(_HERE, "libpdf_gen.so")

# gate codes (pdf.h)
UNKN, INPT, AND, NAND, OR, NOR, XOR, XNOR, BUFF, NOT, FROM, DFF = range(12)
S0, S1, T0, T1 = range(4)
MARK_DEFAULT, MARK_ROBUST, MARK_FIXED_ROBUST, MARK_FIXED_NONROBUST = 0, 1, 2, 3
FLAG_OVERFLOW = 1
BATCH_APPEND, BATCH_NO_GRAPH = 1, 2
INJECT_DEVICE_ALLOC, INJECT_HOST_ALLOC = 1, 2
BENCH_BRANCHES = 1
NONE = 0xFFFFFFFF

STATUS = {0: "OK", 1: "EINVAL", 2: "ENOMEM", 3: "EOVERFLOW", 4: "ETIMEOUT", 5: "ECUDA",
          6: "ENOTSUP", 7: "EBUSY", 8: "ENODEV", 9: "ELIMIT"}


class PdfError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        super().__init__(f"{what}: {STATUS.get(status, status)}")


class Netlist_t(C.Structure):
    _fields_ = [("n_gates", C.c_uint32), ("n_levels", C.c_uint32),
                ("level_offsets", C.POINTER(C.c_uint32)), ("type", C.POINTER(C.c_uint8)),
                ("po", C.POINTER(C.c_uint8)), ("nfi", C.POINTER(C.c_uint32)),
                ("nfo", C.POINTER(C.c_uint32)), ("edge_offset", C.POINTER(C.c_uint64)),
                ("edges", C.POINTER(C.c_uint32)), ("n_edges", C.c_uint64)]


class Pairs_t(C.Structure):
    _fields_ = [("v", C.c_void_p), ("t", C.c_void_p), ("n_pairs", C.c_uint64),
                ("ld", C.c_uint64), ("on_device", C.c_int)]


class Outputs_t(C.Structure):
    _fields_ = [("sim_v", C.c_void_p), ("sim_t", C.c_void_p), ("mark", C.c_void_p),
                ("ld", C.c_uint64), ("on_device", C.c_int)]


class Totals_t(C.Structure):
    _fields_ = [("lo", C.c_uint64), ("hi", C.c_uint64), ("pairs", C.c_uint64),
                ("flags", C.c_uint32), ("reserved", C.c_uint32)]

    @property
    def value(self) -> int:
        return (self.hi << 64) | self.lo


class CircuitOpts_t(C.Structure):
    _fields_ = [("device", C.c_int), ("mark_mode", C.c_int), ("max_pairs", C.c_uint32),
                ("tile_words", C.c_uint32), ("threads", C.c_uint32), ("seg_len", C.c_uint32),
                ("wait_polls", C.c_uint32), ("reserved", C.c_uint32)]


class BatchJob_t(C.Structure):
    _fields_ = [("circuit", C.c_void_p), ("state", C.c_void_p), ("pairs", Pairs_t), ("pair_base", C.c_uint64)]


class BatchInfo_t(C.Structure):
    _fields_ = [("n_jobs", C.c_uint32), ("tile_words", C.c_uint32), ("threads", C.c_uint32),
                ("ctas", C.c_uint32), ("gate_evals", C.c_uint64), ("device_bytes", C.c_uint64),
                ("launches", C.c_uint32), ("forward_launches", C.c_uint32)]


class ServerOpts_t(C.Structure):
    _fields_ = [("device", C.c_int), ("mark_mode", C.c_int), ("tile_words", C.c_uint32),
                ("batch_pairs", C.c_uint32), ("max_jobs", C.c_uint32), ("workers", C.c_uint32),
                ("hbm_budget", C.c_uint64)]


class ServerStats_t(C.Structure):
    _fields_ = [("jobs_done", C.c_uint64), ("jobs_active", C.c_uint64), ("jobs_queued", C.c_uint64),
                ("batches", C.c_uint64), ("steps", C.c_uint64), ("gate_evals", C.c_uint64),
                ("busy_s", C.c_double), ("lat_p50_ms", C.c_double), ("lat_p99_ms", C.c_double),
                ("lat_max_ms", C.c_double), ("bytes_in_use", C.c_uint64), ("launches", C.c_uint64),
                ("gpu_s", C.c_double)]


class CircuitInfo_t(C.Structure):
    _fields_ = [("n_gates", C.c_uint32), ("n_levels", C.c_uint32), ("n_pi", C.c_uint32),
                ("n_po", C.c_uint32), ("max_level_width", C.c_uint32), ("max_nfi", C.c_uint32),
                ("max_nfo", C.c_uint32), ("tile_words", C.c_uint32), ("threads", C.c_uint32),
                ("n_edges", C.c_uint64), ("device_bytes", C.c_uint64), ("max_pairs", C.c_uint64),
                ("seg_len", C.c_uint32), ("reserved", C.c_uint32), ("n_segments", C.c_uint64)]


class GenParams_t(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("n_gates", C.c_uint32), ("n_pi", C.c_uint32),
                ("n_po", C.c_uint32), ("depth", C.c_uint32), ("fanin_min", C.c_uint32),
                ("fanin_max", C.c_uint32), ("fanout_dist", C.c_uint32), ("zipf_s", C.c_double),
                ("fanout_max", C.c_uint32), ("type_mask", C.c_uint32), ("reserved", C.c_uint32 * 4)]


_lib = None

# (name, restype, argtypes) of every symbol include/pdf.h declares.
ABI = [
    ("pdf_status_string", C.c_char_p, [C.c_int]),
    ("pdf_abi_version", C.c_int, []),
    ("pdf_last_error", C.c_char_p, []),
    ("pdf_netlist_check", C.c_int, [C.POINTER(Netlist_t), C.c_char_p, C.c_size_t]),
    ("pdf_test_inject", C.c_int, [C.c_int, C.c_uint32]),
    ("pdf_circuit_create", C.c_int, [C.POINTER(Netlist_t), C.POINTER(CircuitOpts_t), C.POINTER(C.c_void_p)]),
    ("pdf_circuit_destroy", None, [C.c_void_p]),
    ("pdf_circuit_query", C.c_int, [C.c_void_p, C.POINTER(CircuitInfo_t)]),
    ("pdf_state_create", C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    ("pdf_state_destroy", None, [C.c_void_p]),
    ("pdf_state_reset", C.c_int, [C.c_void_p]),
    ("pdf_state_reset_async", C.c_int, [C.c_void_p, C.c_void_p]),
    ("pdf_state_reserve", C.c_int, [C.c_void_p, C.c_uint64]),
    ("pdf_state_profile", C.c_int, [C.c_void_p, C.c_int]),
    ("pdf_state_profile_read", C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_uint32)]),
    ("pdf_state_snapshot", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(Totals_t)]),
    ("pdf_state_snapshot_on", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(Totals_t), C.c_void_p]),
    ("pdf_state_restore", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(Totals_t)]),
    ("pdf_grade_async", C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(Pairs_t), C.c_uint64,
                                  C.POINTER(Outputs_t), C.c_void_p]),
    ("pdf_grade", C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(Pairs_t), C.c_uint64,
                            C.POINTER(Outputs_t), C.POINTER(Totals_t), C.c_void_p]),
    ("pdf_grade_mark_async", C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(Pairs_t), C.c_uint64,
                                       C.POINTER(Outputs_t), C.c_void_p]),
    ("pdf_grade_cover_async", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    ("pdf_state_first_copy", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    ("pdf_sim", C.c_int, [C.c_void_p, C.POINTER(Pairs_t), C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p]),
    ("pdf_mark", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint64,
                           C.c_void_p]),
    ("pdf_merge", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint64,
                            C.c_uint64, C.c_void_p]),
    ("pdf_cover", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint64,
                            C.POINTER(Totals_t), C.c_void_p]),
    ("pdf_cover_counts", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint64,
                                   C.c_void_p, C.POINTER(Totals_t), C.c_void_p]),
    ("pdf_cover_noalloc", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint64, C.c_void_p,
                                    C.c_void_p, C.POINTER(Totals_t), C.c_void_p]),
    ("pdf_batch_create", C.c_int, [C.POINTER(BatchJob_t), C.c_uint32, C.c_uint32, C.POINTER(C.c_void_p)]),
    ("pdf_batch_destroy", None, [C.c_void_p]),
    ("pdf_batch_rebind", C.c_int, [C.c_void_p, C.POINTER(BatchJob_t), C.c_uint32, C.c_uint32]),
    ("pdf_batch_query", C.c_int, [C.c_void_p, C.POINTER(BatchInfo_t)]),
    ("pdf_batch_run_async", C.c_int, [C.c_void_p, C.c_void_p]),
    ("pdf_batch_run", C.c_int, [C.c_void_p, C.c_void_p]),
    ("pdf_batch_profile", C.c_int, [C.c_void_p, C.c_int]),
    ("pdf_batch_profile_read", C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    ("pdf_batch_autotune", C.c_int, [C.POINTER(C.POINTER(Netlist_t)), C.POINTER(C.c_uint64), C.c_uint32,
                                     C.POINTER(CircuitOpts_t), C.c_uint32, C.POINTER(CircuitOpts_t),
                                     C.POINTER(C.c_float)]),
    ("pdf_server_create", C.c_int, [C.POINTER(ServerOpts_t), C.POINTER(C.c_void_p)]),
    ("pdf_server_destroy", None, [C.c_void_p]),
    ("pdf_server_submit", C.c_int, [C.c_void_p, C.POINTER(Netlist_t), C.c_void_p, C.c_void_p, C.c_uint64,
                                    C.c_uint64, C.POINTER(C.c_uint64)]),
    ("pdf_server_step", C.c_int, [C.c_void_p, C.POINTER(C.c_uint32)]),
    ("pdf_server_result", C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(Totals_t), C.c_void_p, C.c_void_p]),
    ("pdf_server_query", C.c_int, [C.c_void_p, C.POINTER(ServerStats_t)]),
    ("pdf_gen_netlist", C.c_int, [C.POINTER(GenParams_t), C.POINTER(C.c_void_p)]),
    ("pdf_netbuf_from", C.c_int, [C.POINTER(Netlist_t), C.POINTER(C.c_void_p)]),
    ("pdf_netbuf_view", None, [C.c_void_p, C.POINTER(Netlist_t)]),
    ("pdf_netbuf_free", None, [C.c_void_p]),
    ("pdf_gen_pairs", C.c_int, [C.c_uint64, C.c_uint32, C.c_uint64, C.c_uint64, C.c_void_p, C.c_void_p]),
    ("pdf_pairs_from_vectors", C.c_int, [C.c_void_p, C.c_uint32, C.c_uint64, C.c_uint64, C.c_void_p,
                                         C.c_void_p]),
    ("pdf_mark_forward", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint64,
                                   C.c_void_p]),
    ("pdf_read_bench", C.c_int, [C.c_char_p, C.c_uint32, C.POINTER(C.c_void_p), C.c_char_p, C.c_size_t]),
    ("pdf_write_bench", C.c_int, [C.POINTER(Netlist_t), C.c_char_p]),
    ("pdf_read_level", C.c_int, [C.c_char_p, C.POINTER(C.c_void_p), C.c_char_p, C.c_size_t]),
    ("pdf_write_level", C.c_int, [C.POINTER(Netlist_t), C.c_char_p]),
    ("pdf_vectors_dim", C.c_int, [C.c_char_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint32)]),
    ("pdf_vectors_read", C.c_int, [C.c_char_p, C.c_uint32, C.c_uint64, C.c_void_p]),
    ("pdf_dump_sim", C.c_int, [C.c_char_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint64, C.c_uint64,
                               C.c_uint64, C.c_int]),
    ("pdf_dump_mark", C.c_int, [C.c_char_p, C.c_void_p, C.c_uint32, C.c_uint64, C.c_uint64, C.c_uint64,
                                C.c_int]),
    ("pdf_dump_merge", C.c_int, [C.c_char_p, C.c_void_p, C.c_void_p, C.c_uint32]),
    ("pdf_dump_cover", C.c_int, [C.c_char_p, C.c_void_p, C.c_uint32, C.c_uint64, C.c_uint64, C.c_int]),
    ("pdf_dump_segments", C.c_int, [C.c_char_p, C.c_void_p, C.c_uint32, C.c_uint64, C.c_void_p, C.c_void_p]),
    ("pdf_circuit_segments", C.c_int, [C.c_void_p, C.c_void_p]),
]


def lib() -> C.CDLL:
    """The grader library.  Raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with __graft_entry__.build()")
        L = C.CDLL(LIB_PATH)
        for name, res, args in ABI:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


_gen_lib = None
GEN_ABI = [("pdf_gen_netlist", C.c_int, [C.POINTER(GenParams_t), C.POINTER(C.c_void_p)]),
           ("pdf_netbuf_view", None, [C.c_void_p, C.POINTER(Netlist_t)]),
           ("pdf_netbuf_free", None, [C.c_void_p]),
           ("pdf_gen_pairs", C.c_int, [C.c_uint64, C.c_uint32, C.c_uint64, C.c_uint64, C.c_void_p, C.c_void_p])]


def gen_lib() -> C.CDLL:
    """The workload generator library (host code only; loads no CUDA code)."""
    global _gen_lib
    if _gen_lib is None:
        if not os.path.exists(GEN_LIB_PATH):
            raise RuntimeError(f"{GEN_LIB_PATH} is missing: build it with __graft_entry__.build()")
        L = C.CDLL(GEN_LIB_PATH)
        for name, res, args in GEN_ABI:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _gen_lib = L
    return _gen_lib


def check(status: int, what: str) -> None:
    if status != 0:
        if status in (2, 5) and _lib is not None:  # ENOMEM, ECUDA: name the CUDA call behind it
            what = f"{what} [{_lib.pdf_last_error().decode(errors='replace')}]"
        raise PdfError(status, what)


def _ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


# ---------------------------------------------------------------------------
# Netlists


class Netlist:
    """A host netlist in the pdf_netlist layout, held as numpy arrays."""

    def __init__(self, level_offsets, type_, po, nfi, nfo, edge_offset, edges):
        self.level_offsets = np.ascontiguousarray(level_offsets, dtype=np.uint32)
        self.type = np.ascontiguousarray(type_, dtype=np.uint8)
        self.po = np.ascontiguousarray(po, dtype=np.uint8)
        self.nfi = np.ascontiguousarray(nfi, dtype=np.uint32)
        self.nfo = np.ascontiguousarray(nfo, dtype=np.uint32)
        self.edge_offset = np.ascontiguousarray(edge_offset, dtype=np.uint64)
        self.edges = np.ascontiguousarray(edges, dtype=np.uint32)
        self._view = Netlist_t(len(self.type), len(self.level_offsets) - 1,
                               _ptr(self.level_offsets, C.c_uint32), _ptr(self.type, C.c_uint8),
                               _ptr(self.po, C.c_uint8), _ptr(self.nfi, C.c_uint32),
                               _ptr(self.nfo, C.c_uint32), _ptr(self.edge_offset, C.c_uint64),
                               _ptr(self.edges if len(self.edges) else np.zeros(1, np.uint32), C.c_uint32),
                               len(self.edges))

    @property
    def n_gates(self) -> int:
        return len(self.type)

    @property
    def n_levels(self) -> int:
        return len(self.level_offsets) - 1

    @property
    def n_pi(self) -> int:
        return int(self.level_offsets[1])

    def view(self) -> Netlist_t:
        return self._view

    def fanins(self, g: int) -> np.ndarray:
        o = int(self.edge_offset[g])
        return self.edges[o:o + int(self.nfi[g])]

    def fanouts(self, g: int) -> np.ndarray:
        o = int(self.edge_offset[g]) + int(self.nfi[g])
        return self.edges[o:o + int(self.nfo[g])]

    def check(self) -> tuple[int, str]:
        buf = C.create_string_buffer(256)
        st = lib().pdf_netlist_check(C.byref(self._view), buf, 256)
        return st, buf.value.decode()

    @classmethod
    def from_fanins(cls, levels: list[list[int]], types: dict | list, fanins: dict | list,
                    pos) -> "Netlist":
        """Build from per-gate fan-in lists; fan-out lists are derived.
        `levels` lists gate ids per level (ids must already be in level order)."""
        G = sum(len(l) for l in levels)
        lo = [0]
        for l in levels:
            lo.append(lo[-1] + len(l))
        fin = [list(fanins[g]) if g < len(fanins) else [] for g in range(G)]
        fo = [[] for _ in range(G)]
        for g in range(G):
            for f in fin[g]:
                fo[f].append(g)
        nfi = [len(x) for x in fin]
        nfo = [len(x) for x in fo]
        eo, edges = [], []
        for g in range(G):
            eo.append(len(edges))
            edges.extend(fin[g])
            edges.extend(fo[g])
        po = np.zeros(G, np.uint8)
        for g in pos:
            po[g] = 1
        return cls(lo, [types[g] for g in range(G)], po, nfi, nfo, eo, edges)


@dataclass
class GenParams:
    seed: int
    n_gates: int
    n_pi: int
    n_po: int
    depth: int
    fanin_min: int = 1
    fanin_max: int = 4
    fanout_dist: int = 0          # 0 geometric, 1 Zipf
    zipf_s: float = 1.5
    fanout_max: int = 0
    type_mask: int = 0


def gen_netlist(p: GenParams) -> Netlist:
    """Seeded synthetic netlist (pdf_gen_netlist)."""
    gp = GenParams_t(p.seed, p.n_gates, p.n_pi, p.n_po, p.depth, p.fanin_min, p.fanin_max,
                     p.fanout_dist, p.zipf_s, p.fanout_max, p.type_mask)
    h = C.c_void_p()
    check(gen_lib().pdf_gen_netlist(C.byref(gp), C.byref(h)), "pdf_gen_netlist")
    return _take_netbuf(h, gen_lib())


def _take_netbuf(h, L=None) -> Netlist:
    """Copy a netlist owned by library L (the grader by default) into a
    Netlist and free it there."""
    L = L or lib()
    try:
        v = Netlist_t()
        L.pdf_netbuf_view(h, C.byref(v))
        G, Lv, E = v.n_gates, v.n_levels, v.n_edges

        def arr(ptr, n, dt):
            return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dt, copy=True)

        return Netlist(arr(v.level_offsets, Lv + 1, np.uint32), arr(v.type, G, np.uint8),
                       arr(v.po, G, np.uint8), arr(v.nfi, G, np.uint32), arr(v.nfo, G, np.uint32),
                       arr(v.edge_offset, G, np.uint64),
                       arr(v.edges, E, np.uint32) if E else np.zeros(0, np.uint32))
    finally:
        L.pdf_netbuf_free(h)


def _read_netlist(call, *args) -> Netlist:
    h = C.c_void_p()
    msg = C.create_string_buffer(512)
    st = call(*args, C.byref(h), msg, len(msg))
    if st != 0:
        raise PdfError(st, msg.value.decode(errors="replace"))
    return _take_netbuf(h)


def read_bench(path: str, branches: bool = False) -> Netlist:
    """ISCAS .bench netlist, levelized, flip-flops cut for full scan (pdf_read_bench)."""
    return _read_netlist(lib().pdf_read_bench, os.fsencode(path), BENCH_BRANCHES if branches else 0)


def read_level(path: str) -> Netlist:
    """Levelized text netlist (pdf_read_level)."""
    return _read_netlist(lib().pdf_read_level, os.fsencode(path))


def write_bench(nl: Netlist, path: str) -> None:
    check(lib().pdf_write_bench(C.byref(nl.view()), os.fsencode(path)), "pdf_write_bench")


def write_level(nl: Netlist, path: str) -> None:
    check(lib().pdf_write_level(C.byref(nl.view()), os.fsencode(path)), "pdf_write_level")


def read_vectors(path: str) -> np.ndarray:
    """A vector file as vec[n_pi][n_vec] of 0/1 bytes (pdf_vectors_dim + pdf_vectors_read)."""
    n, w = C.c_uint64(), C.c_uint32()
    check(lib().pdf_vectors_dim(os.fsencode(path), C.byref(n), C.byref(w)), "pdf_vectors_dim")
    vec = np.zeros((w.value, n.value), np.uint8)
    check(lib().pdf_vectors_read(os.fsencode(path), w.value, n.value, vec.ctypes.data), "pdf_vectors_read")
    return vec


def dump_sim(path: str, sim_v: np.ndarray, sim_t: np.ndarray, n_pairs: int, pair_base: int = 0,
             append: bool = False) -> None:
    """gpusim-p2.log layout from host planes [n_gates][ld] (pdf_dump_sim)."""
    sim_v = np.ascontiguousarray(sim_v, np.uint32)
    sim_t = np.ascontiguousarray(sim_t, np.uint32)
    check(lib().pdf_dump_sim(os.fsencode(path), sim_v.ctypes.data, sim_t.ctypes.data, sim_v.shape[0], n_pairs,
                             sim_v.shape[1], pair_base, int(append)), "pdf_dump_sim")


def dump_mark(path: str, mark: np.ndarray, n_pairs: int, pair_base: int = 0, append: bool = False) -> None:
    """gpumark.log layout from a host plane [n_gates][ld] (pdf_dump_mark)."""
    mark = np.ascontiguousarray(mark, np.uint32)
    check(lib().pdf_dump_mark(os.fsencode(path), mark.ctypes.data, mark.shape[0], n_pairs, mark.shape[1],
                              pair_base, int(append)), "pdf_dump_mark")


def dump_merge(path: str, first_x: np.ndarray, first_y: np.ndarray) -> None:
    """gpumerge.log layout (pdf_dump_merge)."""
    fx = np.ascontiguousarray(first_x, np.uint32)
    fy = np.ascontiguousarray(first_y, np.uint32)
    check(lib().pdf_dump_merge(os.fsencode(path), fx.ctypes.data, fy.ctypes.data, len(fx)), "pdf_dump_merge")


def dump_segments(path: str, segs: np.ndarray, first_x: np.ndarray, first_y: np.ndarray) -> None:
    """gpumerge.log layout of segments (pdf_dump_segments)."""
    sg = np.ascontiguousarray(segs, np.uint32)
    fx = np.ascontiguousarray(first_x, np.uint32)
    fy = np.ascontiguousarray(first_y, np.uint32)
    check(lib().pdf_dump_segments(os.fsencode(path), sg.ctypes.data, sg.shape[1], sg.shape[0], fx.ctypes.data,
                                  fy.ctypes.data), "pdf_dump_segments")


def inject_failures(site: int, count: int) -> None:
    """The next `count` allocations of kind `site` (INJECT_*) fail (pdf_test_inject)."""
    check(lib().pdf_test_inject(site, count), "pdf_test_inject")


def words(n_pairs: int) -> int:
    return (n_pairs + 31) // 32


def gen_pairs(seed: int, n_pi: int, n_pairs: int, ld: int | None = None) -> tuple[np.ndarray, np.ndarray]:
    """Uniform random pairs as (v, t) bit-planes [n_pi][ld] (pdf_gen_pairs)."""
    ld = ld or words(n_pairs)
    v = np.zeros((n_pi, ld), np.uint32)
    t = np.zeros((n_pi, ld), np.uint32)
    check(gen_lib().pdf_gen_pairs(seed, n_pi, n_pairs, ld, v.ctypes.data, t.ctypes.data), "pdf_gen_pairs")
    return v, t


def pairs_from_vectors(vec: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Reference pair formation from a vector stream vec[n_pi][n_vec] of 0/1 bytes."""
    vec = np.ascontiguousarray(vec, dtype=np.uint8)
    n_pi, n_vec = vec.shape
    ld = words(n_vec)
    v = np.zeros((n_pi, ld), np.uint32)
    t = np.zeros((n_pi, ld), np.uint32)
    check(lib().pdf_pairs_from_vectors(vec.ctypes.data, n_pi, n_vec, ld, v.ctypes.data, t.ctypes.data),
          "pdf_pairs_from_vectors")
    return v, t


def codes_from_planes(v: np.ndarray, t: np.ndarray, n_pairs: int) -> np.ndarray:
    """Bit-planes [rows][ld] -> one code byte per (row, pair) (bit0 = v, bit1 = t)."""
    vb = np.unpackbits(np.ascontiguousarray(v).view(np.uint8), axis=1, bitorder="little")[:, :n_pairs]
    tb = np.unpackbits(np.ascontiguousarray(t).view(np.uint8), axis=1, bitorder="little")[:, :n_pairs]
    return (vb | (tb << 1)).astype(np.uint8)


def bits_from_plane(m: np.ndarray, n_pairs: int) -> np.ndarray:
    return np.unpackbits(np.ascontiguousarray(m).view(np.uint8), axis=1, bitorder="little")[:, :n_pairs]


def planes_from_codes(codes: np.ndarray, ld: int | None = None) -> tuple[np.ndarray, np.ndarray]:
    """One code byte per (row, pair) -> (v, t) bit-planes [rows][ld]."""
    codes = np.ascontiguousarray(codes, dtype=np.uint8)
    rows, n = codes.shape
    ld = ld or words(n)
    pad = ld * 32 - n
    vb = np.pad(codes & 1, ((0, 0), (0, pad)))
    tb = np.pad((codes >> 1) & 1, ((0, 0), (0, pad)))
    v = np.packbits(vb, axis=1, bitorder="little").view(np.uint32)
    t = np.packbits(tb, axis=1, bitorder="little").view(np.uint32)
    return np.ascontiguousarray(v), np.ascontiguousarray(t)


# ---------------------------------------------------------------------------
# Device objects


class Circuit:
    """A netlist uploaded to one device (pdf_circuit_create)."""

    def __init__(self, nl: Netlist, device: int = 0, mark_mode: int = MARK_DEFAULT,
                 max_pairs: int = 0, tile_words: int = 0, threads: int = 0, seg_len: int = 1,
                 wait_polls: int = 0):
        self.h = None
        self.netlist = nl
        self.mark_mode = mark_mode
        o = CircuitOpts_t(device, mark_mode, max_pairs, tile_words, threads, seg_len, wait_polls)
        h = C.c_void_p()
        check(lib().pdf_circuit_create(C.byref(nl.view()), C.byref(o), C.byref(h)), "pdf_circuit_create")
        self.h = h
        self.n_first = self.info().n_segments  # entries of a state's first-detect arrays

    def info(self) -> CircuitInfo_t:
        i = CircuitInfo_t()
        check(lib().pdf_circuit_query(self.h, C.byref(i)), "pdf_circuit_query")
        return i

    def segments(self) -> np.ndarray:
        """The segment list [n_segments][seg_len] (pdf_circuit_segments)."""
        i = self.info()
        out = np.zeros((i.n_segments, max(1, i.seg_len)), np.uint32)
        check(lib().pdf_circuit_segments(self.h, out.ctypes.data), "pdf_circuit_segments")
        return out

    def close(self):
        if self.h:
            lib().pdf_circuit_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class State:
    """First-detect ids and running total of one circuit (pdf_state_*)."""

    def __init__(self, c: Circuit):
        self.circuit = c
        h = C.c_void_p()
        check(lib().pdf_state_create(c.h, C.byref(h)), "pdf_state_create")
        self.h = h

    def reset(self):
        check(lib().pdf_state_reset(self.h), "pdf_state_reset")

    def reset_async(self, stream: int = 0):
        check(lib().pdf_state_reset_async(self.h, C.c_void_p(stream)), "pdf_state_reset_async")

    def profile(self, enable: bool):
        check(lib().pdf_state_profile(self.h, int(enable)), "pdf_state_profile")

    def profile_read(self) -> tuple[list[float], int]:
        ms = (C.c_double * 3)()
        n = C.c_uint32()
        check(lib().pdf_state_profile_read(self.h, ms, C.byref(n)), "pdf_state_profile_read")
        return list(ms), n.value

    def snapshot(self, stream: int | None = None):
        """First-detect ids and totals; with a stream, ordered on that stream
        only (pdf_state_snapshot_on) instead of after a device-wide sync."""
        G = self.circuit.n_first
        fx = np.zeros(G, np.uint32)
        fy = np.zeros(G, np.uint32)
        tot = Totals_t()
        if stream is None:
            check(lib().pdf_state_snapshot(self.h, fx.ctypes.data, fy.ctypes.data, C.byref(tot)),
                  "pdf_state_snapshot")
        else:
            check(lib().pdf_state_snapshot_on(self.h, fx.ctypes.data, fy.ctypes.data, C.byref(tot),
                                              C.c_void_p(stream)), "pdf_state_snapshot_on")
        return fx, fy, tot

    def restore(self, fx, fy, tot: Totals_t):
        fx = np.ascontiguousarray(fx, np.uint32)
        fy = np.ascontiguousarray(fy, np.uint32)
        check(lib().pdf_state_restore(self.h, fx.ctypes.data, fy.ctypes.data, C.byref(tot)),
              "pdf_state_restore")

    def close(self):
        if self.h:
            lib().pdf_state_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _addr(x) -> int:
    """Address of a numpy array or torch tensor."""
    if x is None:
        return 0
    if isinstance(x, np.ndarray):
        return x.ctypes.data
    return x.data_ptr()


def _on_device(x) -> int:
    return 0 if isinstance(x, np.ndarray) else int(x.is_cuda)


def make_pairs(v, t, n_pairs: int) -> Pairs_t:
    ld = v.shape[1]
    return Pairs_t(_addr(v), _addr(t), n_pairs, ld, _on_device(v))


def make_outputs(sim_v=None, sim_t=None, mark=None) -> Outputs_t:
    ref = next(x for x in (sim_v, sim_t, mark) if x is not None)
    return Outputs_t(_addr(sim_v), _addr(sim_t), _addr(mark), ref.shape[1], _on_device(ref))


class Batch:
    """Many (circuit, state, device pairs) jobs graded per pass (pdf_batch_*).

    jobs: (Circuit, State, v, t, n_pairs, pair_base) with v, t device tensors
    of shape [n_pi, ld]; the tensors must stay alive (and at their address)
    while the batch exists.  append: each run advances every job's pair_base
    by its pair count."""

    def __init__(self, jobs, append: bool = False, graph: bool = True):
        self.h = None
        self.jobs = list(jobs)  # keeps circuits, states and pair tensors alive
        h = C.c_void_p()
        flags = (BATCH_APPEND if append else 0) | (0 if graph else BATCH_NO_GRAPH)
        check(lib().pdf_batch_create(self._arr(self.jobs), len(self.jobs), flags, C.byref(h)), "pdf_batch_create")
        self.h = h

    @staticmethod
    def _arr(jobs):
        arr = (BatchJob_t * len(jobs))()
        for k, (c, s, v, t, n, base) in enumerate(jobs):
            arr[k] = BatchJob_t(c.h, s.h, make_pairs(v, t, n), base)
        return arr

    def rebind(self, jobs, append: bool = False):
        """Point this batch at another job list (pdf_batch_rebind); no run of
        it may be in flight."""
        jobs = list(jobs)
        check(lib().pdf_batch_rebind(self.h, self._arr(jobs), len(jobs), BATCH_APPEND if append else 0),
              "pdf_batch_rebind")
        self.jobs = jobs

    def info(self) -> BatchInfo_t:
        i = BatchInfo_t()
        check(lib().pdf_batch_query(self.h, C.byref(i)), "pdf_batch_query")
        return i

    def run_async(self, stream: int = 0):
        check(lib().pdf_batch_run_async(self.h, C.c_void_p(stream)), "pdf_batch_run_async")

    def run(self, stream: int = 0):
        check(lib().pdf_batch_run(self.h, C.c_void_p(stream)), "pdf_batch_run")

    def profile(self, enable: bool):
        check(lib().pdf_batch_profile(self.h, int(enable)), "pdf_batch_profile")

    def profile_read(self) -> tuple[float, float]:
        """(forward ms, cover ms) of the most recent run (waits for it)."""
        ms = (C.c_double * 2)()
        check(lib().pdf_batch_profile_read(self.h, ms), "pdf_batch_profile_read")
        return ms[0], ms[1]

    def close(self):
        if self.h:
            lib().pdf_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous-batching grader (pdf_server_*).  Keeps every submitted job's
    netlist and host pair planes alive until its result has been read."""

    def __init__(self, mark_mode: int = MARK_DEFAULT, batch_pairs: int = 4096, tile_words: int = 4,
                 hbm_budget: int = 0, max_jobs: int = 0, device: int = 0, workers: int = 0):
        o = ServerOpts_t(device, mark_mode, tile_words, batch_pairs, max_jobs, workers, hbm_budget)
        h = C.c_void_p()
        check(lib().pdf_server_create(C.byref(o), C.byref(h)), "pdf_server_create")
        self.h = h
        self.keep = {}

    def submit(self, nl: Netlist, v: np.ndarray, t: np.ndarray, n_pairs: int) -> int:
        v = np.ascontiguousarray(v, np.uint32)
        t = np.ascontiguousarray(t, np.uint32)
        jid = C.c_uint64()
        check(lib().pdf_server_submit(self.h, C.byref(nl.view()), v.ctypes.data, t.ctypes.data, v.shape[1],
                                      n_pairs, C.byref(jid)), "pdf_server_submit")
        self.keep[jid.value] = (nl, v, t)
        return jid.value

    def step(self) -> int:
        r = C.c_uint32()
        check(lib().pdf_server_step(self.h, C.byref(r)), "pdf_server_step")
        return r.value

    def result(self, jid: int):
        nl = self.keep[jid][0]
        fx = np.zeros(nl.n_gates, np.uint32)
        fy = np.zeros(nl.n_gates, np.uint32)
        tot = Totals_t()
        check(lib().pdf_server_result(self.h, jid, C.byref(tot), fx.ctypes.data, fy.ctypes.data),
              "pdf_server_result")
        return fx, fy, tot

    def stats(self) -> ServerStats_t:
        s = ServerStats_t()
        check(lib().pdf_server_query(self.h, C.byref(s)), "pdf_server_query")
        return s

    def close(self):
        if self.h:
            lib().pdf_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def batch_autotune(netlists, n_pairs, mark_mode: int = MARK_DEFAULT, reps: int = 3, device: int = 0,
                   threads: int = 0):
    """Best tile width and block size for grading these circuits as one batch:
    (opts, ms per pass); a nonzero `threads` fixes the block size."""
    views = [nl.view() for nl in netlists]
    ptrs = (C.POINTER(Netlist_t) * len(views))(*[C.pointer(v) for v in views])
    npairs = (C.c_uint64 * len(views))(*n_pairs)
    base = CircuitOpts_t(device, mark_mode, 0, 0, threads)
    best = CircuitOpts_t()
    ms = C.c_float()
    check(lib().pdf_batch_autotune(ptrs, npairs, len(views), C.byref(base), reps, C.byref(best), C.byref(ms)),
          "pdf_batch_autotune")
    return best, ms.value


def grade(c: Circuit, s: State, v, t, n_pairs: int, pair_base: int = 0, sim_v=None, sim_t=None,
          mark=None, stream: int = 0) -> Totals_t:
    """Grade one batch and wait; returns the batch's covered-path count."""
    pr = make_pairs(v, t, n_pairs)
    out = make_outputs(sim_v, sim_t, mark) if any(x is not None for x in (sim_v, sim_t, mark)) else None
    tot = Totals_t()
    check(lib().pdf_grade(c.h, s.h, C.byref(pr), pair_base, C.byref(out) if out else None,
                          C.byref(tot), C.c_void_p(stream)), "pdf_grade")
    return tot


def grade_async(c: Circuit, s: State, pairs: Pairs_t, pair_base: int, out: Outputs_t | None,
                stream: int = 0) -> None:
    check(lib().pdf_grade_async(c.h, s.h, C.byref(pairs), pair_base, C.byref(out) if out else None,
                                C.c_void_p(stream)), "pdf_grade_async")


def grade_mark_async(c: Circuit, s: State, pairs: Pairs_t, pair_base: int, out: Outputs_t | None,
                     stream: int = 0) -> None:
    check(lib().pdf_grade_mark_async(c.h, s.h, C.byref(pairs), pair_base, C.byref(out) if out else None,
                                     C.c_void_p(stream)), "pdf_grade_mark_async")


def grade_cover_async(c: Circuit, s: State, stream: int = 0) -> None:
    check(lib().pdf_grade_cover_async(c.h, s.h, C.c_void_p(stream)), "pdf_grade_cover_async")


def first_copy(s: State, fx, fy, to_state: bool, stream: int = 0) -> None:
    check(lib().pdf_state_first_copy(s.h, _addr(fx), _addr(fy), int(to_state), C.c_void_p(stream)),
          "pdf_state_first_copy")


def stage_sim(c: Circuit, v, t, n_pairs, sim_v, sim_t, stream: int = 0):
    pr = make_pairs(v, t, n_pairs)
    check(lib().pdf_sim(c.h, C.byref(pr), _addr(sim_v), _addr(sim_t), sim_v.shape[1], C.c_void_p(stream)),
          "pdf_sim")


def stage_mark(c: Circuit, sim_v, sim_t, mark, n_pairs, stream: int = 0):
    check(lib().pdf_mark(c.h, _addr(sim_v), _addr(sim_t), _addr(mark), n_pairs, mark.shape[1],
                         C.c_void_p(stream)), "pdf_mark")


def stage_mark_forward(c: Circuit, sim_v, sim_t, mark, n_pairs, stream: int = 0):
    """Forward marks before the removal pass (pdf_mark_forward)."""
    check(lib().pdf_mark_forward(c.h, _addr(sim_v), _addr(sim_t), _addr(mark), n_pairs, mark.shape[1],
                                 C.c_void_p(stream)), "pdf_mark_forward")


def stage_merge(c: Circuit, s: State, sim_v, mark, n_pairs, pair_base, stream: int = 0):
    check(lib().pdf_merge(c.h, s.h, _addr(sim_v), _addr(mark), n_pairs, mark.shape[1], pair_base,
                          C.c_void_p(stream)), "pdf_merge")


def stage_cover(c: Circuit, s: State, mark, n_pairs, pair_base, stream: int = 0) -> Totals_t:
    tot = Totals_t()
    check(lib().pdf_cover(c.h, s.h, _addr(mark), n_pairs, mark.shape[1], pair_base, C.byref(tot),
                          C.c_void_p(stream)), "pdf_cover")
    return tot


def stage_cover_counts(c: Circuit, s: State, mark, n_pairs, pair_base, stream: int = 0):
    """pdf_cover_counts: the chunk count and the paths each primary input
    credits to each pair, as Python ints [n_pi][n_pairs]."""
    tot = Totals_t()
    raw = np.zeros((c.netlist.n_pi, n_pairs, 2), np.uint64)
    check(lib().pdf_cover_counts(c.h, s.h, _addr(mark), n_pairs, mark.shape[1], pair_base, raw.ctypes.data,
                                 C.byref(tot), C.c_void_p(stream)), "pdf_cover_counts")
    return tot, raw


def dump_cover(path: str, raw_counts: np.ndarray, pair_base: int = 0, append: bool = False) -> None:
    """gpucover.log layout from pdf_cover_counts' array [n_pi][n_pairs][2] (pdf_dump_cover)."""
    raw = np.ascontiguousarray(raw_counts, np.uint64)
    check(lib().pdf_dump_cover(os.fsencode(path), raw.ctypes.data, raw.shape[0], raw.shape[1], pair_base,
                               int(append)), "pdf_dump_cover")


def stage_cover_noalloc(c: Circuit, mark, n_pairs, pair_base, first_x, first_y, stream: int = 0) -> Totals_t:
    """pdf_cover_noalloc: the chunk count with no allocation (fixed device scratch)."""
    tot = Totals_t()
    check(lib().pdf_cover_noalloc(c.h, _addr(mark), n_pairs, mark.shape[1], pair_base, _addr(first_x),
                                  _addr(first_y), C.byref(tot), C.c_void_p(stream)), "pdf_cover_noalloc")
    return tot


# ---------------------------------------------------------------------------
# The benchmark workloads (synthetic stand-ins; the reference ships no circuits).

SEED_BASE = 0x5EED0000
PAIR_SEED_XOR = 0x9E3779B97F4A7C15

WORKLOADS = {
    # 2,000 gates, 36 PI, 7 PO, depth 40, 1,024 pairs
    "c1": dict(gen=GenParams(SEED_BASE + 1, 2000, 36, 7, 40), pairs=1024),
    # 20,000 gates, 1,500 PI, 1,500 PO, depth 60, 32,768 pairs
    "c2": dict(gen=GenParams(SEED_BASE + 2, 20000, 1500, 1500, 60), pairs=32768),
    # 1,000,000 gates, 8,192 PI/PO, depth 200, Zipf(1.5) fan-out capped at 256, 262,144 pairs
    "c3": dict(gen=GenParams(SEED_BASE + 3, 1_000_000, 8192, 8192, 200, fanout_dist=1, zipf_s=1.5,
                             fanout_max=256), pairs=262144),
}


def batch_workload(seed: int = SEED_BASE + 4, count: int = 256):
    """The mixed-size batch: `count` netlists with gate counts log-uniform in
    500..200,000 (PI and PO about G/13, at least 16), depth uniform in
    20..150, and pair counts log-uniform in 1,024..65,536.  Returns a list of
    (GenParams, n_pairs)."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        g = int(round(np.exp(rng.uniform(np.log(500), np.log(200000)))))
        depth = int(rng.integers(20, 151))
        g = max(g, depth * 4)
        pio = max(16, g // 13)
        n = int(round(np.exp(rng.uniform(np.log(1024), np.log(65536)))))
        out.append((GenParams(seed * 1000 + k, g, pio, pio, depth), n))
    return out


def pair_seed(gen_seed: int) -> int:
    return gen_seed ^ PAIR_SEED_XOR
