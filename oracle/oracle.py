"""ctypes wrapper of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, as the checker.  The product never uses it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        L.pdfo_lut2.restype = C.c_uint8
        L.pdfo_lut2.argtypes = [C.c_int, C.c_uint8, C.c_uint8]
        L.pdfo_stable.restype = C.c_uint8
        L.pdfo_stable.argtypes = [C.c_uint8, C.c_uint8]
        L.pdfo_not.restype = C.c_uint8
        L.pdfo_not.argtypes = [C.c_uint8]
        L.pdfo_sens.restype = C.c_int
        L.pdfo_sens.argtypes = [C.c_int, C.c_int, C.c_uint8, C.c_uint8]
        L.pdfo_sim.argtypes = [P, P, C.c_uint64, P, C.c_int]
        L.pdfo_sim_mode.argtypes = [P, P, C.c_uint64, P, C.c_int, C.c_int]
        L.pdfo_sim_vectors.argtypes = [P, P, C.c_uint64, P, C.c_int]
        L.pdfo_mark.argtypes = [P, P, C.c_uint64, C.c_int, P, C.c_int, C.c_int]
        L.pdfo_merge.argtypes = [P, P, P, C.c_uint64, C.c_uint64, P, P, C.c_int]
        L.pdfo_cover.argtypes = [P, P, C.c_uint64, C.c_uint64, P, P, P, P, P, C.c_int]
        L.pdfo_cover_counts.argtypes = [P, P, C.c_uint64, C.c_uint64, P, P, P, P, P, P, C.c_int]
        L.pdfo_cover_counts.restype = C.c_int
        L.pdfo_grade.argtypes = [P, P, C.c_uint64, C.c_uint64, C.c_int, C.c_uint64, P, P, P, P, P, P, P,
                                 P, C.c_int]
        L.pdfo_segments.restype = C.c_uint64
        L.pdfo_segments.argtypes = [P, C.c_uint32, P, C.c_uint64]
        L.pdfo_grade_seg.argtypes = [P, P, C.c_uint64, C.c_uint64, C.c_int, C.c_uint64, C.c_uint32, P,
                                     C.c_uint64, P, P, P, P, P, C.c_int]
        L.pdfo_grade_seg.restype = C.c_int
        for f in ("pdfo_sim", "pdfo_sim_mode", "pdfo_sim_vectors", "pdfo_mark", "pdfo_merge", "pdfo_cover", "pdfo_grade"):
            getattr(L, f).restype = C.c_int
        _lib = L
    return _lib


def _nl(nl) -> int:
    return C.addressof(nl.view())


class Result:
    def __init__(self, first_x, first_y, total: int, flags: int, sim=None, mark=None, chunk_totals=None):
        self.first_x = first_x
        self.first_y = first_y
        self.total = total
        self.flags = flags
        self.sim = sim
        self.mark = mark
        self.chunk_totals = chunk_totals


def grade(nl, pi_codes: np.ndarray, n_pairs: int, pair_base: int = 0, mark_mode: int = 0,
          chunk: int = 0, first_x=None, first_y=None, total: int = 0, flags: int = 0,
          want_planes: bool = False, threads: int = 0) -> Result:
    """The reference chunk loop over pi_codes[n_pi][n_pairs] (one code byte per pair)."""
    G = nl.n_gates
    pi = np.ascontiguousarray(pi_codes, dtype=np.uint8)
    assert pi.shape == (nl.n_pi, n_pairs)
    fx = np.full(G, 0xFFFFFFFF, np.uint32) if first_x is None else np.array(first_x, np.uint32)
    fy = np.full(G, 0xFFFFFFFF, np.uint32) if first_y is None else np.array(first_y, np.uint32)
    sim = np.zeros((G, n_pairs), np.uint8) if want_planes else None
    mark = np.zeros((G, n_pairs), np.uint8) if want_planes else None
    lo = C.c_uint64(total & ((1 << 64) - 1))
    hi = C.c_uint64(total >> 64)
    fl = C.c_uint32(flags)
    ch = chunk if chunk else n_pairs
    nchunks = (n_pairs + ch - 1) // ch
    ct = np.zeros(2 * nchunks, np.uint64)
    rc = lib().pdfo_grade(_nl(nl), pi.ctypes.data, n_pairs, pair_base, mark_mode, chunk,
                          fx.ctypes.data, fy.ctypes.data, sim.ctypes.data if sim is not None else None,
                          mark.ctypes.data if mark is not None else None, C.addressof(lo), C.addressof(hi),
                          C.addressof(fl), ct.ctypes.data, threads)
    if rc:
        raise MemoryError("oracle allocation failed")
    chunk_totals = [int(ct[2 * i]) | (int(ct[2 * i + 1]) << 64) for i in range(nchunks)]
    return Result(fx, fy, (hi.value << 64) | lo.value, fl.value, sim, mark, chunk_totals)


def segments(nl, seg_len: int) -> np.ndarray:
    """Segments of seg_len nets as [S][seg_len] gate ids (pdfo_segments order)."""
    n = int(lib().pdfo_segments(_nl(nl), seg_len, None, 0))
    out = np.zeros((n, seg_len), np.uint32)
    if n:
        lib().pdfo_segments(_nl(nl), seg_len, out.ctypes.data, n)
    return out


def grade_seg(nl, pi_codes: np.ndarray, n_pairs: int, seg_len: int, pair_base: int = 0, mark_mode: int = 0,
              chunk: int = 0, first_x=None, first_y=None, threads: int = 0) -> Result:
    """The chunk loop with segments of seg_len nets; first_x / first_y are per segment."""
    segs = segments(nl, seg_len)
    S = len(segs)
    pi = np.ascontiguousarray(pi_codes, dtype=np.uint8)
    fx = np.full(S, 0xFFFFFFFF, np.uint32) if first_x is None else np.array(first_x, np.uint32)
    fy = np.full(S, 0xFFFFFFFF, np.uint32) if first_y is None else np.array(first_y, np.uint32)
    lo, hi, fl = C.c_uint64(0), C.c_uint64(0), C.c_uint32(0)
    rc = lib().pdfo_grade_seg(_nl(nl), pi.ctypes.data, n_pairs, pair_base, mark_mode, chunk, seg_len,
                              segs.ctypes.data, S, fx.ctypes.data, fy.ctypes.data, C.addressof(lo),
                              C.addressof(hi), C.addressof(fl), threads)
    if rc:
        raise MemoryError("oracle allocation failed")
    r = Result(fx, fy, (hi.value << 64) | lo.value, fl.value)
    r.segs = segs
    return r


def sim(nl, pi_codes: np.ndarray, n_pairs: int, threads: int = 0, mark_mode: int = 0) -> np.ndarray:
    """Transition codes [n_gates][n_pairs]; mark_mode 2, 3 use the FIXED gate semantics."""
    out = np.zeros((nl.n_gates, n_pairs), np.uint8)
    pi = np.ascontiguousarray(pi_codes, dtype=np.uint8)
    lib().pdfo_sim_mode(_nl(nl), pi.ctypes.data, n_pairs, out.ctypes.data, mark_mode, threads)
    return out


def sim_vectors(nl, vec: np.ndarray, threads: int = 0) -> np.ndarray:
    vec = np.ascontiguousarray(vec, dtype=np.uint8)
    n_vec = vec.shape[1]
    out = np.zeros((nl.n_gates, n_vec), np.uint8)
    lib().pdfo_sim_vectors(_nl(nl), vec.ctypes.data, n_vec, out.ctypes.data, threads)
    return out


def mark(nl, sim_codes: np.ndarray, n_pairs: int, mark_mode: int = 0, prune: bool = True,
         threads: int = 0) -> np.ndarray:
    out = np.zeros((nl.n_gates, n_pairs), np.uint8)
    s = np.ascontiguousarray(sim_codes, dtype=np.uint8)
    lib().pdfo_mark(_nl(nl), s.ctypes.data, n_pairs, mark_mode, out.ctypes.data, int(prune), threads)
    return out


def merge(nl, sim_codes, mark_bits, n_pairs: int, pair_base: int, first_x, first_y) -> None:
    """kernSegmentReduce2<1> restated: folds first ids into first_x/first_y (uint32, in place)."""
    s = np.ascontiguousarray(sim_codes, dtype=np.uint8)
    m = np.ascontiguousarray(mark_bits, dtype=np.uint8)
    assert first_x.dtype == np.uint32 and first_y.dtype == np.uint32
    lib().pdfo_merge(_nl(nl), s.ctypes.data, m.ctypes.data, n_pairs, pair_base, first_x.ctypes.data,
                     first_y.ctypes.data, 0)


def cover(nl, mark_bits, n_pairs: int, pair_base: int, first_x, first_y, threads: int = 0,
          want_counts: bool = False):
    """kernCover<1> + kernSumSingle restated: returns (count, flags) of one
    chunk; with want_counts also the c value of every primary input for every
    pair (what debugCover writes to gpucover.log) as [n_pi][n_pairs][2] u64."""
    m = np.ascontiguousarray(mark_bits, dtype=np.uint8)
    fx = np.ascontiguousarray(first_x, dtype=np.uint32)
    fy = np.ascontiguousarray(first_y, dtype=np.uint32)
    lo, hi, fl = C.c_uint64(0), C.c_uint64(0), C.c_uint32(0)
    counts = np.zeros((nl.n_pi, n_pairs, 2), np.uint64) if want_counts else None
    if want_counts:
        rc = lib().pdfo_cover_counts(_nl(nl), m.ctypes.data, n_pairs, pair_base, fx.ctypes.data, fy.ctypes.data,
                                     counts.ctypes.data, C.addressof(lo), C.addressof(hi), C.addressof(fl), threads)
    else:
        rc = lib().pdfo_cover(_nl(nl), m.ctypes.data, n_pairs, pair_base, fx.ctypes.data, fy.ctypes.data,
                              C.addressof(lo), C.addressof(hi), C.addressof(fl), threads)
    if rc:
        raise MemoryError("oracle allocation failed")
    if want_counts:
        return (hi.value << 64) | lo.value, fl.value, counts
    return (hi.value << 64) | lo.value, fl.value
