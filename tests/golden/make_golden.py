#!/usr/bin/env python
"""Generate golden fixtures from the reference's own kernels.

Runs oracle/_ref/refharness (the reference's simkernel/markkernel/
mergekernel/coverkernel, compiled unmodified from the reference tree by
oracle/refharness/Makefile) on a set of seeded cases on a GPU, and writes one
fixture per case: the netlist, the vector stream, and the reference's
first-detect ids, per-chunk path counts, and per-(net, pair) transition
codes and marks (as SHA-256 digests, plus the full packed planes for the
small cases).  It also grades every case with the oracle and reports any
difference.

Shapes are chosen so the reference is well-defined on them: gate (or, with
segments of N > 1 nets, segment) counts a multiple of 20 and chunks a
multiple of 1,024 vectors (no divergent
__syncthreads, simkernel.cuh:106-110, mergekernel.cuh:130-173), chunks of at
most 4,224 pairs (merge visits 1,056 words, mergekernel.cuh:125), and counts
below 2^16 per (net, pair) (coverkernel.cuh:41-43).  With segments, the
reference's generator (util/segment.cuh) is missing, so the harness is given
this build's segment list; its kernCover<N> initialises each thread's slot of
activeTests with no barrier before other threads may write it
(coverkernel.cuh:181-188), a timing race that the report would show as a
difference.

  python tests/golden/make_golden.py OUT_DIR
"""
from __future__ import annotations

import hashlib
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
import helpers  # noqa: E402

P = helpers.pdf()
O = helpers.oracle()
HARNESS = helpers.ROOT / "oracle" / "_ref" / "refharness"


def gen(seed, G, npi, npo, depth, fmin=1, fmax=4, mask=0, zipf=False, fo_max=0):
    return P.gen_netlist(P.GenParams(seed, G, npi, npo, depth, fmin, fmax, 1 if zipf else 0, 1.5, fo_max, mask))


def hub_260():
    import circuits
    return circuits.hub(217, seed=21)


def diamond_padded(k=10, pad=19):
    """diamond_chain(k) with `pad` extra (dangling) inputs so that the gate
    count is a multiple of 20."""
    import circuits
    d = circuits.diamond_chain(k)
    G = d.n_gates + pad
    shift = lambda x: x + pad if x > 0 else 0  # new PIs take ids 1..pad
    levels = [[0] + list(range(1, pad + 1))]
    for l in range(1, d.n_levels):
        levels.append([shift(g) for g in range(int(d.level_offsets[l]), int(d.level_offsets[l + 1]))])
    types = [P.INPT] * G
    fanins = [[] for _ in range(G)]
    for g in range(1, d.n_gates):
        types[shift(g)] = int(d.type[g])
        fanins[shift(g)] = [shift(int(f)) for f in d.fanins(g)]
    pos = [shift(g) for g in range(d.n_gates) if d.po[g]]
    return P.Netlist.from_fanins(levels, types, fanins, pos)


MARKING = sum(1 << t for t in (P.AND, P.NAND, P.OR, P.NOR, P.NOT, P.BUFF))
WIDE = sum(1 << t for t in (P.AND, P.NAND, P.OR, P.NOR))
FROMDFF = sum(1 << t for t in (P.AND, P.NAND, P.OR, P.NOR, P.XOR, P.XNOR, P.NOT, P.BUFF, P.FROM, P.DFF))


def with_segments(seed, N, *args, **kw):
    """The first netlist from seed, seed + 1, ... whose segments of N nets
    number a multiple of 20 (the reference's merge runs 20 segments per block
    and syncs inside its test of the segment index)."""
    for k in range(400):
        nl = gen(seed + k, *args, **kw)
        if len(O.segments(nl, N)) % 20 == 0:
            return nl
    raise RuntimeError("no netlist with a segment count divisible by 20")


def cases():
    c1 = P.WORKLOADS["c1"]["gen"]
    return [
        # name, netlist, n_vec, chunk, robust, keep full planes
        ("mix_a_default", gen(0x601D0001, 200, 16, 60, 8), 4096, 4096, 0, True),
        ("mix_a_robust", gen(0x601D0001, 200, 16, 60, 8), 4096, 4096, 1, True),
        ("mix_b_chunks", gen(0x601D0002, 400, 30, 100, 10), 8192, 2048, 0, False),
        ("marking_1k", gen(0x601D0003, 300, 20, 120, 9, mask=MARKING), 4096, 1024, 1, False),
        ("wide_fanin", gen(0x601D0004, 240, 24, 80, 6, fmin=3, fmax=6, mask=WIDE), 4096, 4096, 0, False),
        ("wide_fanin_robust", gen(0x601D0004, 240, 24, 80, 6, fmin=3, fmax=6, mask=WIDE), 4096, 4096, 1, False),
        ("from_dff", gen(0x601D0005, 180, 12, 70, 9, mask=FROMDFF), 2048, 1024, 0, False),
        ("zipf", gen(0x601D0006, 400, 24, 120, 7, zipf=True, fo_max=64), 4096, 4096, 0, False),
        ("deep", gen(0x601D0007, 600, 12, 300, 40), 4096, 2048, 0, False),
        ("hub_nfo217", hub_260(), 4096, 4096, 0, False),
        ("diamond10", diamond_padded(10), 1024, 1024, 0, True),
        ("c1_workload", P.gen_netlist(c1), 1024, 1024, 1, False),
        # the default table on the c1 netlist, which marks (the robust one does not)
        ("c1_workload_default", P.gen_netlist(c1), 1024, 1024, 0, False),
        # segments of 2, 3 and 4 nets (gpuMergeSegments<N>, gpuCountPaths<N>)
        ("seg2_mix", with_segments(0x601D0101, 2, 200, 16, 60, 8), 4096, 4096, 0, False, 2),
        ("seg3_marking", with_segments(0x601D0201, 3, 300, 20, 120, 9, mask=MARKING), 4096, 1024, 1, False, 3),
        ("seg4_marking", with_segments(0x601D0501, 4, 300, 20, 120, 9, mask=MARKING), 4096, 2048, 0, False, 4),
    ]


def write_case(path, nl, vec, chunk, robust, segs=None):
    with open(path, "wb") as f:
        hdr = np.array([nl.n_gates, nl.n_levels, nl.n_pi, robust], np.uint32)
        f.write(hdr.tobytes())
        f.write(np.array([vec.shape[1], chunk], np.uint64).tobytes())
        for a in (nl.level_offsets, nl.type, nl.po, nl.nfi, nl.nfo, nl.edge_offset):
            f.write(np.ascontiguousarray(a).tobytes())
        f.write(np.array([len(nl.edges)], np.uint64).tobytes())
        f.write(nl.edges.tobytes())
        f.write(np.ascontiguousarray(vec, np.uint8).tobytes())
        if segs is not None:
            f.write(np.array([segs.shape[1]], np.uint32).tobytes())
            f.write(np.array([segs.shape[0]], np.uint64).tobytes())
            f.write(np.ascontiguousarray(segs, np.uint32).tobytes())


def read_out(path, G, n, S=None):
    b = open(path, "rb").read()
    o = 0
    nc = int(np.frombuffer(b, np.uint64, 1, o)[0]); o += 8
    cov = np.frombuffer(b, np.uint64, nc, o).copy(); o += 8 * nc
    sim = np.frombuffer(b, np.uint8, G * n, o).reshape(G, n).copy(); o += G * n
    mark = np.frombuffer(b, np.uint8, G * n, o).reshape(G, n).copy(); o += G * n
    S = G if S is None else S
    fx = np.frombuffer(b, np.int32, S, o).copy(); o += 4 * S
    fy = np.frombuffer(b, np.int32, S, o).copy()
    return cov, sim, mark, fx.view(np.uint32), fy.view(np.uint32)


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, np.uint8).tobytes()).hexdigest()


def main(out_dir):
    os.makedirs(out_dir, exist_ok=True)
    rng = np.random.default_rng(0x601D)
    report = []
    bad = 0
    for case in cases():
        name, nl, n_vec, chunk, robust, full = case[:6]
        N = case[6] if len(case) > 6 else 1
        segs = O.segments(nl, N) if N > 1 else None
        S = len(segs) if N > 1 else nl.n_gates
        assert S % 20 == 0 and n_vec % 1024 == 0 and chunk % 1024 == 0 and chunk <= 4224, name
        vec = rng.integers(0, 2, size=(nl.n_pi, n_vec), dtype=np.uint8)
        v, t = P.pairs_from_vectors(vec)
        codes = P.codes_from_planes(v, t, n_vec)
        want = O.grade(nl, codes, n_vec, mark_mode=robust, chunk=chunk, want_planes=True)
        if N > 1:  # per-segment first ids and per-chunk counts, chunk by chunk
            wx = wy = None
            seg_counts = []
            for a in range(0, n_vec, chunk):
                r = O.grade_seg(nl, codes[:, a:a + chunk], min(chunk, n_vec - a), N, pair_base=a, mark_mode=robust,
                                first_x=wx, first_y=wy)
                wx, wy = r.first_x, r.first_y
                seg_counts.append(r.total)
        with tempfile.TemporaryDirectory() as td:
            cp, op = os.path.join(td, "case.bin"), os.path.join(td, "out.bin")
            write_case(cp, nl, vec, chunk, robust, segs)
            subprocess.run([str(HARNESS), cp, op], check=True, stderr=subprocess.DEVNULL)
            cov, sim, mark, fx, fy = read_out(op, nl.n_gates, n_vec, S)
        same = {
            "sim": bool(np.array_equal(sim, want.sim)),
            "mark": bool(np.array_equal(mark, want.mark)),
            "first_x": bool(np.array_equal(fx, want.first_x if N == 1 else wx)),
            "first_y": bool(np.array_equal(fy, want.first_y if N == 1 else wy)),
            "chunk_counts": [int(x) for x in cov] == (want.chunk_totals if N == 1 else seg_counts),
        }
        ok = all(same.values())
        bad += not ok
        report.append(f"{name}: G={nl.n_gates} vec={n_vec} chunk={chunk} robust={robust} "
                      f"{f'segs={N}x{S} ' if N > 1 else ''}"
                      f"total={int(cov.sum())} oracle_total={want.total if N == 1 else sum(seg_counts)} "
                      f"marks={int(mark.sum())} {'MATCH' if ok else 'DIFF ' + str(same)}")
        fix = dict(level_offsets=nl.level_offsets, type=nl.type, po=nl.po, nfi=nl.nfi, nfo=nl.nfo,
                   edge_offset=nl.edge_offset, edges=nl.edges, vec=vec,
                   meta=np.array([n_vec, chunk, robust], np.uint64),
                   ref_chunk_counts=cov, ref_first_x=fx, ref_first_y=fy,
                   ref_sim_sha256=np.array(digest(sim)), ref_mark_sha256=np.array(digest(mark)))
        if N > 1:
            fix["seg_len"] = np.array(N, np.uint32)
            fix["segments"] = segs
        if full:
            fix["ref_sim_v"], fix["ref_sim_t"] = P.planes_from_codes(sim)
            fix["ref_mark"] = P.planes_from_codes(mark)[0]
        np.savez_compressed(os.path.join(out_dir, f"ref_{name}.npz"), **fix)
    with open(os.path.join(out_dir, "REPORT.txt"), "w") as f:
        f.write("\n".join(report) + "\n")
    print("\n".join(report))
    return 1 if bad else 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE)))
