"""Golden fixtures produced by the reference's own kernels.

tests/golden/ref_*.npz were written by tests/golden/make_golden.py, which ran
the reference's simkernel/markkernel/mergekernel/coverkernel (compiled
unmodified from the reference tree, oracle/refharness) on a B200.  They pin
the oracle (CPU) and the CUDA path (GPU) to the reference itself: every
transition code and mark (full planes for the small cases, SHA-256 digests
for the rest), every first-detect id and every per-chunk path count.
"""
import glob
import hashlib
import os

import numpy as np
import pytest

import helpers

P = helpers.pdf()
O = helpers.oracle()

FIXTURES = sorted(glob.glob(os.path.join(helpers.ROOT, "tests", "golden", "ref_*.npz")))


def load(path):
    z = np.load(path)
    nl = P.Netlist(z["level_offsets"], z["type"], z["po"], z["nfi"], z["nfo"], z["edge_offset"], z["edges"])
    n_vec, chunk, robust = (int(x) for x in z["meta"])
    v, t = P.pairs_from_vectors(z["vec"])
    return z, nl, n_vec, chunk, robust, v, t


def seg_len(z) -> int:
    """Segments of this many nets (fixtures of gpuMergeSegments<N> /
    gpuCountPaths<N>); 1: single nets."""
    return int(z["seg_len"]) if "seg_len" in z else 1


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, np.uint8).tobytes()).hexdigest()


def test_fixtures_present():
    assert len(FIXTURES) >= 12


@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: os.path.basename(p)[4:-4])
def test_oracle_matches_reference_kernels(path):
    z, nl, n, chunk, robust, v, t = load(path)
    codes = P.codes_from_planes(v, t, n)
    N = seg_len(z)
    if N > 1:  # the segment list given to the reference is the oracle's, and so are the results
        np.testing.assert_array_equal(O.segments(nl, N), z["segments"])
        fx = fy = None
        counts = []
        for a in range(0, n, chunk):
            r = O.grade_seg(nl, codes[:, a:a + chunk], min(chunk, n - a), N, pair_base=a, mark_mode=robust,
                            first_x=fx, first_y=fy)
            fx, fy = r.first_x, r.first_y
            counts.append(r.total)
        np.testing.assert_array_equal(fx, z["ref_first_x"])
        np.testing.assert_array_equal(fy, z["ref_first_y"])
        assert counts == [int(x) for x in z["ref_chunk_counts"]]
    r = O.grade(nl, codes, n, mark_mode=robust, chunk=chunk, want_planes=True)
    assert sha(r.sim) == str(z["ref_sim_sha256"])
    assert sha(r.mark) == str(z["ref_mark_sha256"])
    if N > 1:
        return
    np.testing.assert_array_equal(r.first_x, z["ref_first_x"])
    np.testing.assert_array_equal(r.first_y, z["ref_first_y"])
    assert r.chunk_totals == [int(x) for x in z["ref_chunk_counts"]]
    if "ref_mark" in z:
        np.testing.assert_array_equal(P.codes_from_planes(z["ref_sim_v"], z["ref_sim_t"], n), r.sim)
        np.testing.assert_array_equal(P.bits_from_plane(z["ref_mark"], n), r.mark)


@pytest.mark.gpu
@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: os.path.basename(p)[4:-4])
def test_cuda_path_matches_reference_kernels(path):
    """The CUDA path through the C ABI, batch by batch as the reference's
    chunks, against the reference's own outputs."""
    z, nl, n, chunk, robust, v, t = load(path)
    N = seg_len(z)
    c = P.Circuit(nl, mark_mode=robust, seg_len=N)
    if N > 1:
        np.testing.assert_array_equal(c.segments(), z["segments"])
    s = P.State(c)
    sim = np.zeros((nl.n_gates, n), np.uint8)
    mark = np.zeros((nl.n_gates, n), np.uint8)
    counts = []
    codes = P.codes_from_planes(v, t, n)
    for k, a in enumerate(range(0, n, chunk)):
        b = min(n, a + chunk)
        bv, bt = P.planes_from_codes(codes[:, a:b])
        sv, st, mk = (np.zeros((nl.n_gates, bv.shape[1]), np.uint32) for _ in range(3))
        tot = P.grade(c, s, bv, bt, b - a, a, sv, st, mk)
        counts.append(tot.value)
        sim[:, a:b] = P.codes_from_planes(sv, st, b - a)
        mark[:, a:b] = P.bits_from_plane(mk, b - a)
    fx, fy, total = s.snapshot()
    np.testing.assert_array_equal(fx, z["ref_first_x"])
    np.testing.assert_array_equal(fy, z["ref_first_y"])
    assert counts == [int(x) for x in z["ref_chunk_counts"]]
    assert total.value == int(np.sum(z["ref_chunk_counts"]))
    assert sha(sim) == str(z["ref_sim_sha256"])
    assert sha(mark) == str(z["ref_mark_sha256"])
