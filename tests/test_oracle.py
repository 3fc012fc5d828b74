"""The C oracle against the independent Python model (tests/refmodel.py),
whose cover enumerates paths explicitly; chunk invariance; exact 128-bit
counts and the overflow flag."""
import numpy as np
import pytest

import circuits
import helpers
import refmodel as R

P = helpers.pdf()
O = helpers.oracle()

SUITE = circuits.small_suite() + [("hub", circuits.hub(150)), ("unknown", circuits.unknown_types()),
                                  ("diamond4", circuits.diamond_chain(4))]


def _check(nl, mode, n_pairs, seed):
    rng = np.random.default_rng(seed)
    codes = helpers.rand_codes(rng, nl.n_pi, n_pairs)
    got = O.grade(nl, codes, n_pairs, mark_mode=mode, want_planes=True)
    vals, marks, fx, fy, total = R.grade(nl, codes, n_pairs, mode)
    np.testing.assert_array_equal(got.sim, np.array(vals, np.uint8).T)
    np.testing.assert_array_equal(got.mark, np.array(marks, np.uint8).T)
    np.testing.assert_array_equal(got.first_x, np.array(fx, np.uint32))
    np.testing.assert_array_equal(got.first_y, np.array(fy, np.uint32))
    assert got.total == total and got.flags == 0
    return total


@pytest.mark.parametrize("mode", [0, 1, 2, 3])
def test_oracle_equals_python_model(mode):
    totals = [_check(nl, mode, 40, 17 + i) for i, (_, nl) in enumerate(SUITE)]
    assert sum(totals) > 0, "suite must exercise nonzero path counts"


def test_modes_differ_only_through_folded_nand_nor():
    # the two tables differ only where an on-path and a side input move in
    # opposite directions; on a 3-input folded NAND that still propagates
    nl = circuits.diamond_chain(3)
    codes = np.array([[R.T0, R.T0, R.S0, R.T1]], np.uint8)
    d = O.grade(nl, codes, 4, mark_mode=0)
    r = O.grade(nl, codes, 4, mark_mode=1)
    assert d.total == 3 ** 3 and r.total == 0


@pytest.mark.parametrize("chunk", [1, 3, 32, 50, 0])
def test_chunk_invariance(chunk):
    nl = SUITE[0][1]
    rng = np.random.default_rng(5)
    n = 97
    codes = helpers.rand_codes(rng, nl.n_pi, n)
    whole = O.grade(nl, codes, n)
    part = O.grade(nl, codes, n, chunk=chunk)
    assert part.total == whole.total
    assert sum(part.chunk_totals) == whole.total
    np.testing.assert_array_equal(part.first_x, whole.first_x)
    np.testing.assert_array_equal(part.first_y, whole.first_y)


def test_batches_with_state_carry():
    nl = SUITE[1][1]
    rng = np.random.default_rng(9)
    codes = helpers.rand_codes(rng, nl.n_pi, 120)
    whole = O.grade(nl, codes, 120)
    a = O.grade(nl, codes[:, :50], 50)
    b = O.grade(nl, codes[:, 50:], 70, pair_base=50, first_x=a.first_x, first_y=a.first_y, total=a.total)
    assert b.total == whole.total
    np.testing.assert_array_equal(b.first_x, whole.first_x)


def test_threads_do_not_change_results():
    nl = SUITE[2][1]
    rng = np.random.default_rng(3)
    codes = helpers.rand_codes(rng, nl.n_pi, 300)
    a = O.grade(nl, codes, 300, threads=1, want_planes=True)
    b = O.grade(nl, codes, 300, threads=4, want_planes=True)
    assert a.total == b.total
    np.testing.assert_array_equal(a.mark, b.mark)


@pytest.mark.parametrize("k", [10, 41, 50, 80])
def test_exact_wide_counts(k):
    nl = circuits.diamond_chain(k)
    codes = np.array([[R.T0]], np.uint8)
    r = O.grade(nl, codes, 1)
    assert r.total == 3 ** k and r.flags == 0  # 3^41 > 2^64, 3^80 < 2^128


def test_overflow_flag():
    nl = circuits.diamond_chain(81)  # 3^81 > 2^128
    r = O.grade(nl, np.array([[R.T0]], np.uint8), 1)
    assert r.flags & 1 and r.total == (1 << 128) - 1


def test_vector_stream_pairs():
    # the reference forms pair p from vectors p and p+1, wrapping to vector 0
    nl = SUITE[0][1]
    rng = np.random.default_rng(11)
    vec = rng.integers(0, 2, size=(nl.n_pi, 64), dtype=np.uint8)
    sim = O.sim_vectors(nl, vec)
    v, t = P.pairs_from_vectors(vec)
    codes = P.codes_from_planes(v, t, 64)
    np.testing.assert_array_equal(sim, O.sim(nl, codes, 64))
    v1 = np.roll(vec, 0, axis=1)
    v2 = np.roll(vec, -1, axis=1)
    np.testing.assert_array_equal(codes, (v2 | ((v1 ^ v2) << 1)).astype(np.uint8))


def test_fixed_modes_evaluate_true_gates():
    # a 3-input NAND: the reference folds NAND(NAND(a, b), c); FIXED is NOT(a & b & c)
    nl = P.Netlist([0, 3, 4], [P.INPT] * 3 + [P.NAND], [0, 0, 0, 1], [0, 0, 0, 3], [1, 1, 1, 0],
                   [0, 1, 2, 3], [3, 3, 3, 0, 1, 2])
    codes = np.array([[R.S1], [R.S1], [R.S1]], np.uint8)
    assert O.sim(nl, codes, 1, mark_mode=0)[3, 0] == R.S1  # NAND(NAND(1,1),1) = NAND(0,1) = 1
    assert O.sim(nl, codes, 1, mark_mode=2)[3, 0] == R.S0
    # XOR with two inputs: S0 in the reference, evaluated in FIXED
    nl = P.Netlist([0, 2, 3], [P.INPT] * 2 + [P.XOR], [0, 0, 1], [0, 0, 2], [1, 1, 0], [0, 1, 2], [2, 2, 0, 1])
    codes = np.array([[R.T1], [R.S0]], np.uint8)
    assert O.sim(nl, codes, 1, mark_mode=0)[2, 0] == R.S0
    assert O.sim(nl, codes, 1, mark_mode=3)[2, 0] == R.T1
    assert O.grade(nl, codes, 1, mark_mode=0).total == 0
    assert O.grade(nl, codes, 1, mark_mode=2).total == 1  # the path from input 0, side steady


def test_fixed_marks_follow_any_fanin():
    # AND(a, b) with a steady and b rising: the reference needs fan-in 0's
    # mark (a has no transition, so no mark); FIXED takes the path through b
    nl = P.Netlist([0, 2, 3], [P.INPT] * 2 + [P.AND], [0, 0, 1], [0, 0, 2], [1, 1, 0], [0, 1, 2], [2, 2, 0, 1])
    codes = np.array([[R.S1], [R.T1]], np.uint8)
    assert O.grade(nl, codes, 1, mark_mode=0).total == 0
    assert O.grade(nl, codes, 1, mark_mode=2).total == 1


@pytest.mark.parametrize("N", [2, 3, 5])
@pytest.mark.parametrize("mode", [0, 2])
def test_oracle_segments_equal_python_model(N, mode):
    tot = 0
    for i, (_, nl) in enumerate(SUITE[:8]):
        rng = np.random.default_rng(31 + i)
        codes = helpers.rand_codes(rng, nl.n_pi, 24)
        segs, fx, fy, total = R.grade_seg(nl, codes, 24, N, mode)
        got = O.grade_seg(nl, codes, 24, N, mark_mode=mode)
        assert [tuple(int(x) for x in s) for s in got.segs] == segs
        np.testing.assert_array_equal(got.first_x, np.array(fx, np.uint32))
        np.testing.assert_array_equal(got.first_y, np.array(fy, np.uint32))
        assert got.total == total
        tot += total
    assert tot > 0


def test_segments_of_one_net_are_the_nets():
    nl = SUITE[0][1]
    rng = np.random.default_rng(3)
    codes = helpers.rand_codes(rng, nl.n_pi, 50)
    one = O.grade_seg(nl, codes, 50, 1)
    ref = O.grade(nl, codes, 50)
    assert one.total == ref.total
    np.testing.assert_array_equal(one.first_x, ref.first_x)


@pytest.mark.parametrize("chunk", [1, 7, 0])
def test_segment_chunk_invariance(chunk):
    nl = SUITE[1][1]
    rng = np.random.default_rng(4)
    codes = helpers.rand_codes(rng, nl.n_pi, 60)
    whole = O.grade_seg(nl, codes, 60, 3)
    part = O.grade_seg(nl, codes, 60, 3, chunk=chunk)
    assert part.total == whole.total
    np.testing.assert_array_equal(part.first_x, whole.first_x)
