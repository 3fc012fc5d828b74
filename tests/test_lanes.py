"""GPU parity of the lane forward kernel (tile_words = 32: a warp lane per
word of 32 pairs; 64 and 128: two and four words per lane; a warp per gate,
one barrier per level) against the CPU oracle, bit-exact on every transition
code, mark, first-detect id and count, in every mode and through every entry
point that runs a forward pass."""
import numpy as np
import pytest

import circuits
import helpers
import refmodel as R
from test_gpu_parity import SUITE, assert_same, gpu_grade

pytestmark = pytest.mark.gpu

P = helpers.pdf()
O = helpers.oracle()


@pytest.fixture(params=[32, 64, 128], ids=["lanes32", "lanes64", "lanes128"])
def lanes(request):
    return request.param


@pytest.mark.parametrize("mode", [0, 1, 2, 3])
@pytest.mark.parametrize("idx", range(len(SUITE)))
def test_suite(idx, mode, lanes):
    name, nl = SUITE[idx]
    rng = np.random.default_rng(300 + idx)
    # one block with a ragged tail, and several blocks (the last one partial,
    # the last lane of a wide-lane block partly full)
    for n in (40, 2100, 4100):
        assert_same(nl, helpers.rand_codes(rng, nl.n_pi, n), n, mode, tile_words=lanes)


@pytest.mark.parametrize("n", [1, 31, 32, 33, 63, 64, 65, 1023, 1024, 1025, 1057, 2047, 2048, 2049, 4096 + 7])
def test_pair_counts(n, lanes):
    nl = SUITE[3][1]
    assert_same(nl, helpers.rand_codes(np.random.default_rng(n), nl.n_pi, n), n, 1, tile_words=lanes)


@pytest.mark.parametrize("threads", [256, 512, 1024])
def test_block_sizes(threads, lanes):
    nl = circuits.random_small(4242, n_gates=400, n_pi=30, n_po=120, depth=10)
    rng = np.random.default_rng(7)
    assert_same(nl, helpers.rand_codes(rng, nl.n_pi, 2000), 2000, tile_words=lanes, threads=threads)


@pytest.mark.parametrize("mode", [0, 1, 2, 3])
def test_wide_fanin_and_levels(mode, lanes):
    """Gates of up to 8 fan-ins (past the four kept in the record) on
    1,000-gate levels."""
    nl = circuits.random_small(4343, n_gates=9000, n_pi=600, n_po=1500, depth=9, fmax=8)
    rng = np.random.default_rng(9)
    assert_same(nl, helpers.rand_codes(rng, nl.n_pi, 1500), 1500, mode, tile_words=lanes)


def test_hub_fanout(lanes):
    nl = circuits.hub(200)
    assert_same(nl, helpers.rand_codes(np.random.default_rng(4), nl.n_pi, 900), 900, tile_words=lanes)


def test_unknown_and_single_input_types(lanes):
    nl = circuits.unknown_types()
    assert_same(nl, helpers.rand_codes(np.random.default_rng(5), nl.n_pi, 300), 300, tile_words=lanes)


@pytest.mark.parametrize("k", [41, 80])
def test_wide_counts(k, lanes):
    nl = circuits.diamond_chain(k)
    codes = np.array([[R.T0, R.T1, R.T0, R.S1] * 10], np.uint8)
    got, _ = assert_same(nl, codes, 40, tile_words=lanes)
    assert got["total"] == 3 ** k


def test_overflow_flag(lanes):
    nl = circuits.diamond_chain(81)
    codes = np.array([[R.T0] * 5], np.uint8)
    got, _ = assert_same(nl, codes, 5, tile_words=lanes)
    assert got["flags"] & P.FLAG_OVERFLOW and got["total"] == (1 << 128) - 1


def test_batches_through_the_state(lanes):
    nl = SUITE[3][1]
    rng = np.random.default_rng(3)
    n = 3000
    codes = helpers.rand_codes(rng, nl.n_pi, n)
    got, want = assert_same(nl, codes, n, tile_words=lanes, batches=[0, 700, 701, 2048, 3000])
    assert sum(got["batch_totals"]) == want.total


@pytest.mark.parametrize("mode", [0, 1])
def test_rows_read_back_only(mode, lanes):
    """No plane output asked for: only rows with fan-outs (V, T) and marked
    rows (M) are written; counts and first ids still match."""
    nl = circuits.random_small(77, n_gates=20000, n_pi=400, n_po=2000, depth=90, fmin=1, fmax=8)
    n = 3000
    codes = helpers.rand_codes(np.random.default_rng(31), nl.n_pi, n)
    want = O.grade(nl, codes, n, mark_mode=mode)
    got = gpu_grade(nl, codes, n, mode, outputs=False, tile_words=lanes)
    np.testing.assert_array_equal(got["fx"], want.first_x)
    np.testing.assert_array_equal(got["fy"], want.first_y)
    assert got["total"] == want.total and got["flags"] == want.flags


def test_stage_calls_compose_to_grade(lanes):
    import torch
    nl = SUITE[6][1]
    rng = np.random.default_rng(13)
    n = 2500
    codes = helpers.rand_codes(rng, nl.n_pi, n)
    want = O.grade(nl, codes, n, want_planes=True)
    v, t = P.planes_from_codes(codes)
    c = P.Circuit(nl, tile_words=lanes)
    s = P.State(c)
    W = P.words(n)
    sv, st, mk, fm = (torch.zeros((nl.n_gates, W), dtype=torch.int32, device="cuda") for _ in range(4))
    P.stage_sim(c, v, t, n, sv, st)
    P.stage_mark_forward(c, sv, st, fm, n)
    P.stage_mark(c, sv, st, mk, n)
    P.stage_merge(c, s, sv, mk, n, 0)
    tot = P.stage_cover(c, s, mk, n, 0)
    torch.cuda.synchronize()
    h = lambda x: x.cpu().numpy().view(np.uint32)
    np.testing.assert_array_equal(P.codes_from_planes(h(sv), h(st), n), want.sim)
    np.testing.assert_array_equal(P.bits_from_plane(h(mk), n), want.mark)
    # the forward marks before the removal pass cover the pruned ones
    assert np.all(P.bits_from_plane(h(fm), n) >= want.mark)
    fx, fy, total = s.snapshot()
    np.testing.assert_array_equal(fx, want.first_x)
    np.testing.assert_array_equal(fy, want.first_y)
    assert tot.value == want.total == total.value


@pytest.mark.parametrize("wl", ["c1", "c2"])
def test_benchmark_workloads(wl, lanes):
    w = P.WORKLOADS[wl]
    nl = P.gen_netlist(w["gen"])
    n = w["pairs"]
    v, t = P.gen_pairs(P.pair_seed(w["gen"].seed), nl.n_pi, n)
    codes = P.codes_from_planes(v, t, n)
    assert_same(nl, codes, n, mode=1, tile_words=lanes)


@pytest.mark.parametrize("case", ["uniform_robust", "zipf_default"])
def test_large_circuits(case, lanes):
    """140,000-150,000-gate circuits (levels of thousands of gates, Zipf
    fan-out up to 256) with and without plane outputs."""
    if case.startswith("zipf"):
        g = P.GenParams(0x5EED0300, 150_000, 2048, 2048, 50, fanout_dist=1, zipf_s=1.5, fanout_max=256)
    else:
        g = P.GenParams(0x5EED0301, 140_000, 3000, 3000, 40)
    nl = P.gen_netlist(g)
    mode = 0 if case.endswith("default") else 1
    n = 1100
    codes = helpers.rand_codes(np.random.default_rng(len(case) + 5), nl.n_pi, n)
    assert_same(nl, codes, n, mode, tile_words=lanes)
    want = O.grade(nl, codes, n, mark_mode=mode)
    got = gpu_grade(nl, codes, n, mode, outputs=False, tile_words=lanes)
    np.testing.assert_array_equal(got["fx"], want.first_x)
    np.testing.assert_array_equal(got["fy"], want.first_y)
    assert got["total"] == want.total and got["flags"] == want.flags


def test_bitmap_in_global_memory(lanes):
    """Above about 1.8 million gates a column block's mark bitmap no longer
    fits in the lane kernel's shared memory and is kept in global memory."""
    g = P.GenParams(0x5EED0302, 1_900_000, 4096, 4096, 30)
    nl = P.gen_netlist(g)
    n = 64
    codes = helpers.rand_codes(np.random.default_rng(17), nl.n_pi, n)
    want = O.grade(nl, codes, n, mark_mode=1)
    got = gpu_grade(nl, codes, n, 1, outputs=False, tile_words=lanes)
    np.testing.assert_array_equal(got["fx"], want.first_x)
    np.testing.assert_array_equal(got["fy"], want.first_y)
    assert got["total"] == want.total and got["flags"] == want.flags


@pytest.mark.parametrize("n", [2100, 4096 + 7])
def test_device_planes_in_place(n, lanes):
    """Device pairs and output planes at a pitch the tile divides are used in
    place (no staging copy); the words of each row past the last pair keep
    what the caller left there."""
    import torch
    nl = SUITE[3][1]
    codes = helpers.rand_codes(np.random.default_rng(n + lanes), nl.n_pi, n)
    want = O.grade(nl, codes, n, mark_mode=1, want_planes=True)
    W = P.words(n)
    ld = (W + 127) // 128 * 128
    v, t = P.planes_from_codes(codes, ld)
    dv = torch.from_numpy(v.view(np.int32)).cuda()
    dt = torch.from_numpy(t.view(np.int32)).cuda()
    sentinel = np.int32(np.uint32(0xA5A5A5A5).view(np.int32))
    osv, ost, omk = (torch.full((nl.n_gates, ld), int(sentinel), dtype=torch.int32, device="cuda") for _ in range(3))
    c = P.Circuit(nl, mark_mode=1, tile_words=lanes)
    s = P.State(c)
    tot = P.grade(c, s, dv, dt, n, 0, osv, ost, omk)
    torch.cuda.synchronize()
    h = lambda x: x.cpu().numpy().view(np.uint32)
    np.testing.assert_array_equal(P.codes_from_planes(h(osv), h(ost), n), want.sim)
    np.testing.assert_array_equal(P.bits_from_plane(h(omk), n), want.mark)
    for x in (osv, ost, omk):
        assert np.all(h(x)[:, W:] == 0xA5A5A5A5)
    fx, fy, total = s.snapshot()
    np.testing.assert_array_equal(fx, want.first_x)
    np.testing.assert_array_equal(fy, want.first_y)
    assert tot.value == want.total == total.value
