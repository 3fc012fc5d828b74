"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle,
bit-exact on every transition code, every mark, every first-detect id and
every path count."""
import numpy as np
import pytest

import circuits
import helpers
import refmodel as R

pytestmark = pytest.mark.gpu

P = helpers.pdf()
O = helpers.oracle()


def gpu_grade(nl, codes, n, mode=0, batches=None, outputs=True, **opts):
    c = P.Circuit(nl, mark_mode=mode, **opts)
    s = P.State(c)
    v, t = P.planes_from_codes(codes)
    ld = v.shape[1]
    G = nl.n_gates
    sv, st, mk = (np.zeros((G, ld), np.uint32) for _ in range(3))
    bounds = batches or [0, n]
    batch_totals = []
    for a, b in zip(bounds[:-1], bounds[1:]):
        bv, bt = P.planes_from_codes(codes[:, a:b])
        osv, ost, omk = (np.zeros((G, bv.shape[1]), np.uint32) for _ in range(3))
        tot = P.grade(c, s, bv, bt, b - a, a, osv, ost, omk) if outputs else \
            P.grade(c, s, bv, bt, b - a, a)
        batch_totals.append(tot.value)
        if outputs:
            # stitch the batch planes back together (bit offsets a..b)
            cs = P.codes_from_planes(osv, ost, b - a)
            cm = P.bits_from_plane(omk, b - a)
            full_c = P.codes_from_planes(sv, st, n)
            full_m = P.bits_from_plane(mk, n)
            full_c[:, a:b] = cs
            full_m[:, a:b] = cm
            sv, st = P.planes_from_codes(full_c, ld)
            mk = P.planes_from_codes(full_m, ld)[0]
    fx, fy, tot = s.snapshot()
    return dict(sim=P.codes_from_planes(sv, st, n), mark=P.bits_from_plane(mk, n), fx=fx, fy=fy,
                total=tot.value, flags=tot.flags, pairs=tot.pairs, batch_totals=batch_totals)


def assert_same(nl, codes, n, mode=0, chunk=0, **kw):
    want = O.grade(nl, codes, n, mark_mode=mode, want_planes=True, chunk=chunk)
    got = gpu_grade(nl, codes, n, mode, **kw)
    np.testing.assert_array_equal(got["sim"], want.sim)
    np.testing.assert_array_equal(got["mark"], want.mark)
    np.testing.assert_array_equal(got["fx"], want.first_x)
    np.testing.assert_array_equal(got["fy"], want.first_y)
    assert got["total"] == want.total
    assert got["flags"] == want.flags
    assert got["pairs"] == n
    return got, want


SUITE = circuits.small_suite()


@pytest.mark.parametrize("mode", [0, 1, 2, 3])
@pytest.mark.parametrize("idx", range(len(SUITE)))
def test_suite(idx, mode):
    name, nl = SUITE[idx]
    rng = np.random.default_rng(100 + idx)
    for n in (40, 1000):
        assert_same(nl, helpers.rand_codes(rng, nl.n_pi, n), n, mode)


def test_suite_counts_are_nontrivial():
    rng = np.random.default_rng(1)
    tot = 0
    for _, nl in SUITE:
        tot += gpu_grade(nl, helpers.rand_codes(rng, nl.n_pi, 500), 500)["total"]
    assert tot > 0


@pytest.mark.parametrize("tile_words", [1, 2, 4, 8])
@pytest.mark.parametrize("threads", [128, 512, 1024])
def test_launch_shapes(tile_words, threads):
    nl = circuits.random_small(4242, n_gates=400, n_pi=30, n_po=120, depth=10)
    rng = np.random.default_rng(7)
    assert_same(nl, helpers.rand_codes(rng, nl.n_pi, 2000), 2000, tile_words=tile_words, threads=threads)


@pytest.mark.parametrize("mode", [2, 3])
@pytest.mark.parametrize("tile_words", [1, 2, 4, 8])
def test_fixed_modes_every_tile(tile_words, mode):
    """True n-input gates (XOR evaluated, several fan-ins carrying marks),
    wide fan-in and fan-ins past the ring, against the oracle's FIXED mode."""
    nl = circuits.random_small(4343, n_gates=3000, n_pi=200, n_po=500, depth=9, fmax=6)
    rng = np.random.default_rng(9)
    assert_same(nl, helpers.rand_codes(rng, nl.n_pi, 1500), 1500, mode, tile_words=tile_words)


def test_levels_wider_than_the_ring():
    # 1,500-gate levels exceed the 1,024-gate ring of 8-word tiles: fan-ins
    # beyond the window come from global memory
    nl = circuits.random_small(99, n_gates=12000, n_pi=1500, n_po=3000, depth=7)
    rng = np.random.default_rng(8)
    assert_same(nl, helpers.rand_codes(rng, nl.n_pi, 700), 700, tile_words=8)


@pytest.mark.parametrize("n", [1, 31, 32, 33, 64, 1025])
def test_pair_counts(n):
    nl = SUITE[0][1]
    rng = np.random.default_rng(n)
    assert_same(nl, helpers.rand_codes(rng, nl.n_pi, n), n)


def test_batches_through_the_state():
    nl = SUITE[3][1]
    rng = np.random.default_rng(3)
    n = 3000
    codes = helpers.rand_codes(rng, nl.n_pi, n)
    got, want = assert_same(nl, codes, n, batches=[0, 700, 701, 2048, 3000])
    one = gpu_grade(nl, codes, n)
    assert sum(got["batch_totals"]) == one["total"] == want.total


def test_hub_fanout():
    nl = circuits.hub(200)
    rng = np.random.default_rng(4)
    assert_same(nl, helpers.rand_codes(rng, nl.n_pi, 900), 900)


def test_unknown_and_single_input_types():
    nl = circuits.unknown_types()
    rng = np.random.default_rng(5)
    assert_same(nl, helpers.rand_codes(rng, nl.n_pi, 300), 300)


@pytest.mark.parametrize("k", [41, 80])
def test_wide_counts(k):
    nl = circuits.diamond_chain(k)
    codes = np.array([[R.T0, R.T1, R.T0, R.S1] * 10], np.uint8)
    got, want = assert_same(nl, codes, 40)
    assert got["total"] == 3 ** k


def test_overflow_flag():
    nl = circuits.diamond_chain(81)
    codes = np.array([[R.T0] * 5], np.uint8)
    got, want = assert_same(nl, codes, 5)
    assert got["flags"] & P.FLAG_OVERFLOW and got["total"] == (1 << 128) - 1


def test_no_outputs_requested():
    nl = SUITE[4][1]
    rng = np.random.default_rng(6)
    codes = helpers.rand_codes(rng, nl.n_pi, 500)
    want = O.grade(nl, codes, 500)
    got = gpu_grade(nl, codes, 500, outputs=False)
    assert got["total"] == want.total
    np.testing.assert_array_equal(got["fx"], want.first_x)


@pytest.mark.parametrize("case", ["wide_levels", "deep_wide_fanin", "c2_default", "c2_robust"])
def test_rows_read_back_only(case):
    """With no plane asked for, the forward pass writes only the plane rows
    that are read back (far fan-ins, marked gates).  On circuits larger than
    the shared-memory ring the counts, flags and first ids still match."""
    mode, opts = 0, {}
    if case == "wide_levels":
        nl, n, opts = circuits.random_small(99, n_gates=12000, n_pi=1500, n_po=3000, depth=7), 700, {"tile_words": 8}
    elif case == "deep_wide_fanin":
        nl, n = circuits.random_small(77, n_gates=20000, n_pi=400, n_po=2000, depth=90, fmin=1, fmax=8), 1000
    else:
        w = P.WORKLOADS["c2"]
        nl, n = P.gen_netlist(w["gen"]), 4096
        mode = 1 if case == "c2_robust" else 0
    codes = helpers.rand_codes(np.random.default_rng(len(case)), nl.n_pi, n)
    want = O.grade(nl, codes, n, mark_mode=mode)
    got = gpu_grade(nl, codes, n, mode, outputs=False, **opts)
    np.testing.assert_array_equal(got["fx"], want.first_x)
    np.testing.assert_array_equal(got["fy"], want.first_y)
    assert got["total"] == want.total and got["flags"] == want.flags


def test_device_buffers():
    import torch
    nl = SUITE[5][1]
    rng = np.random.default_rng(12)
    n = 4000
    codes = helpers.rand_codes(rng, nl.n_pi, n)
    want = O.grade(nl, codes, n, want_planes=True)
    v, t = P.planes_from_codes(codes)
    c = P.Circuit(nl)
    s = P.State(c)
    dv, dt = torch.from_numpy(v.view(np.int32)).cuda(), torch.from_numpy(t.view(np.int32)).cuda()
    ld = 128 + 5  # an ld larger than needed
    sv, st, mk = (torch.zeros((nl.n_gates, ld), dtype=torch.int32, device="cuda") for _ in range(3))
    tot = P.grade(c, s, dv, dt, n, 0, sv, st, mk)
    assert tot.value == want.total
    h = lambda x: x.cpu().numpy().view(np.uint32)
    np.testing.assert_array_equal(P.codes_from_planes(h(sv), h(st), n), want.sim)
    np.testing.assert_array_equal(P.bits_from_plane(h(mk), n), want.mark)


def test_stage_calls_compose_to_grade():
    import torch
    nl = SUITE[6][1]
    rng = np.random.default_rng(13)
    n = 2500
    codes = helpers.rand_codes(rng, nl.n_pi, n)
    want = O.grade(nl, codes, n, want_planes=True)
    v, t = P.planes_from_codes(codes)
    c = P.Circuit(nl)
    s = P.State(c)
    W = P.words(n)
    sv, st, mk = (torch.zeros((nl.n_gates, W), dtype=torch.int32, device="cuda") for _ in range(3))
    P.stage_sim(c, v, t, n, sv, st)
    P.stage_mark(c, sv, st, mk, n)
    P.stage_merge(c, s, sv, mk, n, 0)
    tot = P.stage_cover(c, s, mk, n, 0)
    torch.cuda.synchronize()
    h = lambda x: x.cpu().numpy().view(np.uint32)
    np.testing.assert_array_equal(P.codes_from_planes(h(sv), h(st), n), want.sim)
    np.testing.assert_array_equal(P.bits_from_plane(h(mk), n), want.mark)
    fx, fy, total = s.snapshot()
    np.testing.assert_array_equal(fx, want.first_x)
    assert tot.value == want.total == total.value


def test_snapshot_restore_reset():
    nl = SUITE[0][1]
    rng = np.random.default_rng(14)
    codes = helpers.rand_codes(rng, nl.n_pi, 600)
    c = P.Circuit(nl)
    s = P.State(c)
    v1, t1 = P.planes_from_codes(codes[:, :300])
    v2, t2 = P.planes_from_codes(codes[:, 300:])
    P.grade(c, s, v1, t1, 300, 0)
    snap = s.snapshot()
    P.grade(c, s, v2, t2, 300, 300)
    after = s.snapshot()
    s2 = P.State(c)
    s2.restore(*snap)
    P.grade(c, s2, v2, t2, 300, 300)
    again = s2.snapshot()
    np.testing.assert_array_equal(after[0], again[0])
    assert after[2].value == again[2].value == O.grade(nl, codes, 600).total
    s.reset()
    fx, fy, tot = s.snapshot()
    assert np.all(fx == P.NONE) and tot.value == 0 and tot.pairs == 0


@pytest.mark.parametrize("wl", ["c1", "c2"])
def test_benchmark_workloads(wl):
    w = P.WORKLOADS[wl]
    nl = P.gen_netlist(w["gen"])
    n = w["pairs"]
    v, t = P.gen_pairs(P.pair_seed(w["gen"].seed), nl.n_pi, n)
    codes = P.codes_from_planes(v, t, n)
    assert_same(nl, codes, n, mode=1)


@pytest.mark.parametrize("case", ["uniform_robust", "uniform_default", "zipf_robust"])
def test_bitmap_in_global_memory(case):
    """Circuits above 131,072 gates keep each column block's mark bitmap in
    global memory instead of shared memory (it no longer fits in 16 KB);
    levels of several thousand gates also overflow the ring, so fan-ins come
    from far slots and plane rows.  Marks read from each of those places
    must still match the oracle, with and without plane outputs."""
    if case.startswith("zipf"):
        g = P.GenParams(0x5EED0300, 150_000, 2048, 2048, 50, fanout_dist=1, zipf_s=1.5, fanout_max=256)
    else:
        g = P.GenParams(0x5EED0301, 140_000, 3000, 3000, 40)
    nl = P.gen_netlist(g)
    mode = 0 if case.endswith("default") else 1
    n = 300
    codes = helpers.rand_codes(np.random.default_rng(len(case) + 5), nl.n_pi, n)
    assert_same(nl, codes, n, mode)
    want = O.grade(nl, codes, n, mark_mode=mode)
    for tw in (4, 8):
        got = gpu_grade(nl, codes, n, mode, outputs=False, tile_words=tw)
        np.testing.assert_array_equal(got["fx"], want.first_x)
        np.testing.assert_array_equal(got["fy"], want.first_y)
        assert got["total"] == want.total and got["flags"] == want.flags


def test_snapshot_ordered_on_a_stream():
    """pdf_state_snapshot_on reads a state after the grading queued on one
    stream (and waits for that stream only): the same ids and totals as the
    device-wide snapshot and as the oracle."""
    import torch
    nl = SUITE[5][1]
    n = 3000
    codes = helpers.rand_codes(np.random.default_rng(21), nl.n_pi, n)
    want = O.grade(nl, codes, n, mark_mode=1)
    v, t = P.planes_from_codes(codes)
    c = P.Circuit(nl, mark_mode=1)
    s = P.State(c)
    dv, dt = torch.from_numpy(v.view(np.int32)).cuda(), torch.from_numpy(t.view(np.int32)).cuda()
    side = torch.cuda.Stream()
    P.grade_async(c, s, P.make_pairs(dv, dt, n), 0, None, side.cuda_stream)
    fx, fy, tot = s.snapshot(side.cuda_stream)
    np.testing.assert_array_equal(fx, want.first_x)
    np.testing.assert_array_equal(fy, want.first_y)
    assert tot.value == want.total and tot.pairs == n
    fx2, fy2, tot2 = s.snapshot()
    np.testing.assert_array_equal(fx, fx2)
    np.testing.assert_array_equal(fy, fy2)
    assert tot2.value == tot.value and tot2.flags == tot.flags
    s.close()
    c.close()


def test_pending_cuda_error_of_the_caller_is_not_reported():
    """A failure the caller left unchecked on this thread (here a
    cudaSetDevice to a device that does not exist) is not reported as this
    library's error, and the library leaves no error of its own pending."""
    import ctypes
    rt = ctypes.CDLL("libcudart.so.12")
    nl = SUITE[2][1]
    n = 200
    codes = helpers.rand_codes(np.random.default_rng(23), nl.n_pi, n)
    want = O.grade(nl, codes, n)
    assert rt.cudaSetDevice(9999) != 0  # left pending on purpose
    got = gpu_grade(nl, codes, n, outputs=False)
    assert got["total"] == want.total
    np.testing.assert_array_equal(got["fx"], want.first_x)
    assert rt.cudaGetLastError() == 0
