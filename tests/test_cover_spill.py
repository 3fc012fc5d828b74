"""The cover of pairs that mark more nets than its shared-memory table holds
(3,072 on B200): such pairs are counted by the spill cover, with every net's
(h, c) in global memory, instead of failing.  FIXED non-robust marking on a
140,000-gate circuit makes every pair mark about 4,100 nets; a primary input
driving thousands of outputs does it under the reference's own tables."""
import numpy as np
import pytest

import circuits
import helpers

pytestmark = pytest.mark.gpu

P = helpers.pdf()
O = helpers.oracle()


def _grade(nl, codes, n, mode, tile=0):
    c = P.Circuit(nl, mark_mode=mode, tile_words=tile)
    s = P.State(c)
    v, t = P.planes_from_codes(codes)
    P.grade(c, s, v, t, n)
    fx, fy, tot = s.snapshot()
    return fx, fy, tot


@pytest.fixture(scope="module")
def big():
    nl = P.gen_netlist(P.GenParams(0x5EED0301, 140_000, 3000, 3000, 40))
    n = 256
    codes = helpers.rand_codes(np.random.default_rng(77), nl.n_pi, n)
    return nl, codes, n, O.grade(nl, codes, n, mark_mode=3)


@pytest.mark.parametrize("tile", [0, 32, 64, 128])
def test_every_pair_spills(big, tile):
    nl, codes, n, want = big
    per_pair = O.grade(nl, codes, n, mark_mode=3, want_planes=True).mark.sum(axis=0)
    assert per_pair.min() > 3072  # every pair is beyond the table
    fx, fy, tot = _grade(nl, codes, n, 3, tile)
    np.testing.assert_array_equal(fx, want.first_x)
    np.testing.assert_array_equal(fy, want.first_y)
    assert tot.value == want.total and tot.flags == want.flags


def test_spill_in_a_batch(big):
    """A batch mixing a spilling circuit with small ones (both kernels)."""
    import torch
    nl0, codes0, n0, want0 = big
    jobs, want = [], []
    members = [(nl0, codes0, n0, 32)]
    for k in range(3):
        nl = circuits.random_small(50 + k, n_gates=2000, n_pi=60, n_po=300, depth=12)
        members.append((nl, helpers.rand_codes(np.random.default_rng(k), nl.n_pi, 900), 900, (4, 64, 128)[k]))
    for nl, codes, n, tw in members:
        ld = (P.words(n) + 127) // 128 * 128
        v, t = P.planes_from_codes(codes, ld)
        c = P.Circuit(nl, mark_mode=3, tile_words=tw)
        s = P.State(c)
        jobs.append((c, s, torch.from_numpy(v.view(np.int32)).cuda(), torch.from_numpy(t.view(np.int32)).cuda(), n, 0))
        want.append(want0 if nl is nl0 else O.grade(nl, codes, n, mark_mode=3))
    b = P.Batch(jobs)
    b.run()
    b.run()  # replayed: the spill cover's queue starts empty again
    for (c, s, *_), w in zip(jobs, want):
        fx, fy, tot = s.snapshot()
        np.testing.assert_array_equal(fx, w.first_x)
        assert tot.value == 2 * w.total


@pytest.mark.parametrize("mode", [0, 1])
def test_reference_tables_spill_on_a_wide_hub(mode):
    nl = circuits.hub(7000)
    n = 200
    codes = helpers.rand_codes(np.random.default_rng(8), nl.n_pi, n)
    want = O.grade(nl, codes, n, mark_mode=mode, want_planes=True)
    assert want.mark.sum(axis=0).max() > 3072
    for tile in (0, 32, 64):
        fx, fy, tot = _grade(nl, codes, n, mode, tile)
        np.testing.assert_array_equal(fx, want.first_x)
        np.testing.assert_array_equal(fy, want.first_y)
        assert tot.value == want.total


def test_stage_cover_spills():
    """pdf_cover (the stage call) takes the same spill path."""
    import torch
    nl = circuits.hub(7000)
    n = 300
    codes = helpers.rand_codes(np.random.default_rng(9), nl.n_pi, n)
    want = O.grade(nl, codes, n, mark_mode=1, want_planes=True)
    c = P.Circuit(nl, mark_mode=1)
    s = P.State(c)
    W = P.words(n)
    v, t = P.planes_from_codes(codes)
    sv, st, mk = (torch.zeros((nl.n_gates, W), dtype=torch.int32, device="cuda") for _ in range(3))
    P.stage_sim(c, v, t, n, sv, st)
    P.stage_mark(c, sv, st, mk, n)
    P.stage_merge(c, s, sv, mk, n, 0)
    tot = P.stage_cover(c, s, mk, n, 0)
    assert tot.value == want.total
    # the spill cover also reports every input's count for every pair
    s2 = P.State(c)
    P.stage_merge(c, s2, sv, mk, n, 0)
    tot2, raw = P.stage_cover_counts(c, s2, mk, n, 0)
    _, _, counts = O.cover(nl, want.mark, n, 0, want.first_x, want.first_y, want_counts=True)
    np.testing.assert_array_equal(raw, counts)
    assert tot2.value == want.total


def test_fixed_robust_on_c2():
    w = P.WORKLOADS["c2"]
    nl = P.gen_netlist(w["gen"])
    n = 8192
    v, t = P.gen_pairs(P.pair_seed(w["gen"].seed), nl.n_pi, n)
    codes = P.codes_from_planes(v, t, n)
    want = O.grade(nl, codes, n, mark_mode=2)
    for tile in (0, 32, 64):
        fx, fy, tot = _grade(nl, codes, n, 2, tile)
        np.testing.assert_array_equal(fx, want.first_x)
        assert tot.value == want.total


def test_batch_cover_passes(big):
    """A batch's cover runs a small table first (several CTAs per SM), then
    the large table for the pairs that marked more nets, then the spill
    cover: here a 30,000-gate circuit whose pairs mark 670 to 1,330 nets
    each (on both sides of the small table's limit) shares a batch with a
    spilling circuit and a small one; all graded twice, against the oracle."""
    import torch
    nl0, codes0, n0, want0 = big
    mid = P.gen_netlist(P.GenParams(0x5EED0302, 30_000, 700, 700, 40))
    n1 = 256
    codes1 = helpers.rand_codes(np.random.default_rng(5), mid.n_pi, n1)
    want1 = O.grade(mid, codes1, n1, mark_mode=3, want_planes=True)
    per_pair = want1.mark.sum(axis=0)
    assert per_pair.min() < 700 and 1000 < per_pair.max() <= 3072
    small = circuits.random_small(61, n_gates=2000, n_pi=60, n_po=300, depth=12)
    codes2 = helpers.rand_codes(np.random.default_rng(6), small.n_pi, 700)
    members = [(nl0, codes0, n0, 32, want0), (mid, codes1, n1, 64, want1), (mid, codes1, n1, 128, want1),
               (small, codes2, 700, 128, O.grade(small, codes2, 700, mark_mode=3))]
    jobs, want = [], []
    for nl, codes, n, tw, w in members:
        ld = (P.words(n) + 127) // 128 * 128
        v, t = P.planes_from_codes(codes, ld)
        c = P.Circuit(nl, mark_mode=3, tile_words=tw)
        s = P.State(c)
        jobs.append((c, s, torch.from_numpy(v.view(np.int32)).cuda(), torch.from_numpy(t.view(np.int32)).cuda(), n, 0))
        want.append(w)
    b = P.Batch(jobs)
    assert b.info().launches == b.info().forward_launches + 4  # active, two cover tables, spill
    b.run()
    b.run()  # replayed: every pass's queue starts empty again
    for (c, s, *_), w in zip(jobs, want):
        fx, fy, tot = s.snapshot()
        np.testing.assert_array_equal(fx, w.first_x)
        np.testing.assert_array_equal(fy, w.first_y)
        assert tot.value == 2 * w.total and tot.flags == w.flags
