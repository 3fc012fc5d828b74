"""Batched grading (pdf_batch_*): many circuits of uneven size and pair count
in one pass of three launches replayed from a CUDA graph.  Every job's
first-detect ids, count and flags must equal grading that job alone."""
import numpy as np
import pytest

import circuits
import helpers

pytestmark = pytest.mark.gpu

P = helpers.pdf()
O = helpers.oracle()


def _jobs(mode, tile=4, seed=0):
    """Circuits of many shapes and pair counts (including ragged tails).
    tile: one tile width for every job, or a list of widths taken in turn."""
    import torch
    shapes = [s[1] for s in circuits.small_suite()[:6]]
    shapes += [circuits.random_small(500 + seed, n_gates=3000, n_pi=120, n_po=400, depth=25),
               circuits.random_small(600 + seed, n_gates=12000, n_pi=1500, n_po=3000, depth=7),
               circuits.random_small(700 + seed, n_gates=8000, n_pi=300, n_po=800, depth=60, fmax=6),
               circuits.hub(150), circuits.diamond_chain(20)]
    counts = [33, 1000, 1, 2500, 64, 777, 4096, 700, 3001, 900, 40]
    rng = np.random.default_rng(11 + seed)
    jobs, want = [], []
    tiles = tile if isinstance(tile, list) else [tile]
    for k, (nl, n) in enumerate(zip(shapes, counts)):
        tw = tiles[k % len(tiles)]
        codes = helpers.rand_codes(rng, nl.n_pi, n)
        ld = (P.words(n) + tw - 1) // tw * tw
        v, t = P.planes_from_codes(codes, ld)
        c = P.Circuit(nl, mark_mode=mode, tile_words=tw)
        s = P.State(c)
        dv = torch.from_numpy(v.view(np.int32)).cuda()
        dt = torch.from_numpy(t.view(np.int32)).cuda()
        jobs.append((c, s, dv, dt, n, 0))
        want.append((nl, codes, n))
    return jobs, want


@pytest.mark.parametrize("tile", [4, 32, 64, 128, [32, 4, 64, 8, 128, 2]], ids=["walk4", "lanes", "lanes64", "lanes128", "mixed"])
@pytest.mark.parametrize("mode", [0, 1, 2, 3])
def test_batch_equals_each_job_alone(mode, tile):
    """Every tile width in one batch (mixed: one forward launch per class of
    tile width and CTAs per SM)."""
    jobs, want = _jobs(mode, tile)
    b = P.Batch(jobs)
    b.run()
    info = b.info()
    assert info.n_jobs == len(jobs)
    assert info.gate_evals == sum(nl.n_gates * n for nl, _, n in want)
    for (c, s, *_), (nl, codes, n) in zip(jobs, want):
        w = O.grade(nl, codes, n, mark_mode=mode)
        fx, fy, tot = s.snapshot()
        np.testing.assert_array_equal(fx, w.first_x)
        np.testing.assert_array_equal(fy, w.first_y)
        assert tot.value == w.total and tot.flags == w.flags and tot.pairs == n


def test_batch_replay_is_stable():
    """A second replay over the same pairs adds the same counts again."""
    jobs, want = _jobs(1, seed=1)
    b = P.Batch(jobs)
    b.run()
    first = [s.snapshot()[2].value for _, s, *_ in jobs]
    b.run()
    again = [s.snapshot()[2].value for _, s, *_ in jobs]
    assert again == [2 * x for x in first]
    assert sum(first) > 0


def test_batch_append_grades_consecutive_pairs():
    """With append, run k grades pairs [k n, (k+1) n) of each job (the pair
    planes rewritten between runs); the state equals one grading of all."""
    import torch
    jobs, want = _jobs(0, seed=2)
    rng = np.random.default_rng(99)
    extra = []
    b = P.Batch(jobs, append=True)
    b.run()
    for (c, s, dv, dt, n, _), (nl, codes, _) in zip(jobs, want):
        more = helpers.rand_codes(rng, nl.n_pi, n)
        v, t = P.planes_from_codes(more, dv.shape[1])
        dv.copy_(torch.from_numpy(v.view(np.int32)))
        dt.copy_(torch.from_numpy(t.view(np.int32)))
        extra.append(more)
    torch.cuda.synchronize()
    b.run()
    for (c, s, *_), (nl, codes, n), more in zip(jobs, want, extra):
        w = O.grade(nl, np.concatenate([codes, more], axis=1), 2 * n, chunk=n)
        fx, fy, tot = s.snapshot()
        np.testing.assert_array_equal(fx, w.first_x)
        np.testing.assert_array_equal(fy, w.first_y)
        assert tot.value == w.total and tot.pairs == 2 * n


def test_batch_rebind_to_other_jobs():
    """A batch rebound to a different (smaller, then larger) job list grades
    exactly that list; jobs left out are not touched."""
    jobs, want = _jobs(1, seed=3)
    b = P.Batch(jobs[:3])
    b.run()
    b.rebind(jobs[3:])
    b.run()
    b.rebind(jobs[:2])
    b.run()
    assert b.info().n_jobs == 2
    for k, ((c, s, *_), (nl, codes, n)) in enumerate(zip(jobs, want)):
        w = O.grade(nl, codes, n, mark_mode=1)
        fx, fy, tot = s.snapshot()
        runs = 2 if k < 2 else 1
        assert tot.value == runs * w.total and tot.pairs == runs * n
        np.testing.assert_array_equal(fx, w.first_x)


def test_batch_rejects_mixed_mark_modes():
    jobs, _ = _jobs(0)
    c, s, dv, dt, n, base = jobs[0]
    c1 = P.Circuit(c.netlist, mark_mode=1)
    s1 = P.State(c1)
    with pytest.raises(P.PdfError):
        P.Batch([jobs[1], (c1, s1, dv, dt, n, base)])


def test_batch_append_mixed_tiles():
    """Appending runs over a batch whose jobs take different kernels."""
    jobs, want = _jobs(1, [32, 4], seed=4)
    b = P.Batch(jobs, append=True)
    b.run()
    b.run()  # the same planes again: pairs [n, 2n) repeat pairs [0, n)
    for (c, s, *_), (nl, codes, n) in zip(jobs, want):
        w = O.grade(nl, np.concatenate([codes, codes], axis=1), 2 * n, mark_mode=1, chunk=n)
        fx, fy, tot = s.snapshot()
        np.testing.assert_array_equal(fx, w.first_x)
        np.testing.assert_array_equal(fy, w.first_y)
        assert tot.value == w.total and tot.pairs == 2 * n


@pytest.mark.parametrize("graph", [True, False], ids=["graph", "direct"])
def test_batch_profile_times_the_pass(graph):
    """pdf_batch_profile: forward span and cover of the latest pass, from
    events inside the replayed graph or around the direct launches; results
    unchanged."""
    jobs, want = _jobs(1, [32, 4], seed=5)
    b = P.Batch(jobs, graph=graph)
    b.profile(True)
    b.run()
    fwd, cov = b.profile_read()
    assert fwd > 0 and cov > 0
    b.profile(False)
    b.run()
    for (c, s, *_), (nl, codes, n) in zip(jobs, want):
        assert s.snapshot()[2].value == 2 * O.grade(nl, codes, n, mark_mode=1).total


def test_autotune_picks_a_tile():
    nls = [circuits.random_small(800 + k, n_gates=2000 * (k + 1), n_pi=100, n_po=300, depth=20) for k in range(4)]
    opts, ms = P.batch_autotune(nls, [1024, 3000, 5000, 700], mark_mode=1, reps=2)
    assert opts.tile_words in (2, 4, 8, 32, 64, 128) and opts.threads in (0, 256) and ms > 0
    # the picked shape grades the batch like every circuit alone
    counts = [1024, 3000, 5000, 700]
    rng = np.random.default_rng(5)
    for nl, n in zip(nls, counts):
        codes = helpers.rand_codes(rng, nl.n_pi, n)
        c = P.Circuit(nl, mark_mode=1, tile_words=opts.tile_words, threads=opts.threads)
        s = P.State(c)
        v, t = P.planes_from_codes(codes)
        tot = P.grade(c, s, v, t, n)
        assert tot.value == O.grade(nl, codes, n, mark_mode=1).total
    # a fixed block size is kept
    opts2, _ = P.batch_autotune(nls, counts, mark_mode=1, reps=1, threads=384)
    assert opts2.threads == 384
