"""Serving (pdf_server_*): jobs arrive over time, are admitted by device
footprint, graded in batches that append to their device-resident coverage
state, and overlap with other jobs on the device.  Every job's result must be
the same alone and in the mix, and equal to grading all its pairs at once."""
import numpy as np
import pytest

import circuits
import helpers

pytestmark = pytest.mark.gpu

P = helpers.pdf()
O = helpers.oracle()

BATCH = 256


def _jobs():
    shapes = [s[1] for s in circuits.small_suite()[:5]]
    shapes += [circuits.random_small(900, n_gates=3000, n_pi=120, n_po=400, depth=25),
               circuits.random_small(901, n_gates=9000, n_pi=700, n_po=900, depth=40),
               circuits.hub(150)]
    # 1024, 1252, 2048 and 256 pairs have pitches that let each batch be read
    # in place (1252: a short last batch); the others are copied per batch
    counts = [700, 1024, 300, 2 * BATCH + 17, 1252, 1500, 2048, 256]
    rng = np.random.default_rng(21)
    out = []
    for nl, n in zip(shapes, counts):
        codes = helpers.rand_codes(rng, nl.n_pi, n)
        v, t = P.planes_from_codes(codes)
        out.append((nl, codes, v, t, n))
    return out


def _serve(jobs, budget=0, mode=1, arrive_every=2, tile=4):
    srv = P.Server(mark_mode=mode, batch_pairs=BATCH, hbm_budget=budget, tile_words=tile)
    ids, pending = [], list(jobs)
    steps = 0
    while pending or srv.stats().jobs_done < len(jobs):
        # a new job arrives every few steps, while others are on the GPU
        if pending and steps % arrive_every == 0:
            nl, codes, v, t, n = pending.pop(0)
            ids.append(srv.submit(nl, v, t, n))
        srv.step()
        steps += 1
        assert steps < 100000
    res = [srv.result(i) for i in ids]
    return res, srv.stats()


@pytest.mark.parametrize("mode", [0, 1, 3])
def test_served_results_equal_offline_grading(mode):
    jobs = _jobs()
    res, st = _serve(jobs, mode=mode)
    assert st.jobs_done == len(jobs) and st.jobs_active == 0 and st.jobs_queued == 0
    assert st.gate_evals == sum(nl.n_gates * n for nl, _, _, _, n in jobs)
    assert 0 < st.lat_p50_ms <= st.lat_p99_ms <= st.lat_max_ms
    assert 0 < st.gpu_s <= st.busy_s
    for (nl, codes, v, t, n), (fx, fy, tot) in zip(jobs, res):
        w = O.grade(nl, codes, n, mark_mode=mode, chunk=BATCH)
        np.testing.assert_array_equal(fx, w.first_x)
        np.testing.assert_array_equal(fy, w.first_y)
        assert tot.value == w.total and tot.flags == w.flags and tot.pairs == n


def test_served_alone_equals_in_the_mix():
    jobs = _jobs()
    mixed, _ = _serve(jobs)
    for k in (0, 3, 6):
        alone, _ = _serve([jobs[k]])
        np.testing.assert_array_equal(alone[0][0], mixed[k][0])
        np.testing.assert_array_equal(alone[0][1], mixed[k][1])
        assert alone[0][2].value == mixed[k][2].value


def test_admission_by_footprint_queues_jobs():
    """A budget of about one job admits them one at a time (each still served)."""
    jobs = _jobs()[:4]
    res, st = _serve(jobs, budget=1, arrive_every=1)
    assert st.jobs_done == 4
    for (nl, codes, v, t, n), (fx, fy, tot) in zip(jobs, res):
        assert tot.value == O.grade(nl, codes, n, mark_mode=1, chunk=BATCH).total


@pytest.mark.parametrize("tile", [32, 128])
def test_served_on_lane_tiles(tile):
    """Jobs served with the lane kernel (batches narrower than its column
    block: one partial block per job and step)."""
    jobs = _jobs()
    res, st = _serve(jobs, tile=tile)
    assert st.jobs_done == len(jobs)
    for (nl, codes, v, t, n), (fx, fy, tot) in zip(jobs, res):
        w = O.grade(nl, codes, n, mark_mode=1, chunk=BATCH)
        np.testing.assert_array_equal(fx, w.first_x)
        np.testing.assert_array_equal(fy, w.first_y)
        assert tot.value == w.total and tot.flags == w.flags and tot.pairs == n
