"""Parity at the benchmark's own sizes: the 1,000,000-gate Zipf netlist
(c3: Zipf-weighted fan-out, levels of 5,000 gates, far wider than any
on-chip ring, mark bitmaps of 125 KB) and the whole mixed-size batch
of 256 netlists (c4), each graded by the CUDA path and compared with the CPU
oracle on a prefix of its pairs: first-detect ids, counts and flags."""
import numpy as np
import pytest

import helpers

pytestmark = pytest.mark.gpu

P = helpers.pdf()
O = helpers.oracle()


@pytest.fixture(scope="module")
def c3():
    w = P.WORKLOADS["c3"]
    nl = P.gen_netlist(w["gen"])
    n = 2048
    v, t = P.gen_pairs(P.pair_seed(w["gen"].seed), nl.n_pi, n)
    codes = P.codes_from_planes(v, t, n)
    return nl, v, t, codes, n, O.grade(nl, codes, n, mark_mode=1, chunk=1024)


@pytest.mark.parametrize("tile", [0, 8, 32, 64, 128])
def test_c3_prefix_in_two_batches(c3, tile):
    nl, v, t, codes, n, want = c3
    c = P.Circuit(nl, mark_mode=1, max_pairs=n, tile_words=tile)
    s = P.State(c)
    totals = []
    for a in (0, 1024):
        bv, bt = P.planes_from_codes(codes[:, a:a + 1024])
        totals.append(P.grade(c, s, bv, bt, 1024, a).value)
    fx, fy, tot = s.snapshot()
    np.testing.assert_array_equal(fx, want.first_x)
    np.testing.assert_array_equal(fy, want.first_y)
    assert tot.value == want.total and tot.flags == want.flags and tot.pairs == n
    assert totals == want.chunk_totals
    # the same pairs in one batch
    s2 = P.State(c)
    one = P.grade(c, s2, v, t, n)
    assert one.value == sum(totals)


@pytest.mark.parametrize("tile", [0, 32, 64, 128])
def test_c4_batch_against_the_oracle(tile):
    """The 256 circuits of the mixed-size batch in one batched pass, each on
    its first min(n, 1024) pairs; every 8th circuit (32 of them, all sizes)
    checked against the oracle, and every circuit against its own plain call."""
    import torch
    spec = P.batch_workload()
    jobs, hosts = [], []
    for g, n in spec:
        nl = P.gen_netlist(g)
        k = min(n, 1024)
        v, t = P.gen_pairs(P.pair_seed(g.seed), nl.n_pi, k, 128)
        c = P.Circuit(nl, mark_mode=1, max_pairs=k, tile_words=tile)
        jobs.append((c, P.State(c), torch.from_numpy(v.view(np.int32)).cuda(),
                     torch.from_numpy(t.view(np.int32)).cuda(), k, 0))
        hosts.append((nl, v, t, k))
    b = P.Batch(jobs)
    b.run()
    for i, ((c, s, dv, dt, k, _), (nl, v, t, _)) in enumerate(zip(jobs, hosts)):
        fx, fy, tot = s.snapshot()
        if i % 8 == 0:
            want = O.grade(nl, P.codes_from_planes(v, t, k), k, mark_mode=1)
            np.testing.assert_array_equal(fx, want.first_x)
            np.testing.assert_array_equal(fy, want.first_y)
            assert tot.value == want.total and tot.flags == want.flags, i
        s2 = P.State(c)
        alone = P.grade(c, s2, dv, dt, k)
        assert alone.value == tot.value, i
        s2.close()
