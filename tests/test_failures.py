"""Failure paths, made to happen without faulting the GPU: a device-side
wait bounded to one poll runs out (the kernel drains its copies in flight
and reports PDF_ETIMEOUT, the context stays usable), and allocations fail
through the library's host-side fault injection (PDF_ENOMEM, the objects
stay usable).  The reference exits the process on any CUDA error
(HANDLE_ERROR, simkernel.cuh:32-39, coverkernel.cuh:15-25)."""
import numpy as np
import pytest

import circuits
import helpers

pytestmark = pytest.mark.gpu

P = helpers.pdf()
O = helpers.oracle()
ETIMEOUT, ENOMEM = 4, 2


def _case(n=600, seed=3):
    nl = circuits.random_small(4242, n_gates=400, n_pi=30, n_po=120, depth=10)
    codes = helpers.rand_codes(np.random.default_rng(seed), nl.n_pi, n)
    return nl, codes, n


def test_expired_wait_reports_timeout_and_the_device_stays_usable():
    nl, codes, n = _case()
    v, t = P.planes_from_codes(codes)
    c = P.Circuit(nl, mark_mode=1, wait_polls=1)  # one non-blocking poll per staged copy
    s = P.State(c)
    with pytest.raises(P.PdfError) as e:
        P.grade(c, s, v, t, n)
    assert e.value.status == ETIMEOUT
    # the state holds an incomplete batch: it says so until it is reset
    with pytest.raises(P.PdfError) as e:
        s.snapshot()
    assert e.value.status == ETIMEOUT
    s.close()
    c.close()
    # the context is intact: the same grading with the default bound is exact
    c2 = P.Circuit(nl, mark_mode=1)
    s2 = P.State(c2)
    tot = P.grade(c2, s2, v, t, n)
    assert tot.value == O.grade(nl, codes, n, mark_mode=1).total


def test_expired_wait_in_a_stage_call_is_reported_once():
    """pdf_sim with a one-poll bound reports the expired wait; the circuit's
    error word is cleared there, so a later stage call is not blamed."""
    import torch
    nl, codes, n = _case(500, 4)
    v, t = P.planes_from_codes(codes)
    W = P.words(n)
    sv, st = (torch.zeros((nl.n_gates, W), dtype=torch.int32, device="cuda") for _ in range(2))
    c = P.Circuit(nl, wait_polls=1)
    with pytest.raises(P.PdfError) as e:
        P.stage_sim(c, v, t, n, sv, st)
    assert e.value.status == ETIMEOUT
    c.close()
    good = P.Circuit(nl)
    P.stage_sim(good, v, t, n, sv, st)
    torch.cuda.synchronize()
    h = lambda x: x.cpu().numpy().view(np.uint32)
    np.testing.assert_array_equal(P.codes_from_planes(h(sv), h(st), n), O.sim(nl, codes, n))


def test_device_allocation_failure_leaves_the_state_usable():
    nl, codes, n = _case(3000, 5)
    v, t = P.planes_from_codes(codes)
    c = P.Circuit(nl, mark_mode=1)
    s = P.State(c)
    P.inject_failures(P.INJECT_DEVICE_ALLOC, 1)  # the state's first workspace allocation
    try:
        with pytest.raises(P.PdfError) as e:
            P.grade(c, s, v, t, n)
        assert e.value.status == ENOMEM
    finally:
        P.inject_failures(P.INJECT_DEVICE_ALLOC, 0)
    s.reset()
    tot = P.grade(c, s, v, t, n)
    want = O.grade(nl, codes, n, mark_mode=1)
    fx, fy, _ = s.snapshot()
    assert tot.value == want.total
    np.testing.assert_array_equal(fx, want.first_x)


def test_circuit_creation_allocation_failure():
    nl, _, _ = _case()
    P.inject_failures(P.INJECT_DEVICE_ALLOC, 1)
    try:
        with pytest.raises(P.PdfError) as e:
            P.Circuit(nl)
        assert e.value.status == ENOMEM
    finally:
        P.inject_failures(P.INJECT_DEVICE_ALLOC, 0)
    P.Circuit(nl).close()


def test_server_step_survives_a_failed_pinned_allocation():
    """The server's pinned read-back staging cannot be allocated (at creation
    and at the first step that retires a job): that step fails with
    PDF_ENOMEM and retires nothing; the next steps retire every job with the
    same results as offline grading."""
    jobs = []
    for k in range(3):
        nl = circuits.random_small(900 + k, n_gates=1500, n_pi=60, n_po=200, depth=12)
        v, t = P.gen_pairs(77 + k, nl.n_pi, 2048)
        jobs.append((nl, v, t))
    P.inject_failures(P.INJECT_HOST_ALLOC, 2)
    try:
        srv = P.Server(mark_mode=1, batch_pairs=1024)
        ids = [srv.submit(nl, v, t, 2048) for nl, v, t in jobs]
        failed = 0
        for _ in range(200):
            if srv.stats().jobs_done == len(jobs):
                break
            try:
                srv.step()
            except P.PdfError as e:
                assert e.status == ENOMEM
                failed += 1
        assert failed == 1
    finally:
        P.inject_failures(P.INJECT_HOST_ALLOC, 0)
    assert srv.stats().jobs_done == len(jobs)
    for (nl, v, t), jid in zip(jobs, ids):
        fx, fy, tot = srv.result(jid)
        want = O.grade(nl, P.codes_from_planes(v, t, 2048), 2048, mark_mode=1, chunk=1024)
        assert tot.value == want.total and tot.pairs == 2048
        np.testing.assert_array_equal(fx, want.first_x)
        np.testing.assert_array_equal(fy, want.first_y)
    srv.close()
