"""The allocation-free cover call, pdf_cover_noalloc, against pdf_cover.

pdf_cover_noalloc serves callers that may not enter the CUDA allocator while
they grade (a framework that owns every device byte through its own pool, or
a latency-bound loop where cudaMalloc could synchronise the device or fail
under memory pressure).  Its scratch is a fixed device array shared by all
calls, so these tests call it twice in a row and check both counts against
the allocating entry point.  This file is collected last on purpose.
"""
import numpy as np
import pytest
import torch

import circuits
import helpers

pytestmark = pytest.mark.gpu

P = helpers.pdf()
LIMIT = 8 << 20  # bytes of the fixed scratch


def device_free_bytes() -> int:
    import ctypes
    rt = ctypes.CDLL("libcudart.so.12")
    free, total = ctypes.c_size_t(), ctypes.c_size_t()
    assert rt.cudaMemGetInfo(ctypes.byref(free), ctypes.byref(total)) == 0
    return free.value


def noalloc(c, mk, n, base, fx, fy):
    """pdf_cover_noalloc, checking that the device's free memory and torch's
    allocations are the same after the call as before it."""
    torch.cuda.synchronize()
    free0, torch0 = device_free_bytes(), torch.cuda.memory_allocated()
    tot = P.Totals_t()
    st = P.lib().pdf_cover_noalloc(c.h, mk.data_ptr(), n, mk.shape[1], base, fx.data_ptr(), fy.data_ptr(),
                                   P.C.byref(tot), None)
    torch.cuda.synchronize()
    assert device_free_bytes() == free0 and torch.cuda.memory_allocated() == torch0
    return st, tot


def test_noalloc_cover_equals_cover_on_consecutive_calls():
    nl = circuits.random_small(4711, n_gates=600, n_pi=40, n_po=200, depth=8, mask=circuits.MARKING_TYPES)
    c = P.Circuit(nl)
    s = P.State(c)
    G, n = nl.n_gates, 3000
    W = P.words(n)
    rng = np.random.default_rng(12)
    fx = torch.empty(G, dtype=torch.int32, device="cuda")
    fy = torch.empty(G, dtype=torch.int32, device="cuda")
    counts = []
    for k in range(2):
        base = k * n
        v, t = P.planes_from_codes(helpers.rand_codes(rng, nl.n_pi, n))
        sv, st, mk = (torch.zeros((G, W), dtype=torch.int32, device="cuda") for _ in range(3))
        P.stage_sim(c, v, t, n, sv, st)
        P.stage_mark(c, sv, st, mk, n)
        P.stage_merge(c, s, sv, mk, n, base)
        P.first_copy(s, fx, fy, False)
        torch.cuda.synchronize()
        want = P.stage_cover(c, s, mk, n, base)
        st, got = noalloc(c, mk, n, base, fx, fy)
        assert st == 0
        assert got.value == want.value
        assert got.flags == want.flags
        assert got.pairs == n
        counts.append(got.value)
    assert sum(counts) > 0


def test_noalloc_cover_rejects_requests_beyond_its_scratch():
    nl = circuits.random_small(4712, n_gates=200_000, n_pi=2000, n_po=2000, depth=20)
    c = P.Circuit(nl)
    dummy = torch.zeros((1, 8), dtype=torch.int32, device="cuda")
    n = 1 << 20  # 1,024 column blocks x 6,250 bitmap words x 4 B > 8 MiB
    tot = P.Totals_t()
    st = P.lib().pdf_cover_noalloc(c.h, dummy.data_ptr(), n, P.words(n), 0, dummy.data_ptr(),
                                   dummy.data_ptr(), P.C.byref(tot), None)
    assert st == 9  # PDF_ELIMIT, before anything runs on the device


def test_noalloc_cover_accepts_a_chunk_just_under_its_scratch():
    """The largest chunk whose scratch fits the fixed array runs (and
    allocates nothing); one column block more is refused."""
    nl = circuits.random_small(4713, n_gates=200_000, n_pi=2000, n_po=2000, depth=20)
    c = P.Circuit(nl)
    tw, G = c.info().tile_words, nl.n_gates
    bmw = (G + 31) // 32

    def need(n):
        a = lambda x: (x + 255) // 256 * 256
        W = P.words(n)
        nb = -(-W // tw)
        return a(nb * bmw * 4) + a(nb * 4) + a(W * 4 + 16) + a(min(W * 32, 2 * G) * 4) + a(64)

    n = 32 * tw
    while need(n + 32 * tw) <= LIMIT:
        n += 32 * tw
    assert need(n) <= LIMIT < need(n + 32 * tw)
    W = P.words(n + 32 * tw)
    mk = torch.zeros((G, W), dtype=torch.int32, device="cuda")  # no marks: a zero count
    fx = torch.full((G,), -1, dtype=torch.int32, device="cuda")
    st, tot = noalloc(c, mk, n, 0, fx, fx)
    assert st == 0 and tot.value == 0 and tot.pairs == n
    st, _ = noalloc(c, mk, n + 32 * tw, 0, fx, fx)
    assert st == 9  # PDF_ELIMIT
