"""Pair sharding with the first-detect exchange, world size 2 on CPU (gloo).

Each rank marks its own pairs, the ranks reduce first_x/first_y with the
unsigned MIN of gpu-path-delay-coverage_b200/dist.py, each rank counts its
pairs, and the counts sum to one grading of all pairs.  The per-rank compute
is the oracle; what is under test is the exchange.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import circuits
import helpers


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, n_per, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        P = helpers.pdf()
        O = helpers.oracle()
        D = helpers._load("pdf_b200_dist", helpers.PKG_DIR / "dist.py")
        nl = circuits.random_small(2024, n_gates=120, n_pi=10, n_po=50, depth=6, mask=circuits.MARKING_TYPES)
        rng = np.random.default_rng(77)
        codes = helpers.rand_codes(rng, nl.n_pi, world * n_per)
        mine = codes[:, rank * n_per:(rank + 1) * n_per]
        base = rank * n_per
        sim = O.sim(nl, mine, n_per)
        mark = O.mark(nl, sim, n_per)
        fx = np.full(nl.n_gates, 0xFFFFFFFF, np.uint32)
        fy = fx.copy()
        O.merge(nl, sim, mark, n_per, base, fx, fy)
        tx = torch.from_numpy(fx.view(np.int32).copy())
        ty = torch.from_numpy(fy.view(np.int32).copy())
        D.exchange_first_(tx, ty)
        gfx, gfy = tx.numpy().view(np.uint32), ty.numpy().view(np.uint32)
        count, _ = O.cover(nl, mark, n_per, base, gfx, gfy)
        total = D.sum_u128(count, "cpu")
        q.put((rank, total, gfx.copy(), gfy.copy()))
    finally:
        dist.destroy_process_group()


def test_sharded_grading_equals_one_grading():
    world, n_per = 2, 300
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, n_per, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    P = helpers.pdf()
    O = helpers.oracle()
    nl = circuits.random_small(2024, n_gates=120, n_pi=10, n_po=50, depth=6, mask=circuits.MARKING_TYPES)
    rng = np.random.default_rng(77)
    codes = helpers.rand_codes(rng, nl.n_pi, world * n_per)
    want = O.grade(nl, codes, world * n_per)
    assert want.total > 0
    for rank, total, fx, fy in res:
        assert total == want.total
        np.testing.assert_array_equal(fx, want.first_x)
        np.testing.assert_array_equal(fy, want.first_y)


def test_unsigned_min_trick():
    vals = np.array([0, 1, 0x7FFFFFFF, 0x80000000, 0xFFFFFFFE, 0xFFFFFFFF], np.uint32)
    for a in vals:
        for b in vals:
            ta = np.int32(np.uint32(a).view(np.int32) ^ np.int32(-(1 << 31)))
            tb = np.int32(np.uint32(b).view(np.int32) ^ np.int32(-(1 << 31)))
            m = np.int32(min(ta, tb) ^ np.int32(-(1 << 31))).view(np.uint32)
            assert m == min(a, b)
