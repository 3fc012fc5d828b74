"""Pair sharding across ranks (one process per GPU, torch.distributed).

Rank r grades pairs [r * n, (r + 1) * n).  Pairs interact only through the
first-detect ids, so the one exchange is an unsigned MIN of first_x /
first_y between marking and counting; the ranks' counts then add up to the
count of one grading of all the pairs (the batching invariance of the
reference's chunk loop, main.cu:171-231).
"""
from __future__ import annotations

import torch
import torch.distributed as dist

_FLIP = -(1 << 31)  # xor with the sign bit maps unsigned order onto signed order


def allreduce_min_u32_(t: torch.Tensor, group=None) -> torch.Tensor:
    """In-place MIN over ranks of int32 tensors holding uint32 values."""
    t.bitwise_xor_(_FLIP)
    dist.all_reduce(t, op=dist.ReduceOp.MIN, group=group)
    t.bitwise_xor_(_FLIP)
    return t


def sum_u128(value: int, device, group=None) -> int:
    """Exact sum over ranks of a non-negative 128-bit count."""
    parts = torch.tensor([(value >> (32 * i)) & 0xFFFFFFFF for i in range(4)], dtype=torch.int64,
                         device=device)
    dist.all_reduce(parts, op=dist.ReduceOp.SUM, group=group)  # 32-bit limbs cannot overflow int64
    return sum(int(x) << (32 * i) for i, x in enumerate(parts.tolist()))


def exchange_first_(fx: torch.Tensor, fy: torch.Tensor, group=None) -> None:
    allreduce_min_u32_(fx, group)
    allreduce_min_u32_(fy, group)
