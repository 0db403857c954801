"""Shot-parallel gradients over ranks (one process per GPU).

The reference evaluates shots independently (``parfor`` over shots in
w_update_e_.m:32 and w_update_s_.m, each worker calling w_fwd / w_grad on its
own shot) and sums their gradients (w_update_e_.m:38).  Here each rank takes a
round-robin share of the shots, computes their summed gradient with one
batched call on its GPU, and a single all-reduce per evaluation sums the two
gradients and the per-shot misfit vector over the ranks.  No other data moves
between ranks.

The functions work on any ``torch.distributed`` backend: NCCL with CUDA
tensors on the GPUs, gloo with CPU tensors for the host-side tests.
"""
from __future__ import annotations

from typing import Callable, Sequence

import numpy as np


def shard(n: int, rank: int, world: int) -> list[int]:
    """Indices of the shots owned by `rank`: rank, rank + world, ..."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError(f"bad rank {rank} of world {world}")
    return list(range(rank, n, world))


def allreduce_sum(tensors, group=None) -> None:
    """Sums each tensor in place over the ranks (one all-reduce per tensor)."""
    import torch.distributed as dist
    for t in tensors:
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)


def gradient(local: Callable[[list[int]], dict], nshots: int, shape: tuple[int, int], rank: int, world: int,
             group=None, device="cpu") -> dict:
    """Summed (g_eps, g_sig) over all shots and the per-shot misfits.

    `local(indices)` returns ``{"g_eps", "g_sig", "misfit"}`` for the given
    shots: the two gradients summed over those shots (m x n arrays) and one
    misfit per shot, e.g. ``Context.w_gradient`` on that subset.  Every rank
    calls this function; ranks with no shots contribute zeros.
    """
    import torch
    mine = shard(nshots, rank, world)
    m, n = shape
    buf = torch.zeros(2 * m * n + nshots, dtype=torch.float64, device=device)
    if mine:
        r = local(mine)
        ge = np.asarray(r["g_eps"], np.float64).reshape(m, n)
        gs = np.asarray(r["g_sig"], np.float64).reshape(m, n)
        mis = np.zeros(nshots)
        mis[mine] = np.asarray(r["misfit"], np.float64)
        host = np.concatenate([ge.ravel(order="F"), gs.ravel(order="F"), mis])
        buf.copy_(torch.from_numpy(host))
    allreduce_sum([buf], group)
    out = buf.cpu().numpy()
    mn = m * n
    return {"g_eps": out[:mn].reshape((m, n), order="F"), "g_sig": out[mn:2 * mn].reshape((m, n), order="F"),
            "misfit": out[2 * mn:]}


def select(items: Sequence, indices: Sequence[int]) -> list:
    """The items at `indices` (shots, observed traces) in that order."""
    return [items[i] for i in indices]
