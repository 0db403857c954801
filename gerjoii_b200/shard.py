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
             group=None, device="cpu", mean: bool = False) -> dict:
    """Gradient (g_eps, g_sig) over all shots and the per-shot misfits.

    `local(indices)` returns ``{"g_eps", "g_sig", "misfit"}`` for the given
    shots: the two gradients over those shots (m x n arrays) and one misfit per
    shot, e.g. ``Context.w_gradient`` on that subset.  By default the
    gradients are sums over the shots and so is the result.  With
    ``mean=True`` they are means over the given shots (``gj_w_gradient`` with
    per-shot conditioning returns the shot mean, w_update_e_.m:38 divides the
    sum by the number of shots): each rank's mean is turned back into its sum
    before the all-reduce and the total is divided by `nshots` after it, so
    uneven shares average correctly.  Every rank calls this function; ranks
    with no shots contribute zeros.
    """
    import torch
    mine = shard(nshots, rank, world)
    m, n = shape
    buf = torch.zeros(2 * m * n + nshots, dtype=torch.float64, device=device)
    if mine:
        r = local(mine)
        w = float(len(mine)) if mean else 1.0
        ge = w * np.asarray(r["g_eps"], np.float64).reshape(m, n)
        gs = w * np.asarray(r["g_sig"], np.float64).reshape(m, n)
        mis = np.zeros(nshots)
        mis[mine] = np.asarray(r["misfit"], np.float64)
        host = np.concatenate([ge.ravel(order="F"), gs.ravel(order="F"), mis])
        buf.copy_(torch.from_numpy(host))
    allreduce_sum([buf], group)
    out = buf.cpu().numpy()
    mn = m * n
    scale = 1.0 / nshots if mean else 1.0
    return {"g_eps": scale * out[:mn].reshape((m, n), order="F"),
            "g_sig": scale * out[mn:2 * mn].reshape((m, n), order="F"), "misfit": out[2 * mn:]}


def dc_gradient(local: Callable[[list[int]], dict], nsrc: int, shape: tuple[int, int], rank: int, world: int,
                group=None, device="cpu") -> dict:
    """DC sensitivity over all current dipoles, sharded like the radar shots.

    The reference loops over the sources (dc_update2_5d.m per source ``i_e``,
    summed by its caller); every (source, ky) system is independent.
    `local(indices)` returns ``{"g", "misfit"}`` for the given sources: their
    summed gradient (``shape``, the trimmed n x m model of dc_gradient2_5d.m:37-41,
    e.g. ``Context.dc_gradient`` on that subset) and one misfit per source.
    One all-reduce sums the gradients and places the misfits.
    """
    import torch
    mine = shard(nsrc, rank, world)
    n0, m0 = shape
    buf = torch.zeros(n0 * m0 + nsrc, dtype=torch.float64, device=device)
    if mine:
        r = local(mine)
        g = np.asarray(r["g"], np.float64).reshape(n0, m0)
        mis = np.zeros(nsrc)
        mis[mine] = np.asarray(r["misfit"], np.float64)
        buf.copy_(torch.from_numpy(np.concatenate([g.ravel(), mis])))
    allreduce_sum([buf], group)
    out = buf.cpu().numpy()
    return {"g": out[:n0 * m0].reshape(n0, m0), "misfit": out[n0 * m0:]}


def select(items: Sequence, indices: Sequence[int]) -> list:
    """The items at `indices` (shots, observed traces) in that order."""
    return [items[i] for i in indices]
