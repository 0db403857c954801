"""Shot sharding and the gradient all-reduce over two ranks (gloo, CPU).

Each rank computes the exact gradient of its round-robin share of the shots
with the oracle and the ranks sum them with one all-reduce; the result must
equal the single-process gradient over all shots, and the per-shot misfits
must land in their own slots."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from gerjoii_b200 import shard


def test_shard_is_round_robin_and_complete():
    parts = [shard.shard(11, r, 3) for r in range(3)]
    assert parts[0] == [0, 3, 6, 9] and parts[2] == [2, 5, 8]
    assert sorted(sum(parts, [])) == list(range(11))
    assert shard.shard(2, 3, 4) == []
    with pytest.raises(ValueError):
        shard.shard(5, 4, 4)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.join(here, "..", "oracle"))
    import pyoracle as O
    from gerjoii_b200 import synth
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        p = synth.small(m=20, n=36, pml=8, nt=200, nsrc=5, nrec=8, seed=41)
        dobs = [O.forward(p.grid, p.eps_true, p.sig_true, sh)[0] for sh in p.shots]

        def local(idx):
            sh = shard.select(p.shots, idx)
            d = np.stack([x.T for x in shard.select(dobs, idx)])
            ge, gs, mis = O.gradient_batch(p.grid, p.eps0, p.sig0, sh, d, mode="exact", threads=1)
            return {"g_eps": ge, "g_sig": gs, "misfit": mis}

        r = shard.gradient(local, len(p.shots), (p.grid.m, p.grid.n), rank, world)
        np.savez(os.path.join(out_dir, f"r{rank}.npz"), **r)
    finally:
        dist.destroy_process_group()


def test_two_rank_gradient_equals_single_process(oracle, tmp_path):
    world, port = 2, _free_port()
    mp.start_processes(_rank_main, args=(world, port, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    from gerjoii_b200 import synth
    p = synth.small(m=20, n=36, pml=8, nt=200, nsrc=5, nrec=8, seed=41)
    dobs = np.stack([oracle.forward(p.grid, p.eps_true, p.sig_true, sh)[0].T for sh in p.shots])
    ge, gs, mis = oracle.gradient_batch(p.grid, p.eps0, p.sig0, p.shots, dobs, mode="exact", threads=1)
    for rank in range(world):
        r = np.load(tmp_path / f"r{rank}.npz")
        assert np.allclose(r["g_eps"], ge, rtol=1e-12, atol=1e-14 * np.abs(ge).max())
        assert np.allclose(r["g_sig"], gs, rtol=1e-12, atol=1e-14 * np.abs(gs).max())
        assert np.allclose(r["misfit"], mis, rtol=1e-13)
