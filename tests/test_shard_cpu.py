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


def _rank_mean(rank, world, port, out_dir):
    """Each rank returns the MEAN of its shots' (synthetic) per-shot gradients,
    as gj_w_gradient does with per-shot conditioning."""
    import torch.distributed as dist
    import datetime
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        per_shot = np.random.default_rng(7).standard_normal((5, 2, 6, 4))  # 5 shots, (eps, sig) 6 x 4

        def local(idx):
            return {"g_eps": per_shot[idx, 0].mean(0), "g_sig": per_shot[idx, 1].mean(0),
                    "misfit": np.asarray(idx, np.float64) + 0.5}

        r = shard.gradient(local, 5, (6, 4), rank, world, mean=True)
        np.savez(os.path.join(out_dir, f"m{rank}.npz"), **r)
    finally:
        dist.destroy_process_group()


def test_two_rank_conditioned_mean_over_uneven_shares(tmp_path):
    """5 shots over 2 ranks (3 + 2): the all-reduced result is the mean over
    all 5 shots (w_update_e_.m:38), not the sum or mean of the rank means."""
    world, port = 2, _free_port()
    mp.start_processes(_rank_mean, args=(world, port, str(tmp_path)), nprocs=world, join=True, start_method="spawn")
    per_shot = np.random.default_rng(7).standard_normal((5, 2, 6, 4))
    for rank in range(world):
        r = np.load(tmp_path / f"m{rank}.npz")
        assert np.allclose(r["g_eps"], per_shot[:, 0].mean(0), rtol=1e-13, atol=1e-15)
        assert np.allclose(r["g_sig"], per_shot[:, 1].mean(0), rtol=1e-13, atol=1e-15)
        assert np.allclose(r["misfit"], np.arange(5) + 0.5)


def _dc_case():
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, here)
    sys.path.insert(0, os.path.join(here, "..", "oracle"))
    from dc_cases import small_dc
    case = small_dc(seed=3, pairs=3, levels=2)
    rng = np.random.default_rng(4)
    for q in case["srcs"]:
        q.d_obs = rng.standard_normal(q.nd) * 1e-3
    return case


def _dc_local(case, idx):
    import np_dc_oracle as dco
    from dc_cases import oracle_alphas
    n, m = case["n"], case["m"]
    g, mis = 0.0, []
    for i in idx:
        q = case["srcs"][i]
        Mop = dco.measuring_operator(n, m, q.mn)
        al = oracle_alphas(dco, case, q)
        _, uk, _, e = dco.dc_fwd2_5d(case["SIG"], case["DX"], case["DZ"], dco.source_vector(n, m, q.a, q.b, q.current),
                                     al, q.ky_w, Mop, q.d_obs)
        g = g + dco.dc_gradient2_5d(case["SIG"], case["DX"], case["DZ"], al, q.ky_w, Mop, uk, e, case["robin"])
        mis.append(0.5 * float(e @ e))
    return {"g": g, "misfit": mis}


def _rank_dc(rank, world, port, out_dir):
    import torch.distributed as dist
    import datetime
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        case = _dc_case()
        shape = (case["n"] - 2 * case["robin"], case["m"] - case["robin"])
        r = shard.dc_gradient(lambda idx: _dc_local(case, idx), len(case["srcs"]), shape, rank, world)
        np.savez(os.path.join(out_dir, f"dc{rank}.npz"), **r)
    finally:
        dist.destroy_process_group()


def test_two_rank_dc_gradient_equals_single_process(tmp_path):
    """DC sources sharded over 2 ranks (the oracle's direct solves per rank),
    one all-reduce: equal to the single-process sum over all sources."""
    world, port = 2, _free_port()
    mp.start_processes(_rank_dc, args=(world, port, str(tmp_path)), nprocs=world, join=True, start_method="spawn")
    case = _dc_case()
    ref = _dc_local(case, list(range(len(case["srcs"]))))
    for rank in range(world):
        r = np.load(tmp_path / f"dc{rank}.npz")
        assert np.allclose(r["g"], ref["g"], rtol=1e-12, atol=1e-14 * np.abs(ref["g"]).max())
        assert np.allclose(r["misfit"], ref["misfit"], rtol=1e-13)
