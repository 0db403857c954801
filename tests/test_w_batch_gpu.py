"""gj_w_gradient_batch: independent problems of uneven grids, shot counts and
step counts in memory-budgeted waves, all waves one CUDA graph launch.  Every
problem's gradient must equal its own gj_w_gradient call (FP64), with whole
histories and with a pool budget small enough to force several waves (and
checkpointing where a wave's spare memory cannot hold whole histories), and
on a second call with a new model (the cached wave graphs replayed with new
inputs)."""
import numpy as np
import pytest

from conftest import rel_l2
from gerjoii_b200 import synth
from gerjoii_b200 import _native as N

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def problems(oracle):
    specs = [dict(m=24, n=40, pml=8, nt=220, nsrc=2, nrec=8, seed=51),
             dict(m=40, n=28, pml=6, nt=300, nsrc=3, nrec=6, seed=52, free_top=False),
             dict(m=30, n=64, pml=10, nt=180, nsrc=1, nrec=10, seed=53, kind="layer"),
             dict(m=18, n=36, pml=8, nt=260, nsrc=4, nrec=5, seed=54)]
    out = []
    for sp in specs:
        p = synth.small(**sp)
        dobs = [oracle.forward(p.grid, p.eps_true, p.sig_true, sh)[0] for sh in p.shots]
        out.append((p, dobs))
    return out


def _two_wave_budget(ctx, problems, mode):
    """Largest pool budget (of a descending ladder) that splits the batch into
    at least two waves; smaller ones make some problem checkpoint, the
    smallest may be refused (GJ_ENOMEM) before any wave is planned."""
    probs = [(p.grid, p.eps0, p.sig0, p.shots, d) for p, d in problems]
    for mb in (16, 12, 8, 6, 5, 4):
        o = N.OptsC()
        o.mem_budget_bytes = mb << 20
        try:
            _, nwaves = ctx.w_gradient_batch(probs, mode=mode, precision=N.GJ_F64, opts=o)
        except N.GJError:
            break
        if nwaves >= 2:
            return mb << 20
    pytest.fail("no pool budget of the ladder splits the batch into two waves")


@pytest.mark.parametrize("mode", [N.GJ_ADJ_EXACT, N.GJ_ADJ_REFERENCE])
@pytest.mark.parametrize("budget", ["whole_history", "small_pool"])
def test_batch_equals_single_calls(gpu_ctx, problems, mode, budget):
    o = N.OptsC()
    o.mem_budget_bytes = 0 if budget == "whole_history" else _two_wave_budget(gpu_ctx, problems, mode)
    budget = o.mem_budget_bytes
    for scale in (1.0, 1.03):
        probs = [(p.grid, p.eps0 * scale, p.sig0, p.shots, d) for p, d in problems]
        res, nwaves = gpu_ctx.w_gradient_batch(probs, mode=mode, precision=N.GJ_F64, opts=o)
        if budget:
            assert nwaves >= 2
        for (p, d), r in zip(problems, res):
            ref = gpu_ctx.w_gradient(p.grid, p.eps0 * scale, p.sig0, p.shots, d, mode=mode, precision=N.GJ_F64)
            assert rel_l2(r["g_eps"], ref["g_eps"]) < 1e-11
            assert rel_l2(r["g_sig"], ref["g_sig"]) < 1e-11
            assert np.allclose(r["misfit"], ref["misfit"], rtol=1e-12)


def test_batch_fp32_matches_oracle(gpu_ctx, oracle, problems):
    """FP32 batch against the oracle's FP64 exact gradients (every cell)."""
    probs = [(p.grid, p.eps0, p.sig0, p.shots, d) for p, d in problems]
    res, _ = gpu_ctx.w_gradient_batch(probs, mode=N.GJ_ADJ_EXACT, precision=N.GJ_F32)
    for (p, d), r in zip(problems, res):
        ge, gs, _ = oracle.gradient_batch(p.grid, p.eps0, p.sig0, p.shots, np.stack([x.T for x in d]), mode="exact")
        assert rel_l2(r["g_eps"], ge) < 1e-3
        assert rel_l2(r["g_sig"], gs) < 1e-3


def test_batch_rejects_unsupported_options(gpu_ctx, problems):
    o = N.OptsC()
    o.plain = 1
    probs = [(p.grid, p.eps0, p.sig0, p.shots, d) for p, d in problems[:1]]
    with pytest.raises(N.GJError) as ei:
        gpu_ctx.w_gradient_batch(probs, opts=o)
    assert ei.value.status == N.GJ_EUNSUPPORTED


def test_release_frees_the_batch_pool(gpu_ctx, problems):
    """gj_context_release gives the batch's pool and graph back; the next batch
    call plans again and returns the same gradients."""
    import torch
    probs = [(p.grid, p.eps0, p.sig0, p.shots, d) for p, d in problems]
    r1, _ = gpu_ctx.w_gradient_batch(probs, mode=N.GJ_ADJ_EXACT, precision=N.GJ_F64)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    gpu_ctx.release()
    free1 = torch.cuda.mem_get_info()[0]
    assert free1 > free0
    r2, _ = gpu_ctx.w_gradient_batch(probs, mode=N.GJ_ADJ_EXACT, precision=N.GJ_F64)
    for a, b in zip(r1, r2):
        assert rel_l2(a["g_eps"], b["g_eps"]) < 1e-12
        assert rel_l2(a["g_sig"], b["g_sig"]) < 1e-12


@pytest.fixture(scope="module")
def grouped(oracle):
    """One problem whose whole history is large against the pool (8 shots,
    400 steps) beside two small ones."""
    specs = [dict(m=40, n=60, pml=8, nt=400, nsrc=8, nrec=8, seed=61),
             dict(m=20, n=30, pml=6, nt=200, nsrc=2, nrec=5, seed=62),
             dict(m=24, n=28, pml=6, nt=240, nsrc=3, nrec=6, seed=63)]
    out = []
    for sp in specs:
        p = synth.small(**sp)
        dobs = [oracle.forward(p.grid, p.eps_true, p.sig_true, sh)[0] for sh in p.shots]
        out.append((p, dobs))
    return out


@pytest.mark.parametrize("budget_mb", [128, 256])
def test_batch_shot_groups_equal_single_calls(gpu_ctx, grouped, budget_mb):
    """Pool budgets under which the 8-shot problem (whole history about 220 MB
    in FP64) runs its whole history in two groups of 4 shots one after the other
    (128 MB) or in one group (256 MB): every gradient equals its own
    gj_w_gradient call (FP64)."""
    o = N.OptsC()
    o.mem_budget_bytes = budget_mb << 20
    probs = [(p.grid, p.eps0, p.sig0, p.shots, d) for p, d in grouped]
    res, _ = gpu_ctx.w_gradient_batch(probs, mode=N.GJ_ADJ_EXACT, precision=N.GJ_F64, opts=o)
    for (p, d), r in zip(grouped, res):
        ref = gpu_ctx.w_gradient(p.grid, p.eps0, p.sig0, p.shots, d, mode=N.GJ_ADJ_EXACT, precision=N.GJ_F64)
        assert rel_l2(r["g_eps"], ref["g_eps"]) < 1e-11
        assert rel_l2(r["g_sig"], ref["g_sig"]) < 1e-11
        assert np.allclose(r["misfit"], ref["misfit"], rtol=1e-12)
