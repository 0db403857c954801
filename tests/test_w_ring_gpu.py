"""Warp-task ring kernels (the default step kernels for FP32 and FP64)
against the register-marching kernels and the oracle, on grids tall enough
for several row blocks per column, so the halo rows, the fast and general
paths, the column chunks and the imaging windows are all exercised."""
import os

import numpy as np
import pytest

from conftest import rel_l2, edge_cells
from gerjoii_b200 import synth
from gerjoii_b200 import _native as N

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=[True, False], ids=["free_top", "ref_layout"])
def tall(request):
    return synth.small(m=150, n=44, pml=10, nt=260, nsrc=3, nrec=10, free_top=request.param, seed=31)


def _dobs(oracle, p):
    return [oracle.forward(p.grid, p.eps_true, p.sig_true, sh)[0] for sh in p.shots]


@pytest.mark.parametrize("prec", [N.GJ_F64, N.GJ_F32])
def test_ring_kernels_match_marching_kernels(gpu_ctx, oracle, tall, prec):
    p = tall
    dobs = _dobs(oracle, p)
    o = N.OptsC()
    o.no_ring = 1
    a = gpu_ctx.w_gradient(p.grid, p.eps0, p.sig0, p.shots, dobs, mode=N.GJ_ADJ_EXACT, precision=prec, opts=o,
                           want_traces=True)
    b = gpu_ctx.w_gradient(p.grid, p.eps0, p.sig0, p.shots, dobs, mode=N.GJ_ADJ_EXACT, precision=prec,
                           want_traces=True)
    # same arithmetic per node, up to the compiler's fused multiply-adds
    tol = 1e-12 if prec == N.GJ_F64 else 2e-6
    for x, y in zip(a["d"], b["d"]):
        assert rel_l2(y, x) < tol
    if prec == N.GJ_F64:
        # the eps imaging differences consecutive fields; next to the sources
        # that cancellation turns rounding differences into ~1e-10 of the gradient
        assert rel_l2(b["g_eps"], a["g_eps"]) < 1e-9
        assert rel_l2(b["g_sig"], a["g_sig"]) < 1e-9
    # (FP32 gradients: on this short record with sources one row under the
    # surface, FP32 itself -- the C++ oracle in FP32 included -- differs from
    # FP64 by ~10 % in the source rows, so two FP32 roundings are not compared
    # here; the FP32 oracle checks of test_w_gpu.py run through these kernels)


@pytest.mark.parametrize("ckpt", [0, 13])
def test_ring_exact_gradient_matches_oracle(gpu_ctx, oracle, tall, ckpt):
    p = tall
    g = p.grid
    dobs = _dobs(oracle, p)
    ge, gs, _ = oracle.gradient_batch(g, p.eps0, p.sig0, p.shots, np.stack([d.T for d in dobs]), mode="exact")
    o = N.OptsC()
    o.ckpt_every = ckpt
    res = gpu_ctx.w_gradient(g, p.eps0, p.sig0, p.shots, dobs, mode=N.GJ_ADJ_EXACT, precision=N.GJ_F64, opts=o)
    # the eps imaging sums l (E^k - E^{k-1}): cancellation between consecutive
    # fields puts the FP64 agreement near 1e-10 on this 150-row grid; the edge
    # cells (band terms, stronger cancellation) near 1e-9, with the rounding of
    # whichever forward kernels the tuner chose (one step or several per launch)
    assert rel_l2(res["g_eps"], ge) < 1e-9
    assert rel_l2(res["g_sig"], gs) < 1e-9
    assert rel_l2(edge_cells(res["g_eps"]), edge_cells(ge)) < 3e-9


def test_ring_forward_api_matches_oracle(gpu_ctx, oracle, tall):
    p = tall
    out = gpu_ctx.w_forward(p.grid, p.eps0, p.sig0, p.shots, precision=N.GJ_F64, want_u=True)
    for k, sh in enumerate(p.shots):
        d, _, u = oracle.forward(p.grid, p.eps0, p.sig0, sh, store_u=True)
        assert rel_l2(out["d"][k], d) < 1e-12
        assert rel_l2(out["u"][k], u) < 1e-12


def test_ring_edge_receivers_and_sources_match_oracle(gpu_ctx, oracle):
    """Receivers the fused record / injection must handle: the same node twice,
    inside the left and bottom PML, on the Ez = 0 top row, on the last interior
    row, on the boundary column and row; a source inside the PML (no effect,
    w_solve.m:92-94); a shot without receivers.  FP64 traces and per-shot exact
    gradients (all cells) against the oracle."""
    from gerjoii_b200.geometry import Shot
    p = synth.small(m=150, n=44, pml=10, nt=220, nsrc=2, nrec=6, free_top=True, seed=33)
    g = p.grid
    NX, NY = g.NX, g.NY
    node = g.node
    w = p.shots[0].wavelet
    recA = np.array([node(1, 30), node(1, 30), node(50, 3), node(NX - 3, 30), node(0, 20),
                     node(NX - g.pml - 1, 40), node(70, 0), node(NX, 25), node(5, 12)], np.int64)
    shots = [Shot(2, 30, w, recA),
             Shot(100, 5, w, p.shots[1].rec),          # source in the left PML band
             Shot(3, 22, w, np.zeros(0, np.int64))]    # no receivers
    dobs = [oracle.forward(g, p.eps_true, p.sig_true, sh)[0] for sh in shots]
    out = gpu_ctx.w_forward(g, p.eps0, p.sig0, shots, precision=N.GJ_F64)
    o = N.OptsC()
    o.per_shot = 1
    res = gpu_ctx.w_gradient(g, p.eps0, p.sig0, shots, dobs, mode=N.GJ_ADJ_EXACT, precision=N.GJ_F64, opts=o,
                             want_traces=True)
    for k, sh in enumerate(shots):
        d, _, _ = oracle.forward(g, p.eps0, p.sig0, sh)
        if sh.nr:
            assert rel_l2(out["d"][k], d) < 1e-12
            assert rel_l2(res["d"][k], d) < 1e-12
        e = d - dobs[k]
        ge, gs = oracle.grad_exact(g, p.eps0, p.sig0, sh, e)
        if sh.nr == 0:
            assert np.abs(res["g_eps"][k]).max() == 0 and np.abs(res["g_sig"][k]).max() == 0
            continue
        assert rel_l2(res["g_eps"][k], ge) < 1e-9
        assert rel_l2(res["g_sig"][k], gs) < 1e-9


@pytest.mark.parametrize("ckpt", [0, 11])
def test_ring_reference_adjoint_matches_marching_and_oracle(gpu_ctx, oracle, tall, ckpt):
    """w_grad semantics (GJ_ADJ_REFERENCE) on the ring kernels with windowed
    imaging: equal to the register-marching kernels with per-step imaging and
    to the oracle, with and without checkpoints."""
    p = tall
    g = p.grid
    dobs = _dobs(oracle, p)
    o = N.OptsC()
    o.ckpt_every = ckpt
    r = gpu_ctx.w_gradient(g, p.eps0, p.sig0, p.shots, dobs, mode=N.GJ_ADJ_REFERENCE, precision=N.GJ_F64, opts=o)
    o.no_ring = 1
    m = gpu_ctx.w_gradient(g, p.eps0, p.sig0, p.shots, dobs, mode=N.GJ_ADJ_REFERENCE, precision=N.GJ_F64, opts=o)
    assert rel_l2(r["g_eps"], m["g_eps"]) < 1e-10
    assert rel_l2(r["g_sig"], m["g_sig"]) < 1e-10
    ge, gs, _ = oracle.gradient_batch(g, p.eps0, p.sig0, p.shots, np.stack([d.T for d in dobs]), mode="reference")
    assert rel_l2(r["g_eps"], ge) < 1e-9
    assert rel_l2(r["g_sig"], gs) < 1e-9


@pytest.mark.parametrize("mode", ["exact", "reference"])
@pytest.mark.parametrize("nsrc", [4, 5])
def test_split_bottom_tasks_match_oracle(gpu_ctx, oracle, mode, nsrc):
    """A grid whose bottom row block has few live rows (NX + 1 = 152: 24 rows
    past the last full block of 128 (FP32) or 64 (FP64) rows), so that block
    runs as split tasks, two shots per warp, in both precisions; an odd shot
    count leaves the last shot of each launch unpaired."""
    p = synth.small(m=140, n=44, pml=10, nt=200, nsrc=nsrc, nrec=9, seed=37)
    g = p.grid
    assert g.pml_top + g.air + g.m + g.pml + 1 == 152
    dobs = _dobs(oracle, p)
    ge, gs, mis = oracle.gradient_batch(g, p.eps0, p.sig0, p.shots, np.stack([d.T for d in dobs]), mode=mode)
    gm = N.GJ_ADJ_EXACT if mode == "exact" else N.GJ_ADJ_REFERENCE
    r64 = gpu_ctx.w_gradient(g, p.eps0, p.sig0, p.shots, dobs, mode=gm, precision=N.GJ_F64)
    assert rel_l2(r64["g_eps"], ge) < 1e-9
    assert rel_l2(r64["g_sig"], gs) < 1e-9
    assert rel_l2(edge_cells(r64["g_eps"]), edge_cells(ge)) < 1e-9
    assert np.allclose(r64["misfit"], mis, rtol=1e-10)
    # FP32: split tasks against one shot per task everywhere (GJ_NO_SPLIT),
    # both with the same fixed ring configuration (the column chunks decide
    # where a task recomputes its first Hx column, which moves FP32 rounding),
    # in contexts whose plans are made with those variables set
    fixed = {"GJ_RING_STAGES": "2", "GJ_RING_STAGES_FAST": "3", "GJ_RING_CTA_WARPS": "2",
             "GJ_RING_TJF": "32", "GJ_RING_TJS": "8"}
    res = []
    for extra in ({}, {"GJ_NO_SPLIT": "1"}):
        env = dict(fixed, **extra)
        os.environ.update(env)
        try:
            ctx2 = N.Context(0)
            try:
                res.append(ctx2.w_gradient(g, p.eps0, p.sig0, p.shots, dobs, mode=gm, precision=N.GJ_F32))
            finally:
                ctx2.close()
        finally:
            for k in env:
                del os.environ[k]
    for key in ("g_eps", "g_sig"):
        assert rel_l2(res[0][key], res[1][key]) < 1e-6, key


def test_kernel_timing_counts_runs(gpu_ctx, oracle, tall):
    """The optional device timing: every step launch is counted, runs of
    consecutive step launches are sampled, and the average launch time lies
    between zero and the call's wall time per step."""
    import time
    p = tall
    g = p.grid
    dobs = _dobs(oracle, p)
    gpu_ctx.w_gradient(g, p.eps0, p.sig0, p.shots, dobs, mode=N.GJ_ADJ_EXACT, precision=N.GJ_F32)  # plans, graphs
    gpu_ctx.set_kernel_timing(True)
    try:
        t0 = time.perf_counter()
        gpu_ctx.w_gradient(g, p.eps0, p.sig0, p.shots, dobs, mode=N.GJ_ADJ_EXACT, precision=N.GJ_F32)
        wall_ms = 1e3 * (time.perf_counter() - t0)
        kt = {k: gpu_ctx.kernel_time(k) for k in ("fwd_step", "adj_step", "image", "tb_pass")}
    finally:
        gpu_ctx.set_kernel_timing(False)
    # the forward runs one step per launch, or (whole history kept, blocked
    # passes tuned in) up to 4 steps per launch
    fwd = "tb_pass" if kt["tb_pass"]["launches"] > 0 else "fwd_step"
    assert kt[fwd]["launches"] >= (g.nt if fwd == "fwd_step" else -(-g.nt // 4))
    assert kt["adj_step"]["launches"] >= g.nt
    for k in (fwd, "adj_step"):
        assert 0 < kt[k]["sampled"] <= kt[k]["launches"]
        assert 0 < kt[k]["avg_us"] < 1e3 * wall_ms / kt[k]["launches"]
    assert kt["image"]["launches"] >= 1


@pytest.mark.parametrize("env", [
    {"GJ_AUTOTUNE": "0"},
    {"GJ_RING_CTA_WARPS": "4", "GJ_RING_STAGES": "3", "GJ_RING_STAGES_FAST": "4", "GJ_RING_TJF": "16",
     "GJ_RING_TJS": "4"},
    {"GJ_NO_SPLIT": "1", "GJ_SIDE_PRIORITY": "0"},
], ids=["defaults", "fixed", "no_split_no_priority"])
def test_ring_configurations_from_the_environment(gpu_ctx, oracle, tall, env):
    """Plans made with the tuner off, with a fixed ring configuration, or with
    split tasks and the priority stream off give the tuned plan's FP64
    gradient.  The column chunks decide where a task recomputes its first Hx
    column (a different rounding), which the eps imaging's cancellation turns
    into about 1e-10 on this grid, as against the oracle."""
    p = tall
    g = p.grid
    dobs = _dobs(oracle, p)
    ref = gpu_ctx.w_gradient(g, p.eps0, p.sig0, p.shots, dobs, mode=N.GJ_ADJ_EXACT, precision=N.GJ_F64)
    os.environ.update(env)
    try:
        ctx2 = N.Context(0)
        try:
            alt = ctx2.w_gradient(g, p.eps0, p.sig0, p.shots, dobs, mode=N.GJ_ADJ_EXACT, precision=N.GJ_F64)
        finally:
            ctx2.close()
    finally:
        for k in env:
            del os.environ[k]
    assert rel_l2(alt["g_eps"], ref["g_eps"]) < 1e-9
    assert rel_l2(alt["g_sig"], ref["g_sig"]) < 1e-9
    assert np.allclose(alt["misfit"], ref["misfit"], rtol=1e-12)
