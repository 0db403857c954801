"""GPU parity of the radar path against the oracle, through the C ABI."""
import numpy as np
import pytest

from conftest import rel_l2, cosine, edge_cells
from gerjoii_b200 import synth
from gerjoii_b200 import _native as N

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small_ft():
    return synth.small(m=24, n=40, pml=8, nt=300, free_top=True, seed=21)


@pytest.fixture(scope="module")
def small_ref():
    return synth.small(m=20, n=36, pml=8, nt=300, free_top=False, seed=22)


@pytest.mark.parametrize("which", ["small_ft", "small_ref"])
def test_forward_f64_matches_oracle(gpu_ctx, oracle, which, request):
    p = request.getfixturevalue(which)
    g = p.grid
    out = gpu_ctx.w_forward(g, p.eps0, p.sig0, p.shots, precision=N.GJ_F64, want_jz=True, want_u=True)
    for k, sh in enumerate(p.shots):
        d, jz, u = oracle.forward(g, p.eps0, p.sig0, sh, store_u=True)
        assert rel_l2(out["d"][k], d) < 1e-12
        assert rel_l2(out["jz"][k], jz) < 1e-12
        assert rel_l2(out["u"][k], u) < 1e-12


@pytest.mark.parametrize("which", ["small_ft", "small_ref"])
def test_forward_f32_traces_within_1e5(gpu_ctx, oracle, which, request):
    p = request.getfixturevalue(which)
    g = p.grid
    out = gpu_ctx.w_forward(g, p.eps0, p.sig0, p.shots, precision=N.GJ_F32)
    for k, sh in enumerate(p.shots):
        d, _, _ = oracle.forward(g, p.eps0, p.sig0, sh)
        assert rel_l2(out["d"][k], d) < 1e-5


def _dobs(oracle, p):
    return [oracle.forward(p.grid, p.eps_true, p.sig_true, sh)[0] for sh in p.shots]


@pytest.mark.parametrize("prec,tol", [(N.GJ_F64, 1e-10), (N.GJ_F32, 1e-4)])
@pytest.mark.parametrize("ckpt", [0, 7])
def test_reference_gradient_matches_oracle(gpu_ctx, oracle, small_ft, prec, tol, ckpt):
    p = small_ft
    g = p.grid
    dobs = _dobs(oracle, p)
    ge, gs, mis = oracle.gradient_batch(g, p.eps0, p.sig0, p.shots, np.stack([d.T for d in dobs]),
                                        mode="reference")
    o = N.OptsC()
    o.ckpt_every = ckpt
    res = gpu_ctx.w_gradient(g, p.eps0, p.sig0, p.shots, dobs, mode=N.GJ_ADJ_REFERENCE, precision=prec, opts=o)
    assert rel_l2(res["g_eps"], ge) < tol and cosine(res["g_eps"], ge) > 1 - tol
    assert rel_l2(res["g_sig"], gs) < tol and cosine(res["g_sig"], gs) > 1 - tol
    assert np.allclose(res["misfit"], mis, rtol=1e-5 if prec == N.GJ_F32 else 1e-12)


@pytest.mark.parametrize("prec,tol", [(N.GJ_F64, 1e-10), (N.GJ_F32, 1e-4)])
@pytest.mark.parametrize("ckpt", [0, 9])
@pytest.mark.parametrize("which", ["small_ft", "small_ref"])
def test_exact_gradient_matches_oracle(gpu_ctx, oracle, which, request, prec, tol, ckpt):
    """Every model cell, the edge cells (PML-coefficient terms) on their own too."""
    p = request.getfixturevalue(which)
    g = p.grid
    dobs = _dobs(oracle, p)
    ge, gs, _ = oracle.gradient_batch(g, p.eps0, p.sig0, p.shots, np.stack([d.T for d in dobs]), mode="exact")
    o = N.OptsC()
    o.ckpt_every = ckpt
    res = gpu_ctx.w_gradient(g, p.eps0, p.sig0, p.shots, dobs, mode=N.GJ_ADJ_EXACT, precision=prec, opts=o)
    assert rel_l2(res["g_eps"], ge) < tol
    assert rel_l2(res["g_sig"], gs) < tol
    assert rel_l2(edge_cells(res["g_eps"]), edge_cells(ge)) < 10 * tol


def test_w_grad_matches_oracle(gpu_ctx, oracle, small_ref):
    p = small_ref
    g, sh = p.grid, p.shots[0]
    d, _, u = oracle.forward(g, p.eps0, p.sig0, sh, store_u=True)
    e = d - oracle.forward(g, p.eps_true, p.sig_true, sh)[0]
    gr, am = oracle.grad_reference(g, p.eps0, p.sig0, sh, e, u)
    gg, aa = gpu_ctx.w_grad(g, p.eps0, p.sig0, sh, e, u, precision=N.GJ_F64)
    assert rel_l2(gg, gr) < 1e-10 and rel_l2(aa, am) < 1e-10


def test_per_shot_gradients_sum_to_total(gpu_ctx, oracle, small_ft):
    p = small_ft
    dobs = _dobs(oracle, p)
    o = N.OptsC()
    o.per_shot = 1
    r1 = gpu_ctx.w_gradient(p.grid, p.eps0, p.sig0, p.shots, dobs, precision=N.GJ_F64, opts=o)
    r2 = gpu_ctx.w_gradient(p.grid, p.eps0, p.sig0, p.shots, dobs, precision=N.GJ_F64)
    assert r1["g_eps"].shape == (len(p.shots), p.grid.m, p.grid.n)
    assert rel_l2(r1["g_eps"].sum(0), r2["g_eps"]) < 1e-12


def test_invalid_source_is_rejected(gpu_ctx, small_ft):
    p = small_ft
    from gerjoii_b200.geometry import Shot
    bad = Shot(0, 5, p.shots[0].wavelet, p.shots[0].rec)
    with pytest.raises(N.GJError) as ei:
        gpu_ctx.w_forward(p.grid, p.eps0, p.sig0, [bad])
    assert ei.value.status == N.GJ_EINVAL


@pytest.mark.parametrize("mode", [N.GJ_ADJ_REFERENCE, N.GJ_ADJ_EXACT])
def test_plain_fp64_form_matches_fused(gpu_ctx, oracle, small_ft, mode):
    p = small_ft
    dobs = _dobs(oracle, p)
    o = N.OptsC()
    o.plain = 1
    r1 = gpu_ctx.w_gradient(p.grid, p.eps0, p.sig0, p.shots, dobs, mode=mode, precision=N.GJ_F64, opts=o)
    r2 = gpu_ctx.w_gradient(p.grid, p.eps0, p.sig0, p.shots, dobs, mode=mode, precision=N.GJ_F64)
    assert rel_l2(r1["g_eps"], r2["g_eps"]) < 1e-11
    assert rel_l2(r1["g_sig"], r2["g_sig"]) < 1e-11
    assert np.allclose(r1["misfit"], r2["misfit"], rtol=1e-12)
    o.ckpt_every = 11
    r3 = gpu_ctx.w_gradient(p.grid, p.eps0, p.sig0, p.shots, dobs, mode=mode, precision=N.GJ_F64, opts=o)
    assert rel_l2(r3["g_eps"], r2["g_eps"]) < 1e-11


def test_autograd_harness_gradient_matches_finite_difference(gpu_ctx, oracle, small_ft):
    import torch
    from gerjoii_b200.autograd import WGradient
    p = small_ft
    g = p.grid
    dobs = _dobs(oracle, p)
    dev = torch.device("cuda", 0)
    do_t = torch.tensor(np.stack([d.T for d in dobs]), dtype=torch.float64, device=dev)
    eps = torch.tensor(p.eps0, dtype=torch.float64, device=dev, requires_grad=True)
    sig = torch.tensor(p.sig0, dtype=torch.float64, device=dev, requires_grad=True)
    J = WGradient.apply(eps, sig, g, p.shots, do_t, gpu_ctx)
    J.backward()
    # interior cells and edge cells (the latter through the PML coefficients too)
    for (a, b) in [(5, 10), (12, 20), (g.m - 1, 0), (g.m - 1, 17), (7, g.n - 1), (4, 0)]:
        h = 1e-5 * p.eps0[a, b]
        ep, em = p.eps0.copy(), p.eps0.copy()
        ep[a, b] += h
        em[a, b] -= h
        Jp = WGradient.apply(torch.tensor(ep, dtype=torch.float64, device=dev), sig.detach(), g, p.shots, do_t, gpu_ctx)
        Jm = WGradient.apply(torch.tensor(em, dtype=torch.float64, device=dev), sig.detach(), g, p.shots, do_t, gpu_ctx)
        fd = (Jp.item() - Jm.item()) / (2 * h)
        assert abs(eps.grad[a, b].item() - fd) <= 1e-5 * abs(fd), (a, b, eps.grad[a, b].item(), fd)


@pytest.mark.parametrize("prec,tol", [(N.GJ_F64, 1e-9), (N.GJ_F32, 5e-4)])
def test_envelope_residual_and_exact_gradient_match_oracle(gpu_ctx, oracle, small_ft, prec, tol):
    """env_L2 (w_bozdag.m:16-25): residual against the numpy twin, misfit of the
    envelopes (w_E.m after w_fwd.m:34-35), exact gradient against the oracle's
    exact adjoint driven by the same adjoint source (all cells).  The
    residual divides by the envelope E, which magnifies the FP32 trace error
    (~1e-5) where E is small: hence the looser FP32 bound."""
    import np_oracle as npo
    p = small_ft
    g = p.grid
    dobs = _dobs(oracle, p)
    res = gpu_ctx.w_gradient(g, p.eps0, p.sig0, p.shots, dobs, mode=N.GJ_ADJ_EXACT, misfit=N.GJ_MISFIT_ENV_L2,
                             precision=prec, want_traces=True)
    ge = np.zeros((g.m, g.n))
    gs = np.zeros((g.m, g.n))
    for k, sh in enumerate(p.shots):
        d, _, _ = oracle.forward(g, p.eps0, p.sig0, sh)
        e, de, doe = npo.w_bozdag(dobs[k], d, "env_L2")
        assert rel_l2(res["e"][k], e) < tol
        assert abs(res["misfit"][k] - npo.w_E(doe, de)) <= tol * npo.w_E(doe, de)
        a, b = oracle.grad_exact(g, p.eps0, p.sig0, sh, e)
        ge += a
        gs += b
    assert rel_l2(res["g_eps"], ge) < 10 * tol
    assert rel_l2(res["g_sig"], gs) < 10 * tol


@pytest.mark.parametrize("kind", [N.GJ_MISFIT_PHASE_L2, N.GJ_MISFIT_ENV_L22, N.GJ_MISFIT_ENV_LOG],
                         ids=["phase_L2", "env_L22", "env_LOG"])
def test_phase_and_envelope_variants_match_numpy_twin(gpu_ctx, oracle, small_ft, kind):
    """phase_L2, env_L22 and env_LOG (w_bozdag.m:26-54), FP64: the adjoint
    source against the numpy twin applied to the GPU's own modelled traces
    (phase_L2 and env_LOG divide by E^2, so a 1e-12 trace difference already
    moves them by ~1e-8: comparing on the same traces isolates the adjoint-
    source arithmetic), the misfit of w_E.m on the same quantities from the
    gradient call and from the forward-only call, and the exact gradient
    against the oracle's exact adjoint driven by the same adjoint source."""
    import np_oracle as npo
    name = {N.GJ_MISFIT_PHASE_L2: "phase_L2", N.GJ_MISFIT_ENV_L22: "env_L22", N.GJ_MISFIT_ENV_LOG: "env_LOG"}[kind]
    p = small_ft
    g = p.grid
    dobs = _dobs(oracle, p)
    res = gpu_ctx.w_gradient(g, p.eps0, p.sig0, p.shots, dobs, mode=N.GJ_ADJ_EXACT, misfit=kind,
                             precision=N.GJ_F64, want_traces=True)
    mis_only = gpu_ctx.w_misfit(g, p.eps0, p.sig0, p.shots, dobs, misfit=kind, precision=N.GJ_F64)
    ge = np.zeros((g.m, g.n))
    gs = np.zeros((g.m, g.n))
    for k, sh in enumerate(p.shots):
        e, de, doe = npo.w_bozdag(dobs[k], res["d"][k], name)
        assert np.isfinite(res["e"][k]).all()
        assert rel_l2(res["e"][k], e) < 1e-8
        ref = npo.w_E(doe, de, name)
        assert abs(res["misfit"][k] - ref) <= 1e-9 * abs(ref)
        assert abs(mis_only[k] - ref) <= 1e-9 * abs(ref)
        a, b = oracle.grad_exact(g, p.eps0, p.sig0, sh, res["e"][k])
        ge += a
        gs += b
    assert rel_l2(res["g_eps"], ge) < 1e-8
    assert rel_l2(res["g_sig"], gs) < 1e-8


@pytest.mark.parametrize("prec,tol", [(N.GJ_F64, 1e-10), (N.GJ_F32, 2e-4)])
@pytest.mark.parametrize("band", [(-350e6, 350e6), (80e6, 500e6)])
def test_band_filtered_residual_and_gradient_match_oracle(gpu_ctx, oracle, small_ft, prec, tol, band):
    """filt_gauss.m on the residual (w_update_e.m:69-70): the filtered residual
    against the numpy twin of filt_gauss, the misfit of the unfiltered residual,
    and the exact gradient against the oracle's exact adjoint driven by the
    filtered residual (all cells)."""
    import np_oracle as npo
    p = small_ft
    g = p.grid
    dobs = _dobs(oracle, p)
    o = N.OptsC()
    o.filt_low, o.filt_high = band
    res = gpu_ctx.w_gradient(g, p.eps0, p.sig0, p.shots, dobs, mode=N.GJ_ADJ_EXACT, precision=prec, opts=o,
                             want_traces=True)
    ge = np.zeros((g.m, g.n))
    gs = np.zeros((g.m, g.n))
    for k, sh in enumerate(p.shots):
        d, _, _ = oracle.forward(g, p.eps0, p.sig0, sh)
        e = d - dobs[k]
        ef = npo.filt_gauss(e, g.dt, band[0], band[1], 8)
        assert rel_l2(res["e"][k], ef) < tol
        mis = 0.5 * np.sum(e * e) / np.sum(dobs[k] * dobs[k])  # w_update_e.m:75-76, unfiltered
        assert abs(res["misfit"][k] - mis) <= 10 * tol * mis
        a, b = oracle.grad_exact(g, p.eps0, p.sig0, sh, ef)
        ge += a
        gs += b
    assert rel_l2(res["g_eps"], ge) < 10 * tol
    assert rel_l2(res["g_sig"], gs) < 10 * tol


@pytest.mark.parametrize("prec,tol", [(N.GJ_F64, 1e-12), (N.GJ_F32, 1e-5)])
def test_forward_only_misfit_matches_oracle_and_gradient(gpu_ctx, oracle, small_ft, prec, tol):
    """gj_w_misfit (w_objs_e.m, the step-length search's objective): the same
    misfits as the oracle and as the full gradient call, for L2 and env_L2,
    on two trial models in a row."""
    import np_oracle as npo
    p = small_ft
    g = p.grid
    dobs = _dobs(oracle, p)
    for scale in (1.0, 1.05):
        eps = p.eps0 * scale
        m = gpu_ctx.w_misfit(g, eps, p.sig0, p.shots, dobs, precision=prec)
        _, _, mis = oracle.gradient_batch(g, eps, p.sig0, p.shots, np.stack([d.T for d in dobs]), mode="exact")
        assert np.allclose(m, mis, rtol=tol)
        r = gpu_ctx.w_gradient(g, eps, p.sig0, p.shots, dobs, mode=N.GJ_ADJ_EXACT, precision=prec)
        assert np.allclose(m, r["misfit"], rtol=tol)
    me = gpu_ctx.w_misfit(g, p.eps0, p.sig0, p.shots, dobs, misfit=N.GJ_MISFIT_ENV_L2, precision=prec)
    for k, sh in enumerate(p.shots):
        d, _, _ = oracle.forward(g, p.eps0, p.sig0, sh)
        _, de, doe = npo.w_bozdag(dobs[k], d, "env_L2")
        assert abs(me[k] - npo.w_E(doe, de)) <= max(tol, 2e-4) * npo.w_E(doe, de)


def test_gradient_conditioning_matches_numpy_twin(gpu_ctx, oracle, small_ft):
    """Per-shot conditioning (source taper, k-space low-pass, normali, NaN
    guard; w_update_e.m:110-135, w_update_s.m:96-137) and the shot mean
    (w_update_e_.m:38) against the numpy twin applied to the GPU's own
    per-shot gradients."""
    import np_oracle as npo
    from gerjoii_b200.geometry import C_0
    p = small_ft
    g = p.grid
    dobs = _dobs(oracle, p)
    o = N.OptsC()
    o.per_shot = 1
    raw = gpu_ctx.w_gradient(g, p.eps0, p.sig0, p.shots, dobs, mode=N.GJ_ADJ_EXACT, precision=N.GJ_F64, opts=o)
    fo, ax, az = 300e6, 0.2, 0.3
    oc = N.OptsC()
    oc.condition, oc.cond_fo, oc.cond_ax, oc.cond_az = 1, fo, ax, az
    cond = gpu_ctx.w_gradient(g, p.eps0, p.sig0, p.shots, dobs, mode=N.GJ_ADJ_EXACT, precision=N.GJ_F64, opts=oc)
    oc.per_shot = 1
    cps = gpu_ctx.w_gradient(g, p.eps0, p.sig0, p.shots, dobs, mode=N.GJ_ADJ_EXACT, precision=N.GJ_F64, opts=oc)
    te, ts = [], []
    for k, sh in enumerate(p.shots):
        sm = (sh.src_i - g.dom_i0, sh.src_j - g.dom_j0)
        te.append(npo.condition_shot(raw["g_eps"][k], g.dx, g.dy, sm, p.eps0, fo, ax, az, c=C_0))
        ts.append(npo.condition_shot(raw["g_sig"][k], g.dx, g.dy, sm, p.eps0, fo, 2 * ax, 2 * az, c=C_0))
        assert rel_l2(cps["g_eps"][k], te[-1]) < 1e-10
        assert rel_l2(cps["g_sig"][k], ts[-1]) < 1e-10
    assert rel_l2(cond["g_eps"], np.mean(te, axis=0)) < 1e-10
    assert rel_l2(cond["g_sig"], np.mean(ts, axis=0)) < 1e-10
    assert np.abs(cps["g_eps"]).max() == pytest.approx(1.0)


def test_non_finite_results_return_enumeric(gpu_ctx, small_ft):
    """NaN in the conductivity: forward, misfit-only and gradient calls (both
    adjoint modes, FP32 and FP64) return GJ_ENUMERIC; with per-shot
    conditioning the reference's NaN guard (w_update_e.m:131-137) zeroes the
    gradients instead, and the context keeps working afterwards."""
    p = small_ft
    g = p.grid
    sig = p.sig0.copy()
    sig[5, 7] = np.nan
    dobs = [np.zeros((g.nt, sh.nr)) for sh in p.shots]
    for prec in (N.GJ_F32, N.GJ_F64):
        with pytest.raises(N.GJError) as ei:
            gpu_ctx.w_forward(g, p.eps0, sig, p.shots, precision=prec)
        assert ei.value.status == N.GJ_ENUMERIC
        with pytest.raises(N.GJError) as ei:
            gpu_ctx.w_misfit(g, p.eps0, sig, p.shots, dobs, precision=prec)
        assert ei.value.status == N.GJ_ENUMERIC
        for mode in (N.GJ_ADJ_REFERENCE, N.GJ_ADJ_EXACT):
            with pytest.raises(N.GJError) as ei:
                gpu_ctx.w_gradient(g, p.eps0, sig, p.shots, dobs, mode=mode, precision=prec)
            assert ei.value.status == N.GJ_ENUMERIC
    o = N.OptsC()
    o.condition, o.cond_fo, o.cond_ax, o.cond_az, o.per_shot = 1, 300e6, 0.2, 0.3, 1
    with pytest.raises(N.GJError) as ei:  # the misfits themselves are still NaN
        gpu_ctx.w_gradient(g, p.eps0, sig, p.shots, dobs, mode=N.GJ_ADJ_EXACT, precision=N.GJ_F64, opts=o)
    assert ei.value.status == N.GJ_ENUMERIC
    r = gpu_ctx.w_gradient(g, p.eps0, p.sig0, p.shots, dobs, mode=N.GJ_ADJ_EXACT, precision=N.GJ_F64)
    assert np.isfinite(r["g_eps"]).all()


def test_small_memory_budget_checkpoints_with_the_same_result(gpu_ctx, oracle, small_ft):
    """A memory budget too small for the whole u history makes the call
    checkpoint and recompute (more launches) with the same FP64 gradient; a
    grid whose fields cannot be allocated returns GJ_ENOMEM and leaves the
    context usable."""
    p = small_ft
    g = p.grid
    dobs = _dobs(oracle, p)
    r1 = gpu_ctx.w_gradient(g, p.eps0, p.sig0, p.shots, dobs, mode=N.GJ_ADJ_EXACT, precision=N.GJ_F64)
    n1 = gpu_ctx.last_launch_count
    o = N.OptsC()
    o.mem_budget_bytes = 4 << 20
    o.no_graph = 1
    r2 = gpu_ctx.w_gradient(g, p.eps0, p.sig0, p.shots, dobs, mode=N.GJ_ADJ_EXACT, precision=N.GJ_F64, opts=o)
    assert gpu_ctx.last_launch_count > n1
    assert rel_l2(r2["g_eps"], r1["g_eps"]) < 1e-12 and rel_l2(r2["g_sig"], r1["g_sig"]) < 1e-12
    import copy
    huge = copy.copy(g)
    huge.m, huge.n = 120000, 120000
    with pytest.raises(N.GJError) as ei:
        gpu_ctx.w_forward(huge, np.ones((3, 3)), np.ones((3, 3)), p.shots[:1])
    assert ei.value.status in (N.GJ_ENOMEM, N.GJ_EINVAL)
    r3 = gpu_ctx.w_gradient(g, p.eps0, p.sig0, p.shots, dobs, mode=N.GJ_ADJ_EXACT, precision=N.GJ_F64)
    assert rel_l2(r3["g_eps"], r1["g_eps"]) < 1e-12


@pytest.mark.parametrize("mode", [N.GJ_ADJ_EXACT, N.GJ_ADJ_REFERENCE])
@pytest.mark.parametrize("plain", [0, 1])
def test_forward_backward_pair_matches_gradient_and_oracle(gpu_ctx, oracle, small_ft, mode, plain):
    """gj_w_forward -> residual on the host -> gj_w_backward (the MEX
    forward/backward pair) equals the fused gj_w_gradient (FP64, 1e-12) and
    the oracle's exact adjoint of the same adjoint sources (1e-10)."""
    p = small_ft
    g = p.grid
    dobs = _dobs(oracle, p)
    d = gpu_ctx.w_forward(g, p.eps0, p.sig0, p.shots, precision=N.GJ_F64)["d"]
    e = [a - b for a, b in zip(d, dobs)]
    o = N.OptsC()
    o.plain = plain
    bw = gpu_ctx.w_backward(g, p.eps0, p.sig0, p.shots, e, mode=mode, precision=N.GJ_F64, opts=o)
    fu = gpu_ctx.w_gradient(g, p.eps0, p.sig0, p.shots, dobs, mode=mode, precision=N.GJ_F64, opts=o)
    assert rel_l2(bw["g_eps"], fu["g_eps"]) < 1e-12
    assert rel_l2(bw["g_sig"], fu["g_sig"]) < 1e-12
    if mode == N.GJ_ADJ_EXACT:
        ge, gs = np.zeros((g.m, g.n)), np.zeros((g.m, g.n))
        for k, sh in enumerate(p.shots):
            a, b = oracle.grad_exact(g, p.eps0, p.sig0, sh, e[k])
            ge += a
            gs += b
        assert rel_l2(bw["g_eps"], ge) < 1e-10
        assert rel_l2(bw["g_sig"], gs) < 1e-10


@pytest.mark.parametrize("prec,tol", [(N.GJ_F64, 1e-10), (N.GJ_F32, 1e-4)])
def test_misfit_trials_batched_and_band_filtered(gpu_ctx, oracle, small_ft, prec, tol):
    """gj_w_misfit_trials: three trial models in one call equal three single
    calls; with the band filter, each misfit is that of w_objs_e.m:33-36 on
    the oracle's traces: both trace sets filtered (filt_gauss), then
    0.5 |fd - fd_o|^2 / |fd_o|^2."""
    import np_oracle as npo
    p = small_ft
    g = p.grid
    dobs = _dobs(oracle, p)
    models = [p.eps0 * s for s in (0.97, 1.0, 1.04)]
    sigs = [p.sig0] * 3
    band = (80e6, 500e6)
    many = gpu_ctx.w_misfit_trials(g, models, sigs, p.shots, dobs, precision=prec, filt=band)
    assert many.shape == (3, len(p.shots))
    for t, eps in enumerate(models):
        one = gpu_ctx.w_misfit_trials(g, [eps], [p.sig0], p.shots, dobs, precision=prec, filt=band)
        # FP32: the batch and the single call may run different kernels (tuned apart)
        assert np.allclose(one[0], many[t], rtol=1e-12 if prec == N.GJ_F64 else 1e-5)
        for k, sh in enumerate(p.shots):
            d, _, _ = oracle.forward(g, eps, p.sig0, sh)
            fd = npo.filt_gauss(d, g.dt, band[0], band[1], 8)
            fo = npo.filt_gauss(dobs[k], g.dt, band[0], band[1], 8)
            ref = 0.5 * np.sum((fd - fo) ** 2) / np.sum(fo ** 2)
            assert abs(many[t, k] - ref) <= tol * ref
    plain = gpu_ctx.w_misfit_trials(g, models, sigs, p.shots, dobs, precision=prec)
    assert np.allclose(plain[1], gpu_ctx.w_misfit(g, models[1], p.sig0, p.shots, dobs, precision=prec),
                       rtol=1e-12 if prec == N.GJ_F64 else 1e-5)
