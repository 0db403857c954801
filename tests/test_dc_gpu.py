"""GPU parity of the 2.5D DC path against the FP64 direct-solve oracle."""
import numpy as np
import pytest

from conftest import rel_l2
from dc_cases import small_dc, oracle_alphas, oracle_forward
from gerjoii_b200 import _native as N
from gerjoii_b200 import dc
from gerjoii_b200 import synth

pytestmark = pytest.mark.gpu


def test_dc_forward_matches_direct_solve(gpu_ctx):
    """Data, stacked potentials u and the per-wavenumber potentials u_k
    (gerjoii_.dc.u_k of dc_fwd2_5d.m:61, through gj_dc_forward_k) against the
    oracle's FP64 direct solves."""
    import np_dc_oracle as dco
    case = small_dc()
    res = gpu_ctx.dc_forward(case["SIG"], case["DX"], case["DZ"], case["robin"], case["srcs"], want_u=True,
                             want_uk=True)
    ref = oracle_forward(dco, case)
    for k, r in enumerate(ref):
        assert rel_l2(res["d"][k], r[2]) < 1e-9
        assert rel_l2(res["u"][k], r[0].reshape((case["n"], case["m"]), order="F")) < 1e-9
        assert res["u_k"][k].shape == r[1].shape
        assert rel_l2(res["u_k"][k], r[1]) < 1e-9
    assert res["rel_residual"] <= 1e-10


@pytest.mark.parametrize("shape", [
    dict(n0=20, m0=2, n_el=6, spacing=2, first=2, levels=1, pairs=2),   # b = 3, depth fastest
    dict(n0=4, m0=30, n_el=5, spacing=1, first=0, levels=1, pairs=2),   # b = 6, lateral fastest
    dict(n0=150, m0=130, n_el=12, spacing=10, first=5, levels=2, pairs=1, n_ky=2),  # b = 131
], ids=["b3", "b6", "b131"])
def test_dc_forward_band_widths(gpu_ctx, shape):
    """Band widths at the edges of the factor and substitution layouts: windows
    narrower than the factor's panel (b = 3, 6; both unknown orderings) and a
    band wider than 127, which takes the 256-position substitution window."""
    import np_dc_oracle as dco
    case = small_dc(seed=7, **shape)
    res = gpu_ctx.dc_forward(case["SIG"], case["DX"], case["DZ"], case["robin"], case["srcs"], want_u=True)
    assert res["rel_residual"] <= 1e-10
    for k, r in enumerate(oracle_forward(dco, case)):
        assert rel_l2(res["d"][k], r[2]) < 1e-9
        assert rel_l2(res["u"][k], r[0].reshape((case["n"], case["m"]), order="F")) < 1e-9


def test_dc_gradient_matches_oracle(gpu_ctx):
    import np_dc_oracle as dco
    case = small_dc(seed=4)
    n, m, robin = case["n"], case["m"], case["robin"]
    for q, r in zip(case["srcs"], oracle_forward(dco, case, case["SIG"] * 1.3)):
        q.d_obs = r[2]
    g = np.zeros((n - 2 * robin, m - robin))
    mis = []
    for q, r in zip(case["srcs"], oracle_forward(dco, case)):
        g += dco.dc_gradient2_5d(case["SIG"], case["DX"], case["DZ"], oracle_alphas(dco, case, q), q.ky_w,
                                 dco.measuring_operator(n, m, q.mn), r[1], r[3], robin)
        mis.append(0.5 * float(r[3] @ r[3]))
    res = gpu_ctx.dc_gradient(case["SIG"], case["DX"], case["DZ"], robin, case["srcs"])
    assert rel_l2(res["g"], g) < 1e-8
    assert np.allclose(res["misfit"], mis, rtol=1e-8)
    o = N.DcOptsC()
    o.per_source = 1
    res2 = gpu_ctx.dc_gradient(case["SIG"], case["DX"], case["DZ"], robin, case["srcs"], opts=o)
    assert rel_l2(res2["g"].sum(0), res["g"]) < 1e-12


def test_dc_halfspace_matches_analytic_potential(gpu_ctx):
    """dc_analhomo2_5d.m: a homogeneous half-space; the 2.5D solution with the
    designed ky/w (grid units, as the reference's ky_w_) approximates
    I/(2 pi sigma)(1/r_A - 1/r_B) away from the electrodes and the Robin
    boundary (discretisation-limited: a few per cent within 1-2 m of an
    electrode, about 1 % elsewhere)."""
    import np_dc_oracle as dco
    n0, m0, robin, dx = 120, 40, 1, 0.25
    X = np.arange(n0) * dx
    Z = np.arange(m0) * dx
    DX, DZ = dc.deltas(X, Z, robin)
    sigma = 0.01
    SIG = dc.dc_robin(np.full((n0, m0), sigma), robin)
    n, m = SIG.shape
    kyw = dc.ky_weights(dx, n0 * dx, 12, dx=dx)
    la, lb = dc.clean_electrode(51, 70)
    la, lb = la - 1, lb - 1
    al = np.stack([dc.alphas_compact(n, m, DX, DZ, la, lb, ky) for ky in kyw[:, 0]])
    src = dc.DcSource(la, lb, 1.0, np.array([[la + 5, la + 6]], np.int64), kyw, al)
    res = gpu_ctx.dc_forward(SIG, DX, DZ, robin, [src], want_u=True)
    u = res["u"][0]
    ua = dco.analytic_halfspace(n, m, abs(DX), DZ, sigma, la, lb)
    mask = np.zeros_like(u, bool)
    mask[40:85, 2:15] = True
    mask[abs(np.arange(n) - la)[:, None].repeat(m, 1) < 4] = False
    mask[abs(np.arange(n) - lb)[:, None].repeat(m, 1) < 4] = False
    err = np.abs(u[mask] - ua[mask]) / np.abs(ua[mask]).max()
    assert err.max() < 0.10 and np.median(err) < 0.02, (err.max(), np.median(err))


def test_dc_full_survey_converges_in_few_iterations(gpu_ctx):
    """400 x 100 cells, 200 dipole-dipole sources x 20 wavenumbers: the FP64 band
    factor makes the preconditioner (numerically) exact, so CG reaches 1e-10 in a
    handful of iterations for every wavenumber, down to ky dx = 2.5e-4 where the
    operator is nearly singular; the adjoint solves of noisy data converge too,
    and the gradient of two sources matches the direct-solve oracle."""
    import np_dc_oracle as dco
    from gerjoii_b200 import synth
    c = synth.cfg5()
    fw = gpu_ctx.dc_forward(c["SIG"], c["DX"], c["DZ"], c["robin"], c["srcs"])
    assert fw["rel_residual"] <= 1e-10 and fw["iters"] <= 6, (fw["iters"], fw["rel_residual"])
    rng = np.random.default_rng(5)
    for q, d in zip(c["srcs"], fw["d"]):
        q.d_obs = d * (1 + 0.02 * rng.standard_normal(d.shape))
    gr = gpu_ctx.dc_gradient(c["SIG"], c["DX"], c["DZ"], c["robin"], c["srcs"])
    assert gr["rel_residual"] <= 1e-10 and gr["iters"] <= 8, (gr["iters"], gr["rel_residual"])
    case = dict(c, srcs=c["srcs"][:2])
    n, m, robin = c["n"], c["m"], c["robin"]
    g = np.zeros((n - 2 * robin, m - robin))
    for q, r in zip(case["srcs"], oracle_forward(dco, case)):
        g += dco.dc_gradient2_5d(c["SIG"], c["DX"], c["DZ"], oracle_alphas(dco, case, q), q.ky_w,
                                 dco.measuring_operator(n, m, q.mn), r[1], r[3], robin)
    g2 = gpu_ctx.dc_gradient(c["SIG"], c["DX"], c["DZ"], robin, case["srcs"])["g"]
    assert rel_l2(g2, g) < 1e-8


def test_dc_fp32_factor_option(gpu_ctx):
    """factor_fp32 = 1 keeps an FP32 band factor as the preconditioner (half
    the memory); the FP64 iterations still meet the same tolerance."""
    case = small_dc(seed=2)
    o = N.DcOptsC()
    o.factor_fp32 = 1
    o.max_iter = 200
    a = gpu_ctx.dc_forward(case["SIG"], case["DX"], case["DZ"], case["robin"], case["srcs"], opts=o)
    b = gpu_ctx.dc_forward(case["SIG"], case["DX"], case["DZ"], case["robin"], case["srcs"])
    assert a["rel_residual"] <= 1e-10 and b["rel_residual"] <= 1e-10
    assert b["iters"] <= a["iters"]
    for x, y in zip(a["d"], b["d"]):
        assert rel_l2(x, y) < 1e-9


def test_geometric_factor_matches_oracle(gpu_ctx):
    """dc_geomefactor2_5d.m through the GPU solver: k = 1 / d(sigma = 1)
    against the oracle's direct solve, and the apparent resistivity k * d of a
    homogeneous half-space equal to 1 / sigma."""
    import np_dc_oracle as dco
    from gerjoii_b200 import dc as dcm
    case = small_dc(seed=9)
    shape = case["SIG"].shape
    k = dcm.geometric_factor(gpu_ctx, shape, case["DX"], case["DZ"], case["robin"], case["srcs"])
    for kk, r in zip(k, oracle_forward(dco, case, np.ones(shape))):
        assert rel_l2(kk, 1.0 / r[2]) < 1e-9
    d = gpu_ctx.dc_forward(np.full(shape, 0.02), case["DX"], case["DZ"], case["robin"], case["srcs"])["d"]
    for rho in dcm.apparent_resistivity(d, k):
        assert np.allclose(rho, 50.0, rtol=1e-8)


def test_dc_fp32_factor_wide_band(gpu_ctx):
    """factor_fp32 = 1 on a band wider than 127 (b = 131): the FP32 factor
    through the 256-position substitution window meets the FP64 tolerance and
    agrees with the FP64-factor solution."""
    case = small_dc(seed=7, n0=150, m0=130, n_el=12, spacing=10, first=5, levels=2, pairs=1, n_ky=2)
    o = N.DcOptsC()
    o.factor_fp32 = 1
    o.max_iter = 200
    a = gpu_ctx.dc_forward(case["SIG"], case["DX"], case["DZ"], case["robin"], case["srcs"], opts=o)
    b = gpu_ctx.dc_forward(case["SIG"], case["DX"], case["DZ"], case["robin"], case["srcs"])
    assert a["rel_residual"] <= 1e-10 and b["rel_residual"] <= 1e-10
    for x, y in zip(a["d"], b["d"]):
        assert rel_l2(x, y) < 1e-9


def test_dc_ic0_preconditioner_option_matches_direct_solve(gpu_ctx):
    """The FP32 red-black IC(0) preconditioner option (gj_dc_opts.precond = 1):
    FP64 CG refines to the same 1e-10 relative residual, so data, potentials
    and the gradient equal the FP64 direct solve and the band-factor path; it
    needs many more iterations than the band factor's one."""
    import np_dc_oracle as dco
    case = small_dc(seed=11)
    o = N.DcOptsC()
    o.precond = 1
    res = gpu_ctx.dc_forward(case["SIG"], case["DX"], case["DZ"], case["robin"], case["srcs"], opts=o, want_u=True)
    assert res["rel_residual"] <= 1e-10 and res["iters"] > 1
    for k, r in enumerate(oracle_forward(dco, case)):
        assert rel_l2(res["d"][k], r[2]) < 1e-9
        assert rel_l2(res["u"][k], r[0].reshape((case["n"], case["m"]), order="F")) < 1e-9
    for q, r in zip(case["srcs"], oracle_forward(dco, case, case["SIG"] * 1.2)):
        q.d_obs = r[2]
    g1 = gpu_ctx.dc_gradient(case["SIG"], case["DX"], case["DZ"], case["robin"], case["srcs"], opts=o)
    g0 = gpu_ctx.dc_gradient(case["SIG"], case["DX"], case["DZ"], case["robin"], case["srcs"])
    assert rel_l2(g1["g"], g0["g"]) < 1e-8


def test_context_release_frees_cached_buffers_and_keeps_working(gpu_ctx):
    """gj_context_release frees the DC factors and CG vectors the context keeps
    between calls (device memory comes back) and the next call works."""
    import torch
    case = small_dc(seed=12, n0=150, m0=60, pairs=6)
    r1 = gpu_ctx.dc_forward(case["SIG"], case["DX"], case["DZ"], case["robin"], case["srcs"])
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    gpu_ctx.release()
    free1 = torch.cuda.mem_get_info()[0]
    assert free1 > free0
    r2 = gpu_ctx.dc_forward(case["SIG"], case["DX"], case["DZ"], case["robin"], case["srcs"])
    for a, b in zip(r1["d"], r2["d"]):
        assert rel_l2(a, b) < 1e-12


@pytest.mark.parametrize("env", [{"GJ_DC_TILE": "8"}, {"GJ_DC_RING": "16x4"}, {"GJ_DC_RING": "4x8"}],
                         ids=["tile8", "ring16x4", "ring4x8"])
def test_dc_kernel_variants_match_default(gpu_ctx, env):
    """The factor's 4 x 8 trailing tiles and the substitution's other ring
    shapes (chosen per call through the environment) give the default's data."""
    import os
    c = synth.cfg5(n_sources=3, n_ky=4)
    ref = gpu_ctx.dc_forward(c["SIG"], c["DX"], c["DZ"], c["robin"], c["srcs"])
    os.environ.update(env)
    try:
        alt = gpu_ctx.dc_forward(c["SIG"], c["DX"], c["DZ"], c["robin"], c["srcs"])
    finally:
        for k in env:
            del os.environ[k]
    for a, b in zip(alt["d"], ref["d"]):
        assert np.allclose(a, b, rtol=1e-9, atol=0)
    assert alt["rel_residual"] <= 1e-10
