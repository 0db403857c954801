"""DC oracle (CPU): the restated reference gradient is the exact gradient of
0.5*||d - d_obs||^2 (central differences), the host-side Robin coefficients
match the oracle's, and the operator is symmetric positive definite."""
import numpy as np
import pytest

from dc_cases import small_dc, oracle_alphas, oracle_forward


def test_alphas_compact_matches_oracle_layout():
    import np_dc_oracle as dco
    case = small_dc()
    for q in case["srcs"]:
        for k, (AL, co) in enumerate(oracle_alphas(dco, case, q)):
            n, m = case["n"], case["m"]
            comp = np.concatenate([AL[0, 1:m - 1], AL[1:n - 1, m - 1], AL[n - 1, 1:m - 1],
                                   [co[0, 0], co[1, 0], co[0, 1], co[1, 1]]])
            assert np.allclose(comp, q.alpha[k], rtol=1e-13, atol=0)


def test_operator_symmetric_positive_definite():
    import np_dc_oracle as dco
    case = small_dc()
    q = case["srcs"][0]
    for k, (AL, co) in enumerate(oracle_alphas(dco, case, q)):
        A = dco.dc_Lk(case["SIG"], case["DX"], case["DZ"], AL, co, q.ky_w[k, 0]).toarray()
        assert np.abs(A - A.T).max() == 0
        assert np.linalg.eigvalsh(A).min() > 0


def test_reference_gradient_matches_finite_differences():
    import np_dc_oracle as dco
    case = small_dc(seed=3)
    n, m, robin = case["n"], case["m"], case["robin"]
    for q, r in zip(case["srcs"], oracle_forward(dco, case, case["SIG"] * 1.2)):
        q.d_obs = r[2]

    def J(S):
        return sum(0.5 * float(r[3] @ r[3]) for r in oracle_forward(dco, case, S))

    g = np.zeros((n - 2 * robin, m - robin))
    for q, r in zip(case["srcs"], oracle_forward(dco, case)):
        g += dco.dc_gradient2_5d(case["SIG"], case["DX"], case["DZ"], oracle_alphas(dco, case, q), q.ky_w,
                                 dco.measuring_operator(n, m, q.mn), r[1], r[3], robin)
    for (l, h) in [(5, 3), (12, 5), (20, 1), (8, 8)]:
        hh = 1e-5 * case["SIG"][l, h]
        Sp, Sm = case["SIG"].copy(), case["SIG"].copy()
        Sp[l, h] += hh
        Sm[l, h] -= hh
        fd = (J(Sp) - J(Sm)) / (2 * hh)
        assert abs(g[l - robin, h] - fd) <= 1e-5 * abs(fd), (l, h, g[l - robin, h], fd)


class _OracleSolver:
    """Stands in for a Context on CPU: dc_forward by the oracle's direct solves."""

    def __init__(self, case):
        self.case = case

    def dc_forward(self, SIG, DX, DZ, robin, srcs, opts=None):
        import np_dc_oracle as dco
        from dc_cases import oracle_forward
        return {"d": [r[2] for r in oracle_forward(dco, self.case, SIG)]}


def test_geometric_factor_and_apparent_resistivity_of_a_half_space():
    """dc_geomefactor2_5d.m: k = 1 / d(sigma = 1); over a homogeneous half-space
    Lk scales with sigma (the Robin terms do not depend on it), so the apparent
    resistivity k * d is exactly 1 / sigma."""
    from dc_cases import small_dc
    from gerjoii_b200 import dc as dcm
    case = small_dc(seed=9)
    solver = _OracleSolver(case)
    shape = case["SIG"].shape
    k = dcm.geometric_factor(solver, shape, case["DX"], case["DZ"], case["robin"], case["srcs"])
    sigma0 = 0.02
    d = solver.dc_forward(np.full(shape, sigma0), case["DX"], case["DZ"], case["robin"], case["srcs"])["d"]
    for rho in dcm.apparent_resistivity(d, k):
        assert np.allclose(rho, 1.0 / sigma0, rtol=1e-10)


def _halfspace_grid():
    from gerjoii_b200 import dc as dcm
    n0, m0, robin, dx = 120, 40, 1, 0.25
    DX, DZ = dcm.deltas(np.arange(n0) * dx, np.arange(m0) * dx, robin)
    return n0 + 2 * robin, m0 + robin, DX, DZ, dx


def test_kfourier_fits_the_dipole_kernel():
    """dc_kfourier.m's design: with the final wavenumbers and weights,
    (2/pi) R sum_k w_k (K0(ky_k r) - K0(ky_k r_)) reproduces 1 over the
    distance pairs of dc_coca.m (rms misfit below 1 %)."""
    import scipy.special as ss
    from gerjoii_b200 import dc as dcm
    n, m, DX, DZ, dx = _halfspace_grid()
    la, lb = dcm.clean_electrode(41, 60)
    r, r_, R = dcm.coca_radius(n, m, DX, DZ, la - 1, lb - 1)
    kw = dcm.kfourier(n, m, DX, DZ, la - 1, lb - 1, 12, dx)
    assert kw.shape == (12, 2) and np.isfinite(kw).all() and (kw[:, 0] > 0).all()
    ky = kw[:, 0] / dx
    v = (2 / np.pi) * R[:, None] * (ss.k0(np.outer(r, ky)) - ss.k0(np.outer(r_, ky))) @ kw[:, 1]
    assert np.sqrt(np.mean((1 - v) ** 2)) < 0.01
    # the reference reuses the first source's distances once finite_.dc.radius is set
    assert np.array_equal(dcm.kfourier(n, m, DX, DZ, 0, 1, 12, dx, radius=(r, r_, R)), kw)


def test_kfourier_halfspace_matches_analytic_potential():
    """The 2.5D potential of a homogeneous half-space (oracle direct solves)
    with dc_kfourier.m's wavenumbers and weights against dc_analhomo2_5d.m's
    I/(2 pi sigma)(1/r_A - 1/r_B), away from the electrodes and the Robin
    boundary (discretisation-limited)."""
    import np_dc_oracle as dco
    from gerjoii_b200 import dc as dcm
    n, m, DX, DZ, dx = _halfspace_grid()
    sigma = 0.01
    SIG = np.full((n, m), sigma)
    la, lb = dcm.clean_electrode(41, 60)
    la, lb = la - 1, lb - 1
    kyw = dcm.kfourier(n, m, DX, DZ, la, lb, 12, dx)
    al = [dco.alphas(n, m, DX, DZ, dco.source_vector(n, m, la, lb)[:n], ky) for ky in kyw[:, 0]]
    u = dco.dc_fwd2_5d(SIG, DX, DZ, dco.source_vector(n, m, la, lb, 1.0), al, kyw,
                       dco.measuring_operator(n, m, np.array([[la + 5, la + 6]])), None)[0]
    u = np.asarray(u).reshape((n, m), order="F")
    ua = dco.analytic_halfspace(n, m, abs(DX), DZ, sigma, la, lb)
    mask = np.zeros_like(u, bool)
    mask[40:85, 2:15] = True
    mask[abs(np.arange(n) - la)[:, None].repeat(m, 1) < 4] = False
    mask[abs(np.arange(n) - lb)[:, None].repeat(m, 1) < 4] = False
    err = np.abs(u[mask] - ua[mask]) / np.abs(ua[mask]).max()
    assert err.max() < 0.10 and np.median(err) < 0.02, (err.max(), np.median(err))


def test_kfourier_rejects_symmetric_electrodes():
    """Electrodes placed symmetrically in the grid leave dc_kfourier.m's
    resampled distances r and r_ identical (every R infinite): an error here,
    where the reference would return NaN weights."""
    from gerjoii_b200 import dc as dcm
    n, m, DX, DZ, dx = _halfspace_grid()
    la, lb = dcm.clean_electrode(51, 70)
    with pytest.raises(ValueError, match="symmetric"):
        dcm.kfourier(n, m, DX, DZ, la - 1, lb - 1, 12, dx)


def test_host_alphas_match_the_python_restatement():
    """gj_dc_alphas (the library's host computation of dc_Lk.m's private alphas,
    for callers that cannot reach it) equals dc.alphas_compact, across grids,
    signed spacings and wavenumbers from ky dx = 2.5e-4 to arguments where
    besselk underflows (large-argument expansion); a node midway between the
    electrodes is 0/0 in both."""
    from gerjoii_b200 import _native as N
    from gerjoii_b200 import dc as dcm
    ky = np.array([2.5e-4, 1e-3, 0.01, 0.1, 1.0, 3.0, 20.0, 80.0])
    for (n, m, DX, DZ, a, b) in [(122, 41, -0.25, 0.25, 40, 59), (32, 11, 0.5, 0.25, 3, 9),
                                 (402, 101, -0.25, 0.25, 100, 107), (7, 5, 1.0, 1.0, 1, 4)]:
        with np.errstate(invalid="ignore"):
            ref = np.stack([dcm.alphas_compact(n, m, DX, DZ, a, b, k) for k in ky])
        got = N.dc_alphas(n, m, DX, DZ, a, b, ky)
        assert got.shape == ref.shape
        assert np.array_equal(np.isnan(got), np.isnan(ref))
        ok = ~np.isnan(ref)
        assert np.allclose(got[ok], ref[ok], rtol=1e-10, atol=0)


def test_redesigned_sources_carry_their_own_design():
    """redesign_sources gives every source dc_kfourier.m's wavenumbers and
    weights (the first source's equal a direct kfourier call) with Robin
    coefficients for those wavenumbers, and the oracle solves the redesigned
    survey to finite, nonzero data."""
    import np_dc_oracle as dco
    from dc_cases import small_dc
    from gerjoii_b200 import dc as dcm
    case = small_dc(seed=11, n0=40, m0=12, n_el=14, pairs=2, levels=2)
    n, m = case["n"], case["m"]
    srcs = dcm.redesign_sources(case["srcs"], n, m, case["DX"], case["DZ"], 8, 0.25)
    assert all(q.ky_w.shape == (8, 2) and q.alpha.shape == (8, dcm.nalpha(n, m)) for q in srcs)
    assert np.array_equal(srcs[0].ky_w, dcm.kfourier(n, m, case["DX"], case["DZ"], srcs[0].a, srcs[0].b, 8, 0.25))
    for q in srcs:
        al = [dco.alphas(n, m, case["DX"], case["DZ"], dco.source_vector(n, m, q.a, q.b)[:n], ky) for ky in q.ky_w[:, 0]]
        d = dco.dc_fwd2_5d(case["SIG"], case["DX"], case["DZ"], dco.source_vector(n, m, q.a, q.b, q.current), al,
                           q.ky_w, dco.measuring_operator(n, m, q.mn), None)[2]
        assert np.isfinite(d).all() and np.abs(d).max() > 0


@pytest.mark.parametrize("sig1,sig2", [(0.01, 0.05), (0.05, 0.01)], ids=["conductive", "resistive"])
def test_two_layer_surface_potential_matches_image_series(sig1, sig2):
    """dc_analbi2_5d.m's known answer: over a 2 m layer on a half-space, the
    oracle's 2.5D surface potential (16 wavenumbers of ky_weights) against the
    image series, away from the electrodes and the Robin boundary."""
    import np_dc_oracle as dco
    from gerjoii_b200 import dc as dcm
    n0, m0, robin, dx, rows = 160, 60, 1, 0.25, 8
    DX, DZ = dcm.deltas(np.arange(n0) * dx, np.arange(m0) * dx, robin)
    sig0 = np.full((n0, m0), sig2)
    sig0[:, :rows] = sig1
    SIG = dcm.dc_robin(sig0, robin)
    n, m = SIG.shape
    la, lb = dcm.clean_electrode(61, 90)
    la, lb = la - 1, lb - 1
    kyw = dcm.ky_weights(dx, n0 * dx, 16, dx=dx)
    al = [dco.alphas(n, m, DX, DZ, dco.source_vector(n, m, la, lb)[:n], ky) for ky in kyw[:, 0]]
    u = dco.dc_fwd2_5d(SIG, DX, DZ, dco.source_vector(n, m, la, lb, 1.0), al, kyw,
                       dco.measuring_operator(n, m, np.array([[la + 5, la + 6]])), None)[0]
    u = np.asarray(u).reshape((n, m), order="F")[:, 0]
    ua = dco.analytic_two_layer(n, dx, sig1, sig2, rows * dx, la, lb)
    l = np.arange(n)
    mask = (np.abs(l - la) >= 4) & (np.abs(l - lb) >= 4) & (l > 30) & (l < n - 30)
    err = np.abs(u[mask] - ua[mask]) / np.abs(ua[mask]).max()
    assert err.max() < 0.03 and np.median(err) < 0.005, (err.max(), np.median(err))
