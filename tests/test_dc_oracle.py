"""DC oracle (CPU): the restated reference gradient is the exact gradient of
0.5*||d - d_obs||^2 (central differences), the host-side Robin coefficients
match the oracle's, and the operator is symmetric positive definite."""
import numpy as np

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
