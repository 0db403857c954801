"""Oracle self-consistency (CPU): the C++ restatement against the numpy twin
that follows the MATLAB slicing, known-answer checks, and the exact adjoint
against central finite differences."""
import numpy as np
import pytest

from conftest import rel_l2
from gerjoii_b200 import synth
from gerjoii_b200.geometry import Shot


def _np_run(npo, p, shot):
    g = p.grid
    f = npo.w_layout(g.m, g.n, g.pml, g.air, g.pml_top)
    er, sz = npo.w_exp2pml(p.eps0, p.sig0, g.pml, g.air, g.pml_top)
    d, u, jz = npo.w_solve(er, sz, f, (shot.src_i + 1, shot.src_j + 1), shot.rec + 1, shot.wavelet, g.nt,
                           g.dx, g.dy, g.dt, g.eps0, g.mu0)
    return f, er, sz, d, u, jz


@pytest.mark.parametrize("free_top", [True, False])
def test_forward_and_reference_adjoint_match_numpy_twin(oracle, free_top):
    import np_oracle as npo
    p = synth.small(m=14, n=20, pml=6, nt=160, free_top=free_top, seed=3)
    g, shot = p.grid, p.shots[1]
    d, jz, u = oracle.forward(g, p.eps0, p.sig0, shot, store_u=True)
    f, er, sz, d2, u2, jz2 = _np_run(npo, p, shot)
    assert rel_l2(d, d2) < 1e-13 and rel_l2(u, u2) < 1e-13 and rel_l2(jz, jz2) < 1e-13
    e = d - 0.5 * np.roll(d, 7, axis=0)
    gr, am = oracle.grad_reference(g, p.eps0, p.sig0, shot, e, u)
    gr2, am2 = npo.w_grad(u2, e, er, sz, f, (shot.src_i + 1, shot.src_j + 1), shot.rec + 1, g.nt, g.dx, g.dy,
                          g.dt, g.eps0, g.mu0)
    assert rel_l2(gr, gr2) < 1e-12 and rel_l2(am, am2) < 1e-12


def test_differentiate_cube_known_answer(oracle):
    # differentiate_line.m:52-56: derivative of sin is cos to second order.
    import np_oracle as npo
    nt, dt = 400, 1e-3
    t = np.arange(nt) * dt
    v = np.sin(2 * np.pi * 5 * t)[None, None, :] * np.ones((3, 2, 1))
    dv = oracle.differentiate_cube(v, dt)
    ref = 2 * np.pi * 5 * np.cos(2 * np.pi * 5 * t)
    assert np.max(np.abs(dv[1, 1, 1:-1] - ref[1:-1])) < 2e-2 * np.max(np.abs(ref))
    assert rel_l2(dv, npo.differentiate_cube(v, dt)) < 1e-14
    # exact on quadratics in the interior and at both one-sided ends
    q = (3 * t ** 2 - t)[None, None, :]
    assert np.allclose(oracle.differentiate_cube(q, dt)[0, 0], 6 * t - 1, rtol=0, atol=1e-9)


@pytest.mark.parametrize("free_top", [True, False])
def test_exact_adjoint_matches_finite_differences(oracle, free_top):
    p = synth.small(m=10, n=14, pml=5, nt=140, free_top=free_top, seed=11)
    g = p.grid
    sh = p.shots[1]
    rec = np.concatenate([sh.rec, [g.node(*g.model_node(9, 0)), g.node(g.NX - 2, 3)]])
    sh = Shot(sh.src_i, sh.src_j, sh.wavelet, rec)
    dobs, _, _ = oracle.forward(g, p.eps_true, p.sig_true, sh)

    def J(e_, s_):
        d, _, _ = oracle.forward(g, e_, s_, sh)
        return 0.5 * np.sum((d - dobs) ** 2)

    d, _, _ = oracle.forward(g, p.eps0, p.sig0, sh)
    ge, gs = oracle.grad_exact(g, p.eps0, p.sig0, sh, d - dobs)
    # interior cell, model corners and edges (PML-replicated), first column (PML band)
    for (a, b) in [(4, 6), (0, 0), (9, 13), (9, 0), (5, 0), (5, 13), (9, 7), (0, 8)]:
        h = 1e-4 * p.eps0[a, b]
        ep, em = p.eps0.copy(), p.eps0.copy()
        ep[a, b] += h
        em[a, b] -= h
        fd = (J(ep, p.sig0) - J(em, p.sig0)) / (2 * h)
        assert abs(ge[a, b] - fd) <= 1e-5 * abs(fd) + 1e-12 * np.abs(ge).max(), (a, b, ge[a, b], fd)
        hs = 1e-3 * p.sig0[a, b]
        sp, sm = p.sig0.copy(), p.sig0.copy()
        sp[a, b] += hs
        sm[a, b] -= hs
        fds = (J(p.eps0, sp) - J(p.eps0, sm)) / (2 * hs)
        assert abs(gs[a, b] - fds) <= 1e-5 * abs(fds) + 1e-9 * np.abs(gs).max(), (a, b, gs[a, b], fds)


def test_exact_adjoint_dot_product(oracle):
    """<J'(m) dm> from the adjoint equals the directional derivative."""
    p = synth.small(m=10, n=14, pml=5, nt=120, seed=5)
    g, sh = p.grid, p.shots[0]
    rng = np.random.default_rng(0)
    dm = rng.standard_normal(p.eps0.shape)
    dobs, _, _ = oracle.forward(g, p.eps_true, p.sig_true, sh)
    d, _, _ = oracle.forward(g, p.eps0, p.sig0, sh)
    ge, _ = oracle.grad_exact(g, p.eps0, p.sig0, sh, d - dobs)
    h = 1e-5
    dp, _, _ = oracle.forward(g, p.eps0 + h * dm, p.sig0, sh)
    dmn, _, _ = oracle.forward(g, p.eps0 - h * dm, p.sig0, sh)
    fd = (0.5 * np.sum((dp - dobs) ** 2) - 0.5 * np.sum((dmn - dobs) ** 2)) / (2 * h)
    assert abs(np.sum(ge * dm) - fd) < 1e-6 * abs(fd)


def test_reference_adjoint_differs_from_exact_in_lossy_media(oracle):
    """The reference adjoint (sigma flipped, hard-set residual) is not the
    exact transpose; record the cosine between the two sigma gradients."""
    p = synth.small(m=12, n=18, pml=6, nt=200, seed=9)
    g, sh = p.grid, p.shots[1]
    dobs, _, _ = oracle.forward(g, p.eps_true, p.sig_true, sh)
    d, _, u = oracle.forward(g, p.eps0, p.sig0, sh, store_u=True)
    e = d - dobs
    ge, gs = oracle.grad_exact(g, p.eps0, p.sig0, sh, e)
    gr, _ = oracle.grad_reference(g, p.eps0, p.sig0, sh, e, u)
    c = float(np.sum(gr * gs) / (np.linalg.norm(gr) * np.linalg.norm(gs)))
    assert np.isfinite(c)


def _smooth_traces(seed=3, nt=64, nr=3):
    rng = np.random.default_rng(seed)
    t = np.arange(nt)[:, None]
    d = (np.sin(0.3 * t + rng.random(nr)) * np.exp(-((t - 30) / 15.0) ** 2)
         + 0.3 * np.cos(0.11 * t + rng.random(nr)))
    do = 0.9 * d + 0.05 * np.sin(0.2 * t)
    return d, do


@pytest.mark.parametrize("kind,scale", [("env_L2", 1.0), ("env_L22", 2.0), ("env_LOG", 1.0)])
def test_envelope_adjoint_sources_are_misfit_gradients(kind, scale):
    """w_bozdag.m's envelope adjoint sources are the derivatives of their
    unnormalised misfits 0.5 sum (f(E) - f(Eo))^2 (f = identity, square, log;
    w_E.m:8-16) with respect to the traces; env_L22's is half of it.  Central
    differences on smooth traces pin the restatement without MATLAB."""
    import np_oracle as npo
    d, do = _smooth_traces()
    f = {"env_L2": lambda v: v, "env_L22": lambda v: v ** 2, "env_LOG": np.log}[kind]

    def J(x):
        _, de, doe = npo.w_bozdag(do, x, kind)
        r = f(de) - f(doe)
        return 0.5 * float(np.sum(r * r))

    e, _, _ = npo.w_bozdag(do, d, kind)
    h = 1e-6
    for (i, j) in [(5, 0), (30, 1), (47, 2), (63, 0)]:
        dp, dm = d.copy(), d.copy()
        dp[i, j] += h
        dm[i, j] -= h
        fd = (J(dp) - J(dm)) / (2 * h)
        assert abs(scale * e[i, j] - fd) <= 1e-6 * max(abs(fd), np.abs(scale * e).max())


@pytest.mark.parametrize("kind", ["L2", "env_L2", "phase_L2", "env_L22", "env_LOG"])
def test_adjoint_sources_vanish_at_the_data(kind):
    """Every objective's adjoint source and misfit are zero when the modelled
    traces equal the observed ones (w_bozdag.m:13-54, w_E.m)."""
    import np_oracle as npo
    d, _ = _smooth_traces(seed=5)
    e, de, doe = npo.w_bozdag(d, d, kind)
    assert np.abs(e).max() <= 1e-12 * np.abs(d).max()
    assert npo.w_E(doe, de, kind) == 0.0


def test_forward_matches_the_2d_greens_function(oracle):
    """Known answer: w_wavelet.m:15-18's 2D impulse response (1/2 pi) /
    sqrt((v t)^2 - R^2) driven by the injected source.  The soft source adds
    -dt/eps w(t) to one Ez node (Cezj, w_coeff.m), a line current w dx dy, so in
    vacuum E(R, t) = -(mu dx dy / 2 pi) int_0^acosh(ct/R) w'(t - (R/c) cosh s) ds
    (the substitution removes the singularity at t = R/c).  The oracle's traces
    (reference layout, PML all round) at 15-35 cells equal it half a time step
    later (the leapfrog staggering) to correlation 1 - 1e-5 and amplitude 0.5 %."""
    import math
    from gerjoii_b200.geometry import WGrid, Shot, w_wavelet, MU_0, C_0
    m = n = 90
    pml, air, dx, fo, nt = 20, 10, 0.05, 100e6, 520
    dt = WGrid(m=m, n=n, pml=pml, pml_top=pml, air=air, nt=1, dx=dx, dy=dx, dt=1.0).cfl_dt(1.0, 0.95)
    g = WGrid(m=m, n=n, pml=pml, pml_top=pml, air=air, nt=nt, dx=dx, dy=dx, dt=dt)
    t = np.arange(nt) * dt
    w = w_wavelet(t, 1e3, 1 / fo)
    si, sj = g.model_node(45, 30)
    cells = [(45, 50), (45, 65), (60, 30)]
    rec = np.array([g.node(*g.model_node(a, b)) for a, b in cells])
    d, _, _ = oracle.forward(g, np.ones((m, n)), np.zeros((m, n)), Shot(si, sj, w, rec))
    tf = np.arange(-2000, 20 * nt) * (dt / 20)
    wpf = np.gradient(w_wavelet(tf, 1e3, 1 / fo), tf)
    for k, (a, b) in enumerate(cells):
        R = math.hypot((a - 45) * dx, (b - 30) * dx)
        an = np.zeros(nt)
        for i, ti in enumerate(t + 0.5 * dt):
            if C_0 * ti > R:
                s = np.linspace(0.0, math.acosh(C_0 * ti / R), 4000)
                an[i] = np.trapezoid(np.interp(ti - (R / C_0) * np.cosh(s), tf, wpf), s)
        an *= -(MU_0 * dx * dx / (2 * math.pi))
        cc = float(an @ d[:, k] / (np.linalg.norm(an) * np.linalg.norm(d[:, k])))
        assert cc > 1 - 1e-5, (R, cc)
        assert abs(np.abs(d[:, k]).max() / np.abs(an).max() - 1) < 5e-3, R


@pytest.mark.parametrize("sigma", [2e-3, 1e-2])
def test_forward_matches_the_lossy_2d_solution(oracle, sigma):
    """Known answer in a lossy dielectric (eps_r = 4): the line-source field
    E(w) = -(w mu / 4) I(w) H0^(2)(k R), k^2 = w^2 mu eps - i w mu sigma (time
    dependence e^{iwt}, Im k < 0), with I = w dx dy as above and the half-step
    staggering.  The model is deep enough that the reflection from the air
    layer arrives after the record; numerical dispersion (about 30 cells per
    wavelength at the air-limited time step) bounds the match: correlation
    1 - 5e-4, amplitude 1.5 %, at 20 and 35 cells."""
    import math
    import scipy.special as ss
    from gerjoii_b200.geometry import WGrid, Shot, w_wavelet, MU_0, EPS_0
    m, n, pml, air, dx, fo, nt, epsr = 200, 160, 20, 10, 0.05, 100e6, 700, 4.0
    dt = WGrid(m=m, n=n, pml=pml, pml_top=pml, air=air, nt=1, dx=dx, dy=dx, dt=1.0).cfl_dt(1.0, 0.95)
    g = WGrid(m=m, n=n, pml=pml, pml_top=pml, air=air, nt=nt, dx=dx, dy=dx, dt=dt)
    w = w_wavelet(np.arange(nt) * dt, 1e3, 1 / fo)
    a0, b0 = 140, 60
    cells = [(140, 80), (140, 95)]
    rec = np.array([g.node(*g.model_node(a, b)) for a, b in cells])
    d, _, _ = oracle.forward(g, np.full((m, n), epsr), np.full((m, n), sigma), Shot(*g.model_node(a0, b0), w, rec))
    npad = 8 * nt
    om = 2 * np.pi * np.fft.rfftfreq(npad, dt)
    Iw = np.fft.rfft(w * dx * dx, npad) * np.exp(0.5j * om * dt)
    k = np.sqrt(om ** 2 * MU_0 * epsr * EPS_0 - 1j * om * MU_0 * sigma)
    k = np.where(k.imag > 0, -k, k)
    for j, (a, b) in enumerate(cells):
        R = math.hypot((a - a0) * dx, (b - b0) * dx)
        H = np.zeros_like(Iw)
        H[1:] = -(om[1:] * MU_0 / 4) * Iw[1:] * ss.hankel2(0, k[1:] * R)
        an = np.fft.irfft(H, npad)[:nt]
        cc = float(an @ d[:, j] / (np.linalg.norm(an) * np.linalg.norm(d[:, j])))
        assert cc > 1 - 5e-4, (R, cc)
        assert abs(np.abs(d[:, j]).max() / np.abs(an).max() - 1) < 0.015, R


@pytest.mark.parametrize("pml,bound", [(10, 2e-3), (20, 5e-4)])
def test_pml_absorbs(oracle, pml, bound):
    """The split-field PML of w_cpml.m (order 2, R0 = 1e-8, wdc_geom.m:98-99)
    absorbs: traces 10 cells from the PML of a 60 x 60 model equal those of a
    300 x 300 model (no boundary within reach during the record) to `bound` of
    the direct wave's peak (measured 5e-4 at 10 cells, 1e-4 at 20)."""
    from gerjoii_b200.geometry import WGrid, Shot, w_wavelet
    dx, fo, air, nt = 0.05, 100e6, 10, 600

    def run(m, n, src, recs):
        dt = WGrid(m=m, n=n, pml=pml, pml_top=pml, air=air, nt=1, dx=dx, dy=dx, dt=1.0).cfl_dt(1.0, 0.95)
        g = WGrid(m=m, n=n, pml=pml, pml_top=pml, air=air, nt=nt, dx=dx, dy=dx, dt=dt)
        w = w_wavelet(np.arange(nt) * dt, 1e3, 1 / fo)
        rec = np.array([g.node(*g.model_node(a, b)) for a, b in recs])
        return oracle.forward(g, np.ones((m, n)), np.zeros((m, n)), Shot(*g.model_node(*src), w, rec))[0]

    small = run(60, 60, (30, 20), [(30, 50), (50, 20)])
    big = run(300, 300, (150, 140), [(150, 170), (170, 140)])
    for j in range(2):
        assert np.abs(small[:, j] - big[:, j]).max() <= bound * np.abs(big[:, j]).max()
