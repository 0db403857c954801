"""Host side of the 2.5D DC-resistivity path (mirrors src/dc of the reference).

The solves run in the CUDA library (gj_dc_forward / gj_dc_gradient); this
module prepares their inputs the way the reference's MATLAB does:

* :func:`dc_robin` pads sigma with the Robin columns/rows (dc_robin.m:36-46);
* :func:`deltas` returns the spacings do_grid.m stores in DELTAS;
* :func:`clean_electrode` applies dc_electrodes.m's parity clean (:66-75);
* :func:`alphas_compact` evaluates the Robin coefficients of dc_Lk.m's
  private ``alphas`` (:820-960) in the compact layout of the C ABI;
* :func:`ky_weights` designs wavenumbers and weights for the inverse cosine
  transform u = (2/pi) sum_k w_k u_k (a least-squares fit of the half-space
  kernel on fixed log-spaced wavenumbers);
* :func:`kfourier` is the reference's own per-source design (dc_kfourier.m,
  Gauss-Newton on the wavenumbers over the distances of :func:`coca_radius`).
"""
from __future__ import annotations

import dataclasses

import numpy as np
import scipy.special as ss


def dc_robin(sigma: np.ndarray, robin: int) -> np.ndarray:
    """Pad an (n0 x m0) lateral-by-depth conductivity with `robin` replicated
    columns left/right and rows at the bottom (dc_robin.m:36-46)."""
    s = np.asarray(sigma, np.float64)
    s = np.vstack([np.repeat(s[:1, :], robin, 0), s, np.repeat(s[-1:, :], robin, 0)])
    return np.hstack([s, np.repeat(s[:, -1:], robin, 1)])


def deltas(X: np.ndarray, Z: np.ndarray, robin: int) -> tuple[float, float]:
    """DELTAS(:,:,1) and DELTAS(:,:,2) of do_grid.m: x_robin(2)-x_robin(1) and
    z_robin(2)-z_robin(1) with x_robin = [(1:robin)*dx, X, (1:robin)*dx]."""
    X = np.asarray(X, np.float64)
    Z = np.asarray(Z, np.float64)
    xr = np.concatenate([np.arange(1, robin + 1) * (X[1] - X[0]), X, np.arange(1, robin + 1) * (X[-1] - X[-2])])
    zr = np.concatenate([Z, np.arange(1, robin + 1) * (Z[-1] - Z[-2])])
    return float(xr[1] - xr[0]), float(zr[1] - zr[0])


def clean_electrode(la_1based: int, lb_1based: int) -> tuple[int, int]:
    """dc_electrodes.m:66-75: the +I electrode moves to an even lateral index
    and the -I electrode to an odd one (1-based), so that no node is
    equidistant from both."""
    if la_1based % 2 == 1:
        la_1based += 1
    if lb_1based % 2 == 0:
        lb_1based += 1
    return la_1based, lb_1based


def nalpha(n: int, m: int) -> int:
    return 2 * (m - 2) + (n - 2) + 4


def alphas_compact(n: int, m: int, DX: float, DZ: float, a_node: int, b_node: int, ky: float) -> np.ndarray:
    """Robin coefficients alpha = sum_e beta_e ky K1(ky r) (ca/r) / sum_e beta_e
    K0(ky r) for the two surface electrodes (beta = +1 at A, -1 at B), on the
    left side, bottom, right side and bottom corners, in the compact layout
    [left h=2..m-1 | bottom l=2..n-1 | right h=2..m-1 | c11 c21 c12 c22].

    Distances follow dc_Lk.m's alphas (co/ca built from DELTAS, signs included).
    Only the two electrode columns carry weight, so only they are evaluated,
    and K0/K1 are taken exponentially scaled (k0e, k1e) relative to the nearer
    electrode: where ky*r is large enough for besselk to underflow (0/0 in
    the reference) this returns the limit of the same ratio."""
    la, lb = a_node % n, b_node % n
    cols = np.array([la, lb])
    beta = np.array([1.0, -1.0])
    hh = np.arange(1, m)
    co_left = np.outer(hh * DZ, np.ones(2))
    co_down = np.abs(np.arange(n)[:, None] - cols[None, :]) * DX
    co_right = np.outer(hh[::-1] * DZ, np.ones(2))
    co = np.vstack([co_left, co_down, co_right])
    ca_left = np.outer(np.ones(m - 1), cols * DX)
    ca_right = np.outer(np.ones(m - 1), (n - 1 - cols) * DX)
    ca = np.vstack([ca_left, (m - 1) * DZ * np.ones((n, 2)), ca_right])
    r = np.sqrt(co ** 2 + ca ** 2)
    x = ky * r
    x0 = x.min(axis=1, keepdims=True)
    sc = np.exp(-(x - x0))
    numer = (ky * ss.k1e(x) * sc * (ca / r)) @ beta
    denom = (ss.k0e(x) * sc) @ beta
    a = numer / denom
    left = a[0:m - 2]
    bottom = a[m:m + n - 2]
    right = a[m + n:][::-1]
    corners = np.array([a[m - 2], a[m - 1], a[m + n - 2], a[m + n - 1]])  # c11 c21 c12 c22
    return np.concatenate([left, bottom, right, corners])


def ky_weights(r_min: float, r_max: float, n_ky: int, dx: float | None = None, n_fit: int = 200):
    """Wavenumbers (log-spaced over [0.1/r_max, 10/r_min]) and weights w_k >= 0
    chosen by least squares so that (2/pi) sum_k w_k K0(ky_k r) ~ 1/r over
    [r_min, r_max] (relative error), the half-space form of the 2.5D inverse
    transform.  Returns an (n_ky, 2) array like finite_.dc.ky_w_.  With `dx`
    the wavenumbers are returned in grid units (ky*|dx|), the convention of
    the reference's ky_w_ (dc_kfourier.m:197): its operator adds ky^2 sigma
    without a cell area (dc_Lk.m:809)."""
    from scipy.optimize import nnls
    ky = np.geomspace(0.1 / r_max, 10.0 / r_min, n_ky)
    r = np.geomspace(r_min, r_max, n_fit)
    A = (2 / np.pi) * ss.k0(np.outer(r, ky)) * r[:, None]  # relative: times r
    w, _ = nnls(A, np.ones(n_fit), maxiter=50 * n_ky * n_fit)
    if dx is not None:
        ky = ky * abs(dx)
    return np.column_stack([ky, w])


@dataclasses.dataclass
class DcSource:
    a: int  # +I node (0-based, vectorised l + h*n)
    b: int  # -I node
    current: float
    mn: np.ndarray  # (nd, 2) receiver node pairs
    ky_w: np.ndarray  # (n_ky, 2)
    alpha: np.ndarray  # (n_ky, nalpha)
    d_obs: np.ndarray | None = None

    @property
    def nd(self) -> int:
        return int(len(self.mn))


def dipole_dipole(n: int, m: int, robin: int, DX: float, DZ: float, n_electrodes: int, spacing_nodes: int,
                  first_node: int, pairs: int, levels: int, ky_w: np.ndarray, rng=None, current: float = 1.0,
                  dipole_lengths=(1, 2, 3)):
    """Surface dipole-dipole survey: AB dipoles of length a electrode spacings
    (a in dipole_lengths), each with MN dipoles of the same length at
    separations a*1..a*levels beyond B.  `pairs` AB dipoles are drawn (seeded
    by rng) from every complete combination.  Electrode lateral node indices
    are 0-based surface nodes; the source pair is parity-cleaned like
    dc_electrodes.m."""
    elec = first_node + robin + spacing_nodes * np.arange(n_electrodes)
    combos = [(i, a) for a in dipole_lengths for i in range(n_electrodes)
              if i + a + a * levels + a < n_electrodes]
    if rng is not None:
        combos = [combos[k] for k in rng.permutation(len(combos))]
    srcs = []
    for (i, a) in combos[:pairs]:
        la, lb = clean_electrode(int(elec[i]) + 1, int(elec[i + a]) + 1)
        la, lb = la - 1, lb - 1
        mn = [(int(elec[i + a + a * lev]), int(elec[i + 2 * a + a * lev])) for lev in range(1, levels + 1)]
        al = np.stack([alphas_compact(n, m, DX, DZ, la, lb, ky) for ky in ky_w[:, 0]])
        srcs.append(DcSource(la, lb, current, np.asarray(mn, np.int64), ky_w, al))
    return srcs


def geometric_factor(ctx, shape: tuple[int, int], DX: float, DZ: float, robin: int, srcs, opts=None) -> list:
    """Geometric factors of a survey (dc_geomefactor2_5d.m:44-49): the data of a
    forward run on the Robin-padded grid with sigma = 1 everywhere, inverted,
    k = 1 / d.  `ctx` is a Context (its dc_forward runs the GPU solver);
    returns one array of nd factors per source."""
    fw = ctx.dc_forward(np.ones(shape), DX, DZ, robin, srcs, opts=opts)
    return [1.0 / np.asarray(d, np.float64) for d in fw["d"]]


def apparent_resistivity(d: list, k: list) -> list:
    """rho_a = k * d per datum (dc_geomefactor2_5d.m:36-43): the resistivity of
    the homogeneous half-space that would produce the measured data."""
    return [np.asarray(x, np.float64) * np.asarray(kk, np.float64) for x, kk in zip(d, k)]


def coca_radius(n: int, m: int, DX: float, DZ: float, a_node: int, b_node: int):
    """The distance pairs the wavenumber design fits (dc_coca.m:12-39,
    dc_kfourier.m:43-65) on a uniform grid: for every node the distances r, r_
    to the lower- and higher-index surface electrode (the lateral distance sums
    the spacings over the inclusive index range, as dc_coca.m:18-21 does; the
    depth of row h is h*DZ), unique pairs with both nonzero, then each of r and
    r_ resampled on its own to fix(N^0.7) evenly spaced values, and
    R = 1 / (1/r - 1/r_) where finite.  Returns (r, r_, R)."""
    nodes = sorted(int(x) for x in (a_node, b_node))
    if nodes[1] >= n:
        raise ValueError("the wavenumber design needs both source electrodes on the surface row")
    l = np.arange(n)
    co = [np.where(l == s, 0.0, (np.abs(s - l) + 1) * DX) for s in nodes]
    ca = np.arange(m) * DZ
    r = np.sqrt(co[0][:, None] ** 2 + ca[None, :] ** 2).ravel(order="F")
    r_ = np.sqrt(co[1][:, None] ** 2 + ca[None, :] ** 2).ravel(order="F")
    RR = np.unique(np.column_stack([r, r_]), axis=0)
    RR = RR[RR[:, 0] != 0]
    RR = RR[RR[:, 1] != 0]
    cnt = int(np.fix(10 ** (np.log10(len(RR)) * 0.7)))
    r = np.linspace(RR[:, 0].min(), RR[:, 0].max(), cnt)
    r_ = np.linspace(RR[:, 1].min(), RR[:, 1].max(), cnt)
    with np.errstate(divide="ignore"):
        R = 1.0 / (1.0 / r - 1.0 / r_)
    keep = ~np.isinf(R)
    if not keep.any():
        # electrodes placed symmetrically in the grid give r and r_ the same
        # range, so the two resampled lists coincide and every R is infinite;
        # the reference's design is then left without distances (NaN weights)
        raise ValueError("symmetric electrode placement: no distance pairs left for the wavenumber design")
    return r[keep], r_[keep], R[keep]


def _ridge_solve(A: np.ndarray, b: np.ndarray) -> np.ndarray:
    try:
        return np.linalg.solve(A, b)
    except np.linalg.LinAlgError:  # MATLAB's backslash warns and returns Inf/NaN
        return np.full(A.shape[1], np.nan)


def kfourier(n: int, m: int, DX: float, DZ: float, a_node: int, b_node: int, n_ky: int, dx: float,
             radius=None) -> np.ndarray:
    """Wavenumbers and weights of the 2.5D inverse transform for one source, as
    dc_kfourier.m:26-197 designs them.  K(ky) = (2/pi) R (K0(ky r) - K0(ky r_))
    (the real part of besselk, which for a negative argument is K0 of its
    magnitude); the fit v = K (K'K + 1e-8 I)^-1 K' 1 of the dipole kernel
    should be 1.  From ky = logspace(-2, 0.5, n_ky) * dx, Gauss-Newton steps
    (forward-difference Jacobian at 1.05 ky, ridge 1e-8, smallness 1e-8 ky)
    with a 20-point line search over [0.01, 0.9] run while every objective so
    far exceeds 1e-5, fewer than 25 iterations have run and each reduced the
    objective by more than 5 %; an ill-conditioned K'K (reciprocal 1-norm
    condition below 1e-15) or a NaN fit restores the previous ky and stops.
    Weights w = (K'K + 5e-8 I)^-1 K' 1 at |ky|.  Returns [ky*dx, w] (n_ky x 2),
    the reference's ky_w_.  `radius` = (r, r_, R) reuses the distances of an
    earlier source, as the reference does once finite_.dc.radius is set
    (dc_kfourier.m:43, 66-69).  The design fits resampled distance pairs, not
    the grid's own: on the grids tried, 12 wavenumbers gave half-space
    potentials within 1 % (median) of the analytic ones and 16 within 10 %."""
    r, r_, R = coca_radius(n, m, DX, DZ, a_node, b_node) if radius is None else radius
    beta_v, beta_g, beta_dky, beta_wky = 1e-8, 1e-8, 1e-8, 5e-8
    eye = np.eye(n_ky)
    one = np.ones(len(r))

    def kmat(ky):
        with np.errstate(invalid="ignore"):
            return (2 / np.pi) * R[:, None] * (ss.k0(np.abs(np.outer(r, ky))) - ss.k0(np.abs(np.outer(r_, ky))))

    def fit(K):
        return K @ _ridge_solve(K.T @ K + beta_v * eye, K.T @ one)

    ky = np.logspace(-2, 0.5, n_ky) * dx
    v = fit(kmat(ky))
    obj = [float((1 - v) @ (1 - v))]
    its, stopper, reduction = 1, False, 1.0
    ls = np.linspace(0.01, 0.9, 20)
    while all(o > 1e-5 for o in obj) and its < 25 and not stopper and reduction > 0.05:
        ky_prev = ky.copy()
        J = np.empty((len(r), n_ky))
        for ii in range(n_ky):
            k_ = ky.copy()
            k_[ii] = 1.05 * k_[ii]
            J[:, ii] = (fit(kmat(k_)) - v) / (k_[ii] - ky[ii])
        grad = J.T @ (1 - v) + beta_g * ky
        dky = _ridge_solve(J.T @ J + beta_dky * eye, grad)
        res = np.array([float((1 - f) @ (1 - f)) for f in (fit(kmat(ky + a * dky)) for a in ls)])
        jj = int(np.nanargmin(res)) if not np.isnan(res).all() else 0  # MATLAB min skips NaN
        ky = ky + ls[jj] * dky
        K = kmat(ky)
        v = fit(K)
        obj.append(float((1 - v) @ (1 - v)))
        reduction = obj[its - 1] / obj[its] - 1
        its += 1
        with np.errstate(divide="ignore"):
            rc = 1.0 / np.linalg.cond(K.T @ K, 1) if np.isfinite(K).all() else 0.0
        if rc < 1e-15 or np.isnan(v).any():
            ky = ky_prev
            stopper = True
    ky = np.abs(ky)
    K = kmat(ky)
    w = _ridge_solve(K.T @ K + beta_wky * eye, K.T @ one)
    return np.column_stack([ky * dx, w])


def redesign_sources(srcs, n: int, m: int, DX: float, DZ: float, n_ky: int, dx: float,
                     reuse_first_radius: bool = True) -> list:
    """The survey's sources with the reference's per-source wavenumbers and
    weights (dc_kfourier.m for each source, as ky_w(:,:,i_e) of dc_load2_5d.m:33
    holds them) and the matching Robin coefficients.  With reuse_first_radius
    every source after the first uses the first source's distances, as the
    reference does once finite_.dc.radius is set (dc_kfourier.m:43, 66-69)."""
    out, radius = [], None
    for q in srcs:
        if radius is None or not reuse_first_radius:
            radius = coca_radius(n, m, DX, DZ, q.a, q.b)
        kyw = kfourier(n, m, DX, DZ, q.a, q.b, n_ky, dx, radius=radius)
        al = np.stack([alphas_compact(n, m, DX, DZ, q.a, q.b, ky) for ky in kyw[:, 0]])
        out.append(dataclasses.replace(q, ky_w=kyw, alpha=al))
    return out


def binning(x, r) -> np.ndarray:
    """binning.m: for each value of r, the 1-based index of the nearest entry of
    the sorted grid x; on a tie the lower index (its forward scan stops at the
    first entry that is no nearer than the previous one)."""
    x = np.asarray(x, np.float64)
    r = np.atleast_1d(np.asarray(r, np.float64))
    return np.array([int(np.argmin(np.abs(x - v))) + 1 for v in r], np.int64)


def electrode_nodes(X, Z, electr_real, ab, mn, robin: int, n: int):
    """dc_electrodes.m:29-52: electrode numbers (1-based rows of the coordinate
    table electr_real, columns x and z) to grid nodes.  Coordinates are binned
    onto the model grid X (lateral) and Z (depth), shifted by the Robin columns,
    the source pair gets the parity clean (:66-75), and nodes are vectorised as
    l + n (h - 1) (:76-83) with n the padded lateral size.  Returns 0-based
    (a, b) and an (nd, 2) array of 0-based (M, N) nodes."""
    E = np.asarray(electr_real, np.float64).reshape(-1, 2)

    def nodes(nums):
        nums = np.asarray(nums, np.int64).reshape(-1)
        l = binning(X, E[nums - 1, 0]) + robin
        h = binning(Z, E[nums - 1, 1])
        return l, h

    l, h = nodes(ab)
    la, lb = clean_electrode(int(l[0]), int(l[1]))
    a = (la - 1) + n * (int(h[0]) - 1)
    b = (lb - 1) + n * (int(h[1]) - 1)
    mn = np.asarray(mn, np.int64).reshape(-1, 2)
    lm, hm = nodes(mn[:, 0])
    ln, hn = nodes(mn[:, 1])
    pairs = np.column_stack([(lm - 1) + n * (hm - 1), (ln - 1) + n * (hn - 1)])
    return a, b, pairs


def sources_from_survey(gathers, ky_w, X, Z, electr_real, robin: int, n: int, m: int, DX: float, DZ: float) -> list:
    """DcSource list of a field survey: the gathers of s_i_r_d_std.mat
    (matio.load_dc_survey), the per-source wavenumbers of ky_w.mat (n_ky x 2 x
    nsrc, one shared when nsrc = 1) and the electrode coordinate table, as
    dc_load2_5d.m:8-33 and dc_electrodes.m assemble them; observed data go to
    d_obs and the Robin coefficients are computed for each source."""
    kw = np.asarray(ky_w, np.float64)
    if kw.ndim == 2:
        kw = kw[:, :, None]
    out = []
    for ie, gth in enumerate(gathers):
        a, b, pairs = electrode_nodes(X, Z, electr_real, gth["ab"], gth["mn"], robin, n)
        k = kw[:, :, ie if kw.shape[2] > 1 else 0]
        al = np.stack([alphas_compact(n, m, DX, DZ, a, b, ky) for ky in k[:, 0]])
        out.append(DcSource(a, b, float(gth["current"]), pairs, k.copy(), al, np.asarray(gth["d"], np.float64)))
    return out
