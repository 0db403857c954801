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
  kernel, standing in for dc_kfourier.m's Gauss-Newton design).
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
