"""ORACLE — TEST INFRASTRUCTURE ONLY (2.5D DC resistivity, FP64).

A numpy/scipy restatement of the reference's 2.5D finite-volume DC forward and
sensitivity solves.  Arrays follow the reference: (n x m) with n = nx the
lateral node count including the Robin columns (first index) and m = nz the
depth node count including the bottom Robin row; node (l, h) (1-based) is the
vectorised unknown i = l + (h-1)*n (coordP.m), i.e. numpy ravel(order="F").
Only tests/, the smoke check and the benchmark's CPU-baseline leg import this.

The sparse solves use scipy.sparse.linalg.spsolve (SuperLU) in FP64 in place
of MATLAB's `\\` (dc_fwd_k.m:43, dc_adjoint.m:10); Bessel K0/K1 come from
scipy.special in place of MATLAB's besselk (dc_Lk.m:949-950).
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla
import scipy.special as ss


def dc_robin(sigma, robin):
    """dc_robin.m:36-46: replicate the first/last lateral columns `robin` times
    on each side and the last depth row `robin` times below."""
    s = np.asarray(sigma, np.float64)
    s = np.vstack([np.repeat(s[:1, :], robin, 0), s, np.repeat(s[-1:, :], robin, 0)])
    s = np.hstack([s, np.repeat(s[:, -1:], robin, 1)])
    return s


def do_grid_spacing(X, Z, robin):
    """dc_robin.m:21-35 + do_grid.m:6-7: the constant spacings the reference
    stores in DELTAS.  x_robin = [(1:robin)*dx1, X, (1:robin)*dx2] and
    dx = x_robin(2) - x_robin(1), which for robin = 1 is X(1) - dx1 (negative
    when X starts at 0); dz = z_robin(2) - z_robin(1)."""
    X = np.asarray(X, np.float64)
    Z = np.asarray(Z, np.float64)
    dx1 = X[1] - X[0]
    dx2 = X[-1] - X[-2]
    dz2 = Z[-1] - Z[-2]
    xr = np.concatenate([np.arange(1, robin + 1) * dx1, X, np.arange(1, robin + 1) * dx2])
    zr = np.concatenate([Z, np.arange(1, robin + 1) * dz2])
    return xr[1] - xr[0], zr[1] - zr[0]


def alphas(n, m, DX, DZ, s_surface, ky):
    """dc_Lk.m:820-960 (private `alphas`): Robin coefficients
    alpha = sum_e beta_e ky K1(ky r) cos / sum_e beta_e K0(ky r) for the left
    side (h = 2..m-1), the bottom (l = 2..n-1), the right side and the corners.
    Returns (ALPHAS (n x m), corners (2 x 2))."""
    beta = np.sign(np.asarray(s_surface, np.float64))
    co_left = np.outer(np.arange(1, m) * DZ, np.ones(n))               # (m-1, n)
    idx = np.arange(n)
    co_down = np.abs(idx[:, None] - idx[None, :]) * DX                  # (n, n), DX may be negative
    co_right = co_left[::-1, ::-1]
    co = np.vstack([co_left, co_down, co_right])
    ca_left = np.outer(np.ones(m - 1), np.arange(n) * DX)
    ca_down = (m - 1) * DZ * np.ones((n, n))
    ca_right = ca_left[::-1, ::-1]
    ca = np.vstack([ca_left, ca_down, ca_right])
    r = np.sqrt(co ** 2 + ca ** 2)
    # K0/K1 exponentially scaled relative to the nearest electrode of each row:
    # identical to besselk where it does not underflow, and its limit where
    # the reference's besselk would give 0/0.
    x = ky * r
    on = beta != 0
    x0 = np.min(np.where(on[None, :], x, np.inf), axis=1, keepdims=True)
    sc = np.where(on[None, :], np.exp(-np.where(on[None, :], x - x0, 0.0)), 0.0)
    numer = (ky * ss.k1e(x) * sc * (ca / r)) @ beta
    denom = (ss.k0e(x) * sc) @ beta
    a = numer / denom
    AL = np.zeros((n, m))
    AL[0, 1:m - 1] = a[0:m - 2]
    AL[1:n - 1, m - 1] = a[m:m + n - 2]
    AL[n - 1, 1:m - 1] = a[m + n:][::-1]
    corners = np.array([[a[m - 2], a[m + n - 2]], [a[m - 1], a[m + n - 1]]])
    return AL, corners


def _H(a, b):
    return 2.0 * a * b / (a + b)


def dc_Lk(SIG, DX, DZ, ALPHAS, corners, ky):
    """dc_Lk.m:35-817: Lk = -L + ky^2 diag(sigma) as a scipy CSR matrix.
    L has harmonic-mean face conductances (offdiag MM1..MM4), a Neumann top
    (h = 1), Robin ghost terms MM5 on the sides, bottom and bottom corners,
    and diagonal MM6 = -(MM1+...+MM5)."""
    n, m = SIG.shape
    N = n * m
    idx = lambda l, h: l + h * n  # 0-based
    rows, cols, vals = [], [], []
    diag = np.zeros((n, m))
    # lateral faces (l, h)-(l+1, h): MM = -H * DZ/DX
    cx = -_H(SIG[:-1, :], SIG[1:, :]) * (DZ / DX)  # (n-1, m)
    # depth faces (l, h)-(l, h+1): MM = -H * DX/DZ
    cz = -_H(SIG[:, :-1], SIG[:, 1:]) * (DX / DZ)  # (n, m-1)
    L, Hh = np.meshgrid(np.arange(n - 1), np.arange(m), indexing="ij")
    for a_, b_ in ((0, 1), (1, 0)):
        ii = idx(L + a_, Hh).ravel()
        jj = idx(L + b_, Hh).ravel()
        rows.append(ii); cols.append(jj); vals.append(cx.ravel())
    L, Hh = np.meshgrid(np.arange(n), np.arange(m - 1), indexing="ij")
    for a_, b_ in ((0, 1), (1, 0)):
        ii = idx(L, Hh + a_).ravel()
        jj = idx(L, Hh + b_).ravel()
        rows.append(ii); cols.append(jj); vals.append(cz.ravel())
    diag[:-1, :] += cx
    diag[1:, :] += cx
    diag[:, :-1] += cz
    diag[:, 1:] += cz
    # Robin ghosts MM5
    mm5 = np.zeros((n, m))
    mm5[0, 1:m - 1] = -SIG[0, 1:m - 1] * DZ * ALPHAS[0, 1:m - 1]
    mm5[n - 1, 1:m - 1] = -SIG[n - 1, 1:m - 1] * DZ * ALPHAS[n - 1, 1:m - 1]
    mm5[1:n - 1, m - 1] = -SIG[1:n - 1, m - 1] * DX * ALPHAS[1:n - 1, m - 1]
    mm5[0, m - 1] = -SIG[0, m - 1] * DZ * corners[0, 0] - SIG[0, m - 1] * DX * corners[1, 0]
    mm5[n - 1, m - 1] = -SIG[n - 1, m - 1] * DZ * corners[0, 1] - SIG[n - 1, m - 1] * DX * corners[1, 1]
    diag += mm5
    # L(i,j) = MM_dir (offdiag), L(i,i) = MM6 = -(sum MM); Lk = -L + ky^2 diag(sigma)
    r = np.concatenate(rows)
    c = np.concatenate(cols)
    v = -np.concatenate(vals)
    dvals = diag.ravel(order="F") + ky ** 2 * SIG.ravel(order="F")
    Lk = sp.coo_matrix((np.concatenate([v, dvals]), (np.concatenate([r, np.arange(N)]),
                                                        np.concatenate([c, np.arange(N)]))), shape=(N, N))
    return Lk.tocsr()


def dc_Sk_apply(SIG, DX, DZ, ALPHAS, corners, U, A, ky):
    """dc_Sk.m: g = Sdc * a with Sdc = -S - ky^2 diag(U), where S has
    offdiag SIJ = (face/spacing) (U_i - U_j) 2 (sigma_j/(sigma_i+sigma_j))^2 and
    diag SII = -sum SIJ - SR, SR = face * alpha * U on the Robin nodes.
    Equivalently g_i = sum_j SIJ_ij (a_i - a_j) + SR_i a_i - ky^2 U_i a_i."""
    n, m = SIG.shape
    g = np.zeros((n, m))
    # lateral faces: ratio DZ/DX; derivative wrt sigma of node i of H(si, sj)
    r = DZ / DX
    si, sj = SIG[:-1, :], SIG[1:, :]
    du, da = U[:-1, :] - U[1:, :], A[:-1, :] - A[1:, :]
    g[:-1, :] += r * 2 * (sj / (si + sj)) ** 2 * du * da
    g[1:, :] += r * 2 * (si / (si + sj)) ** 2 * du * da
    r = DX / DZ
    si, sj = SIG[:, :-1], SIG[:, 1:]
    du, da = U[:, :-1] - U[:, 1:], A[:, :-1] - A[:, 1:]
    g[:, :-1] += r * 2 * (sj / (si + sj)) ** 2 * du * da
    g[:, 1:] += r * 2 * (si / (si + sj)) ** 2 * du * da
    SR = np.zeros((n, m))
    SR[0, 1:m - 1] = DZ * ALPHAS[0, 1:m - 1] * U[0, 1:m - 1]
    SR[n - 1, 1:m - 1] = DZ * ALPHAS[n - 1, 1:m - 1] * U[n - 1, 1:m - 1]
    SR[1:n - 1, m - 1] = DX * ALPHAS[1:n - 1, m - 1] * U[1:n - 1, m - 1]
    SR[0, m - 1] = DZ * corners[0, 0] * U[0, m - 1] + DX * corners[1, 0] * U[0, m - 1]
    SR[n - 1, m - 1] = DZ * corners[0, 1] * U[n - 1, m - 1] + DX * corners[1, 1] * U[n - 1, m - 1]
    g += SR * A
    g -= ky ** 2 * U * A
    return g


def source_vector(n, m, a_node, b_node, current=1.0):
    """dc_electrodes.m:54-55: +I at node A, -I at node B (0-based vectorised)."""
    s = np.zeros(n * m)
    s[a_node] += current
    s[b_node] -= current
    return s


def measuring_operator(n, m, mn_pairs):
    """dc_M.m:45-53: one row per datum, +1 at M and -1 at N (0-based nodes)."""
    mn_pairs = np.asarray(mn_pairs, np.int64).reshape(-1, 2)
    nd = len(mn_pairs)
    rows = np.repeat(np.arange(nd), 2)
    cols = mn_pairs.ravel()
    vals = np.tile([1.0, -1.0], nd)
    return sp.csr_matrix((vals, (rows, cols)), shape=(nd, n * m))


def dc_fwd2_5d(SIG, DX, DZ, src, alphas_k, ky_w, Mop, d_obs=None):
    """dc_fwd2_5d.m:44-57 / dc_fwd_k.m:35-43 for one source: u_k = Lk \\ (0.5 s),
    u = (2/pi) sum_k w_k u_k, d = M u, e = d - d_o.
    alphas_k: list of (ALPHAS, corners) per ky; ky_w: (n_ky, 2)."""
    n, m = SIG.shape
    uk = np.zeros((n * m, len(ky_w)))
    for k, (ky, _) in enumerate(ky_w):
        AL, co = alphas_k[k]
        Lk = dc_Lk(SIG, DX, DZ, AL, co, ky)
        uk[:, k] = spla.spsolve(Lk.tocsc(), 0.5 * src)
    u = (2 / np.pi) * uk @ np.asarray(ky_w)[:, 1]
    d = Mop @ u
    e = d - d_obs if d_obs is not None else None
    return u, uk, d, e


def dc_gradient2_5d(SIG, DX, DZ, alphas_k, ky_w, Mop, uk, e, robin):
    """dc_gradient2_5d.m:18-41 for one source: a_k = Lk' \\ (M' e),
    g_k = Sk(u_k) a_k, g = (2/pi) sum_k w_k g_k, trimmed of the Robin padding."""
    n, m = SIG.shape
    g = np.zeros((n, m))
    rhs = Mop.T @ e
    for k, (ky, w) in enumerate(ky_w):
        AL, co = alphas_k[k]
        Lk = dc_Lk(SIG, DX, DZ, AL, co, ky)
        ak = spla.spsolve(Lk.T.tocsc(), rhs)
        gk = dc_Sk_apply(SIG, DX, DZ, AL, co, uk[:, k].reshape((n, m), order="F"),
                         ak.reshape((n, m), order="F"), ky)
        g += (2 / np.pi) * w * gk
    return g[robin:n - robin, 0:m - robin]


def analytic_halfspace(n, m, DXabs, DZ, sigma, a_l, b_l, current=1.0):
    """dc_analhomo2_5d.m:20-25: surface dipole potential in a homogeneous
    half-space, I/(2 pi sigma) (1/r_A - 1/r_B), at every node (lateral index l,
    depth index h, 0-based), spacings taken positive.  Distances are the
    physical ones, |l - l_A| dx; dc_coca.m's sum over the inclusive index range
    would add one spacing."""
    l = np.arange(n)[:, None]
    h = np.arange(m)[None, :]
    rA = np.sqrt(((l - a_l) * DXabs) ** 2 + (h * DZ) ** 2)
    rB = np.sqrt(((l - b_l) * DXabs) ** 2 + (h * DZ) ** 2)
    with np.errstate(divide="ignore"):
        return current / (2 * np.pi * sigma) * (1 / rA - 1 / rB)


def analytic_two_layer(n, DXabs, sigma1, sigma2, depth, a_l, b_l, current=1.0, terms=200):
    """dc_analbi2_5d.m:23-44 on the surface row: the image series of a surface
    dipole over a layer of conductivity sigma1 and thickness `depth` on a
    half-space of sigma2, I/(2 pi sigma1) (a(r_A) - a(r_B)) with
    a(r) = 1/r + sum_i 2 k^i / sqrt(r^2 + (2 i depth)^2), k = (sigma1 - sigma2) /
    (sigma1 + sigma2); physical lateral distances (see analytic_halfspace)."""
    l = np.arange(n)
    k = (sigma1 - sigma2) / (sigma1 + sigma2)

    def a(r):
        with np.errstate(divide="ignore"):
            return 1.0 / r + sum(2.0 * k ** i / np.sqrt(r ** 2 + (2.0 * i * depth) ** 2) for i in range(1, terms + 1))
    return current / (2 * np.pi * sigma1) * (a(np.abs(l - a_l) * DXabs) - a(np.abs(l - b_l) * DXabs))
