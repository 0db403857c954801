"""ORACLE — TEST INFRASTRUCTURE ONLY (numpy twin of oracle/gj_oracle.hpp).

A second CPU restatement of the reference's radar path, written to follow the
MATLAB source slice by slice: the eight split-field PML strip arrays of
w_solve.m, the strip coefficient blocks of w_cpml.m, and the same loop order.
The C++ oracle uses a per-node formulation instead, so agreement between the
two pins that reformulation.  Only tests/, the smoke check and the benchmark's
CPU-baseline leg may import this module; the product path never does.

Indexing helper: ``S(a, b)`` is the MATLAB range ``a:b`` (1-based, inclusive).
Structs are plain dicts mirroring geome_/parame_/finite_/gerjoii_.
"""
from __future__ import annotations

import numpy as np


def S(a, b):
    """MATLAB a:b (1-based inclusive) as a Python slice."""
    return slice(int(a) - 1, int(b))


# ---------------------------------------------------------------- geometry
def w_layout(m, n, pml, air, pml_top=None):
    """Index quantities of wdc_geom.m:69-110 (1-based, as in MATLAB).

    ``pml_top`` generalises the reference (which always pads pml_w rows on top)
    to a free top (pml_top = 0)."""
    if pml_top is None:
        pml_top = pml
    nx = pml_top + air + m + pml
    ny = n + 2 * pml
    pis = pml_top + 1
    pie = nx - pml + 1
    pjs = pml + 1
    pje = ny - pml + 1
    domain_i = np.arange(pis + air, pie)  # pis+air : pie-1
    domain_j = np.arange(pjs, pje)        # pjs : pje-1
    return dict(nx=nx, ny=ny, pis=pis, pie=pie, pjs=pjs, pje=pje, pml_w=pml, pml_d=pml,
                pml_top=pml_top, air=air, domain_i=domain_i, domain_j=domain_j)


def w_exp2pml(epsilon, sigma, pml, air, pml_top=None, dtype=np.float64):
    """w_exp2pml.m:19-34: air rows on top, edge-replicated eps_r in the PML,
    zero sigma outside the model."""
    if pml_top is None:
        pml_top = pml
    m, n = epsilon.shape
    eps_r_z = np.vstack([np.ones((air, n)), epsilon]).astype(np.float64)
    sigma_e_z = np.vstack([np.zeros((air, n)), sigma]).astype(np.float64)
    left = np.repeat(eps_r_z[:, :1], pml, axis=1)
    right = np.repeat(eps_r_z[:, -1:], pml, axis=1)
    eps_r_z = np.hstack([left, eps_r_z, right])
    sigma_e_z = np.hstack([np.zeros((air + m, pml)), sigma_e_z, np.zeros((air + m, pml))])
    up = np.repeat(eps_r_z[:1, :], pml_top, axis=0)
    down = np.repeat(eps_r_z[-1:, :], pml, axis=0)
    eps_r_z = np.vstack([up, eps_r_z, down])
    sigma_e_z = np.vstack([np.zeros((pml_top, n + 2 * pml)), sigma_e_z, np.zeros((pml, n + 2 * pml))])
    return eps_r_z.astype(dtype), sigma_e_z.astype(dtype)


def w_cpml(eps_r_z, fin, dx, dy, dt, eps_0, mu_0, pml_order=2, R_0=1e-8):
    """w_cpml.m:11-185, strip by strip (xn = top, xp = bottom, yn = left, yp = right)."""
    nx, ny, pis, pie, pjs, pje = (fin[k] for k in ("nx", "ny", "pis", "pie", "pjs", "pje"))
    pml_w, pml_d, pml_top = fin["pml_w"], fin["pml_d"], fin["pml_top"]
    c = 1.0 / np.sqrt(mu_0 * eps_0)
    nym1 = ny - 1
    nxm1 = nx - 1
    cp = {}
    # ---- left side in the reference's words: the top (xn) strip, pml_top rows
    if pml_top > 0:
        smax = -(pml_order + 1) * eps_0 * c * np.log(R_0) / (2 * dx * pml_top)
        rho_e = (np.arange(pml_top, 0, -1) - 0.75) / pml_top
        rho_m = (np.arange(pml_top, 0, -1) - 0.25) / pml_top
        spex = np.repeat((smax * rho_e ** pml_order)[:, None], nym1, axis=1)
        spmx = np.repeat(((mu_0 / eps_0) * smax * rho_m ** pml_order)[:, None], nym1, axis=1)
        cp["Chyh_xn"] = (2 * mu_0 - dt * spmx) / (2 * mu_0 + dt * spmx)
        cp["Chyez_xn"] = (2 * dt / dx) / (2 * mu_0 + dt * spmx)
        cp["Cezxe_xn"] = (2 * eps_0 - dt * spex) / (2 * eps_0 + dt * spex)
        cp["Cezxhy_xn"] = (2 * dt / dx) / (2 * eps_0 + dt * spex)
        cp["Cezye_xn"] = 1.0
        cp["Cezyhx_xn"] = -dt / (dy * eps_0)
    # ---- bottom (xp)
    smax = -(pml_order + 1) * eps_0 * c * np.log(R_0) / (2 * dx * pml_w)
    rho_e = (np.arange(1, pml_w + 1) - 0.75) / pml_w
    rho_m = (np.arange(1, pml_w + 1) - 0.25) / pml_w
    spex = np.repeat((smax * rho_e ** pml_order)[:, None], nym1, axis=1)
    spmx = np.repeat(((mu_0 / eps_0) * smax * rho_m ** pml_order)[:, None], nym1, axis=1)
    spmx = spmx / eps_r_z[S(pie, nx), S(2, ny)]
    cp["Chyh_xp"] = (2 * mu_0 - dt * spmx) / (2 * mu_0 + dt * spmx)
    cp["Chyez_xp"] = (2 * dt / dx) / (2 * mu_0 + dt * spmx)
    e = eps_r_z[S(pie, nx), S(2, ny)]
    cp["Cezxe_xp"] = (2 * eps_0 * e - dt * spex) / (2 * eps_0 * e + dt * spex)
    cp["Cezxhy_xp"] = (2 * dt / dx) / (2 * eps_0 * e + dt * spex)
    cp["Cezye_xp"] = 1.0
    cp["Cezyhx_xp"] = -dt / (dy * eps_0 * eps_r_z[S(pie, nx), S(pjs + 1, pje - 1)])
    # ---- left (yn)
    smax = -(pml_order + 1) * eps_0 * c * np.log(R_0) / (2 * dy * pml_d)
    rho_e = (np.arange(pml_d, 0, -1) - 0.75) / pml_d
    rho_m = (np.arange(pml_d, 0, -1) - 0.25) / pml_d
    spey = np.repeat((smax * rho_e ** pml_order)[None, :], nxm1, axis=0)
    spmy = np.repeat(((mu_0 / eps_0) * smax * rho_m ** pml_order)[None, :], nxm1, axis=0)
    spmy = spmy / eps_r_z[S(2, nx), S(1, pjs - 1)]
    cp["Chxh_yn"] = (2 * mu_0 - dt * spmy) / (2 * mu_0 + dt * spmy)
    cp["Chxez_yn"] = -(2 * dt / dy) / (2 * mu_0 + dt * spmy)
    cp["Cezxe_yn"] = 1.0
    cp["Cezxhy_yn"] = dt / (dx * eps_0 * eps_r_z[S(pis + 1, pie - 1), S(2, pjs)])
    e = eps_r_z[S(2, nx), S(2, pjs)]
    cp["Cezye_yn"] = (2 * eps_0 * e - dt * spey) / (2 * eps_0 * e + dt * spey)
    cp["Cezyhx_yn"] = -(2 * dt / dy) / (2 * eps_0 * e + dt * spey)
    # ---- right (yp)
    rho_e = (np.arange(1, pml_d + 1) - 0.75) / pml_d
    rho_m = (np.arange(1, pml_d + 1) - 0.25) / pml_d
    spey = np.repeat((smax * rho_e ** pml_order)[None, :], nxm1, axis=0)
    spmy = np.repeat(((mu_0 / eps_0) * smax * rho_m ** pml_order)[None, :], nxm1, axis=0)
    spmy = spmy / eps_r_z[S(2, nx), S(pje, ny)]
    cp["Chxh_yp"] = (2 * mu_0 - dt * spmy) / (2 * mu_0 + dt * spmy)
    cp["Chxez_yp"] = -(2 * dt / dy) / (2 * mu_0 + dt * spmy)
    cp["Cezxe_yp"] = 1.0
    cp["Cezxhy_yp"] = dt / (dx * eps_0 * eps_r_z[S(pis + 1, pie - 1), S(pje, ny)])
    e = eps_r_z[S(2, nx), S(pje, ny)]
    cp["Cezye_yp"] = (2 * eps_0 * e - dt * spey) / (2 * eps_0 * e + dt * spey)
    cp["Cezyhx_yp"] = -(2 * dt / dy) / (2 * eps_0 * e + dt * spey)
    return cp


def w_coeff(eps_r_z, sigma_e_z, s_w, dx, dy, dt, eps_0, mu_0):
    """w_coeff.m:28-45 with mu_r = 1, sigma_m = 0 (w_magmat.m:10-13)."""
    co = {}
    D = 2 * eps_r_z * eps_0 + dt * sigma_e_z
    co["Ceze"] = (2 * eps_r_z * eps_0 - dt * sigma_e_z) / D
    co["Cezhy"] = (2 * dt / dx) / D
    co["Cezhx"] = -(2 * dt / dy) / D
    co["Chxh"] = 1.0
    co["Chxez"] = -(2 * dt / dy) / (2 * mu_0)
    co["Chyh"] = 1.0
    co["Chyez"] = (2 * dt / dx) / (2 * mu_0)
    i, j = s_w
    co["Cezj"] = -(2 * dt) / (2 * eps_r_z[i - 1, j - 1] * eps_0 + dt * sigma_e_z[i - 1, j - 1])
    return co


def _new_H(Hx, Hy, Ez, co, f):
    """w_solve.m:136-148."""
    pis, pie, pjs, pje = f["pis"], f["pie"], f["pjs"], f["pje"]
    Hx[:, S(pjs, pje - 1)] = co["Chxh"] * Hx[:, S(pjs, pje - 1)] + co["Chxez"] * (
        Ez[:, S(pjs + 1, pje)] - Ez[:, S(pjs, pje - 1)])
    Hy[S(pis, pie - 1), :] = co["Chyh"] * Hy[S(pis, pie - 1), :] + co["Chyez"] * (
        Ez[S(pis + 1, pie), :] - Ez[S(pis, pie - 1), :])


def _new_H_pml(Hx, Hy, Ez, cp, f):
    """w_solve.m:154-187."""
    pis, pie, pjs, pje, nx, ny = (f[k] for k in ("pis", "pie", "pjs", "pje", "nx", "ny"))
    nxp1, nyp1 = nx + 1, ny + 1
    if pis > 1:
        Hy[S(1, pis - 1), S(2, ny)] = cp["Chyh_xn"] * Hy[S(1, pis - 1), S(2, ny)] + cp["Chyez_xn"] * (
            Ez[S(2, pis), S(2, ny)] - Ez[S(1, pis - 1), S(2, ny)])
    Hy[S(pie, nx), S(2, ny)] = cp["Chyh_xp"] * Hy[S(pie, nx), S(2, ny)] + cp["Chyez_xp"] * (
        Ez[S(pie + 1, nxp1), S(2, ny)] - Ez[S(pie, nx), S(2, ny)])
    Hx[S(2, nx), S(1, pjs - 1)] = cp["Chxh_yn"] * Hx[S(2, nx), S(1, pjs - 1)] + cp["Chxez_yn"] * (
        Ez[S(2, nx), S(2, pjs)] - Ez[S(2, nx), S(1, pjs - 1)])
    Hx[S(2, nx), S(pje, ny)] = cp["Chxh_yp"] * Hx[S(2, nx), S(pje, ny)] + cp["Chxez_yp"] * (
        Ez[S(2, nx), S(pje + 1, nyp1)] - Ez[S(2, nx), S(pje, ny)])


def _new_Ez(Hx, Hy, Ez, co, f):
    """w_solve.m:193-207."""
    pis, pie, pjs, pje = f["pis"], f["pie"], f["pjs"], f["pje"]
    I, J = S(pis + 1, pie - 1), S(pjs + 1, pje - 1)
    Ez[I, J] = (co["Ceze"][I, J] * Ez[I, J]
                + co["Cezhy"][I, J] * (Hy[I, J] - Hy[S(pis, pie - 2), J])
                + co["Cezhx"][I, J] * (Hx[I, J] - Hx[I, S(pjs, pje - 2)]))


def _new_Ez_pml(Hx, Hy, Ez, cp, E, f):
    """w_solve.m:215-268; E holds the eight split strips."""
    pis, pie, pjs, pje, nx, ny = (f[k] for k in ("pis", "pie", "pjs", "pje", "nx", "ny"))
    nxm1, nym1 = nx - 1, ny - 1
    if pis > 1:
        E["Ezx_xn"] = cp["Cezxe_xn"] * E["Ezx_xn"] + cp["Cezxhy_xn"] * (
            Hy[S(2, pis), S(2, ny)] - Hy[S(1, pis - 1), S(2, ny)])
        E["Ezy_xn"] = cp["Cezye_xn"] * E["Ezy_xn"] + cp["Cezyhx_xn"] * (
            Hx[S(2, pis), S(pjs + 1, pje - 1)] - Hx[S(2, pis), S(pjs, pje - 2)])
    E["Ezx_xp"] = cp["Cezxe_xp"] * E["Ezx_xp"] + cp["Cezxhy_xp"] * (
        Hy[S(pie, nx), S(2, ny)] - Hy[S(pie - 1, nx - 1), S(2, ny)])
    E["Ezy_xp"] = cp["Cezye_xp"] * E["Ezy_xp"] + cp["Cezyhx_xp"] * (
        Hx[S(pie, nx), S(pjs + 1, pje - 1)] - Hx[S(pie, nx), S(pjs, pje - 2)])
    E["Ezx_yn"] = cp["Cezxe_yn"] * E["Ezx_yn"] + cp["Cezxhy_yn"] * (
        Hy[S(pis + 1, pie - 1), S(2, pjs)] - Hy[S(pis, pie - 2), S(2, pjs)])
    E["Ezy_yn"] = cp["Cezye_yn"] * E["Ezy_yn"] + cp["Cezyhx_yn"] * (
        Hx[S(2, nx), S(2, pjs)] - Hx[S(2, nx), S(1, pjs - 1)])
    E["Ezx_yp"] = cp["Cezxe_yp"] * E["Ezx_yp"] + cp["Cezxhy_yp"] * (
        Hy[S(pis + 1, pie - 1), S(pje, ny)] - Hy[S(pis, pie - 2), S(pje, ny)])
    E["Ezy_yp"] = cp["Cezye_yp"] * E["Ezy_yp"] + cp["Cezyhx_yp"] * (
        Hx[S(2, nx), S(pje, ny)] - Hx[S(2, nx), S(pje - 1, ny - 1)])
    if pis > 1:
        Ez[S(2, pis), S(2, pjs)] = E["Ezx_xn"][:, S(1, pjs - 1)] + E["Ezy_yn"][S(1, pis - 1), :]
        Ez[S(2, pis), S(pje, ny)] = E["Ezx_xn"][:, S(pje - 1, nym1)] + E["Ezy_yp"][S(1, pis - 1), :]
        Ez[S(2, pis), S(pjs + 1, pje - 1)] = E["Ezx_xn"][:, S(pjs, pje - 2)] + E["Ezy_xn"]
    Ez[S(pie, nx), S(pje, ny)] = E["Ezx_xp"][:, S(pje - 1, nym1)] + E["Ezy_yp"][S(pie - 1, nxm1), :]
    Ez[S(pie, nx), S(2, pjs)] = E["Ezx_xp"][:, S(1, pjs - 1)] + E["Ezy_yn"][S(pie - 1, nxm1), :]
    Ez[S(pis + 1, pie - 1), S(2, pjs)] = E["Ezx_yn"] + E["Ezy_yn"][S(pis, pie - 2), :]
    Ez[S(pis + 1, pie - 1), S(pje, ny)] = E["Ezx_yp"] + E["Ezy_yp"][S(pis, pie - 2), :]
    Ez[S(pie, nx), S(pjs + 1, pje - 1)] = E["Ezx_xp"][:, S(pjs, pje - 2)] + E["Ezy_xp"]


def _init_fields(f, dtype):
    nx, ny, pml_w, pml_d, pt = f["nx"], f["ny"], f["pml_w"], f["pml_d"], f["pml_top"]
    nxm1, nym1 = nx - 1, ny - 1
    E = {
        "Ezx_xn": np.zeros((pt, nym1), dtype), "Ezy_xn": np.zeros((pt, nym1 - 2 * pml_d), dtype),
        "Ezx_xp": np.zeros((pml_w, nym1), dtype), "Ezy_xp": np.zeros((pml_w, nym1 - 2 * pml_d), dtype),
        "Ezx_yn": np.zeros((nxm1 - pt - pml_w, pml_d), dtype), "Ezy_yn": np.zeros((nxm1, pml_d), dtype),
        "Ezx_yp": np.zeros((nxm1 - pt - pml_w, pml_d), dtype), "Ezy_yp": np.zeros((nxm1, pml_d), dtype),
    }
    Hx = np.zeros((nx + 1, ny), dtype)
    Hy = np.zeros((nx, ny + 1), dtype)
    Ez = np.zeros((nx + 1, ny + 1), dtype)
    return Hx, Hy, Ez, E


def _cast(d, dtype):
    return {k: (np.asarray(v, dtype=dtype) if np.ndim(v) else dtype(v)) for k, v in d.items()}


def w_solve(eps_r_z, sigma_e_z, f, s_w, r_lin, wvlet, nt, dx, dy, dt, eps_0, mu_0,
            store_u=True, dtype=np.float64):
    """w_solve.m:80-105.  s_w = (i, j) 1-based source node; r_lin = 1-based
    linear Ez indices (w_M.m:20).  Returns d (nt x nr), u (m x n x nt), Jz."""
    cp = _cast(w_cpml(eps_r_z, f, dx, dy, dt, eps_0, mu_0), dtype)
    co = _cast(w_coeff(eps_r_z, sigma_e_z, s_w, dx, dy, dt, eps_0, mu_0), dtype)
    Hx, Hy, Ez, E = _init_fields(f, dtype)
    nr = len(r_lin)
    d = np.zeros((nt, nr), dtype)
    di, dj = f["domain_i"] - 1, f["domain_j"] - 1
    u = np.zeros((len(di), len(dj), nt), dtype) if store_u else None
    Jz = np.zeros(nt, dtype)
    rr = np.asarray(r_lin) - 1
    ri, rj = rr % (f["nx"] + 1), rr // (f["nx"] + 1)
    si, sj = s_w[0] - 1, s_w[1] - 1
    for it in range(nt):
        _new_H(Hx, Hy, Ez, co, f)
        _new_H_pml(Hx, Hy, Ez, cp, f)
        _new_Ez(Hx, Hy, Ez, co, f)
        Ez[si, sj] = Ez[si, sj] + co["Cezj"] * dtype(wvlet[it])
        _new_Ez_pml(Hx, Hy, Ez, cp, E, f)
        d[it, :] = Ez[ri, rj]
        if store_u:
            u[:, :, it] = Ez[np.ix_(di, dj)]
        Jz[it] = Ez[si, sj]
    return d, u, Jz


def w_grad(u, e, eps_r_z, sigma_e_z, f, s_w, r_lin, nt, dx, dy, dt, eps_0, mu_0, dtype=np.float64):
    """w_grad.m:24-112 (reference adjoint).  Returns (g, a_max)."""
    cp = _cast(w_cpml(eps_r_z, f, dx, dy, dt, eps_0, mu_0), dtype)
    co = _cast(w_coeff(eps_r_z, -sigma_e_z, s_w, dx, dy, dt, eps_0, mu_0), dtype)
    Hx, Hy, Ez, E = _init_fields(f, dtype)
    di, dj = f["domain_i"] - 1, f["domain_j"] - 1
    g = np.zeros((len(di), len(dj)), dtype)
    rr = np.asarray(r_lin) - 1
    ri, rj = rr % (f["nx"] + 1), rr // (f["nx"] + 1)
    a = None
    for it in range(nt):
        Ez[ri, rj] = e[nt - it - 1, :]
        _new_H(Hx, Hy, Ez, co, f)
        _new_H_pml(Hx, Hy, Ez, cp, f)
        _new_Ez(Hx, Hy, Ez, co, f)
        _new_Ez_pml(Hx, Hy, Ez, cp, E, f)
        a = Ez[np.ix_(di, dj)]
        g = g - u[:, :, nt - it - 1] * a
    g = dtype(dt) * g
    return g, np.abs(a)


def differentiate_cube(v, dt):
    """differentiate_cube.m:23-51 (second-order, one-sided ends), along axis 2."""
    v = np.asarray(v, dtype=np.float64)
    out = np.empty_like(v)
    out[:, :, 0] = (-1.5 * v[:, :, 0] + 2.0 * v[:, :, 1] - 0.5 * v[:, :, 2]) / dt
    out[:, :, 1:-1] = (v[:, :, 2:] - v[:, :, :-2]) * (0.5 / dt)
    out[:, :, -1] = (0.5 * v[:, :, -3] - 2.0 * v[:, :, -2] + 1.5 * v[:, :, -1]) / dt
    return out


def hilbert(x, axis=0):
    """Analytic signal along ``axis`` with MATLAB's hilbert definition."""
    x = np.asarray(x, dtype=np.float64)
    n = x.shape[axis]
    X = np.fft.fft(x, axis=axis)
    h = np.zeros(n)
    if n % 2 == 0:
        h[0] = h[n // 2] = 1
        h[1:n // 2] = 2
    else:
        h[0] = 1
        h[1:(n + 1) // 2] = 2
    shape = [1] * x.ndim
    shape[axis] = n
    return np.fft.ifft(X * h.reshape(shape), axis=axis)


def instant_(u):
    """instant_.m:14-20: envelope, phase, Hilbert transform (column-wise)."""
    ua = hilbert(u, axis=0)
    return np.abs(ua), np.angle(ua), np.imag(ua)


def w_bozdag(d_o, d, obj_fnc="L2"):
    """w_bozdag.m:13-54: adjoint source for each objective (L2, env_L2,
    phase_L2, env_L22, env_LOG). Returns (e, d_e, d_oe), the quantities whose
    misfit w_E measures (w_fwd.m:34-35 stores d_e and d_oe in place of d and
    d_o).  With hilbert's imaginary part H (an antisymmetric circulant):
    env_L2 and env_LOG are the gradients of their misfits with respect to d,
    env_L22 is half of it; phase_L2 is -g + H(g d), g = (phi - phi_o) / E^2, as
    the reference writes it (w_bozdag.m:32-34)."""
    if obj_fnc == "L2":
        return d - d_o, d, d_o
    with np.errstate(divide="ignore", invalid="ignore"):
        if obj_fnc == "env_L2":
            d_e, _, d_H = instant_(d)
            d_oe, _, _ = instant_(d_o)
            dedoe = (d_e - d_oe) / d_e
            e_ = d * dedoe - np.imag(hilbert(dedoe * d_H, axis=0))
            e_[np.isnan(e_)] = 0
            return e_, d_e, d_oe
        if obj_fnc == "phase_L2":
            d_e, d_p, _ = instant_(d)
            _, d_op, _ = instant_(d_o)
            g = (d_p - d_op) / d_e ** 2
            e_ = -g + np.imag(hilbert(g * d, axis=0))
            return e_, d_p, d_op
        if obj_fnc == "env_L22":
            d_e, _, d_H = instant_(d)
            d_oe, _, _ = instant_(d_o)
            dedoe = d_e ** 2 - d_oe ** 2
            e_ = d * dedoe - np.imag(hilbert(dedoe * d_H, axis=0))
            return e_, d_e, d_oe
        if obj_fnc == "env_LOG":
            d_e, _, d_H = instant_(d)
            d_oe, _, _ = instant_(d_o)
            dedoe = np.real(np.log((d_oe / d_e).astype(np.complex128)))
            e_ = -dedoe * (d / d_e ** 2) + np.imag(hilbert(dedoe * (d_H / d_e ** 2), axis=0))
            e_[np.isnan(e_)] = 0
            return e_, d_e, d_oe
    raise ValueError(obj_fnc)


def w_E(d_o, d, obj_fnc="L2"):
    """w_E.m:7-16 with N = identity (env_L22 squares, env_LOG takes logs of
    both arguments), normalised by d_o.d_o as w_update_e.m:75-76; after
    w_fwd.m:34-35 the arguments are w_bozdag's d_oe and d_e."""
    d = np.asarray(d, np.float64).ravel()
    do = np.asarray(d_o, np.float64).ravel()
    if obj_fnc == "env_L22":
        a, b = d ** 2, do ** 2
    elif obj_fnc == "env_LOG":
        with np.errstate(divide="ignore"):
            a, b = np.log(d), np.log(do)
    else:
        a, b = d, do
    e = a - b
    return 0.5 * float(e @ e) / float(do @ do)


def w_wavelet(t, ampli, tau):
    """w_wavelet.m:11-33: -(t-t0)*exp(-(t-t0)^2/tau^2), tau = tau/pi, t0 = 5 tau,
    normalised to peak |ampli|."""
    tau = tau / np.pi
    to = 5 * tau
    w = -(t - to) * np.exp(-((t - to) ** 2) / tau ** 2)
    return ampli * (w / np.max(np.abs(w)))


def filt_gauss(d, dt, f_low, f_high, steep=8):
    """filt_gauss.m:16-47: Tukey(0.1) taper, zero-pad to 2^k, Gaussian band filter."""
    d = np.asarray(d, np.float64)
    nt, nr = d.shape
    d = d * tukeywin(nt, 0.1)[:, None]
    nt_ = 1 << int(np.ceil(np.log2(nt)))
    dx = np.vstack([d, np.zeros((nt_ - nt, nr))])
    F = np.fft.fft(dx, axis=0)
    df = 1.0 / dt / nt_
    f = np.arange(-nt_ // 2, nt_ // 2) * df
    width = f_high - f_low
    middle = f_low + width * 0.5
    gauss = np.exp(-((f - middle) ** steep) / ((df * 0.5) * width ** (steep - 1)))
    gauss = np.fft.fftshift(gauss)
    out = np.real(np.fft.ifft(F * gauss[:, None], axis=0))
    return out[:nt, :]


def tukeywin(n, r=0.5):
    """MATLAB tukeywin(n, r)."""
    if r <= 0:
        return np.ones(n)
    if r >= 1:
        return 0.5 * (1 - np.cos(2 * np.pi * np.arange(n) / (n - 1)))
    t = np.linspace(0, 1, n)
    per = r / 2
    tl = int(np.floor(per * (n - 1))) + 1
    th = n - tl + 1
    w = np.ones(n)
    w[:tl] = (1 + np.cos(np.pi / per * (t[:tl] - per))) / 2
    w[th - 1:] = (1 + np.cos(np.pi / per * (t[th - 1:] - 1 + per))) / 2
    return w


# ---------------------------------------------------------------------------
# Gradient conditioning of w_update_e.m:99-137 / w_update_s.m:96-137.

def normali(a):
    """normali.m: a / max|a| (1 when that is 0)."""
    a = np.asarray(a, np.float64)
    mx = np.nanmax(np.abs(a)) if a.size else 0.0
    return a / (mx if mx != 0 else 1.0)


def gaussi(x, z, s, lo):
    """gaussi.m with s = (iz, ix) 0-based: normali(1 - exp(-r^2)), r measured in
    units of 2*lo (the caller passes 2*lo, gaussi doubles it again)."""
    X, Z = np.meshgrid(np.asarray(x, np.float64), np.asarray(z, np.float64))
    lo = 2 * lo
    g = ((X - x[s[1]]) / lo) ** 2 + ((Z - z[s[0]]) / lo) ** 2
    return normali(1 - np.exp(-g))


def image_gaussian_low(img, a, b):
    """image_gaussian.m with filt_TYPE 'LOW_PASS'."""
    img = np.asarray(img, np.float64)
    m, n = img.shape
    m_ = 1 << int(np.ceil(np.log2(m)))
    n_ = 1 << int(np.ceil(np.log2(n)))
    pad = np.zeros((m_, n_))
    pad[:m, :n] = img
    K = np.fft.fft2(pad)
    A = n_ * (a / 2) * np.sqrt(2)
    B = m_ * (b / 2) * np.sqrt(2)
    XY, YX = np.meshgrid(np.arange(n_), np.arange(m_))
    kk = np.exp(-(((XY - n_ / 2) / A) ** 2 + ((YX - m_ / 2) / B) ** 2))
    kk = kk / np.max(np.abs(kk))
    out = np.real(np.fft.ifft2(np.fft.fftshift(kk) * K))
    return out[:m, :n]


def condition_shot(g, dx, dz, src_model, eps_model, fo, ax, az, c=299792458.0):
    """One shot's gradient through the taper, the k-space low-pass, normali and
    the NaN guard (w_update_e.m:110-135).  src_model = (row, column) of the
    source in the model, 0-based."""
    m, n = g.shape
    x = np.arange(n) * dx
    z = np.arange(m) * dz
    lo = c / np.sqrt(eps_model[src_model[0], src_model[1]]) / fo
    g = gaussi(x, z, src_model, 2 * lo) * g
    g = normali(image_gaussian_low(g, ax, az))
    if np.isnan(g).any():
        g = np.zeros_like(g)
    return g
