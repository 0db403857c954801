"""Seeded synthetic models and acquisitions for the radar workloads.

Every workload here is generated from ``numpy.random.default_rng(seed)``; no
field data is involved.  Sizes follow the five benchmark configurations:

* ``cfg1``: 200 x 100 model at 0.05 m, free top, 20 PML cells, 2000 steps,
  100 MHz Ricker, 5 sources and 50 receivers on the surface row; blob model.
* ``cfg2``: 1000 x 400 at 0.02 m, 30 PML, 6000 steps, 250 MHz, 30 sources,
  200 receivers; five-layer model with sinusoidal interfaces plus blobs.
* ``cfg3``: 2000 x 800 at 0.02 m, 30 PML, 8000 steps, 250 MHz, one shot; blobs.
* ``cfg4``: 48 uneven problems (see :func:`cfg4_problems`).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from .geometry import WGrid, Shot, ricker, surface_acquisition


@dataclasses.dataclass
class WProblem:
    grid: WGrid
    eps_true: np.ndarray
    sig_true: np.ndarray
    eps0: np.ndarray  # starting model
    sig0: np.ndarray
    shots: list
    name: str = ""
    fo: float = 0.0


def gaussian_smooth(a: np.ndarray, sigma_cells: float) -> np.ndarray:
    """Separable Gaussian smoothing with edge replication (truncated at 3 sigma)."""
    if sigma_cells <= 0:
        return a.copy()
    r = int(math.ceil(3 * sigma_cells))
    x = np.arange(-r, r + 1)
    k = np.exp(-0.5 * (x / sigma_cells) ** 2)
    k /= k.sum()
    out = np.asarray(a, np.float64)
    for ax in (0, 1):
        pad = [(0, 0), (0, 0)]
        pad[ax] = (r, r)
        p = np.pad(out, pad, mode="edge")
        out = np.apply_along_axis(lambda v: np.convolve(v, k, mode="valid"), ax, p)
    return out


def blob_model(m, n, dx, rng, base_eps=5.0, nblob=6, eps_clip=(3.0, 25.0), sig_base=1e-3,
               sig_clip=(1e-3, 1e-2), r_range=(0.3, 1.5), a_range=(-2.0, 20.0)):
    """eps_r = clip(base + sum A exp(-r^2/R^2)), sigma likewise (R ~ U[0.3, 1.5] m)."""
    zz, xx = np.meshgrid(np.arange(m) * dx, np.arange(n) * dx, indexing="ij")
    eps = np.full((m, n), base_eps)
    sig = np.full((m, n), sig_base)
    for _ in range(nblob):
        cz, cx = rng.uniform(0, m * dx), rng.uniform(0, n * dx)
        R = rng.uniform(*r_range)
        A = rng.uniform(*a_range)
        eps += A * np.exp(-((zz - cz) ** 2 + (xx - cx) ** 2) / R ** 2)
    for _ in range(nblob):
        cz, cx = rng.uniform(0, m * dx), rng.uniform(0, n * dx)
        R = rng.uniform(*r_range)
        B = rng.uniform(0.0, sig_clip[1] - sig_base)
        sig += B * np.exp(-((zz - cz) ** 2 + (xx - cx) ** 2) / R ** 2)
    return np.clip(eps, *eps_clip), np.clip(sig, *sig_clip)


def layer_model(m, n, dx, rng, eps_layers=(4, 9, 16, 6, 25), sig_layers=(0.5e-3, 2e-3, 5e-3, 1e-3, 20e-3),
                amp=0.2, nblob=10):
    """Five layers with interfaces at equal depths perturbed by +-amp sinusoids, plus blobs."""
    depth = m * dx
    x = np.arange(n) * dx
    z = np.arange(m) * dx
    nl = len(eps_layers)
    idx = np.zeros((m, n), int)
    for L in range(1, nl):
        lam = rng.uniform(0.2, 1.0) * n * dx
        ph = rng.uniform(0, 2 * np.pi)
        zi = depth * L / nl + amp * np.sin(2 * np.pi * x / lam + ph)
        idx += (z[:, None] >= zi[None, :]).astype(int)
    eps = np.asarray(eps_layers, float)[idx]
    sig = np.asarray(sig_layers, float)[idx]
    zz, xx = np.meshgrid(z, x, indexing="ij")
    for _ in range(nblob):
        cz, cx = rng.uniform(0, depth), rng.uniform(0, n * dx)
        R = rng.uniform(0.1, 0.5)
        A = rng.uniform(-2.0, 8.0)
        eps += A * np.exp(-((zz - cz) ** 2 + (xx - cx) ** 2) / R ** 2)
    return np.clip(eps, 2.0, 30.0), sig


def _problem(name, m, n, dx, pml, nt, fo, nsrc, nrec, kind, seed, free_top=True, courant=0.95,
             smooth_m=1.0, blob_kw=None):
    rng = np.random.default_rng(seed)
    if kind == "blob":
        eps, sig = blob_model(m, n, dx, rng, **(blob_kw or {}))
    else:
        eps, sig = layer_model(m, n, dx, rng)
    g = WGrid(m=m, n=n, pml=pml, pml_top=0 if free_top else pml, air=1 if free_top else 10, nt=nt,
              dx=dx, dy=dx, dt=1.0)
    eps_min = float(eps.min()) if free_top else 1.0
    g.dt = g.cfl_dt(eps_min, courant)
    w = ricker(nt, g.dt, fo, ampli=1e3)
    shots = surface_acquisition(g, nsrc, nrec, w)
    s_cells = smooth_m / dx
    eps0 = gaussian_smooth(eps, s_cells)
    sig0 = gaussian_smooth(sig, s_cells)
    g.check()
    return WProblem(g, eps, sig, eps0, sig0, shots, name, fo)


def cfg1(seed=1001):
    return _problem("cfg1", 100, 200, 0.05, 20, 2000, 100e6, 5, 50, "blob", seed)


def cfg2(seed=1002, nshots=30, nt=6000):
    """1000 x 400 at 0.02 m, 30 PML cells, free top; 30 surface sources (more when
    nshots asks for more), 200 receivers, 250 MHz, five layers + blobs."""
    p = _problem("cfg2", 400, 1000, 0.02, 30, nt, 250e6, max(30, nshots), 200, "layer", seed)
    p.shots = p.shots[:nshots]
    return p


def cfg3(seed=1003, nt=8000):
    return _problem("cfg3", 800, 2000, 0.02, 30, nt, 250e6, 1, 200, "blob", seed)


def small(seed=7, m=24, n=40, pml=8, nt=300, nsrc=3, nrec=12, free_top=True, kind="blob", dx=0.05,
          fo=300e6):
    """Small test problem (seconds on the oracle): blobs sized to the domain."""
    L = min(m, n) * dx
    return _problem("small", m, n, dx, pml, nt, fo, nsrc, nrec, kind, seed, free_top=free_top,
                    smooth_m=0.15 * L, blob_kw=dict(r_range=(0.1 * L, 0.3 * L), a_range=(-2.0, 8.0),
                                                   nblob=4))


def cfg4_problems(seed=2000, count=48):
    """48 uneven problems: NX ~ U{256..1536}, NZ ~ U{128..512}, dx ~ U[0.02, 0.05],
    nt ~ U{1500..5000}, shots ~ U{4..24}; blob and layer models alternate."""
    out = []
    for k in range(count):
        rng = np.random.default_rng(seed + k)
        n = int(rng.integers(256, 1537))
        m = int(rng.integers(128, 513))
        dx = float(rng.uniform(0.02, 0.05))
        nt = int(rng.integers(1500, 5001))
        ns = int(rng.integers(4, 25))
        fo = 250e6 * 0.02 / dx
        out.append(_problem(f"cfg4_{k}", m, n, dx, 20, nt, fo, ns, min(100, n // 4),
                            "blob" if k % 2 == 0 else "layer", seed + k))
    return out


def cfg5(seed=1005, n_sources=200, n_ky=20):
    """2.5D DC: 400 x 100 cells at 0.25 m, one Robin cell (402 x 101 nodes),
    96 surface electrodes at 1 m, `n_sources` seeded dipole-dipole AB pairs x
    6 MN levels, n_ky wavenumbers (grid units).  log10 sigma ~ N(log10 0.01,
    0.5) smoothed over 1 m, plus 4 seeded resistive/conductive blocks."""
    from . import dc
    n0, m0, dx, robin = 400, 100, 0.25, 1
    rng = np.random.default_rng(seed)
    ls = np.log10(0.01) + 0.5 * rng.standard_normal((n0, m0))
    ls = gaussian_smooth(ls, 1.0 / dx)
    ls = np.log10(0.01) + (ls - ls.mean()) * (0.5 / max(ls.std(), 1e-12))
    for _ in range(4):
        l0, h0 = rng.integers(20, n0 - 60), rng.integers(4, m0 - 30)
        L, H = rng.integers(12, 40), rng.integers(6, 20)
        ls[l0:l0 + L, h0:h0 + H] += rng.choice([-1.0, 1.0]) * rng.uniform(0.5, 1.0)
    sig = 10 ** ls
    X = np.arange(n0) * dx
    Z = np.arange(m0) * dx
    DX, DZ = dc.deltas(X, Z, robin)
    SIG = dc.dc_robin(sig, robin)
    n, m = SIG.shape
    kyw = dc.ky_weights(dx, n0 * dx, n_ky, dx=dx)
    srcs = dc.dipole_dipole(n, m, robin, DX, DZ, n_electrodes=96, spacing_nodes=4, first_node=8,
                            pairs=n_sources, levels=6, ky_w=kyw, rng=np.random.default_rng(seed + 1))
    return dict(SIG=SIG, sig=sig, DX=DX, DZ=DZ, robin=robin, srcs=srcs, n=n, m=m, ky_w=kyw)
