"""Grid and acquisition geometry for the radar (GPR) path.

Mirrors the index bookkeeping of the reference's wdc_geom.m:35-125 and w_M.m
with one generalisation: the number of PML rows on top (``pml_top``) is either
``pml`` (the reference layout: PML on all four sides plus ``air`` rows, as in
w_exp2pml.m:19-34) or 0 (a free, reflecting top: the Yee grid's Ez = 0 row sits
directly above the air rows).

All indices handed to the C ABI are 0-based.  MATLAB-facing helpers take and
return 1-based indices, as the reference does.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

EPS_0 = 8.854187817e-12  # param_wdc.m:28
MU_0 = 4 * math.pi * 1e-7  # param_wdc.m:29
C_0 = 1.0 / math.sqrt(MU_0 * EPS_0)


@dataclasses.dataclass
class WGrid:
    """Padded Yee grid.  Field order matches ``gj_w_grid`` in include/gerjoii_gpu.h."""

    m: int  # model rows (depth, fastest index)
    n: int  # model columns (lateral)
    pml: int  # PML cells on the bottom, left and right (pml_w == pml_d)
    pml_top: int  # PML rows on top: pml (reference layout) or 0 (free top)
    air: int  # air rows (eps_r = 1, sigma = 0) above the model
    nt: int
    dx: float
    dy: float
    dt: float
    eps0: float = EPS_0
    mu0: float = MU_0
    order: int = 2  # wdc_geom.m:98
    R0: float = 1e-8  # wdc_geom.m:99

    @property
    def NX(self) -> int:
        """Depth cells incl. PML and air ("nx", wdc_geom.m:70)."""
        return self.pml_top + self.air + self.m + self.pml

    @property
    def NY(self) -> int:
        """Lateral cells incl. PML ("ny", wdc_geom.m:69)."""
        return self.n + 2 * self.pml

    @property
    def nodes(self) -> int:
        return (self.NX + 1) * (self.NY + 1)

    @property
    def dom_i0(self) -> int:
        """0-based Ez row of the first model row (pis+air-1)."""
        return self.pml_top + self.air

    @property
    def dom_j0(self) -> int:
        """0-based Ez column of the first model column (pjs-1)."""
        return self.pml

    def node(self, i: int, j: int) -> int:
        """0-based linear Ez node index (column-major, leading dimension NX+1)."""
        return int(i) + int(j) * (self.NX + 1)

    def model_node(self, a: int, b: int) -> tuple[int, int]:
        """Ez node (0-based) of model cell (a, b) (0-based row, column)."""
        return self.dom_i0 + int(a), self.dom_j0 + int(b)

    def check(self) -> None:
        if min(self.m, self.n) < 3 or self.pml < 1 or self.nt < 3:
            raise ValueError("grid too small (need m, n >= 3, pml >= 1, nt >= 3)")
        if self.pml_top not in (0, self.pml):
            raise ValueError("pml_top must be 0 (free top) or equal to pml")
        if self.pml_top == 0 and self.air < 1:
            raise ValueError("a free top needs air >= 1 so the model starts below the Ez = 0 row")
        if not (self.dx > 0 and self.dy > 0 and self.dt > 0):
            raise ValueError("dx, dy, dt must be positive")

    def cfl_dt(self, eps_min: float, courant: float = 0.95) -> float:
        """dt = courant / (v_max * sqrt(1/dx^2 + 1/dy^2)) (wdc_geom.m:54-56)."""
        vmax = C_0 / math.sqrt(eps_min)
        return courant / (vmax * math.sqrt(1.0 / self.dx ** 2 + 1.0 / self.dy ** 2))


def w_M(grid: WGrid, r_ji_1based: np.ndarray) -> np.ndarray:
    """w_M.m:20: receivers given as [j_lateral, i_depth] (1-based) -> 1-based
    linear Ez indices sub2ind([nx+1, ny+1], i, j)."""
    r = np.asarray(r_ji_1based, dtype=np.int64).reshape(-1, 2)
    return (r[:, 1] - 1) + (r[:, 0] - 1) * (grid.NX + 1) + 1


@dataclasses.dataclass
class Shot:
    """One source and its receivers, 0-based Ez nodes."""

    src_i: int
    src_j: int
    wavelet: np.ndarray  # (nt,)
    rec: np.ndarray  # (nr,) 0-based linear Ez node indices

    @property
    def nr(self) -> int:
        return int(len(self.rec))


def ricker(nt: int, dt: float, fo: float, t0: float | None = None, ampli: float = 1.0) -> np.ndarray:
    """Ricker wavelet (1 - 2 (pi fo tau)^2) exp(-(pi fo tau)^2), tau = t - t0."""
    t = np.arange(nt) * dt
    if t0 is None:
        t0 = 1.5 / fo
    a = (math.pi * fo * (t - t0)) ** 2
    return ampli * (1 - 2 * a) * np.exp(-a)


def w_wavelet(t: np.ndarray, ampli: float, tau: float) -> np.ndarray:
    """w_wavelet.m:11-33: -(t - t0) exp(-(t - t0)^2 / tau'^2), tau' = tau/pi,
    t0 = 5 tau', normalised to peak |ampli|."""
    tau = tau / math.pi
    to = 5 * tau
    w = -(t - to) * np.exp(-((t - to) ** 2) / tau ** 2)
    return ampli * (w / np.max(np.abs(w)))


def surface_acquisition(grid: WGrid, nsrc: int, nrec: int, wavelet: np.ndarray,
                        row: int = 0, margin: int = 2) -> list[Shot]:
    """Sources and receivers evenly spaced on model row ``row`` (0-based); a
    single source sits at the centre, and no source shares a receiver's node."""
    i = grid.dom_i0 + row
    jr = np.linspace(margin, grid.n - 1 - margin, nrec).round().astype(int) + grid.dom_j0
    # keep receivers off the model's first column (it lies in the PML band)
    jr = np.clip(jr, grid.dom_j0 + 1, grid.dom_j0 + grid.n - 1)
    if nsrc == 1:
        js = np.array([grid.dom_j0 + grid.n // 2])
    else:
        js = np.linspace(margin, grid.n - 1 - margin, nsrc).round().astype(int) + grid.dom_j0
    # no source on a receiver node: move it to the next free column
    taken = set(int(j) for j in jr)
    js = np.array([j + 1 if int(j) in taken and int(j) + 1 < grid.dom_j0 + grid.n else j for j in js])
    rec = np.array([grid.node(i, j) for j in jr], dtype=np.int64)
    return [Shot(int(i), int(j), np.asarray(wavelet, np.float64), rec) for j in js]
