"""The reference's MAT-file formats, read and written from Python.

Field data and surveys reach the reference's solvers through four kinds of
MATLAB files; these functions read them into plain numpy arrays (and the radar
shots into this library's ``Shot`` objects) and write them back in the same
layout, so a survey prepared for the reference runs here unchanged.

    line<is>.mat      struct ``radargram`` of shot ``is`` (written by
                      w_natur_.m:42-65, read by w_load.m:9-15): d (nt x nr
                      observed traces), std_ (data weights), dr, and t, dt, fo,
                      dx, r, s, dsr, wvlet_, Jy
    s_r.mat, s_r_.mat cell ns x 2 (experim_w.m:119-135): {is,1} the source,
                      {is,2} the receivers (nr x 2); s_r in metres, s_r_ in
                      model-cell indices, source [iz ix] and receivers [ix iz]
                      (w_load.m:31-35)
    s_i_r_d_std.mat   cell of DC source gathers (dc_load2_5d.m:8-13): {ie}{1} =
                      [electrode A, electrode B, current], {ie}{2} = one row
                      [electrode M, electrode N, datum, std] per datum
    ky_w.mat          ky_w, n_ky x 2 x nsrc wavenumbers and weights per source
                      (dc_load2_5d.m:24-33)

MATLAB v5 files (MATLAB's default ``save``) go through scipy.io.  v7.3 files
are HDF5 containers and need h5py, which this environment does not have:
reading one raises an error that says so.
"""
from __future__ import annotations

import numpy as np

from .geometry import Shot, WGrid, w_M


def _loadmat(path: str) -> dict:
    import scipy.io
    try:
        return scipy.io.loadmat(path, squeeze_me=False, struct_as_record=False)
    except NotImplementedError as ex:  # scipy's answer to a v7.3 (HDF5) file
        raise ValueError(f"{path}: MATLAB v7.3 (HDF5) files need h5py; save with -v7 instead") from ex


def _savemat(path: str, variables: dict) -> None:
    import scipy.io
    scipy.io.savemat(path, variables, format="5", do_compression=False, oned_as="column")


def _cell(rows: list[list[np.ndarray]]) -> np.ndarray:
    out = np.empty((len(rows), len(rows[0]) if rows else 0), dtype=object)
    for i, row in enumerate(rows):
        for j, v in enumerate(row):
            out[i, j] = np.asarray(v, np.float64)
    return out


def load_radargram(path: str) -> dict:
    """line<is>.mat -> dict of the struct's fields (arrays as stored; 1 x 1
    values as floats)."""
    m = _loadmat(path)
    if "radargram" not in m:
        raise ValueError(f"{path}: no variable 'radargram'")
    st = m["radargram"].reshape(-1)[0]
    out = {}
    for name in st._fieldnames:
        v = np.asarray(getattr(st, name))
        out[name] = float(v.reshape(-1)[0]) if v.size == 1 and v.dtype.kind in "fiu" else v
    return out


def save_radargram(path: str, d, t, dt: float, fo: float, dx: float, r, s, wvlet, Jy=None, std=None) -> None:
    """Writes line<is>.mat as w_natur_.m:42-65 does: dr is the first receiver
    spacing and dsr the source to first receiver distance; std_ defaults to
    ones (nt*nr x 1)."""
    d = np.asarray(d, np.float64)
    r = np.asarray(r, np.float64).reshape(-1, 2)
    s = np.asarray(s, np.float64).reshape(1, 2)
    rg = {"d": d, "t": np.asarray(t, np.float64).reshape(-1, 1), "dt": float(dt), "fo": float(fo), "dx": float(dx),
          "r": r, "s": s,
          "dr": float(abs(r[0, 0] - r[1, 0])) if len(r) > 1 else 0.0,
          "dsr": float(np.hypot(s[0, 0] - r[0, 0], s[0, 1] - r[0, 1])),
          "wvlet_": np.asarray(wvlet, np.float64).reshape(-1, 1),
          "Jy": np.zeros((d.shape[0], 1)) if Jy is None else np.asarray(Jy, np.float64).reshape(-1, 1),
          "std_": np.ones((d.size, 1)) if std is None else np.asarray(std, np.float64).reshape(-1, 1)}
    _savemat(path, {"radargram": rg})


def load_s_r(path: str) -> list[tuple[np.ndarray, np.ndarray]]:
    """s_r.mat or s_r_.mat -> per shot (source (2,), receivers (nr, 2))."""
    m = _loadmat(path)
    name = "s_r_" if "s_r_" in m else "s_r"
    if name not in m:
        raise ValueError(f"{path}: no variable 's_r' or 's_r_'")
    c = m[name]
    return [(np.asarray(c[i, 0], np.float64).reshape(-1), np.asarray(c[i, 1], np.float64).reshape(-1, 2))
            for i in range(c.shape[0])]


def save_s_r(path: str, pairs, indexed: bool) -> None:
    """Writes s_r_.mat (indexed = True) or s_r.mat as experim_w.m:119-135."""
    rows = [[np.asarray(s, np.float64).reshape(1, 2), np.asarray(r, np.float64).reshape(-1, 2)] for s, r in pairs]
    _savemat(path, {"s_r_" if indexed else "s_r": _cell(rows)})


def shots_from_s_r_(grid: WGrid, pairs, wavelets) -> list[Shot]:
    """Shots on this library's grid from s_r_ indices, with the offsets of
    w_load.m:31-35: the source row pis + air + iz and column pjs + ix, the
    receivers [pjs + ix, pis + air + iz] (1-based, pis = pml_top + 1 and
    pjs = pml + 1 as wdc_geom.m:100-102), receivers through w_M.m:20.
    `wavelets` is the nt x ns matrix parame_.w.wvlets_ (w_load.m:50)."""
    wv = np.asarray(wavelets, np.float64)
    if wv.ndim == 1:
        wv = wv[:, None]
    shots = []
    pis, pjs = grid.pml_top + 1, grid.pml + 1
    for k, (s, r) in enumerate(pairs):
        iz, ix = int(round(s[0])), int(round(s[1]))
        rr = np.rint(np.asarray(r)).astype(np.int64).reshape(-1, 2)
        rec_ji = np.stack([pjs + rr[:, 0], pis + grid.air + rr[:, 1]], axis=1)
        shots.append(Shot(src_i=pis + grid.air + iz - 1, src_j=pjs + ix - 1,
                          wavelet=wv[:, k if wv.shape[1] > 1 else 0].copy(), rec=w_M(grid, rec_ji) - 1))
    return shots


def load_dc_survey(path: str) -> list[dict]:
    """s_i_r_d_std.mat -> per source gather {"ab": electrode numbers (2,),
    "current", "mn": (nd, 2) electrode numbers, "d": (nd,), "std": (nd,)}
    (dc_load2_5d.m:9-13).  Electrode numbers index the survey's electrode
    coordinate table, as in dc_electrodes.m:31-35."""
    m = _loadmat(path)
    if "s_i_r_d_std" not in m:
        raise ValueError(f"{path}: no variable 's_i_r_d_std'")
    out = []
    for g in m["s_i_r_d_std"].reshape(-1):
        g = g.reshape(-1)
        src = np.asarray(g[0], np.float64).reshape(-1)
        rec = np.asarray(g[1], np.float64).reshape(-1, 4)
        out.append({"ab": src[:2].astype(np.int64), "current": float(src[2]), "mn": rec[:, :2].astype(np.int64),
                    "d": rec[:, 2].copy(), "std": rec[:, 3].copy()})
    return out


def save_dc_survey(path: str, gathers) -> None:
    """Writes s_i_r_d_std.mat in the layout dc_load2_5d.m:8-13 reads."""
    c = np.empty((1, len(gathers)), dtype=object)
    for i, g in enumerate(gathers):
        inner = np.empty((1, 2), dtype=object)
        inner[0, 0] = np.array([[g["ab"][0], g["ab"][1], g["current"]]], np.float64)
        inner[0, 1] = np.column_stack([np.asarray(g["mn"], np.float64).reshape(-1, 2), g["d"], g["std"]])
        c[0, i] = inner
    _savemat(path, {"s_i_r_d_std": c})


def load_ky_w(path: str) -> np.ndarray:
    """ky_w.mat -> (n_ky, 2, nsrc) wavenumbers and weights (dc_load2_5d.m:33)."""
    m = _loadmat(path)
    if "ky_w" not in m:
        raise ValueError(f"{path}: no variable 'ky_w'")
    k = np.asarray(m["ky_w"], np.float64)
    return k[:, :, None] if k.ndim == 2 else k


def save_ky_w(path: str, ky_w) -> None:
    _savemat(path, {"ky_w": np.asarray(ky_w, np.float64)})
