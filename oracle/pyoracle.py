"""ORACLE — TEST INFRASTRUCTURE ONLY.

ctypes bindings for oracle/_build/libgj_oracle.so (the C++ restatement in
gj_oracle.hpp).  Importable only by tests/, the smoke check and the benchmark's
CPU-baseline leg.  ``build()`` compiles it with oracle/Makefile.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libgj_oracle.so")


class GridC(C.Structure):
    _fields_ = [("m", C.c_int), ("n", C.c_int), ("pml", C.c_int), ("pml_top", C.c_int),
                ("air", C.c_int), ("nt", C.c_int), ("dx", C.c_double), ("dy", C.c_double),
                ("dt", C.c_double), ("eps0", C.c_double), ("mu0", C.c_double),
                ("order", C.c_int), ("R0", C.c_double)]


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = C.CDLL(LIB_PATH)
    return _lib


def _grid(g) -> GridC:
    return GridC(g.m, g.n, g.pml, g.pml_top, g.air, g.nt, g.dx, g.dy, g.dt, g.eps0, g.mu0,
                 g.order, g.R0)


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _f64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel(order="F"))


def forward(g, eps, sig, shot, precision="f64", store_u=False):
    """Traces d (nt x nr), source trace Jz (nt) and optional history u (m x n x nt)."""
    T = np.float64 if precision == "f64" else np.float32
    e, s = _f64(eps), _f64(sig)
    rec = np.ascontiguousarray(shot.rec, dtype=np.int64)
    d = np.zeros((g.nt, shot.nr), T, order="F")
    jz = np.zeros(g.nt, T)
    u = np.zeros((g.m, g.n, g.nt), T, order="F") if store_u else None
    fn = getattr(lib(), f"gjo_w_forward_{precision}")
    gc = _grid(g)
    fn(C.byref(gc), _p(e), _p(s), C.c_int(shot.src_i), C.c_int(shot.src_j),
       _p(_f64(shot.wavelet)), C.c_int(shot.nr), _p(rec), _p(d), _p(jz),
       _p(u) if u is not None else None)
    return d, jz, u


def grad_reference(g, eps, sig, shot, e, u, precision="f64"):
    """w_grad.m: returns (g, a_max), both m x n."""
    T = np.float64 if precision == "f64" else np.float32
    ea = np.asfortranarray(e, dtype=T)
    ua = np.asfortranarray(u, dtype=T)
    out = np.zeros((g.m, g.n), T, order="F")
    amax = np.zeros((g.m, g.n), T, order="F")
    rec = np.ascontiguousarray(shot.rec, dtype=np.int64)
    fn = getattr(lib(), f"gjo_w_grad_reference_{precision}")
    gc = _grid(g)
    fn(C.byref(gc), _p(_f64(eps)), _p(_f64(sig)), C.c_int(shot.src_i), C.c_int(shot.src_j),
       C.c_int(shot.nr), _p(rec), _p(ea), _p(ua), _p(out), _p(amax))
    return out, amax


def grad_exact(g, eps, sig, shot, e, precision="f64"):
    """Exact discrete gradient of 0.5*||d - d_obs||^2 given e = dJ/dd."""
    T = np.float64 if precision == "f64" else np.float32
    ea = np.asfortranarray(e, dtype=T)
    ge = np.zeros((g.m, g.n), np.float64, order="F")
    gs = np.zeros((g.m, g.n), np.float64, order="F")
    rec = np.ascontiguousarray(shot.rec, dtype=np.int64)
    fn = getattr(lib(), f"gjo_w_grad_exact_{precision}")
    gc = _grid(g)
    fn(C.byref(gc), _p(_f64(eps)), _p(_f64(sig)), C.c_int(shot.src_i), C.c_int(shot.src_j),
       _p(_f64(shot.wavelet)), C.c_int(shot.nr), _p(rec), _p(ea), _p(ge), _p(gs))
    return ge, gs


def differentiate_cube(v, dt, precision="f64"):
    T = np.float64 if precision == "f64" else np.float32
    a = np.array(v, dtype=T, order="F", copy=True)
    npix = int(np.prod(a.shape[:-1]))
    getattr(lib(), f"gjo_differentiate_cube_{precision}")(_p(a), C.c_long(npix), C.c_int(a.shape[-1]),
                                                         C.c_double(dt))
    return a


def _pack_shots(g, shots):
    nr = shots[0].nr
    if any(s.nr != nr for s in shots):
        raise ValueError("batched oracle calls need the same nr for every shot")
    si = np.array([s.src_i for s in shots], np.int32)
    sj = np.array([s.src_j for s in shots], np.int32)
    wav = np.ascontiguousarray(np.stack([np.asarray(s.wavelet, np.float64) for s in shots]))
    rec = np.ascontiguousarray(np.stack([np.asarray(s.rec, np.int64) for s in shots]))
    return nr, si, sj, wav, rec


def forward_batch(g, eps, sig, shots, precision="f64", threads=0):
    """d: (nshots, nr, nt) view of the nt x nr traces per shot."""
    nr, si, sj, wav, rec = _pack_shots(g, shots)
    d = np.zeros((len(shots), nr, g.nt), np.float64)
    gc = _grid(g)
    lib().gjo_w_forward_batch(C.byref(gc), C.c_int(1 if precision == "f64" else 0), _p(_f64(eps)),
                              _p(_f64(sig)), C.c_int(len(shots)), _p(si), _p(sj), _p(wav), C.c_int(nr),
                              _p(rec), C.c_int(threads), _p(d))
    return d


def gradient_batch(g, eps, sig, shots, dobs, mode="reference", precision="f64", threads=0):
    """Summed (g_eps, g_sig) over shots plus per-shot misfits.  dobs: (nshots, nr, nt)."""
    nr, si, sj, wav, rec = _pack_shots(g, shots)
    dobs = np.ascontiguousarray(dobs, dtype=np.float64)
    ge = np.zeros((g.m, g.n), np.float64, order="F")
    gs = np.zeros((g.m, g.n), np.float64, order="F")
    mis = np.zeros(len(shots), np.float64)
    gc = _grid(g)
    lib().gjo_w_gradient_batch(C.byref(gc), C.c_int(1 if precision == "f64" else 0), _p(_f64(eps)),
                               _p(_f64(sig)), C.c_int(len(shots)), _p(si), _p(sj), _p(wav), C.c_int(nr),
                               _p(rec), _p(dobs), C.c_int(0 if mode == "reference" else 1),
                               C.c_int(threads), _p(ge), _p(gs), _p(mis))
    return ge, gs, mis

