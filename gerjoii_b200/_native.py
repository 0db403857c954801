"""ctypes bindings for the in-tree sm_100a library (include/gerjoii_gpu.h).

Loading fails loudly when the library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import build as _build

GJ_OK, GJ_EINVAL, GJ_ENOMEM, GJ_ENUMERIC, GJ_ETIMEOUT, GJ_ECUDA, GJ_EUNSUPPORTED = range(7)
GJ_F32, GJ_F64 = 0, 1
GJ_ADJ_REFERENCE, GJ_ADJ_EXACT = 0, 1
GJ_MISFIT_L2, GJ_MISFIT_ENV_L2, GJ_MISFIT_PHASE_L2, GJ_MISFIT_ENV_L22, GJ_MISFIT_ENV_LOG = 0, 1, 2, 3, 4
# the reference's obj_FNC names (w_bozdag.m:13-54); FREQstp is L2 there
MISFIT_KINDS = {"L2": GJ_MISFIT_L2, "FREQstp": GJ_MISFIT_L2, "env_L2": GJ_MISFIT_ENV_L2,
                "phase_L2": GJ_MISFIT_PHASE_L2, "env_L22": GJ_MISFIT_ENV_L22, "env_LOG": GJ_MISFIT_ENV_LOG}


def misfit_kind(misfit) -> int:
    """A gj_misfit_kind from its value or the reference's obj_FNC name."""
    if isinstance(misfit, str):
        if misfit not in MISFIT_KINDS:
            raise ValueError(f"unknown obj_FNC {misfit!r}; one of {sorted(MISFIT_KINDS)}")
        return MISFIT_KINDS[misfit]
    return int(misfit)

STATUS_NAMES = {0: "GJ_OK", 1: "GJ_EINVAL", 2: "GJ_ENOMEM", 3: "GJ_ENUMERIC", 4: "GJ_ETIMEOUT",
                5: "GJ_ECUDA", 6: "GJ_EUNSUPPORTED"}


class GJError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class GridC(C.Structure):
    _fields_ = [("m", C.c_int), ("n", C.c_int), ("pml", C.c_int), ("pml_top", C.c_int),
                ("air", C.c_int), ("nt", C.c_int), ("dx", C.c_double), ("dy", C.c_double),
                ("dt", C.c_double), ("eps0", C.c_double), ("mu0", C.c_double), ("order", C.c_int),
                ("R0", C.c_double)]


class ShotC(C.Structure):
    _fields_ = [("src_i", C.c_int), ("src_j", C.c_int), ("wavelet", C.POINTER(C.c_double)),
                ("nr", C.c_int), ("rec", C.POINTER(C.c_long))]


class DcGridC(C.Structure):
    _fields_ = [("n", C.c_int), ("m", C.c_int), ("robin", C.c_int), ("n_ky", C.c_int), ("dx", C.c_double),
                ("dz", C.c_double)]


class DcSrcC(C.Structure):
    _fields_ = [("a", C.c_long), ("b", C.c_long), ("current", C.c_double), ("nd", C.c_int),
                ("mn", C.POINTER(C.c_long)), ("ky", C.POINTER(C.c_double)), ("w", C.POINTER(C.c_double)),
                ("alpha", C.POINTER(C.c_double)), ("d_obs", C.POINTER(C.c_double))]


class DcOptsC(C.Structure):
    _fields_ = [("tol", C.c_double), ("max_iter", C.c_int), ("per_source", C.c_int),
                ("sources_per_batch", C.c_int), ("mem_budget_bytes", C.c_size_t), ("factor_fp32", C.c_int),
                ("precond", C.c_int)]


class DcStatsC(C.Structure):
    _fields_ = [("max_iterations", C.c_int), ("max_rel_residual", C.c_double)]


class OptsC(C.Structure):
    _fields_ = [("ckpt_every", C.c_int), ("mem_budget_bytes", C.c_size_t),
                ("shots_per_launch", C.c_int), ("no_kahan", C.c_int), ("no_graph", C.c_int),
                ("per_shot", C.c_int), ("plain", C.c_int), ("no_ring", C.c_int),
                ("filt_low", C.c_double), ("filt_high", C.c_double), ("filt_steep", C.c_int),
                ("condition", C.c_int), ("cond_fo", C.c_double), ("cond_ax", C.c_double), ("cond_az", C.c_double)]


_DP_ = C.POINTER(C.c_double)


class ProblemC(C.Structure):
    _fields_ = [("grid", GridC), ("eps_r", _DP_), ("sigma", _DP_), ("shots", C.c_void_p), ("nshots", C.c_int),
                ("d_obs", _DP_), ("g_eps", _DP_), ("g_sig", _DP_), ("misfit", _DP_)]


# Every symbol the header declares, with its signature.
_VP, _DP, _I, _L = C.c_void_p, C.POINTER(C.c_double), C.c_int, C.c_long
SIGNATURES = {
    "gj_version": (C.c_char_p, []),
    "gj_context_create": (_I, [C.POINTER(_VP), _I]),
    "gj_context_destroy": (_I, [_VP]),
    "gj_context_release": (_I, [_VP]),
    "gj_last_error": (C.c_char_p, [_VP]),
    "gj_last_launch_count": (_L, [_VP]),
    "gj_set_kernel_timing": (_I, [_VP, _I]),
    "gj_kernel_time": (_I, [_VP, _I, _DP, C.POINTER(C.c_long), C.POINTER(C.c_long), C.POINTER(C.c_long)]),
    "gj_w_forward": (_I, [_VP, C.POINTER(GridC), _I, _DP, _DP, C.POINTER(ShotC), _I, _DP, _DP, _DP]),
    "gj_w_gradient": (_I, [_VP, C.POINTER(GridC), _I, _DP, _DP, C.POINTER(ShotC), _I, _DP, _I, _I,
                           C.POINTER(OptsC), _DP, _DP, _DP, _DP, _DP]),
    "gj_w_misfit": (_I, [_VP, C.POINTER(GridC), _I, _DP, _DP, C.POINTER(ShotC), _I, _DP, _I, _DP]),
    "gj_w_misfit_trials": (_I, [_VP, C.POINTER(GridC), _I, _I, _DP, _DP, C.POINTER(ShotC), _I, _DP, _I,
                                C.POINTER(OptsC), _DP]),
    "gj_w_gradient_batch": (_I, [_VP, _I, C.POINTER(ProblemC), _I, _I, C.POINTER(OptsC), C.POINTER(C.c_int)]),
    "gj_w_backward": (_I, [_VP, C.POINTER(GridC), _I, _DP, _DP, C.POINTER(ShotC), _I, _DP, _I, C.POINTER(OptsC),
                           _DP, _DP]),
    "gj_w_grad": (_I, [_VP, C.POINTER(GridC), _I, _DP, _DP, C.POINTER(ShotC), _DP, _DP, _DP, _DP]),
    "gj_w_gradient_dev": (_I, [_VP, C.POINTER(GridC), _I, _VP, _VP, C.POINTER(ShotC), _I, _VP, _I, _I,
                               C.POINTER(OptsC), _VP, _VP, _DP, _VP]),
    "gj_dc_forward": (_I, [_VP, C.POINTER(DcGridC), _DP, C.POINTER(DcSrcC), _I, C.POINTER(DcOptsC), _DP, _DP,
                           C.POINTER(DcStatsC)]),
    "gj_dc_forward_k": (_I, [_VP, C.POINTER(DcGridC), _DP, C.POINTER(DcSrcC), _I, C.POINTER(DcOptsC), _DP, _DP,
                             _DP, C.POINTER(DcStatsC)]),
    "gj_dc_gradient": (_I, [_VP, C.POINTER(DcGridC), _DP, C.POINTER(DcSrcC), _I, C.POINTER(DcOptsC), _DP, _DP, _DP,
                            _DP, C.POINTER(DcStatsC)]),
    "gj_dc_alphas": (_I, [C.POINTER(DcGridC), C.c_long, C.c_long, _DP, _DP]),
    "gj_w_forward_noalloc": (_I, [C.POINTER(GridC), _VP, _VP, _I, _I, _VP, _I, _VP, _VP, _VP, C.c_char_p,
                                  C.c_size_t]),
}

_lib = None


def library_path() -> str:
    return _build.LIB


def load(build_if_missing: bool = False):
    """Loads libgerjoii_b200.so; raises if it is absent (no fallback path)."""
    global _lib
    if _lib is not None:
        return _lib
    path = os.environ.get("GERJOII_B200_LIB", _build.LIB)
    if not os.path.exists(path):
        if build_if_missing:
            _build.build()
        else:
            raise ImportError(f"gerjoii_b200 CUDA library not built: {path} "
                              "(run python -m gerjoii_b200.build)")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _dp(a):
    return a.ctypes.data_as(_DP) if a is not None else None


def grid_c(g) -> GridC:
    return GridC(g.m, g.n, g.pml, g.pml_top, g.air, g.nt, g.dx, g.dy, g.dt, g.eps0, g.mu0, g.order, g.R0)


class _ShotPack:
    """Keeps the numpy buffers behind a ShotC array alive."""

    def __init__(self, shots, nt):
        self.wav = [np.ascontiguousarray(np.asarray(s.wavelet, np.float64)[:nt]) for s in shots]
        self.rec = [np.ascontiguousarray(np.asarray(s.rec, np.int64)) for s in shots]
        arr = (ShotC * len(shots))()
        for k, s in enumerate(shots):
            if len(self.wav[k]) < nt:
                raise ValueError(f"shot {k}: wavelet has {len(self.wav[k])} < nt samples")
            arr[k].src_i = int(s.src_i)
            arr[k].src_j = int(s.src_j)
            arr[k].wavelet = self.wav[k].ctypes.data_as(_DP)
            arr[k].nr = len(self.rec[k])
            arr[k].rec = self.rec[k].ctypes.data_as(C.POINTER(C.c_long))
        self.arr = arr
        self.n = len(shots)


def _f(a):
    """Column-major float64 copy of a model / trace array."""
    return np.asfortranarray(np.asarray(a, dtype=np.float64))


class Context:
    """One gj_ctx on a device."""

    def __init__(self, device: int = 0):
        self.lib = load()
        h = _VP()
        st = self.lib.gj_context_create(C.byref(h), int(device))
        if st != GJ_OK:
            raise GJError(st, f"gj_context_create(device={device}) failed")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.gj_context_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def release(self):
        """gj_context_release: free the cached plans and DC buffers."""
        self._check(self.lib.gj_context_release(self.h))

    def _check(self, st):
        if st != GJ_OK:
            raise GJError(st, self.lib.gj_last_error(self.h).decode())

    @property
    def last_launch_count(self) -> int:
        return int(self.lib.gj_last_launch_count(self.h))

    KERNEL_KINDS = {"fwd_step": 0, "ref_step": 1, "adj_step": 2, "io": 3, "plain": 4, "dc_factor": 5, "image": 6,
                    "dc_precond": 7, "tb_pass": 8}

    def set_kernel_timing(self, on: bool):
        self._check(self.lib.gj_set_kernel_timing(self.h, int(bool(on))))

    def kernel_time(self, kind: str):
        """Accumulated timing of a kernel kind while timing is on: dict with the
        summed ms of the sampled launches, their number, all launches of the
        kind and the sum of shots over those launches."""
        ms = C.c_double(0)
        smp, n, sl = C.c_long(0), C.c_long(0), C.c_long(0)
        self._check(self.lib.gj_kernel_time(self.h, self.KERNEL_KINDS[kind], C.byref(ms), C.byref(smp),
                                            C.byref(n), C.byref(sl)))
        return {"ms": ms.value, "sampled": smp.value, "launches": n.value, "shot_launches": sl.value,
                "avg_us": 1e3 * ms.value / smp.value if smp.value else 0.0}

    # ------------------------------------------------------------------ radar
    def w_forward(self, g, eps, sig, shots, precision=GJ_F32, want_jz=False, want_u=False):
        """Traces per shot (nt x nr), optional Jz (nt) and u (m x n x nt)."""
        sp = _ShotPack(shots, g.nt)
        d = np.zeros(sum(g.nt * len(r) for r in sp.rec), np.float64)
        jz = np.zeros(len(shots) * g.nt, np.float64) if want_jz else None
        u = np.zeros(len(shots) * g.m * g.n * g.nt, np.float64) if want_u else None
        gc = grid_c(g)
        e, s = _f(eps), _f(sig)
        self._check(self.lib.gj_w_forward(self.h, C.byref(gc), precision, _dp(e), _dp(s), sp.arr, sp.n,
                                          _dp(d), _dp(jz), _dp(u)))
        out, o = [], 0
        for r in sp.rec:
            out.append(d[o:o + g.nt * len(r)].reshape((g.nt, len(r)), order="F"))
            o += g.nt * len(r)
        res = {"d": out}
        if want_jz:
            res["jz"] = jz.reshape(len(shots), g.nt)
        if want_u:
            res["u"] = [u[k * g.m * g.n * g.nt:(k + 1) * g.m * g.n * g.nt].reshape((g.m, g.n, g.nt), order="F")
                        for k in range(len(shots))]
        return res

    def w_gradient(self, g, eps, sig, shots, d_obs, mode=GJ_ADJ_REFERENCE, misfit=GJ_MISFIT_L2,
                   precision=GJ_F32, opts=None, want_traces=False):
        """Gradient (g_eps, g_sig) summed over shots (or per shot), misfits, optional d and e."""
        sp = _ShotPack(shots, g.nt)
        o = opts or OptsC()
        per = len(shots) if o.per_shot else 1
        ge = np.zeros(per * g.m * g.n, np.float64)
        gs = np.zeros_like(ge)
        mis = np.zeros(len(shots), np.float64)
        dobs = np.concatenate([_f(x).ravel(order="F") for x in d_obs])
        ntr = sum(g.nt * len(r) for r in sp.rec)
        if dobs.size != ntr:
            raise ValueError("d_obs does not match the shots' receivers")
        dd = np.zeros(ntr) if want_traces else None
        ee = np.zeros(ntr) if want_traces else None
        gc = grid_c(g)
        e, s = _f(eps), _f(sig)
        self._check(self.lib.gj_w_gradient(self.h, C.byref(gc), precision, _dp(e), _dp(s), sp.arr, sp.n,
                                           _dp(dobs), int(mode), misfit_kind(misfit), C.byref(o), _dp(ge), _dp(gs),
                                           _dp(mis), _dp(dd), _dp(ee)))
        shape = (g.m, g.n) if per == 1 else (per, g.m, g.n)
        res = {"g_eps": ge.reshape(shape, order="F") if per == 1 else
               np.stack([ge[k * g.m * g.n:(k + 1) * g.m * g.n].reshape((g.m, g.n), order="F") for k in range(per)]),
               "g_sig": gs.reshape(shape, order="F") if per == 1 else
               np.stack([gs[k * g.m * g.n:(k + 1) * g.m * g.n].reshape((g.m, g.n), order="F") for k in range(per)]),
               "misfit": mis}
        if want_traces:
            outd, oute, q = [], [], 0
            for r in sp.rec:
                n_ = g.nt * len(r)
                outd.append(dd[q:q + n_].reshape((g.nt, len(r)), order="F"))
                oute.append(ee[q:q + n_].reshape((g.nt, len(r)), order="F"))
                q += n_
            res["d"], res["e"] = outd, oute
        return res

    def w_backward(self, g, eps, sig, shots, e, mode=GJ_ADJ_EXACT, precision=GJ_F32, opts=None):
        """gj_w_backward: the adjoint of the forward map applied to the given
        adjoint sources e (list of nt x nr arrays, one per shot): g_eps, g_sig
        (summed over shots, or per shot with opts.per_shot)."""
        sp = _ShotPack(shots, g.nt)
        o = opts or OptsC()
        per = len(shots) if o.per_shot else 1
        ge = np.zeros(per * g.m * g.n, np.float64)
        gs = np.zeros_like(ge)
        ea = np.concatenate([_f(x).ravel(order="F") for x in e])
        if ea.size != sum(g.nt * len(r) for r in sp.rec):
            raise ValueError("e does not match the shots' receivers")
        gc = grid_c(g)
        self._check(self.lib.gj_w_backward(self.h, C.byref(gc), precision, _dp(_f(eps)), _dp(_f(sig)), sp.arr, sp.n,
                                           _dp(ea), int(mode), C.byref(o), _dp(ge), _dp(gs)))
        if per == 1:
            return {"g_eps": ge.reshape((g.m, g.n), order="F"), "g_sig": gs.reshape((g.m, g.n), order="F")}
        mn = g.m * g.n
        return {"g_eps": np.stack([ge[k * mn:(k + 1) * mn].reshape((g.m, g.n), order="F") for k in range(per)]),
                "g_sig": np.stack([gs[k * mn:(k + 1) * mn].reshape((g.m, g.n), order="F") for k in range(per)])}

    def w_grad(self, g, eps, sig, shot, e, u, precision=GJ_F32):
        """w_grad.m for one shot: (g, a_max)."""
        sp = _ShotPack([shot], g.nt)
        out = np.zeros(g.m * g.n)
        amax = np.zeros(g.m * g.n)
        gc = grid_c(g)
        ea, ua = _f(e), _f(u)
        self._check(self.lib.gj_w_grad(self.h, C.byref(gc), precision, _dp(_f(eps)), _dp(_f(sig)), sp.arr,
                                       _dp(ea), _dp(ua), _dp(out), _dp(amax)))
        return out.reshape((g.m, g.n), order="F"), amax.reshape((g.m, g.n), order="F")

    # --------------------------------------------------------------------- DC
    @staticmethod
    def _dc_pack(srcs, with_dobs):
        keep, arr = [], (DcSrcC * len(srcs))()
        for k, q in enumerate(srcs):
            mn = np.ascontiguousarray(np.asarray(q.mn, np.int64).reshape(-1, 2))
            ky = np.ascontiguousarray(q.ky_w[:, 0], np.float64)
            w = np.ascontiguousarray(q.ky_w[:, 1], np.float64)
            al = np.ascontiguousarray(q.alpha, np.float64)
            do = np.ascontiguousarray(q.d_obs, np.float64) if (with_dobs and q.d_obs is not None) else None
            keep += [mn, ky, w, al, do]
            arr[k].a, arr[k].b, arr[k].current, arr[k].nd = int(q.a), int(q.b), float(q.current), len(mn)
            arr[k].mn = mn.ctypes.data_as(C.POINTER(C.c_long))
            arr[k].ky = ky.ctypes.data_as(_DP)
            arr[k].w = w.ctypes.data_as(_DP)
            arr[k].alpha = al.ctypes.data_as(_DP)
            arr[k].d_obs = do.ctypes.data_as(_DP) if do is not None else None
        return arr, keep

    def dc_forward(self, sigma_robin, dx, dz, robin, srcs, opts=None, want_u=False, want_uk=False):
        """Data per source (list of nd arrays), optional stacked u (nsrc x n x m),
        optional per-wavenumber u_k (nsrc x N x n_ky, N = n*m in the vectorised
        order l + h*n of dc_fwd2_5d.m:61), stats."""
        n, m = sigma_robin.shape
        nky = len(srcs[0].ky_w)
        g = DcGridC(n, m, robin, nky, dx, dz)
        arr, keep = self._dc_pack(srcs, False)
        nd = sum(q.nd for q in srcs)
        d = np.zeros(max(nd, 1))
        u = np.zeros(len(srcs) * n * m) if want_u else None
        uk = np.zeros(len(srcs) * nky * n * m) if want_uk else None
        st = DcStatsC()
        sg = np.asfortranarray(sigma_robin, np.float64)
        self._check(self.lib.gj_dc_forward_k(self.h, C.byref(g), _dp(sg), arr, len(srcs),
                                             C.byref(opts) if opts else None, _dp(d), _dp(u), _dp(uk),
                                             C.byref(st)))
        out, o = [], 0
        for q in srcs:
            out.append(d[o:o + q.nd].copy())
            o += q.nd
        res = {"d": out, "iters": st.max_iterations, "rel_residual": st.max_rel_residual}
        if want_u:
            res["u"] = u.reshape((len(srcs), m, n)).transpose(0, 2, 1)
        if want_uk:
            res["u_k"] = uk.reshape((len(srcs), nky, n * m)).transpose(0, 2, 1)
        return res

    def dc_gradient(self, sigma_robin, dx, dz, robin, srcs, opts=None):
        """Gradient (n-2robin x m-robin, summed or per source), data, residuals, misfits, stats."""
        n, m = sigma_robin.shape
        g = DcGridC(n, m, robin, len(srcs[0].ky_w), dx, dz)
        arr, keep = self._dc_pack(srcs, True)
        nd = sum(q.nd for q in srcs)
        per = len(srcs) if (opts is not None and opts.per_source) else 1
        n0, m0 = n - 2 * robin, m - robin
        gout = np.zeros(per * n0 * m0)
        d = np.zeros(max(nd, 1))
        e = np.zeros(max(nd, 1))
        mis = np.zeros(len(srcs))
        st = DcStatsC()
        sg = np.asfortranarray(sigma_robin, np.float64)
        self._check(self.lib.gj_dc_gradient(self.h, C.byref(g), _dp(sg), arr, len(srcs),
                                            C.byref(opts) if opts else None, _dp(gout), _dp(d), _dp(e), _dp(mis),
                                            C.byref(st)))
        gg = gout.reshape((per, m0, n0)).transpose(0, 2, 1)
        return {"g": gg[0] if per == 1 else gg, "d": d[:nd], "e": e[:nd], "misfit": mis,
                "iters": st.max_iterations, "rel_residual": st.max_rel_residual}

    def w_misfit(self, g, eps, sig, shots, dobs, misfit=GJ_MISFIT_L2, precision=GJ_F32):
        """Per-shot misfits of forward runs only (the step-length search's
        objective evaluations); dobs: list of nt x nr arrays."""
        sp = _ShotPack(shots, g.nt)
        gc = grid_c(g)
        ob = np.concatenate([_f(d).ravel(order="F") for d in dobs])
        out = np.zeros(len(shots))
        e, s_ = _f(eps), _f(sig)
        self._check(self.lib.gj_w_misfit(self.h, C.byref(gc), precision, _dp(e), _dp(s_), sp.arr, sp.n, _dp(ob),
                                          misfit_kind(misfit), _dp(out)))
        return out

    def w_misfit_trials(self, g, eps_list, sig_list, shots, dobs, misfit=GJ_MISFIT_L2, precision=GJ_F32,
                        filt=None, steep=0):
        """gj_w_misfit_trials: misfits (ntrial x nshots) of several trial
        models; filt = (f_low, f_high) band-filters both trace sets first
        (w_objs_e.m:33-36)."""
        sp = _ShotPack(shots, g.nt)
        gc = grid_c(g)
        ob = np.concatenate([_f(d).ravel(order="F") for d in dobs])
        nt_ = len(eps_list)
        e = np.concatenate([_f(x).ravel(order="F") for x in eps_list])
        s_ = np.concatenate([_f(x).ravel(order="F") for x in sig_list])
        o = OptsC()
        if filt is not None:
            o.filt_low, o.filt_high = filt
            o.filt_steep = steep
        out = np.zeros(nt_ * len(shots))
        self._check(self.lib.gj_w_misfit_trials(self.h, C.byref(gc), precision, nt_, _dp(e), _dp(s_), sp.arr, sp.n,
                                                _dp(ob), misfit_kind(misfit), C.byref(o), _dp(out)))
        return out.reshape(nt_, len(shots))

    def w_gradient_batch(self, problems, mode=GJ_ADJ_EXACT, precision=GJ_F32, opts=None):
        """gj_w_gradient_batch: problems is a list of (grid, eps, sig, shots,
        d_obs) tuples (d_obs: list of nt x nr arrays); returns a list of
        {"g_eps", "g_sig", "misfit"} and the number of waves used."""
        keep, arr = [], (ProblemC * len(problems))()
        outs = []
        for k, (g, eps, sig, shots, dobs) in enumerate(problems):
            sp = _ShotPack(shots, g.nt)
            e, s_ = _f(eps), _f(sig)
            ob = np.concatenate([_f(d).ravel(order="F") for d in dobs])
            ge = np.zeros(g.m * g.n)
            gs = np.zeros(g.m * g.n)
            mis = np.zeros(len(shots))
            keep += [sp, e, s_, ob]
            arr[k].grid = grid_c(g)
            arr[k].eps_r, arr[k].sigma = _dp(e), _dp(s_)
            arr[k].shots = C.cast(sp.arr, C.c_void_p)
            arr[k].nshots = len(shots)
            arr[k].d_obs = _dp(ob)
            arr[k].g_eps, arr[k].g_sig, arr[k].misfit = _dp(ge), _dp(gs), _dp(mis)
            outs.append((g, ge, gs, mis))
        nw = C.c_int(0)
        self._check(self.lib.gj_w_gradient_batch(self.h, precision, arr, len(problems), int(mode),
                                                 C.byref(opts) if opts else None, C.byref(nw)))
        res = [{"g_eps": ge.reshape((g.m, g.n), order="F"), "g_sig": gs.reshape((g.m, g.n), order="F"),
                "misfit": mis} for (g, ge, gs, mis) in outs]
        return res, nw.value

    def w_gradient_dev(self, g, eps_t, sig_t, shots, dobs_t, ge_t, gs_t, mode=GJ_ADJ_REFERENCE,
                       misfit=GJ_MISFIT_L2, opts=None, stream=0):
        """Device-pointer gradient: arguments are torch CUDA tensors (float32 or float64)."""
        import torch
        prec = GJ_F64 if eps_t.dtype == torch.float64 else GJ_F32
        sp = _ShotPack(shots, g.nt)
        o = opts or OptsC()
        mis = np.zeros(len(shots), np.float64)
        gc = grid_c(g)
        self._check(self.lib.gj_w_gradient_dev(self.h, C.byref(gc), prec, eps_t.data_ptr(), sig_t.data_ptr(),
                                               sp.arr, sp.n, dobs_t.data_ptr(), int(mode), misfit_kind(misfit),
                                               C.byref(o), ge_t.data_ptr(), gs_t.data_ptr(), _dp(mis),
                                               C.c_void_p(stream)))
        return mis


def dc_alphas(n: int, m: int, dx: float, dz: float, a_node: int, b_node: int, ky) -> np.ndarray:
    """gj_dc_alphas: the Robin coefficients of one source (n_ky x GJ_DC_NALPHA,
    the layout of DcSource.alpha), computed by the library on the host."""
    lib = load()
    ky = np.ascontiguousarray(ky, np.float64).ravel()
    na = 2 * (m - 2) + (n - 2) + 4
    out = np.zeros((len(ky), na))
    g = DcGridC(n, m, 0, len(ky), dx, dz)
    st = lib.gj_dc_alphas(C.byref(g), int(a_node), int(b_node), _dp(ky), _dp(out))
    if st != 0:
        raise ValueError(f"gj_dc_alphas failed with status {st}")
    return out
