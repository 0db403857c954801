"""Step lengths of the radar permittivity and conductivity updates, as the
reference chooses them around its objective evaluations (w_stepparabola_e.m,
w_stepparabola_s.m, w_boundstep2.m, w_objs_e.m:24-25, w_objs_s.m:22-25).  The
trial objectives are forward-only runs of all shots; all trial models of one
search run in one ``Context.w_misfit_trials`` call (gj_w_misfit_trials), which
band-filters the observed and modelled traces first as w_objs_e.m:33-36 does.
This module holds the host logic around them.
"""
from __future__ import annotations

import math
from typing import Callable

import numpy as np


def perturb_eps(eps: np.ndarray, g_e: np.ndarray, ke: float) -> np.ndarray:
    """The trial model eps * exp(-ke * eps * g_e) (w_objs_e.m:24-25)."""
    eps = np.asarray(eps, np.float64)
    return eps * np.exp(-ke * eps * np.asarray(g_e, np.float64))


def _in_bounds(eps, deps, k, eps_max, eps_min) -> bool:
    e = eps * np.exp(k * eps * deps)
    return not (e.max() > eps_max or e.min() < eps_min)


def boundstep2(eps, deps, eps_max: float, eps_min: float, k_) -> float:
    """The largest step k for which eps * exp(k * eps * deps) stays within
    [eps_min, eps_max] (w_boundstep2.m:5-23): a reverse search over 13
    log-spaced steps from max(k_) down to min(k_) for the first one in bounds,
    then a forward search over 20 linear steps between it and the previous,
    out-of-bounds one, for the last one in bounds.  If even min(k_) is out of
    bounds the first search ends there and its value is returned."""
    eps = np.asarray(eps, np.float64).ravel()
    deps = np.asarray(deps, np.float64).ravel()
    k_ = np.atleast_1d(np.asarray(k_, np.float64))
    k = np.logspace(math.log10(k_.max()), math.log10(k_.min()), 13)
    ik = 0  # first in bounds, or the last entry (w_boundstep2.m:28-43)
    while not _in_bounds(eps, deps, k[ik], eps_max, eps_min):
        if ik + 1 >= len(k):
            break
        ik += 1
    if ik == 0:
        return float(k[0])
    k = np.linspace(k[ik], k[ik - 1], 20)
    ik = 0  # last in bounds (w_boundstep2.m:44-63)
    while _in_bounds(eps, deps, k[ik], eps_max, eps_min):
        if ik + 1 >= len(k):
            return float(k[ik])
        ik += 1
    return float(k[max(ik - 1, 0)])


def stepparabola(eps, g_e, objective: Callable[[float], float], E0: float, eps_max: float, eps_min: float,
                 k_e, keprct_: float, keprct__: float, nparabo: int) -> tuple[float, np.ndarray, np.ndarray]:
    """w_stepparabola_e.m: trial steps ke from -keprct_ * boundstep2(eps, g_e)
    to keprct__ * boundstep2(eps, -g_e) (nparabo of them), their objectives
    beside E0 at ke = 0, a least-squares parabola through the points and its
    vertex as the step; a flat (zero or NaN) or negative vertex gives 0.
    `objective(ke)` evaluates the trial model perturb_eps(eps, g_e, ke).
    Returns (step, ke, E) with ke and E including the ke = 0 point first."""
    ke_ = -boundstep2(eps, g_e, eps_max, eps_min, k_e) * keprct_
    ke__ = boundstep2(eps, -np.asarray(g_e, np.float64), eps_max, eps_min, k_e) * keprct__
    ks = np.linspace(ke_, ke__, nparabo)
    E = np.concatenate([[float(E0)], _evaluate(objective, ks)])
    ke = np.concatenate([[0.0], ks])
    with np.errstate(all="ignore"):
        p = np.polyfit(ke, E, 2)
        step = -p[1] / (2 * p[0])
    if not np.isfinite(step) or step == 0 or step < 0:
        step = 0.0
    return float(step), ke, E


def stepparabola_s(sig, g_s, objective: Callable[[float], float], E0: float, sig_max: float, sig_min: float,
                   k_s, ksprct_: float, ksprct__: float, nparabo: int) -> tuple[float, np.ndarray, np.ndarray]:
    """w_stepparabola_s.m: the conductivity's trial steps all lie on the
    positive side, from ksprct_ to ksprct__ times boundstep2(sig, -g_s)
    (nparabo + 2 of them); the vertex of the least-squares parabola through
    them and E0 at ks = 0 is the step, 0 when flat (zero or NaN).  Unlike the
    permittivity's, a negative vertex is returned as it is (w_stepparabola_s.m
    only reports it).  `objective(ks)` evaluates perturb_eps(sig, g_s, ks), the
    same exponential update (w_objs_s.m:22-25)."""
    kb = boundstep2(sig, -np.asarray(g_s, np.float64), sig_max, sig_min, k_s)
    ks = np.linspace(kb * ksprct_, kb * ksprct__, nparabo + 2)
    E = np.concatenate([[float(E0)], _evaluate(objective, ks)])
    k = np.concatenate([[0.0], ks])
    with np.errstate(all="ignore"):
        p = np.polyfit(k, E, 2)
        step = -p[1] / (2 * p[0])
    if not np.isfinite(step) or step == 0:
        step = 0.0
    return float(step), k, E


def _evaluate(objective, ks) -> np.ndarray:
    """Objective values at the trial steps ks: one batched call when the
    objective offers ``many`` (all trial models in one GPU call), else one
    call per step."""
    many = getattr(objective, "many", None)
    if many is not None:
        return np.asarray(many(np.asarray(ks, np.float64)), np.float64)
    return np.array([float(objective(float(k))) for k in ks])


class MisfitObjective:
    """The trial objective of w_objs_e.m (which = "eps") or w_objs_s.m
    (which = "sig") on the GPU: the summed normalised misfit of all shots with
    that parameter perturbed as x exp(-k x g).  ``many(ks)`` evaluates all
    trial steps of a search in one gj_w_misfit_trials call (forward runs
    only); calling the object evaluates one step.  ``filt = (f_, f__)`` are
    regu.f_ and regu.f__ of w_objs_e.m:33-36: both trace sets are band-filtered
    (filt_gauss.m, exponent 8) before the misfit."""

    def __init__(self, ctx, grid, eps, sig, shots, d_obs, g, misfit=0, precision=0, which="eps", filt=None):
        if which not in ("eps", "sig"):
            raise ValueError("which must be 'eps' or 'sig'")
        self.ctx, self.grid, self.eps, self.sig, self.shots, self.d_obs = ctx, grid, eps, sig, shots, d_obs
        self.g, self.misfit, self.precision, self.which, self.filt = g, misfit, precision, which, filt

    def _models(self, ks):
        if self.which == "eps":
            return [perturb_eps(self.eps, self.g, k) for k in ks], [self.sig] * len(ks)
        return [self.eps] * len(ks), [perturb_eps(self.sig, self.g, k) for k in ks]

    def many(self, ks) -> np.ndarray:
        e, s_ = self._models(ks)
        m = self.ctx.w_misfit_trials(self.grid, e, s_, self.shots, self.d_obs, misfit=self.misfit,
                                     precision=self.precision, filt=self.filt)
        return m.sum(axis=1)

    def __call__(self, k: float) -> float:
        return float(self.many([k])[0])


def misfit_objective(ctx, grid, eps, sig, shots, d_obs, g, misfit=0, precision=0, which: str = "eps",
                     filt=None) -> MisfitObjective:
    """The trial objective of w_objs_e.m / w_objs_s.m (see MisfitObjective)."""
    return MisfitObjective(ctx, grid, eps, sig, shots, d_obs, g, misfit, precision, which, filt)


def dc_stepparabola(sig, g, objective: Callable[[float], float], E0: float, sig_max: float, sig_min: float,
                    k_s, kprct_: float, kprct__: float) -> tuple[float, np.ndarray, np.ndarray]:
    """dc_stepparabola2_5d.m: four trial steps from -kprct_ boundstep2(sig, g)
    to kprct__ boundstep2(sig, -g) (dc_boundstep2.m is w_boundstep2.m), the
    vertex of the least-squares parabola through them and E0 at k = 0; 0 when
    flat (zero or NaN); a negative vertex falls back to the trial step of least
    objective if that step is positive, else 0.  `objective(k)` evaluates the
    model sig exp(-k sig g) (dc_objs2_5d.m)."""
    g = np.asarray(g, np.float64)
    k_ = -boundstep2(sig, g, sig_max, sig_min, k_s) * kprct_
    k__ = boundstep2(sig, -g, sig_max, sig_min, k_s) * kprct__
    ks = np.linspace(k_, k__, 4)
    E = np.concatenate([[float(E0)], _evaluate(objective, ks)])
    k = np.concatenate([[0.0], ks])
    with np.errstate(all="ignore"):
        p = np.polyfit(k, E, 2)
        step = -p[1] / (2 * p[0])
    if not np.isfinite(step) or step == 0:
        step = 0.0
    if step < 0:
        kb = k[int(np.argmin(E))]
        step = float(kb) if kb > 0 else 0.0
    return float(step), k, E


def dc_E(d_o, d, w=None, obj_fnc: str = "L2") -> float:
    """dc_E.m: 0.5 e' N e with e = d - d_o, on the squared data for 'env_L22'
    and on the log data for 'env_LOG'; N = diag(w) (ones when None)."""
    d = np.asarray(d, np.float64).ravel()
    d_o = np.asarray(d_o, np.float64).ravel()
    if obj_fnc == "env_L22":
        d, d_o = d ** 2, d_o ** 2
    elif obj_fnc == "env_LOG":
        d, d_o = np.log(d), np.log(d_o)
    elif obj_fnc != "L2":
        raise ValueError(f"unknown DC obj_FNC {obj_fnc!r}")
    e = d - d_o
    w = np.ones_like(e) if w is None else np.asarray(w, np.float64).ravel()
    return 0.5 * float(e @ (w * e))


def dc_misfit_objective(ctx, sig, robin: int, DX: float, DZ: float, srcs, g, std=None,
                        obj_fnc: str = "L2") -> Callable[[float], float]:
    """The trial objective of dc_objs2_5d.m on the GPU: the model sig (n0 x m0,
    before the Robin padding) perturbed as sig exp(-k sig g), padded (dc_robin),
    one gj_dc_forward over the sources, and per source dc_E(d_o, d, std,
    obj_fnc) / (d_o' d_o) (the normaliser uses the untransformed data,
    dc_objs2_5d.m).  The reference runs this search per source inside
    dc_update2_5d(i_e); pass a one-source list for that; with several sources
    the per-source objectives are summed.  `std` is a list of per-datum
    weights (ones when None)."""
    from .dc import dc_robin

    def objective(k: float) -> float:
        d = ctx.dc_forward(dc_robin(perturb_eps(sig, g, k), robin), DX, DZ, robin, srcs)["d"]
        total = 0.0
        for j, (q, dj) in enumerate(zip(srcs, d)):
            do = np.asarray(q.d_obs, np.float64)
            total += dc_E(do, dj, None if std is None else std[j], obj_fnc) / float(do @ do)
        return total
    return objective
