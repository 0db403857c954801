"""Step-length host logic (CPU): w_boundstep2.m's bound search and
w_stepparabola_e.m's parabola vertex, on models and objectives with known
answers."""
import numpy as np
import pytest

from gerjoii_b200 import steplen


def test_boundstep2_finds_the_largest_step_in_bounds():
    """For a uniform model eps = 4 and direction 1, eps exp(4k) reaches the
    upper bound 9 at k* = ln(9/4)/4: the search returns the last of its linear
    candidates below k* (w_boundstep2.m:14-15), so within one candidate spacing."""
    eps = np.full((5, 6), 4.0)
    g = np.ones_like(eps)
    k_star = np.log(9.0 / 4.0) / 4.0
    k = steplen.boundstep2(eps, g, 9.0, 1.0, [1e-3, 10.0])
    k_log = np.logspace(1, -3, 13)
    i = int(np.argmax(k_log < k_star))  # first log candidate in bounds
    assert k <= k_star and k_star - k <= (k_log[i - 1] - k_log[i]) / 19 + 1e-12
    assert steplen.boundstep2(eps, g, 9.0, 1.0, [1e-3, 0.01]) == 0.01  # largest candidate already in bounds
    assert steplen.perturb_eps(eps, -g, k).max() <= 9.0 + 1e-12


def test_stepparabola_vertex_of_a_quadratic_objective():
    """A quadratic objective in ke: the parabola through the trial points is
    exact, so the step is its vertex; a vertex on the negative side gives 0."""
    eps = np.full((4, 4), 5.0)
    g = np.full((4, 4), 0.01)

    def obj(ke, c=0.3):
        return 2.0 + 3.0 * (ke - c) ** 2

    step, ke, E = steplen.stepparabola(eps, g, obj, obj(0.0), 20.0, 1.0, [1e-3, 10.0], 0.5, 0.5, 5)
    assert len(ke) == 6 and ke[0] == 0.0 and ke.min() < 0 < ke.max()
    assert abs(step - 0.3) < 1e-9
    step, _, _ = steplen.stepparabola(eps, g, lambda k: obj(k, -0.2), obj(0.0, -0.2), 20.0, 1.0, [1e-3, 10.0],
                                      0.5, 0.5, 5)
    assert step == 0.0
    step, _, _ = steplen.stepparabola(eps, g, lambda k: 1.0 + k, 1.0, 20.0, 1.0, [1e-3, 10.0], 0.5, 0.5, 5)
    assert step == 0.0  # a line: no vertex


def test_stepparabola_s_samples_positive_steps_and_keeps_a_negative_vertex():
    """w_stepparabola_s.m: nparabo + 2 trial steps, all positive (both ends come
    from boundstep2(sig, -g_s)); the vertex of a quadratic objective is the step,
    and a negative vertex is returned rather than zeroed."""
    sig = np.full((4, 4), 0.01)
    g = np.full((4, 4), 1.0)

    def obj(k, c):
        return 1.0 + 2.0 * (k - c) ** 2

    step, ks, E = steplen.stepparabola_s(sig, g, lambda k: obj(k, 0.2), obj(0.0, 0.2), 0.1, 1e-4, [1e-2, 1e3],
                                         0.1, 0.9, 3)
    assert len(ks) == 6 and ks[0] == 0.0 and (ks[1:] > 0).all()
    assert abs(step - 0.2) < 1e-9
    step, _, _ = steplen.stepparabola_s(sig, g, lambda k: obj(k, -0.3), obj(0.0, -0.3), 0.1, 1e-4, [1e-2, 1e3],
                                        0.1, 0.9, 3)
    assert abs(step + 0.3) < 1e-9


def test_dc_stepparabola_vertex_and_negative_fallback():
    """dc_stepparabola2_5d.m: four trials around 0, the parabola vertex of a
    quadratic objective; a negative vertex falls back to the best positive
    trial step, or to 0 when the best trial is not positive."""
    sig = np.full((5, 5), 0.01)
    g = np.full((5, 5), 1.0)

    def obj(k, c):
        return 1.0 + 5.0 * (k - c) ** 2

    step, k, E = steplen.dc_stepparabola(sig, g, lambda x: obj(x, 1.0), obj(0.0, 1.0), 0.1, 1e-4, [1e-2, 1e4],
                                         0.5, 0.5)
    assert len(k) == 5 and k.min() < 0 < k.max()
    assert abs(step - 1.0) < 1e-9
    step, k, E = steplen.dc_stepparabola(sig, g, lambda x: obj(x, -1.0), obj(0.0, -1.0), 0.1, 1e-4, [1e-2, 1e4],
                                         0.5, 0.5)
    assert step == 0.0  # vertex at -1, best trial negative
    # a concave objective has a "vertex" that is a maximum; here on the negative side
    step, k, E = steplen.dc_stepparabola(sig, g, lambda x: 10.0 - (x + 1.0) ** 2, 10.0 - 1.0, 0.1, 1e-4,
                                         [1e-2, 1e4], 0.5, 0.5)
    assert step == float(k[int(np.argmin(E))]) and step > 0


def test_dc_misfit_objective_on_the_oracle():
    """dc_objs2_5d.m's trial objective, with the oracle's direct solves standing
    in for the GPU context: at k = 0 it is the normalised misfit of the model,
    0.5 sum e^2 / sum d_obs^2 per source, and data weights scale it."""
    import np_dc_oracle as dco
    from dc_cases import small_dc, oracle_forward
    from gerjoii_b200 import dc as dcm

    case = small_dc(seed=13, pairs=2)
    sig0 = case["SIG"][case["robin"]:-case["robin"], :-case["robin"]]
    for q, r in zip(case["srcs"], oracle_forward(dco, case, case["SIG"] * 1.2)):
        q.d_obs = r[2]

    class Oracle:
        def dc_forward(self, SIG, DX, DZ, robin, srcs):
            return {"d": [r[2] for r in oracle_forward(dco, dict(case, srcs=srcs), SIG)]}

    g = np.ones_like(sig0)
    obj = steplen.dc_misfit_objective(Oracle(), sig0, case["robin"], case["DX"], case["DZ"], case["srcs"], g)
    ref = sum(0.5 * float((r[2] - q.d_obs) @ (r[2] - q.d_obs)) / float(q.d_obs @ q.d_obs)
              for q, r in zip(case["srcs"], oracle_forward(dco, case)))
    assert abs(obj(0.0) - ref) <= 1e-12 * ref
    w = [np.full(q.nd, 2.0) for q in case["srcs"]]
    obj2 = steplen.dc_misfit_objective(Oracle(), sig0, case["robin"], case["DX"], case["DZ"], case["srcs"], g, std=w)
    assert abs(obj2(0.0) - 2 * ref) <= 1e-12 * ref
    assert np.isfinite(obj(1.0)) and obj(1.0) != obj(0.0)


def test_dc_E_objective_transforms():
    """dc_E.m: 0.5 e'Ne on the data, the squared data (env_L22) or the log
    data (env_LOG)."""
    rng = np.random.default_rng(3)
    d_o = rng.uniform(0.5, 2.0, 20)
    d = d_o * (1 + 0.1 * rng.standard_normal(20))
    w = rng.uniform(0.5, 1.5, 20)
    assert abs(steplen.dc_E(d_o, d, w) - 0.5 * np.sum(w * (d - d_o) ** 2)) < 1e-14
    assert abs(steplen.dc_E(d_o, d, None, "env_L22") - 0.5 * np.sum((d ** 2 - d_o ** 2) ** 2)) < 1e-14
    assert abs(steplen.dc_E(d_o, d, w, "env_LOG") - 0.5 * np.sum(w * (np.log(d) - np.log(d_o)) ** 2)) < 1e-14
    with pytest.raises(ValueError):
        steplen.dc_E(d_o, d, None, "L1")


def test_batched_objective_is_used_by_the_searches():
    """An objective with ``many`` is called once per search with all trial
    steps (the batched GPU call) and gives the same step as per-step calls."""
    eps = np.full((6, 7), 9.0)
    g = np.full((6, 7), 0.01)
    calls = []

    class Obj:
        def __call__(self, k):
            return 1.0 + 3.0 * (k - 0.5) ** 2

        def many(self, ks):
            calls.append(len(ks))
            return np.array([self(k) for k in ks])

    s1, _, _ = steplen.stepparabola(eps, g, Obj(), 1.75, 25.0, 1.0, [1e-3, 1e2], 0.5, 0.9, 5)
    s2, _, _ = steplen.stepparabola(eps, g, lambda k: Obj()(k), 1.75, 25.0, 1.0, [1e-3, 1e2], 0.5, 0.9, 5)
    assert calls == [5] and s1 == s2
