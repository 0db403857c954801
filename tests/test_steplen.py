"""Step-length host logic (CPU): w_boundstep2.m's bound search and
w_stepparabola_e.m's parabola vertex, on models and objectives with known
answers."""
import numpy as np

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
