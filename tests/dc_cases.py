"""Small seeded DC problems shared by the DC tests."""
import numpy as np

from gerjoii_b200 import dc


def small_dc(seed=0, n0=30, m0=10, robin=1, dx=0.25, n_el=12, pairs=3, levels=3, n_ky=6, blocks=True, spacing=2,
             first=2):
    X = np.arange(n0) * dx
    Z = np.arange(m0) * dx
    DX, DZ = dc.deltas(X, Z, robin)
    rng = np.random.default_rng(seed)
    sig0 = 10 ** (np.log10(0.01) + 0.3 * rng.standard_normal((n0, m0)))
    if blocks:
        sig0[n0 // 3:n0 // 3 + 4, 2:5] *= 5.0
        sig0[2 * n0 // 3:2 * n0 // 3 + 3, 4:7] *= 0.2
    SIG = dc.dc_robin(sig0, robin)
    n, m = SIG.shape
    kyw = dc.ky_weights(dx, n0 * dx, n_ky, dx=dx)
    srcs = dc.dipole_dipole(n, m, robin, DX, DZ, n_electrodes=n_el, spacing_nodes=spacing, first_node=first, pairs=pairs,
                            levels=levels, ky_w=kyw, rng=np.random.default_rng(seed + 1))
    return dict(SIG=SIG, DX=DX, DZ=DZ, robin=robin, srcs=srcs, n=n, m=m)


def oracle_alphas(dco, case, q):
    n, m, DX, DZ = case["n"], case["m"], case["DX"], case["DZ"]
    out = []
    for ky in q.ky_w[:, 0]:
        s = dco.source_vector(n, m, q.a, q.b)
        out.append(dco.alphas(n, m, DX, DZ, s[:n], ky))
    return out


def oracle_forward(dco, case, SIG=None):
    SIG = case["SIG"] if SIG is None else SIG
    n, m = case["n"], case["m"]
    res = []
    for q in case["srcs"]:
        Mop = dco.measuring_operator(n, m, q.mn)
        res.append(dco.dc_fwd2_5d(SIG, case["DX"], case["DZ"], dco.source_vector(n, m, q.a, q.b, q.current),
                                  oracle_alphas(dco, case, q), q.ky_w, Mop, q.d_obs))
    return res
