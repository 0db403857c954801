"""Warp-task ring kernels (the default step kernels for FP32 and FP64)
against the register-marching kernels and the oracle, on grids tall enough
for several row blocks per column, so the halo rows, the fast and general
paths, the column chunks and the imaging windows are all exercised."""
import numpy as np
import pytest

from conftest import rel_l2, edge_cells
from gerjoii_b200 import synth
from gerjoii_b200 import _native as N

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=[True, False], ids=["free_top", "ref_layout"])
def tall(request):
    return synth.small(m=150, n=44, pml=10, nt=260, nsrc=3, nrec=10, free_top=request.param, seed=31)


def _dobs(oracle, p):
    return [oracle.forward(p.grid, p.eps_true, p.sig_true, sh)[0] for sh in p.shots]


@pytest.mark.parametrize("prec", [N.GJ_F64, N.GJ_F32])
def test_ring_kernels_match_marching_kernels(gpu_ctx, oracle, tall, prec):
    p = tall
    dobs = _dobs(oracle, p)
    o = N.OptsC()
    o.no_ring = 1
    a = gpu_ctx.w_gradient(p.grid, p.eps0, p.sig0, p.shots, dobs, mode=N.GJ_ADJ_EXACT, precision=prec, opts=o,
                           want_traces=True)
    b = gpu_ctx.w_gradient(p.grid, p.eps0, p.sig0, p.shots, dobs, mode=N.GJ_ADJ_EXACT, precision=prec,
                           want_traces=True)
    # same arithmetic per node, up to the compiler's fused multiply-adds
    tol = 1e-12 if prec == N.GJ_F64 else 2e-6
    for x, y in zip(a["d"], b["d"]):
        assert rel_l2(y, x) < tol
    if prec == N.GJ_F64:
        # the eps imaging differences consecutive fields; next to the sources
        # that cancellation turns rounding differences into ~1e-10 of the gradient
        assert rel_l2(b["g_eps"], a["g_eps"]) < 1e-9
        assert rel_l2(b["g_sig"], a["g_sig"]) < 1e-9
    # (FP32 gradients: on this short record with sources one row under the
    # surface, FP32 itself -- the C++ oracle in FP32 included -- differs from
    # FP64 by ~10 % in the source rows, so two FP32 roundings are not compared
    # here; the FP32 oracle checks of test_w_gpu.py run through these kernels)


@pytest.mark.parametrize("ckpt", [0, 13])
def test_ring_exact_gradient_matches_oracle(gpu_ctx, oracle, tall, ckpt):
    p = tall
    g = p.grid
    dobs = _dobs(oracle, p)
    ge, gs, _ = oracle.gradient_batch(g, p.eps0, p.sig0, p.shots, np.stack([d.T for d in dobs]), mode="exact")
    o = N.OptsC()
    o.ckpt_every = ckpt
    res = gpu_ctx.w_gradient(g, p.eps0, p.sig0, p.shots, dobs, mode=N.GJ_ADJ_EXACT, precision=N.GJ_F64, opts=o)
    # the eps imaging sums l (E^k - E^{k-1}): cancellation between consecutive
    # fields puts the FP64 agreement near 1e-10 on this 150-row grid
    assert rel_l2(res["g_eps"], ge) < 1e-9
    assert rel_l2(res["g_sig"], gs) < 1e-9
    assert rel_l2(edge_cells(res["g_eps"]), edge_cells(ge)) < 1e-9


def test_ring_forward_api_matches_oracle(gpu_ctx, oracle, tall):
    p = tall
    out = gpu_ctx.w_forward(p.grid, p.eps0, p.sig0, p.shots, precision=N.GJ_F64, want_u=True)
    for k, sh in enumerate(p.shots):
        d, _, u = oracle.forward(p.grid, p.eps0, p.sig0, sh, store_u=True)
        assert rel_l2(out["d"][k], d) < 1e-12
        assert rel_l2(out["u"][k], u) < 1e-12


def test_ring_edge_receivers_and_sources_match_oracle(gpu_ctx, oracle):
    """Receivers the fused record / injection must handle: the same node twice,
    inside the left and bottom PML, on the Ez = 0 top row, on the last interior
    row, on the boundary column and row; a source inside the PML (no effect,
    w_solve.m:92-94); a shot without receivers.  FP64 traces and per-shot exact
    gradients (all cells) against the oracle."""
    from gerjoii_b200.geometry import Shot
    p = synth.small(m=150, n=44, pml=10, nt=220, nsrc=2, nrec=6, free_top=True, seed=33)
    g = p.grid
    NX, NY = g.NX, g.NY
    node = g.node
    w = p.shots[0].wavelet
    recA = np.array([node(1, 30), node(1, 30), node(50, 3), node(NX - 3, 30), node(0, 20),
                     node(NX - g.pml - 1, 40), node(70, 0), node(NX, 25), node(5, 12)], np.int64)
    shots = [Shot(2, 30, w, recA),
             Shot(100, 5, w, p.shots[1].rec),          # source in the left PML band
             Shot(3, 22, w, np.zeros(0, np.int64))]    # no receivers
    dobs = [oracle.forward(g, p.eps_true, p.sig_true, sh)[0] for sh in shots]
    out = gpu_ctx.w_forward(g, p.eps0, p.sig0, shots, precision=N.GJ_F64)
    o = N.OptsC()
    o.per_shot = 1
    res = gpu_ctx.w_gradient(g, p.eps0, p.sig0, shots, dobs, mode=N.GJ_ADJ_EXACT, precision=N.GJ_F64, opts=o,
                             want_traces=True)
    for k, sh in enumerate(shots):
        d, _, _ = oracle.forward(g, p.eps0, p.sig0, sh)
        if sh.nr:
            assert rel_l2(out["d"][k], d) < 1e-12
            assert rel_l2(res["d"][k], d) < 1e-12
        e = d - dobs[k]
        ge, gs = oracle.grad_exact(g, p.eps0, p.sig0, sh, e)
        if sh.nr == 0:
            assert np.abs(res["g_eps"][k]).max() == 0 and np.abs(res["g_sig"][k]).max() == 0
            continue
        assert rel_l2(res["g_eps"][k], ge) < 1e-9
        assert rel_l2(res["g_sig"][k], gs) < 1e-9


@pytest.mark.parametrize("ckpt", [0, 11])
def test_ring_reference_adjoint_matches_marching_and_oracle(gpu_ctx, oracle, tall, ckpt):
    """w_grad semantics (GJ_ADJ_REFERENCE) on the ring kernels with windowed
    imaging: equal to the register-marching kernels with per-step imaging and
    to the oracle, with and without checkpoints."""
    p = tall
    g = p.grid
    dobs = _dobs(oracle, p)
    o = N.OptsC()
    o.ckpt_every = ckpt
    r = gpu_ctx.w_gradient(g, p.eps0, p.sig0, p.shots, dobs, mode=N.GJ_ADJ_REFERENCE, precision=N.GJ_F64, opts=o)
    o.no_ring = 1
    m = gpu_ctx.w_gradient(g, p.eps0, p.sig0, p.shots, dobs, mode=N.GJ_ADJ_REFERENCE, precision=N.GJ_F64, opts=o)
    assert rel_l2(r["g_eps"], m["g_eps"]) < 1e-10
    assert rel_l2(r["g_sig"], m["g_sig"]) < 1e-10
    ge, gs, _ = oracle.gradient_batch(g, p.eps0, p.sig0, p.shots, np.stack([d.T for d in dobs]), mode="reference")
    assert rel_l2(r["g_eps"], ge) < 1e-9
    assert rel_l2(r["g_sig"], gs) < 1e-9
