"""The radar workloads at their own sizes against the C++ oracle.

- The plain FP64 small-size workload in full: 100 x 200 model at 0.05 m, 20 PML
  cells with a free top, 2000 steps, 100 MHz, 5 surface sources and 50
  receivers, observed traces modelled by the oracle on the true model.  Both
  adjoint modes, every model cell: FP64 gradients within 1e-10 (rel-L2) of the
  oracle's FP64 ones, FP32 within 1e-4 with cosine >= 0.9999, misfits within
  1e-10 (FP64).
- One shot of the 1000 x 400 benchmark acquisition (0.02 m, 30 PML cells,
  6000 steps, 250 MHz, 200 receivers): FP32 traces within 1e-5 (rel-L2) of the
  oracle's FP64 traces, FP64 traces within 1e-12.
"""
import numpy as np
import pytest

from conftest import rel_l2, cosine, edge_cells
from gerjoii_b200 import synth
from gerjoii_b200 import _native as N

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small_workload(oracle):
    p = synth.cfg1()
    dobs = oracle.forward_batch(p.grid, p.eps_true, p.sig_true, p.shots)  # (shots, nr, nt)
    refs = {mode: oracle.gradient_batch(p.grid, p.eps0, p.sig0, p.shots, dobs, mode=mode)
            for mode in ("exact", "reference")}
    return p, [d.T.copy() for d in dobs], refs


@pytest.mark.parametrize("mode", ["exact", "reference"])
def test_small_workload_gradients_match_oracle(gpu_ctx, small_workload, mode):
    p, dobs, refs = small_workload
    ge, gs, mis = refs[mode]
    gm = N.GJ_ADJ_EXACT if mode == "exact" else N.GJ_ADJ_REFERENCE
    r64 = gpu_ctx.w_gradient(p.grid, p.eps0, p.sig0, p.shots, dobs, mode=gm, precision=N.GJ_F64)
    assert rel_l2(r64["g_eps"], ge) <= 1e-10
    assert rel_l2(r64["g_sig"], gs) <= 1e-10
    assert rel_l2(edge_cells(r64["g_eps"]), edge_cells(ge)) <= 1e-9
    assert np.allclose(r64["misfit"], mis, rtol=1e-10)
    r32 = gpu_ctx.w_gradient(p.grid, p.eps0, p.sig0, p.shots, dobs, mode=gm, precision=N.GJ_F32)
    for key, ref in (("g_eps", ge), ("g_sig", gs)):
        assert rel_l2(r32[key], ref) <= 1e-4, key
        assert cosine(r32[key], ref) >= 0.9999, key


def test_benchmark_shot_traces_match_oracle(gpu_ctx, oracle):
    p = synth.cfg2(nshots=1)
    d_ref = oracle.forward_batch(p.grid, p.eps_true, p.sig_true, p.shots)[0].T  # nt x nr
    d32 = gpu_ctx.w_forward(p.grid, p.eps_true, p.sig_true, p.shots, precision=N.GJ_F32)["d"][0]
    d64 = gpu_ctx.w_forward(p.grid, p.eps_true, p.sig_true, p.shots, precision=N.GJ_F64)["d"][0]
    assert rel_l2(d64, d_ref) <= 1e-12
    assert rel_l2(d32, d_ref) <= 1e-5
