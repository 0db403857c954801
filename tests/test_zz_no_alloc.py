"""gj_w_forward_noalloc: the forward model for callers that cannot allocate
device memory when they call in (a MEX function inside MATLAB, whose GPU
memory belongs to MATLAB's pool; an application that reserves the whole device
up front).  Its buffers live in a fixed per-device array inside the library.

The test hands it device buffers it allocated itself, calls it twice in a row
through the C ABI and compares each result with gj_w_forward, the allocating
entry point, and with the oracle; a receiver outside the grid is rejected.
The file name sorts last so a run that stops at the first failure has already
run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import rel_l2
from gerjoii_b200 import synth
from gerjoii_b200 import _native as N

pytestmark = pytest.mark.gpu


def _call_noalloc(lib, g, eps_t, sig_t, shot, wav_t, rec_t, d_t):
    import torch
    err = C.create_string_buffer(512)
    gc = N.grid_c(g)
    st = lib.gj_w_forward_noalloc(C.byref(gc), eps_t.data_ptr(), sig_t.data_ptr(), int(shot.src_i),
                                  int(shot.src_j), wav_t.data_ptr(), int(rec_t.numel()), rec_t.data_ptr(),
                                  d_t.data_ptr(), None, err, len(err))
    torch.cuda.synchronize()
    return st, err.value.decode()


@pytest.mark.parametrize("free_top", [True, False])
def test_noalloc_forward_matches_allocating_forward_twice(gpu_ctx, free_top):
    import torch
    p = synth.small(m=24, n=40, pml=8, nt=300, free_top=free_top, seed=31)
    g = p.grid
    lib = N.load()
    dev = torch.device("cuda", 0)
    ref = gpu_ctx.w_forward(g, p.eps0, p.sig0, p.shots, precision=N.GJ_F32)["d"]
    eps_t = torch.tensor(np.asfortranarray(p.eps0).ravel(order="F"), dtype=torch.float32, device=dev)
    sig_t = torch.tensor(np.asfortranarray(p.sig0).ravel(order="F"), dtype=torch.float32, device=dev)
    for k, shot in enumerate(p.shots):
        wav_t = torch.tensor(shot.wavelet[:g.nt], dtype=torch.float32, device=dev)
        rec_nx1 = np.asarray(shot.rec, np.int64)  # 0-based (NX+1)-linear indices
        rec_t = torch.tensor(rec_nx1, dtype=torch.int64, device=dev)
        for _ in range(2):
            d_t = torch.full((shot.nr, g.nt), float("nan"), dtype=torch.float32, device=dev)
            st, msg = _call_noalloc(lib, g, eps_t, sig_t, shot, wav_t, rec_t, d_t)
            assert st == N.GJ_OK, msg
            d = d_t.cpu().numpy().T  # nt x nr
            assert np.isfinite(d).all()
            assert rel_l2(d, ref[k]) < 1e-5


def test_noalloc_rejects_grids_above_its_scratch_limit(gpu_ctx):
    import torch
    p = synth.small(m=24, n=40, pml=8, nt=50, seed=32)
    g = p.grid
    g.m, g.n = 2000, 2000  # far above the fixed scratch size
    lib = N.load()
    dev = torch.device("cuda", 0)
    eps_t = torch.ones(g.m * g.n, dtype=torch.float32, device=dev)
    shot = p.shots[0]
    wav_t = torch.zeros(g.nt, dtype=torch.float32, device=dev)
    rec_t = torch.zeros(1, dtype=torch.int64, device=dev)
    d_t = torch.zeros((1, g.nt), dtype=torch.float32, device=dev)
    st, msg = _call_noalloc(lib, g, eps_t, eps_t, shot, wav_t, rec_t, d_t)
    assert st == N.GJ_EINVAL
    assert "limit" in msg


def test_noalloc_forward_matches_oracle_with_last_node_receiver(gpu_ctx, oracle):
    """Traces against the FP64 oracle (FP32 bound 1e-5 rel-L2), with one
    receiver on the last Ez node of the padded grid ((NX+1)(NY+1) - 1, on the
    PEC corner: an all-zero trace) beside surface receivers."""
    import torch
    from gerjoii_b200.geometry import Shot
    p = synth.small(m=24, n=40, pml=8, nt=300, free_top=True, seed=34)
    g = p.grid
    last = (g.NX + 1) * (g.NY + 1) - 1
    sh = p.shots[0]
    shot = Shot(sh.src_i, sh.src_j, sh.wavelet, np.concatenate([np.asarray(sh.rec, np.int64), [last]]))
    d_ref, _, _ = oracle.forward(g, p.eps0, p.sig0, shot)
    dev = torch.device("cuda", 0)
    eps_t = torch.tensor(np.asfortranarray(p.eps0).ravel(order="F"), dtype=torch.float32, device=dev)
    sig_t = torch.tensor(np.asfortranarray(p.sig0).ravel(order="F"), dtype=torch.float32, device=dev)
    wav_t = torch.tensor(shot.wavelet[:g.nt], dtype=torch.float32, device=dev)
    rec_t = torch.tensor(np.asarray(shot.rec, np.int64), dtype=torch.int64, device=dev)
    for _ in range(2):
        d_t = torch.full((shot.nr, g.nt), float("nan"), dtype=torch.float32, device=dev)
        st, msg = _call_noalloc(N.load(), g, eps_t, sig_t, shot, wav_t, rec_t, d_t)
        assert st == N.GJ_OK, msg
        d = d_t.cpu().numpy().T
        assert rel_l2(d, d_ref) < 1e-5
        assert np.all(d[:, -1] == 0)


def test_noalloc_rejects_receivers_outside_the_grid(gpu_ctx):
    """A receiver index past the last Ez node (or negative) is never read:
    the call returns GJ_EINVAL and every trace sample is NaN; the next call
    with valid receivers works again."""
    import torch
    p = synth.small(m=24, n=40, pml=8, nt=60, free_top=True, seed=35)
    g = p.grid
    dev = torch.device("cuda", 0)
    eps_t = torch.tensor(np.asfortranarray(p.eps0).ravel(order="F"), dtype=torch.float32, device=dev)
    sig_t = torch.tensor(np.asfortranarray(p.sig0).ravel(order="F"), dtype=torch.float32, device=dev)
    shot = p.shots[0]
    wav_t = torch.tensor(shot.wavelet[:g.nt], dtype=torch.float32, device=dev)
    lib = N.load()
    for bad in ((g.NX + 1) * (g.NY + 1), -1):
        rec = np.asarray(shot.rec, np.int64).copy()
        rec[1] = bad
        rec_t = torch.tensor(rec, dtype=torch.int64, device=dev)
        d_t = torch.zeros((len(rec), g.nt), dtype=torch.float32, device=dev)
        st, msg = _call_noalloc(lib, g, eps_t, sig_t, shot, wav_t, rec_t, d_t)
        assert st == N.GJ_EINVAL and "outside" in msg, msg
        assert torch.isnan(d_t).all()
    rec_t = torch.tensor(np.asarray(shot.rec, np.int64), dtype=torch.int64, device=dev)
    d_t = torch.zeros((shot.nr, g.nt), dtype=torch.float32, device=dev)
    st, msg = _call_noalloc(lib, g, eps_t, sig_t, shot, wav_t, rec_t, d_t)
    assert st == N.GJ_OK, msg
    assert torch.isfinite(d_t).all()
