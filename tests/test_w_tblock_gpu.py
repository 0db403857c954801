"""Temporally blocked forward passes (k_fwd_tb: D = 1..4 Yee steps per launch
on shared-memory tiles with a D-node halo) against the oracle and against the
one-step ring kernels, through the C ABI.  The grids span several tiles in
both directions, the step counts are not multiples of D (a shorter last
pass), and receivers sit on tile boundaries, in the PML and on the grid's
PEC corners."""
import numpy as np
import pytest

from conftest import rel_l2
from gerjoii_b200 import synth
from gerjoii_b200 import _native as N
from gerjoii_b200.geometry import Shot

pytestmark = pytest.mark.gpu


def _with_receivers(p, extra):
    g = p.grid
    NX1 = g.NX + 1
    lin = [i + j * NX1 for i, j in extra]
    p.shots = [Shot(sh.src_i, sh.src_j, sh.wavelet, np.concatenate([np.asarray(sh.rec, np.int64), lin]))
               for sh in p.shots]
    p.corner0 = [sh.nr - len(lin) for sh in p.shots]  # first of the four corner receivers
    return p


def _extra_nodes(g):
    """Nodes on tile edges of every tile shape (rows 27-34, 55-66, 119-126;
    columns 27-30, 55-62) and on streaming-task row edges (rows 60-66,
    119-130, 240-250), in the bottom and side PML, and the four corners."""
    pts = [(0, 0), (g.NX, g.NY), (g.NX, 0), (0, g.NY), (g.NX - 3, g.NY // 2), (g.NX // 2, 2), (g.NX // 2, g.NY - 2)]
    for i in (27, 28, 33, 34, 55, 56, 60, 61, 62, 63, 65, 66, 119, 120, 121, 122, 123, 124, 125, 126, 127, 128, 130,
              240, 243, 244, 245, 246, 247, 250):
        for j in (27, 28, 29, 30, 55, 56, 61, 62):
            if i < g.NX and j < g.NY:
                pts.append((i, j))
    return pts


@pytest.fixture(scope="module")
def multi_ft():
    p = synth.small(m=130, n=150, pml=10, nt=157, free_top=True, seed=41, nsrc=3, nrec=20)
    return _with_receivers(p, _extra_nodes(p.grid))


@pytest.fixture(scope="module")
def multi_ref():
    p = synth.small(m=110, n=90, pml=12, nt=103, free_top=False, seed=42, nsrc=2, nrec=10)
    return _with_receivers(p, _extra_nodes(p.grid))


@pytest.fixture(scope="module")
def tall_ft():
    """Tall enough for several FP32 streaming row tasks (128 loaded rows each)."""
    p = synth.small(m=290, n=100, pml=10, nt=91, free_top=True, seed=43, nsrc=2, nrec=12)
    return _with_receivers(p, _extra_nodes(p.grid))


@pytest.fixture(scope="module")
def oracle_out(oracle, multi_ft, multi_ref, tall_ft):
    out = {}
    for name, p in (("ft", multi_ft), ("ref", multi_ref), ("tall", tall_ft)):
        out[name] = [oracle.forward(p.grid, p.eps0, p.sig0, sh) for sh in p.shots]
    return out


CFGS = [(D, shape, spb) for D in (1, 2, 3, 4) for shape in (0, 1, 2) for spb in (1, 2)]


def _set(monkeypatch, D, shape, spb):
    monkeypatch.setenv("GJ_TB_DEPTH", str(D))
    monkeypatch.setenv("GJ_TB_SHAPE", str(shape))
    monkeypatch.setenv("GJ_TB_SPB", str(spb))


@pytest.mark.parametrize("D,shape,spb", CFGS)
def test_blocked_forward_f64_matches_oracle(gpu_ctx, multi_ft, oracle_out, monkeypatch, D, shape, spb):
    p = multi_ft
    _set(monkeypatch, D, shape, spb)
    out = gpu_ctx.w_forward(p.grid, p.eps0, p.sig0, p.shots, precision=N.GJ_F64, want_jz=True)
    for k in range(len(p.shots)):
        d, jz, _ = oracle_out["ft"][k]
        assert rel_l2(out["d"][k], d) < 1e-12
        assert rel_l2(out["jz"][k], jz) < 1e-12
        c0 = p.corner0[k]
        assert np.all(out["d"][k][:, c0:c0 + 4] == 0)  # the four PEC corners


@pytest.mark.parametrize("D,shape", [(1, 0), (2, 1), (3, 2), (4, 1)])
def test_blocked_forward_reference_layout_f64(gpu_ctx, multi_ref, oracle_out, monkeypatch, D, shape):
    p = multi_ref
    _set(monkeypatch, D, shape, 1)
    out = gpu_ctx.w_forward(p.grid, p.eps0, p.sig0, p.shots, precision=N.GJ_F64, want_jz=True)
    for k in range(len(p.shots)):
        d, jz, _ = oracle_out["ref"][k]
        assert rel_l2(out["d"][k], d) < 1e-12
        assert rel_l2(out["jz"][k], jz) < 1e-12


@pytest.mark.parametrize("D,shape,spb", [(1, 1, 1), (2, 1, 2), (3, 0, 1), (4, 2, 2)])
def test_blocked_forward_f32_traces(gpu_ctx, multi_ft, oracle_out, monkeypatch, D, shape, spb):
    """FP32 traces within 1e-5 rel-L2 of the FP64 oracle and of the FP32 ring
    kernels (one step per launch)."""
    p = multi_ft
    monkeypatch.setenv("GJ_TB_DEPTH", "0")
    ring = gpu_ctx.w_forward(p.grid, p.eps0, p.sig0, p.shots, precision=N.GJ_F32)
    _set(monkeypatch, D, shape, spb)
    out = gpu_ctx.w_forward(p.grid, p.eps0, p.sig0, p.shots, precision=N.GJ_F32)
    for k in range(len(p.shots)):
        d, _, _ = oracle_out["ft"][k]
        assert rel_l2(out["d"][k], d) < 1e-5
        assert rel_l2(out["d"][k], ring["d"][k]) < 1e-5


STREAM = [(D, lc, shape, ss) for D in (1, 2, 3, 4) for lc, shape, ss in ((8, 0, 3), (20, 1, 6), (64, 0, 6))]


def _set_stream(monkeypatch, D, lc, shape, ss):
    _set(monkeypatch, D, shape, 1)
    monkeypatch.setenv("GJ_TB_STREAM", "1")
    monkeypatch.setenv("GJ_TB_CHUNK", str(lc))
    monkeypatch.setenv("GJ_TB_STAGES", str(ss))


@pytest.mark.parametrize("D,lc,shape,ss", STREAM)
@pytest.mark.parametrize("which", ["ft", "ref", "tall"])
def test_streamed_forward_f64_matches_oracle(gpu_ctx, multi_ft, multi_ref, tall_ft, oracle_out, monkeypatch, D, lc,
                                             shape, ss, which):
    """Streaming warp tasks over the interior (k_fwd_tbs, D levels in
    registers) with clipped tiles around them, FP64 against the oracle."""
    p = {"ft": multi_ft, "ref": multi_ref, "tall": tall_ft}[which]
    _set_stream(monkeypatch, D, lc, shape, ss)
    out = gpu_ctx.w_forward(p.grid, p.eps0, p.sig0, p.shots, precision=N.GJ_F64, want_jz=True)
    for k in range(len(p.shots)):
        d, jz, _ = oracle_out[which][k]
        assert rel_l2(out["d"][k], d) < 1e-12
        assert rel_l2(out["jz"][k], jz) < 1e-12


@pytest.mark.parametrize("D,lc,shape,ss", STREAM)
@pytest.mark.parametrize("which", ["ft", "tall"])
def test_streamed_forward_f32_matches_ring(gpu_ctx, multi_ft, tall_ft, oracle_out, monkeypatch, D, lc, shape, ss,
                                           which):
    """FP32 streaming passes (128-row tasks) against the FP64 oracle (1e-5)
    and the FP32 one-step ring kernels."""
    p = {"ft": multi_ft, "tall": tall_ft}[which]
    monkeypatch.setenv("GJ_TB_DEPTH", "0")
    ring = gpu_ctx.w_forward(p.grid, p.eps0, p.sig0, p.shots, precision=N.GJ_F32, want_jz=True)
    _set_stream(monkeypatch, D, lc, shape, ss)
    out = gpu_ctx.w_forward(p.grid, p.eps0, p.sig0, p.shots, precision=N.GJ_F32, want_jz=True)
    for k in range(len(p.shots)):
        d, jz, _ = oracle_out[which][k]
        assert rel_l2(out["d"][k], d) < 1e-5
        assert rel_l2(out["d"][k], ring["d"][k]) < 1e-5
        assert rel_l2(out["jz"][k], ring["jz"][k]) < 1e-5


def test_blocked_misfit_equals_ring_misfit(gpu_ctx, multi_ft, oracle, monkeypatch):
    p = multi_ft
    dobs = [oracle.forward(p.grid, p.eps_true, p.sig_true, sh)[0] for sh in p.shots]
    monkeypatch.setenv("GJ_TB_DEPTH", "0")
    ring = gpu_ctx.w_misfit(p.grid, p.eps0, p.sig0, p.shots, dobs, precision=N.GJ_F64)
    for D in (2, 4):
        _set(monkeypatch, D, 1, 1)
        tb = gpu_ctx.w_misfit(p.grid, p.eps0, p.sig0, p.shots, dobs, precision=N.GJ_F64)
        assert np.allclose(tb, ring, rtol=1e-12, atol=0)
        trials = gpu_ctx.w_misfit_trials(p.grid, [p.eps0, p.eps_true], [p.sig0, p.sig_true], p.shots, dobs,
                                         precision=N.GJ_F64)
        assert np.allclose(trials[0], ring, rtol=1e-12, atol=0)
        assert np.all(trials[1] < 1e-20)


@pytest.mark.parametrize("misfit,band", [("L2", None), ("env_L2", None), ("L2", (80e6, 500e6))])
@pytest.mark.parametrize("cfg", [(3, 16, 0, 3, 2), (2, 0, 1, 0, 1)])
def test_trial_models_in_one_blocked_run(gpu_ctx, multi_ft, oracle, monkeypatch, misfit, band, cfg):
    """gj_w_misfit_trials with three models: one blocked run whose every pass
    is one launch over the 3 x 3 (model, shot) pairs, each model with its own
    coefficient set, equals the models run one by one with one step per
    launch (FP64, 1e-11), band-filtered and envelope objectives included."""
    p = multi_ft
    g = p.grid
    dobs = [oracle.forward(g, p.eps_true, p.sig_true, sh)[0] for sh in p.shots]
    models = [p.eps0 * f for f in (0.95, 1.0, 1.05)]
    sigs = [p.sig0 * f for f in (1.0, 1.2, 0.8)]
    monkeypatch.setenv("GJ_TB_DEPTH", "0")
    ref = np.stack([gpu_ctx.w_misfit_trials(g, [e], [s_], p.shots, dobs, misfit=misfit, precision=N.GJ_F64,
                                            filt=band)[0] for e, s_ in zip(models, sigs)])
    D, lc, shape, ss, stream = cfg
    _set(monkeypatch, D, shape, 2)
    monkeypatch.setenv("GJ_TB_STREAM", str(stream))
    monkeypatch.setenv("GJ_TB_CHUNK", str(max(lc, 4)))
    monkeypatch.setenv("GJ_TB_STAGES", str(max(ss, 3)))
    got = gpu_ctx.w_misfit_trials(g, models, sigs, p.shots, dobs, misfit=misfit, precision=N.GJ_F64, filt=band)
    launches = gpu_ctx.last_launch_count
    assert got.shape == (3, len(p.shots))
    assert np.allclose(got, ref, rtol=1e-11, atol=0)
    # at most three launches per pass for all three models together (three
    # models run one by one would take at least six per pass)
    passes = -(-g.nt // D)
    assert launches < 5 * passes


@pytest.mark.parametrize("mode", [N.GJ_ADJ_EXACT, N.GJ_ADJ_REFERENCE])
@pytest.mark.parametrize("cfg", [(3, 1, 16, 3), (2, 0, 0, 3), (4, 1, 64, 6), (1, 1, 8, 3)])
@pytest.mark.parametrize("which", ["ft", "tall"])
def test_gradient_with_blocked_forward(gpu_ctx, multi_ft, tall_ft, oracle, monkeypatch, mode, cfg, which):
    """The gradient's forward (whole u history kept) as blocked passes
    (GJ_TB_GRAD=1) that write the u history and the band history of the exact
    adjoint at every step: FP64 gradients of every model cell (edge cells
    included) equal the oracle's to 1e-10 and the one-step ring kernels'
    (GJ_TB_GRAD=0) to 1e-12."""
    p = {"ft": multi_ft, "tall": tall_ft}[which]
    g = p.grid
    dobs = [oracle.forward(g, p.eps_true, p.sig_true, sh)[0] for sh in p.shots]
    ge, gs, mis = oracle.gradient_batch(g, p.eps0, p.sig0, p.shots, np.stack([d.T for d in dobs]),
                                        mode="exact" if mode == N.GJ_ADJ_EXACT else "reference")
    D, stream, lc, ss = cfg
    monkeypatch.setenv("GJ_TB_GRAD", "1")
    _set(monkeypatch, D, 0, 1)
    monkeypatch.setenv("GJ_TB_STREAM", str(stream))
    monkeypatch.setenv("GJ_TB_CHUNK", str(max(lc, 4)))
    monkeypatch.setenv("GJ_TB_STAGES", str(ss))
    res = gpu_ctx.w_gradient(g, p.eps0, p.sig0, p.shots, dobs, mode=mode, precision=N.GJ_F64)
    assert rel_l2(res["g_eps"], ge) < 1e-10 and rel_l2(res["g_sig"], gs) < 1e-10
    assert np.allclose(res["misfit"], mis, rtol=1e-10)
    monkeypatch.setenv("GJ_TB_GRAD", "0")
    ring = gpu_ctx.w_gradient(g, p.eps0, p.sig0, p.shots, dobs, mode=mode, precision=N.GJ_F64)
    assert rel_l2(res["g_eps"], ring["g_eps"]) < 1e-12 and rel_l2(res["g_sig"], ring["g_sig"]) < 1e-12


@pytest.mark.parametrize("mode", [N.GJ_ADJ_EXACT, N.GJ_ADJ_REFERENCE])
def test_gradient_with_blocked_forward_f32(gpu_ctx, multi_ft, oracle, monkeypatch, mode):
    """FP32 gradient with the blocked forward: 1e-4 rel-L2 and cosine >= 1 - 1e-4
    against the FP64 oracle."""
    from conftest import cosine
    p = multi_ft
    g = p.grid
    dobs = [oracle.forward(g, p.eps_true, p.sig_true, sh)[0] for sh in p.shots]
    ge, gs, _ = oracle.gradient_batch(g, p.eps0, p.sig0, p.shots, np.stack([d.T for d in dobs]),
                                      mode="exact" if mode == N.GJ_ADJ_EXACT else "reference")
    monkeypatch.setenv("GJ_TB_GRAD", "1")
    _set_stream(monkeypatch, 3, 16, 0, 3)
    res = gpu_ctx.w_gradient(g, p.eps0, p.sig0, p.shots, dobs, mode=mode, precision=N.GJ_F32)
    for a_, b_ in ((res["g_eps"], ge), (res["g_sig"], gs)):
        assert rel_l2(a_, b_) < 1e-4 and cosine(a_, b_) > 1 - 1e-4


def test_tuned_forward_matches_oracle(gpu_ctx, multi_ft, oracle_out, monkeypatch):
    """No configuration fixed: the tuner picks one (the ring kernels or a
    blocked depth) and the traces still equal the oracle's."""
    p = multi_ft
    for k in ("GJ_TB_DEPTH", "GJ_TB_SHAPE", "GJ_TB_SPB", "GJ_TB_STREAM", "GJ_TB_CHUNK", "GJ_TB_STAGES", "GJ_TB_GRAD",
              "GJ_AUTOTUNE"):
        monkeypatch.delenv(k, raising=False)
    out = gpu_ctx.w_forward(p.grid, p.eps0, p.sig0, p.shots, precision=N.GJ_F64)
    for k in range(len(p.shots)):
        assert rel_l2(out["d"][k], oracle_out["ft"][k][0]) < 1e-12
