#!/usr/bin/env python
"""Benchmark: FWI shot-gradients/s on one B200 (FP32 + checkpointing + batched shots).

Workload (one "step" = one whole FWI gradient over all shots): the 1000 x 400
radar model at dx = 0.02 m with 30 PML cells and a free top (padded 431 x 1060
Yee grid), 6000 time steps, 250 MHz Ricker source, 30 surface sources and 200
receivers, five-layer + blob permittivity, layered conductivity; seeded
synthetic data (no field data).  Each step runs the whole gradient of the 30
shots: the forward solve (shots batched per launch; the u history kept in HBM
in shot groups when it fits, else checkpoints every K steps and a segment
recompute), the residual and misfit, the exact adjoint with the imaging
condition (Kahan-compensated FP32 sums) and the PML-coefficient terms of the
edge cells, and returns the epsilon and sigma gradients.

The timed region runs with kernel timing off; the per-kernel figures and the
roofline come from one more step run afterwards with sampled CUDA events on.
A forward leg times the same acquisition's forward solve alone (temporally
blocked passes against the one-step ring kernels), a cfg1 leg the plain FP64
small-size gradient (GPU plain FP64, GPU FP32 and the oracle), a cfg3 leg the checkpointed
single-shot gradient on the 2000 x 800 grid
(8000 steps, checkpoints every 90 steps), a cfg4 leg the 48 uneven problems in
one gj_w_gradient_batch call (--no-cfg4 skips it; --cfg4 prints it as a line of
its own), and a dc leg the 2.5D DC survey (--no-dc).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Under torchrun (N > 1) the acquisition has 30 x N sources; every rank takes a
round-robin share of 30 shots (gerjoii_b200/shard.py, weak scaling) and the
gradients are summed with one NCCL all-reduce per step.
The reference arm (--impl reference) times the CPU restatement of the
reference (oracle/) on the host cores; rank 0 alone runs it.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "FWI shot-gradients/s & Gcell-upd/s, 1 B200: FP32+ckpt+batch vs plain FP64"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="gerjoii", choices=["gerjoii", "reference"])
    ap.add_argument("--nt", type=int, default=6000)
    ap.add_argument("--nshots", type=int, default=30)
    ap.add_argument("--mode", default="exact", choices=["exact", "reference"])
    ap.add_argument("--no-extras", action="store_true", help="skip the e2e, plain-FP64, DC and CPU legs")
    ap.add_argument("--no-dc", action="store_true", help="skip the DC leg")
    ap.add_argument("--no-cfg4", action="store_true", help="skip the 48-problem batch leg")
    ap.add_argument("--dc-only", action="store_true", help="only the DC leg (JSON line of its own)")
    ap.add_argument("--dc-sources", type=int, default=200, help="DC sources (x 20 wavenumbers)")
    ap.add_argument("--forward-only", action="store_true",
                    help="only the forward leg on --nshots x --nt (JSON line of its own; the profiling case)")
    ap.add_argument("--cfg4", action="store_true",
                    help="the 48 uneven problems instead (one gradient call each, vs plain FP64 on a sample)")
    return ap.parse_args()


def workload(args, world=1):
    from gerjoii_b200 import synth
    p = synth.cfg2(nshots=args.nshots * world, nt=args.nt)
    g = p.grid
    cfg = {"workload": f"radar FWI gradient, {g.n}x{g.m} model (padded {g.NX}x{g.NY} Yee grid), "
                       f"{args.nshots} shots x {len(p.shots[0].rec)} receivers, {g.nt} steps, FP32, "
                       f"{args.mode} adjoint",
           "grid": [g.NX, g.NY], "model": [g.m, g.n], "nt": g.nt, "shots": args.nshots,
           "receivers": len(p.shots[0].rec), "adjoint": args.mode,
           "l2": "working set (fields, checkpoints, history ring) larger than the 126 MB L2; no flush needed",
           "memory_plan": "u history (and the PML band history of the exact adjoint) in HBM in shot groups when "
                          "it fits the memory budget, else checkpoints + segment recompute"}
    return p, cfg


def synth_dobs(p, device=0):
    """Observed traces: the true model's forward response, from the library itself."""
    from gerjoii_b200 import _native as N
    ctx = N.Context(device)
    out = ctx.w_forward(p.grid, p.eps_true, p.sig_true, p.shots, precision=N.GJ_F32)
    ctx.close()
    return out["d"]


class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev):
        self.dev = dev
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) >= 9 and r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            if len(r) < 9:
                continue
            for k, nm in enumerate(names):
                if r[5 + k].strip().lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def band_counts(g):
    """PML band Ez nodes (split fields) and band-frame entries per shot-step
    (the band history of the exact adjoint, csrc/w_band.cuh band_geometry)."""
    NX, NY, P, Pt = g.NX, g.NY, g.pml, g.pml_top
    interior = (NX - P - 1 - Pt) * (NY - 2 * P - 1)
    bnodes = (NX - 1) * (NY - 1) - interior
    bR0, bRB = (NX - P) // 4 * 4, (NX + 3) // 4 * 4
    bsz = 3 * (bRB * 2 * (P + 1) + (bRB - bR0) * (NY + 1))
    return bnodes, bsz


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0}, "fallback"


def traffic_per_unit(kernel):
    """dram bytes per (shot x cell) for `kernel` from the committed ncu summary, or None."""
    try:
        t = json.load(open(os.path.join(ROOT, "profiles", "ncu_traffic.json")))
        e = t[kernel]
        return e["dram_bytes_per_launch"] / e["units_per_launch"]
    except Exception:
        return None


def _cpu_worker(job):
    """One shot of the oracle in a worker process (the reference's parfor worker)."""
    import copy
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from gerjoii_b200 import synth
    from gerjoii_b200.geometry import Shot
    nshots, nt_full, nt_sample, k, mode = job
    p = synth.cfg2(nshots=nshots, nt=nt_full)
    g = copy.copy(p.grid)
    g.nt = nt_sample
    s = p.shots[k % len(p.shots)]
    shot = Shot(s.src_i, s.src_j, s.wavelet[:nt_sample], s.rec)
    dobs = np.random.default_rng(k).standard_normal((1, shot.nr, nt_sample)) * 1e-3
    t0 = time.perf_counter()
    pyoracle.gradient_batch(g, p.eps0, p.sig0, [shot], dobs, mode=mode, precision="f32", threads=1)
    return time.perf_counter() - t0


class CpuPool:
    """Spawned worker processes running the oracle, one shot each per round (the
    reference's parfor pool).  Freed memory stays in each worker's heap, so
    rounds after the first do not pay first-touch page faults again."""

    def __init__(self, threads):
        import multiprocessing as mp
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import pyoracle
        pyoracle.build()
        os.environ.setdefault("MALLOC_MMAP_MAX_", "0")
        os.environ.setdefault("MALLOC_TRIM_THRESHOLD_", str(1 << 40))
        self.threads = threads
        self.pool = mp.get_context("spawn").Pool(threads)

    def sample(self, p, mode, nt_sample):
        """`threads` shots at nt_sample steps; returns (seconds, shot-gradients/s
        scaled to the full nt)."""
        jobs = [(len(p.shots), p.grid.nt, nt_sample, k, mode) for k in range(self.threads)]
        t0 = time.perf_counter()
        self.pool.map(_cpu_worker, jobs, chunksize=1)
        dt = time.perf_counter() - t0
        return dt, self.threads / dt * (nt_sample / p.grid.nt)

    def close(self):
        self.pool.close()
        self.pool.join()


_DC_CASE = {}


def _dc_cpu_worker(job):
    """One DC source (all its wavenumbers) through the oracle's FP64 sparse
    direct solves, in a worker process (one source per host core)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import np_dc_oracle as dco
    from gerjoii_b200 import synth
    n_sources, k = job
    if n_sources not in _DC_CASE:
        _DC_CASE[n_sources] = synth.cfg5(n_sources=n_sources)
    c = _DC_CASE[n_sources]
    q = c["srcs"][k]
    n, m = c["n"], c["m"]
    t0 = time.perf_counter()
    al = [dco.alphas(n, m, c["DX"], c["DZ"], dco.source_vector(n, m, q.a, q.b)[:n], ky) for ky in q.ky_w[:, 0]]
    dco.dc_fwd2_5d(c["SIG"], c["DX"], c["DZ"], dco.source_vector(n, m, q.a, q.b), al, q.ky_w,
                   dco.measuring_operator(n, m, q.mn))
    return time.perf_counter() - t0


def dc_cpu_baseline(n_sources, threads):
    """DC forward solves/s of the oracle on the host cores: `threads` spawned
    workers, one source (x its wavenumbers) each, as BASELINE plans (one
    source per core).  The first round starts the workers and builds the
    survey in each; the second is timed."""
    import multiprocessing as mp
    pool = mp.get_context("spawn").Pool(threads)
    jobs = [(n_sources, k % n_sources) for k in range(threads)]
    pool.map(_dc_cpu_worker, jobs, chunksize=1)
    t0 = time.perf_counter()
    pool.map(_dc_cpu_worker, jobs, chunksize=1)
    dt = time.perf_counter() - t0
    pool.close()
    pool.join()
    return dt


def dc_leg(ctx, n_sources=200):
    """Timed DC forward + sensitivity on the survey; accuracy on one source."""
    import torch
    from gerjoii_b200 import synth
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import np_dc_oracle as dco
    c = synth.cfg5(n_sources=n_sources)
    srcs = c["srcs"]
    fw = ctx.dc_forward(c["SIG"], c["DX"], c["DZ"], c["robin"], srcs)  # warm-up and observed data
    rng = np.random.default_rng(5)
    for q, d in zip(srcs, fw["d"]):
        q.d_obs = d * (1 + 0.02 * rng.standard_normal(d.shape))
    torch.cuda.synchronize()
    ctx.set_kernel_timing(True)
    t0 = time.perf_counter()
    fw = ctx.dc_forward(c["SIG"], c["DX"], c["DZ"], c["robin"], srcs)
    t_f = time.perf_counter() - t0
    kt = {k: ctx.kernel_time(k) for k in ("dc_factor", "dc_precond")}
    ctx.set_kernel_timing(False)
    t0 = time.perf_counter()
    gr = ctx.dc_gradient(c["SIG"], c["DX"], c["DZ"], c["robin"], srcs)
    t_g = time.perf_counter() - t0
    # the FP32 red-black IC(0) preconditioner option on the same forward solves
    from gerjoii_b200 import _native as N
    oi = N.DcOptsC()
    oi.precond = 1
    try:
        t0 = time.perf_counter()
        fi = ctx.dc_forward(c["SIG"], c["DX"], c["DZ"], c["robin"], srcs, opts=oi)
        t_i = time.perf_counter() - t0
        ic0 = {"forward_solves_per_s": len(srcs) * len(srcs[0].ky_w) / t_i, "forward_s": t_i,
               "cg_iterations_max": fi["iters"], "max_rel_residual": fi["rel_residual"],
               "data_rel_diff_vs_band_factor": float(np.linalg.norm(np.concatenate(fi["d"]) - np.concatenate(fw["d"]))
                                                     / np.linalg.norm(np.concatenate(fw["d"]))),
               "preconditioner": "FP32 IC(0), red-black ordering, in FP64 flexible CG (gj_dc_opts.precond = 1)"}
    except Exception as exc:  # reported, not fatal: the default path stays the band factor
        ic0 = {"error": str(exc)[:300]}
    nky = len(srcs[0].ky_w)
    q = srcs[0]
    n, m = c["n"], c["m"]
    al = []
    for ky in q.ky_w[:, 0]:
        s_ = dco.source_vector(n, m, q.a, q.b)
        al.append(dco.alphas(n, m, c["DX"], c["DZ"], s_[:n], ky))
    t0 = time.perf_counter()
    _, _, d_ref, _ = dco.dc_fwd2_5d(c["SIG"], c["DX"], c["DZ"], dco.source_vector(n, m, q.a, q.b), al, q.ky_w,
                                    dco.measuring_operator(n, m, q.mn))
    t_cpu = time.perf_counter() - t0
    rel = float(np.linalg.norm(fw["d"][0] - d_ref) / np.linalg.norm(d_ref))
    threads = min(os.cpu_count() or 1, 32)
    t_par = dc_cpu_baseline(n_sources, threads)
    dc_cpu = {"forward_solves_per_s": threads * nky / t_par, "cores": threads, "kind": "port",
              "sample": f"{threads} sources x {nky} ky on {threads} worker processes (one source each), FP64 "
                        f"sparse direct solves (scipy SuperLU) of the restated operator, operator assembly "
                        f"included ({t_par:.1f} s); one source alone on one core: {nky / t_cpu:.2f} solves/s"}
    # per-kernel device time of the timed forward; algorithmic work per system:
    # factor b(b+1)/2 FMA per unknown, substitution reads the FP64 factor twice
    # (N rounded up to 32 columns of b+1 rounded up to even entries) and moves
    # r (twice), z (write, read, write) in FP64
    N_, b_ = n * m, min(n, m)
    wp_, nq_ = (b_ + 2) // 2 * 2, (N_ + 31) // 32 * 32
    pk, pk_src = peaks()
    kern = {}
    f, pc = kt["dc_factor"], kt["dc_precond"]
    if f["sampled"]:
        sys_per = f["shot_launches"] / f["launches"]
        flops = 2.0 * N_ * b_ * (b_ + 1) / 2 * sys_per
        kern["k_dc_factor"] = {"avg_ms": f["ms"] / f["sampled"], "launches": f["launches"], "systems_per_launch": sys_per,
                               "achieved_fp64_tflops": flops / (f["ms"] / f["sampled"] * 1e-3) / 1e12,
                               "bound": "fp64 issue / shared memory"}
    if pc["sampled"]:
        sys_per = pc["shot_launches"] / pc["launches"]
        byts = (2.0 * nq_ * wp_ * 8 + 5.0 * 8 * N_) * sys_per
        gbs = byts / (pc["ms"] / pc["sampled"] * 1e-3) / 1e9
        kern["k_dc_precond"] = {"avg_ms": pc["ms"] / pc["sampled"], "launches": pc["launches"],
                                "systems_per_launch": sys_per, "bytes_per_launch": byts, "achieved_gbs": gbs,
                                "peak_gbs": pk["hbm_gbs"], "frac": gbs / pk["hbm_gbs"], "peak_source": pk_src,
                                "bound": "hbm"}
    return {"workload": f"2.5D DC, {n - 2}x{m - 1} cells (+Robin), {len(srcs)} sources x {nky} ky, "
                        f"{sum(x.nd for x in srcs)} data",
            "forward_solves_per_s": len(srcs) * nky / t_f, "forward_s": t_f,
            "gradient_solves_per_s": 2 * len(srcs) * nky / t_g, "gradient_s": t_g,
            "cg_iterations_max": max(fw["iters"], gr["iters"]),
            "ic0_option": ic0,
            "max_rel_residual": max(fw["rel_residual"], gr["rel_residual"]),
            "data_rel_err_vs_fp64_direct_solve": rel,
            "kernels": kern,
            "cpu_baseline": dc_cpu,
            "path": "gj_dc_forward / gj_dc_gradient, host buffers"}


def cfg3_leg(ctx):
    """cfg3: the single-shot FP32 exact gradient on the 2000 x 800 grid (30
    PML cells, free top, 8000 steps, 250 MHz), with checkpoints every 90
    steps and the segment recompute (the ~51 GB u history is never held).
    Device-resident inputs, one call timed with CUDA events, kernel timing
    off; then one instrumented call for the per-kernel averages.  Algorithmic
    bytes per shot-gradient (shot-cells of the padded grid per step): forward
    32 B + recompute 32 B + adjoint 32 B + imaging, u slots and adjoint ring
    per model cell."""
    import torch
    from gerjoii_b200 import synth
    from gerjoii_b200 import _native as N
    p = synth.cfg3()
    g = p.grid
    dev = torch.device("cuda", 0)
    d = ctx.w_forward(g, p.eps_true, p.sig_true, p.shots, precision=N.GJ_F32)["d"]
    dobs_t = torch.tensor(np.stack([x.T for x in d]), dtype=torch.float32, device=dev).contiguous()
    eps_t = torch.tensor(np.asfortranarray(p.eps0).ravel(order="F"), dtype=torch.float32, device=dev)
    sig_t = torch.tensor(np.asfortranarray(p.sig0).ravel(order="F"), dtype=torch.float32, device=dev)
    ge = torch.zeros(g.m * g.n, dtype=torch.float32, device=dev)
    gs = torch.zeros_like(ge)
    o = N.OptsC()
    o.ckpt_every = 90
    st = torch.cuda.current_stream(dev)
    run = lambda: ctx.w_gradient_dev(g, eps_t, sig_t, p.shots, dobs_t, ge, gs, mode=N.GJ_ADJ_EXACT, opts=o,
                                     stream=st.cuda_stream)
    ctx.set_kernel_timing(False)
    run()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(st)
    run()
    e1.record(st)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    ctx.set_kernel_timing(True)
    run()
    torch.cuda.synchronize()
    ctx.set_kernel_timing(True)
    run()
    torch.cuda.synchronize()
    kt = {k: ctx.kernel_time(k) for k in ("fwd_step", "adj_step", "image")}
    ctx.set_kernel_timing(False)
    cells, mn = g.NX * g.NY, g.m * g.n
    steps = kt["fwd_step"]["shot_launches"] + kt["adj_step"]["shot_launches"]
    byts = (kt["fwd_step"]["shot_launches"] * (cells * 32.0 + mn * 4.0)
            + kt["adj_step"]["shot_launches"] * (cells * 32.0 + mn * 4.0)
            + kt["adj_step"]["shot_launches"] * mn * 8.0 + kt["image"]["shot_launches"] * mn * 36.0)
    pk, pk_src = peaks()
    per = {k: {"avg_launch_us": v["avg_us"], "launches": v["launches"]} for k, v in kt.items()}
    return {"workload": f"radar FWI gradient, 1 shot, {g.n}x{g.m} model (padded {g.NX}x{g.NY}), {g.nt} steps, "
                        "FP32, exact adjoint, checkpoints every 90 steps + segment recompute",
            "shot_gradients_per_s": 1e3 / ms, "ms_per_gradient": ms,
            "gcell_updates_per_s": steps * cells / (ms / 1e3) / 1e9,
            "forward_plus_recompute_steps": kt["fwd_step"]["shot_launches"], "adjoint_steps": kt["adj_step"]["shot_launches"],
            "recompute_overhead": kt["fwd_step"]["shot_launches"] / g.nt - 1.0,
            "roofline": {"bound": "hbm", "achieved": byts / (ms / 1e3) / 1e9, "peak": pk["hbm_gbs"], "unit": "GB/s",
                         "frac": byts / (ms / 1e3) / 1e9 / pk["hbm_gbs"], "peak_source": pk_src,
                         "algorithmic_bytes_per_gradient": byts,
                         "units": "per shot-step 32 B x NX*NY (forward, recompute, adjoint) + per model cell 4 B "
                                  "(u slot, adjoint ring) + 8 B per imaged step + 36 B per imaging pass"},
            "kernels": per}


def _leg(fn, *args):
    """An extra leg of the bench line; its failure is reported in the line
    instead of losing the line."""
    try:
        return fn(*args)
    except Exception as e:  # reported, not hidden: the key holds the error
        return {"error": f"{type(e).__name__}: {e}"}


def _cfg1_worker(k):
    """One shot of the small-size workload's FP64 exact gradient on the oracle
    (one worker process per shot, the reference's parfor)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from gerjoii_b200 import synth
    p = synth.cfg1()
    g, sh = p.grid, p.shots[k]
    dobs = pyoracle.forward(g, p.eps_true, p.sig_true, sh)[0]
    t0 = time.perf_counter()
    ge, gs, mis = pyoracle.gradient_batch(g, p.eps0, p.sig0, [sh], dobs.T[None], mode="exact", precision="f64",
                                          threads=1)
    return time.perf_counter() - t0, np.asarray(ge), np.asarray(gs)


def cfg1_leg(ctx):
    """The plain FP64 small-size workload (100 x 200 model, 20 PML cells, free
    top, 2000 steps, 5 shots x 50 receivers) in full: the exact gradient of
    the 5 shots as the plain per-shot FP64 GPU form, as the batched FP32 GPU
    form, and on the oracle in FP64 with one host process per shot; the GPU
    gradients against the oracle's."""
    import multiprocessing as mp
    import torch
    from gerjoii_b200 import synth
    from gerjoii_b200 import _native as N
    p = synth.cfg1()
    g = p.grid
    dobs = ctx.w_forward(g, p.eps_true, p.sig_true, p.shots, precision=N.GJ_F64)["d"]
    o_pl = N.OptsC()
    o_pl.plain = 1

    def timed(prec, o):
        ctx.w_gradient(g, p.eps0, p.sig0, p.shots, dobs, mode=N.GJ_ADJ_EXACT, precision=prec, opts=o)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = ctx.w_gradient(g, p.eps0, p.sig0, p.shots, dobs, mode=N.GJ_ADJ_EXACT, precision=prec, opts=o)
        torch.cuda.synchronize()
        return r, time.perf_counter() - t0

    r64, t64 = timed(N.GJ_F64, o_pl)
    r32, t32 = timed(N.GJ_F32, None)
    ctx.release()
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    pyoracle.build()
    with mp.get_context("spawn").Pool(len(p.shots)) as pool:
        t0 = time.perf_counter()
        res = pool.map(_cfg1_worker, range(len(p.shots)), chunksize=1)
        t_cpu = time.perf_counter() - t0
    ge = sum(r[1] for r in res)
    gs = sum(r[2] for r in res)
    rel = lambda a, b: float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b)))
    cos = lambda a, b: float(np.ravel(a) @ np.ravel(b) / (np.linalg.norm(a) * np.linalg.norm(b)))
    ns = len(p.shots)
    upd = 2 * ns * g.nt * g.NX * g.NY
    return {"workload": f"plain FP64 small-size gradient, {g.n}x{g.m} model (padded {g.NX}x{g.NY}), {ns} shots x "
                        f"{len(p.shots[0].rec)} receivers, {g.nt} steps, exact adjoint",
            "gpu_plain_fp64": {"shot_gradients_per_s": ns / t64, "gcell_updates_per_s": upd / t64 / 1e9,
                               "g_eps_rel_l2_vs_oracle": rel(r64["g_eps"], ge),
                               "g_sig_rel_l2_vs_oracle": rel(r64["g_sig"], gs)},
            "gpu_fp32_batched": {"shot_gradients_per_s": ns / t32, "gcell_updates_per_s": upd / t32 / 1e9,
                                 "g_eps_rel_l2_vs_oracle": rel(r32["g_eps"], ge),
                                 "g_eps_cosine_vs_oracle": cos(r32["g_eps"], ge),
                                 "g_sig_rel_l2_vs_oracle": rel(r32["g_sig"], gs)},
            "cpu_oracle_fp64": {"shot_gradients_per_s": ns / t_cpu, "cores": ns, "kind": "port",
                                "sample": f"all {ns} shots, full {g.nt} steps, one process per shot"}}


def forward_leg(ctx, p):
    """The benchmark acquisition's forward solve alone (the plain-forward
    workload: 30 shots x 6000 steps on the 1000 x 400 model, traces of 200
    receivers, FP32), through gj_w_forward with host buffers.  The library's
    tuner picks the temporally blocked passes (k_fwd_tb, D steps per launch on
    shared-memory tiles) or the one-step ring kernels; the ring kernels are
    timed beside it (GJ_TB_DEPTH=0), and the FP32 traces of one shot are
    compared with FP64.  Device time per launch from sampled CUDA events
    (a separate instrumented call); algorithmic bytes per blocked pass: the
    state read and written once (24 B per padded cell) + Ceze, Cezhy (8 B) +
    the split fields of the PML band (16 B per band node), per shot, for D steps."""
    import torch
    from gerjoii_b200 import _native as N
    g = p.grid
    cells = g.NX * g.NY
    bnodes, _ = band_counts(g)
    pk, pk_src = peaks()

    def timed(kind):
        ctx.set_kernel_timing(False)
        ctx.w_forward(g, p.eps0, p.sig0, p.shots, precision=N.GJ_F32)  # plans (and tunes)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        out = ctx.w_forward(g, p.eps0, p.sig0, p.shots, precision=N.GJ_F32)
        t = time.perf_counter() - t0
        launches = ctx.last_launch_count
        ctx.set_kernel_timing(True)
        ctx.w_forward(g, p.eps0, p.sig0, p.shots, precision=N.GJ_F32)
        kt = ctx.kernel_time(kind)
        ctx.set_kernel_timing(False)
        dev_s = kt["avg_us"] * kt["launches"] / 1e6
        return out, t, launches, kt, dev_s

    saved = os.environ.get("GJ_TB_DEPTH")  # a depth fixed by the caller (profiling) stays in force
    out, t, launches, kt, dev_s = timed("tb_pass")
    ns = len(p.shots)
    upd = ns * g.nt * cells
    res = {"workload": f"radar forward, {ns} shots x {len(p.shots[0].rec)} receivers, {g.n}x{g.m} model "
                       f"(padded {g.NX}x{g.NY}), {g.nt} steps, FP32, traces only (gj_w_forward, host buffers)",
           "e2e_shot_forwards_per_s": ns / t, "e2e_s": t, "gpu_launches": launches}
    if kt["launches"] > 0:
        steps_per_pass = g.nt / kt["launches"]
        b = ns * (cells * 32.0 + bnodes * 16.0)
        res.update({
            "kernel": "k_fwd_tb<float,D> (interior and PML tiles of a pass)",
            "steps_per_pass": steps_per_pass, "passes": kt["launches"], "avg_pass_us": kt["avg_us"],
            "device_s": dev_s, "gcell_updates_per_s": upd / dev_s / 1e9,
            "roofline": {"bound": "hbm", "achieved": b / (kt["avg_us"] / 1e6) / 1e9, "peak": pk["hbm_gbs"],
                         "unit": "GB/s", "frac": b / (kt["avg_us"] / 1e6) / 1e9 / pk["hbm_gbs"],
                         "peak_source": pk_src, "algorithmic_bytes_per_pass": b,
                         # DRAM bytes per pass from the ncu capture of a 3-step pass, scaled per shot-cell
                         "traffic": (traffic_per_unit("k_fwd_tb+k_fwd_tbs<float,3>") * ns * cells
                                     if round(steps_per_pass) == 3 and traffic_per_unit("k_fwd_tb+k_fwd_tbs<float,3>")
                                     else None),
                         "step_equivalent_gbs": steps_per_pass * b / (kt["avg_us"] / 1e6) / 1e9,
                         "units": "per shot and pass: 32 B x NX*NY (state once in and out, Ceze/Cezhy) + 16 B x "
                                  "PML band nodes; step_equivalent: the bytes one-step-per-launch kernels move "
                                  "for the same steps"}})
    os.environ["GJ_TB_DEPTH"] = "0"
    try:
        out_r, t_r, _, kt_r, dev_r = timed("fwd_step")
    finally:
        if saved is None:
            os.environ.pop("GJ_TB_DEPTH", None)
        else:
            os.environ["GJ_TB_DEPTH"] = saved
    res["ring_one_step_per_launch"] = {"e2e_s": t_r, "device_s": dev_r, "avg_step_us": kt_r["avg_us"],
                                       "gcell_updates_per_s": upd / dev_r / 1e9 if dev_r > 0 else None}
    if kt["launches"] > 0 and dev_r > 0:
        res["speedup_device_over_ring"] = dev_r / dev_s
    rel = lambda a, b_: float(np.linalg.norm(a - b_) / np.linalg.norm(b_))
    res["traces_rel_l2_blocked_vs_ring"] = max(rel(a, b_) for a, b_ in zip(out["d"], out_r["d"]))
    d64 = ctx.w_forward(g, p.eps0, p.sig0, p.shots[:1], precision=N.GJ_F64)["d"][0]
    res["traces_rel_l2_fp32_vs_fp64_shot0"] = rel(out["d"][0], d64)
    ctx.release()
    return res


def cfg4_leg(ctx=None):
    """cfg4: 48 uneven problems (grids 256..1536 x 128..512, dx 0.02..0.05 m,
    1500..5000 steps, 4..24 shots; blob / layer models), FP32 exact gradients
    with Kahan sums, all of them in one gj_w_gradient_batch call: the problems
    run concurrently in memory-budgeted waves, all waves one CUDA graph launch.
    Timed: one call after a warm-up call (which plans, tunes and captures the
    graph).  Baseline: the plain per-shot FP64 form on one shot of
    every 12th problem, compared per cell-update.  Returns the figures as a
    dict (the bench line's "cfg4" key, or a line of its own with --cfg4)."""
    import torch
    from gerjoii_b200 import synth
    from gerjoii_b200 import _native as N
    probs = synth.cfg4_problems()
    own = ctx is None
    if own:
        ctx = N.Context(0)
    ctx.release()  # the caller's cached plans give their memory back
    data = []
    for p in probs:
        d = ctx.w_forward(p.grid, p.eps_true, p.sig_true, p.shots, precision=N.GJ_F32)["d"]
        data.append(d)
    ctx.release()
    batch = [(p.grid, p.eps0, p.sig0, p.shots, d) for p, d in zip(probs, data)]
    t0 = time.perf_counter()
    ctx.w_gradient_batch(batch, mode=N.GJ_ADJ_EXACT, precision=N.GJ_F32)
    torch.cuda.synchronize()
    t_first = time.perf_counter() - t0
    clocks = Clocks(0)
    clocks.start()
    t0 = time.perf_counter()
    _, nwaves = ctx.w_gradient_batch(batch, mode=N.GJ_ADJ_EXACT, precision=N.GJ_F32)
    torch.cuda.synchronize()
    t = time.perf_counter() - t0
    clk = clocks.stop()
    launches = ctx.last_launch_count
    shots = sum(len(p.shots) for p in probs)
    upd = sum(2 * len(p.shots) * p.grid.nt * p.grid.NX * p.grid.NY for p in probs)
    ctx.release()
    # plain FP64 sample
    o = N.OptsC()
    o.plain = 1
    s_upd, s_t = 0, 0.0
    for p, d in list(zip(probs, data))[::12]:
        ctx.w_gradient(p.grid, p.eps0, p.sig0, p.shots[:1], d[:1], mode=N.GJ_ADJ_EXACT, precision=N.GJ_F64,
                       opts=o)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ctx.w_gradient(p.grid, p.eps0, p.sig0, p.shots[:1], d[:1], mode=N.GJ_ADJ_EXACT, precision=N.GJ_F64,
                       opts=o)
        torch.cuda.synchronize()
        s_t += time.perf_counter() - t0
        s_upd += 2 * p.grid.nt * p.grid.NX * p.grid.NY
    ctx.release()
    if own:
        ctx.close()
    return {"workload": "48 uneven problems (cfg4), one gj_w_gradient_batch call, exact adjoint, FP32",
            "shot_gradients_per_s": shots / t, "ms_per_call": t * 1e3, "gcell_updates_per_s": upd / t / 1e9,
            "problems": len(probs), "shots": shots, "cell_updates": upd, "waves": nwaves,
            "graph_launches_per_call": 1, "gpu_launches": launches, "first_call_s": t_first, "clocks": clk,
            "plain_fp64_sample": {"gcell_updates_per_s": s_upd / s_t / 1e9,
                                  "sample": "1 shot of problems 0, 12, 24, 36, plain per-shot FP64 form",
                                  "speedup_fp32_over_plain_fp64": (upd / t) / (s_upd / s_t)}}


def cfg4_line():
    r = cfg4_leg()
    line = {"metric": "cfg4: 48 uneven radar gradients, shot-gradients/s & Gcell-upd/s, 1 B200",
            "value": r["shot_gradients_per_s"], "unit": "shot-gradients/s", "n_gpus": 1, "steps": 1, "warmup": 1,
            "ms_per_step": r["ms_per_call"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded blob / layer models, observed traces modelled on the device)",
            "config": {"workload": r["workload"], "problems": r["problems"], "shots": r["shots"],
                       "cell_updates": r["cell_updates"], "waves": r["waves"], "first_call_s": r["first_call_s"]},
            "gcell_updates_per_s": r["gcell_updates_per_s"], "gpu_launches": r["gpu_launches"], "clocks": r["clocks"],
            "plain_fp64_sample": r["plain_fp64_sample"]}
    print(json.dumps(line), flush=True)


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    p, cfg = workload(args)
    threads = min(os.cpu_count() or 1, 32)
    nt_sample = max(50, min(args.nt, 150))
    vals = []
    pool = CpuPool(threads)
    for k in range(max(args.warmup, 1) + args.steps):
        dt, v = pool.sample(p, args.mode, nt_sample)
        if k >= max(args.warmup, 1):
            vals.append((dt, v))
    pool.close()
    v = statistics.median([x[1] for x in vals])
    ms = statistics.median([x[0] for x in vals]) * 1e3
    sample = (f"{threads} shots x {nt_sample} of {args.nt} steps per step on {threads} threads "
              f"(C++ oracle, FP32, {args.mode} adjoint); value scaled to the full step count")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "shot-gradients/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded layered model)", "config": cfg,
            "cpu_baseline": {"value": v, "unit": "shot-gradients/s", "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": v, "unit": "shot-gradients/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.cfg4:
        return cfg4_line()
    if args.forward_only:
        from gerjoii_b200 import _native as N
        p, _ = workload(args)
        ctx = N.Context(0)
        print(json.dumps({"metric": "radar forward solve, shot-forwards/s, 1 B200", "forward": forward_leg(ctx, p)}),
              flush=True)
        ctx.close()
        return
    if args.dc_only:
        from gerjoii_b200 import _native as N
        ctx = N.Context(0)
        print(json.dumps({"metric": "2.5D DC solves/s, 1 B200", "dc": dc_leg(ctx, args.dc_sources)}), flush=True)
        return
    import torch
    import torch.distributed as dist
    from gerjoii_b200 import _native as N

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev = torch.device("cuda", local)
    from gerjoii_b200 import shard
    p, cfg = workload(args, world)
    g = p.grid
    if world > 1:
        p.shots = shard.select(p.shots, shard.shard(len(p.shots), rank, world))
        cfg["parallelism"] = (f"dp{world}: shots sharded round-robin, {args.nshots} per GPU (weak), "
                              "one gradient all-reduce per step")
    else:
        cfg["parallelism"] = "1 GPU"
    mode = N.GJ_ADJ_EXACT if args.mode == "exact" else N.GJ_ADJ_REFERENCE
    dobs = synth_dobs(p, local)
    nr = len(p.shots[0].rec)
    dobs_t = torch.tensor(np.stack([d.T for d in dobs]), dtype=torch.float32, device=dev).contiguous()
    eps_t = torch.tensor(np.asfortranarray(p.eps0).ravel(order="F"), dtype=torch.float32, device=dev)
    sig_t = torch.tensor(np.asfortranarray(p.sig0).ravel(order="F"), dtype=torch.float32, device=dev)
    ge_t = torch.zeros(g.m * g.n, dtype=torch.float32, device=dev)
    gs_t = torch.zeros_like(ge_t)
    ctx = N.Context(local)
    stream = torch.cuda.current_stream(dev)

    def step():
        ctx.w_gradient_dev(g, eps_t, sig_t, p.shots, dobs_t, ge_t, gs_t, mode=mode, stream=stream.cuda_stream)
        if world > 1:
            shard.allreduce_sum([ge_t, gs_t])

    # the warm-up captures the CUDA graphs (one per shot group) that the timed
    # steps replay; kernel timing stays off for both, so the timed graphs hold
    # no event nodes
    ctx.set_kernel_timing(False)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    launches = 0
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
        launches += ctx.last_launch_count
    e1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    # instrumented pass after the timed region: one step (after one more that
    # captures the graphs with the timing events) with CUDA events around runs
    # of 8 consecutive launches of a step kernel (one run per 16 launches) and
    # single imaging launches; per-kernel averages and the roofline come from
    # here
    ctx.set_kernel_timing(True)
    step()
    torch.cuda.synchronize()
    ctx.set_kernel_timing(True)  # clears the counters
    isteps = 1
    for _ in range(isteps):
        step()
    torch.cuda.synchronize()
    ktimes = {k: ctx.kernel_time(k) for k in ("fwd_step", "ref_step", "adj_step", "image", "tb_pass")}
    ktimes = {k: v for k, v in ktimes.items() if v["launches"] > 0}
    # a temporally blocked forward (whole history kept) runs every step of every
    # shot in passes of several steps: its shot-steps are the acquisition's
    tb_steps = args.nshots * g.nt * isteps if "tb_pass" in ktimes else 0
    ctx.set_kernel_timing(False)
    if world > 1:
        t = torch.tensor([ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    shots_total = args.nshots * world * args.steps
    value = shots_total / (ms / 1e3)
    cells = g.NX * g.NY
    mn = g.m * g.n
    bnodes, bsz = band_counts(g)
    # cell-updates in the timed region: every forward, recompute and adjoint
    # launch (counted per step in the instrumented pass, which runs the same plan)
    upd = ((sum(ktimes[k]["shot_launches"] for k in ktimes if k not in ("image", "tb_pass")) + tb_steps) / isteps
           * args.steps * cells * world)
    gcell = upd / (ms / 1e3) / 1e9
    # Algorithmic DRAM bytes of each kernel kind over the timed region.
    #  fwd_step (k_fwdw): read Ez, Hx, Hy, Ceze, Cezhy + write Ez, Hx, Hy = 32 B per
    #    padded cell, + 4 B per model node for the history write, + 16 B per PML
    #    band node (split fields Ezx, Ezy read and written), + 4 B per band-frame
    #    entry for the band history write (exact adjoint).
    #  adj_step (k_adjw): the transposed stencil, 32 B per padded cell, + 4 B per
    #    model node for the adjoint-field ring write, + 16 B per band node (split
    #    adjoints), + 4 B per band-frame entry (adjoint band ring write).
    #  image (k_image + k_image_band): per imaged step 8 B per model node and 8 B
    #    per band-frame entry (adjoint ring + history), per launch 36 B per model
    #    node and 20 B per band-frame entry (one more history slot, the
    #    compensated accumulators read and written).
    #  ref_step (k_stepv<float,1>): 32 B per cell + 48 B per model node (4 history
    #    reads, 4 accumulators read and written).
    adj_sl = ktimes.get("adj_step", {}).get("shot_launches", 0)
    exact = args.mode == "exact"
    bz = bsz if exact else 0
    alg = {
        "fwd_step": lambda k: k["shot_launches"] * (cells * 32.0 + mn * 4.0 + bnodes * 16.0 + bz * 4.0),
        "adj_step": lambda k: k["shot_launches"] * (cells * 32.0 + mn * 4.0 + bnodes * 16.0 + bz * 4.0),
        "image": lambda k: adj_sl * (mn + bz) * 8.0 + k["shot_launches"] * (mn * 36.0 + bz * 20.0),
        "ref_step": lambda k: k["shot_launches"] * (cells * 32.0 + mn * 48.0),
        # per shot and pass the state once in and out with Ceze/Cezhy, the split
        # fields of the band; per shot-step the history and band-history writes
        "tb_pass": lambda k: k["shot_launches"] * (cells * 32.0 + bnodes * 16.0) + tb_steps * (mn * 4.0 + bz * 4.0),
    }
    # (a forward or adjoint "launch" is one step: the fast-only and the general
    # ring kernel of that step together)
    kname = {"fwd_step": "k_fwdw<float,2>", "adj_step": "k_adjw<float,2>", "image": "k_image<float>",
             "ref_step": "k_stepv<float,1>", "tb_pass": "k_fwd_tb+k_fwd_tbs<float,3>"}
    pk, pk_src = peaks()
    kern = {}
    for kk, kt in ktimes.items():
        tot_s = kt["avg_us"] * kt["launches"] / 1e6
        b = alg[kk](kt)
        kern[kk] = {"kernel": kname[kk], "launches": kt["launches"], "timed_launches": kt["sampled"],
                    "avg_launch_us": kt["avg_us"], "ms_per_step": tot_s * 1e3 / isteps,
                    "algorithmic_bytes_per_launch": b / max(kt["launches"], 1),
                    "achieved_gbs": b / tot_s / 1e9 if tot_s > 0 else 0.0,
                    "frac_of_measured_hbm": (b / tot_s / 1e9) / pk["hbm_gbs"] if tot_s > 0 else 0.0}
    dom = max(ktimes, key=lambda k: ktimes[k]["avg_us"] * ktimes[k]["launches"])
    kt = ktimes[dom]
    shots_per_launch = kt["shot_launches"] / max(kt["launches"], 1)
    achieved = kern[dom]["achieved_gbs"]
    tpu = traffic_per_unit(kname[dom])
    roof = {"kernel": kname[dom], "bound": "hbm", "achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s",
            "frac": achieved / pk["hbm_gbs"], "peak_source": pk_src,
            "traffic": (tpu * shots_per_launch * cells if tpu is not None else None),
            "algorithmic_bytes_per_launch": kern[dom]["algorithmic_bytes_per_launch"],
            "shots_per_launch": shots_per_launch,
            "launches": kt["launches"], "timed_launches": kt["sampled"], "avg_launch_us": kt["avg_us"],
            "units": {"fwd_step": "per shot: 32 B x NX*NY cells (stencil) + 4 B x m*n history write + 16 B x PML "
                                  "band nodes (split fields) + 4 B x band-frame entries (band history)",
                      "adj_step": "per shot: 32 B x NX*NY cells (stencil) + 4 B x m*n adjoint-field ring write + 16 B "
                                  "x PML band nodes + 4 B x band-frame entries (adjoint band ring)",
                      "image": "per imaged shot-step 8 B x (m*n + band-frame entries), per shot-launch 36 B x m*n + "
                               "20 B x band-frame entries",
                      "ref_step": "per shot: 32 B x NX*NY cells + 48 B x m*n (4 history reads, 4 sums r/w)",
                      "tb_pass": "per shot and pass (several steps): 32 B x NX*NY + 16 B x PML band nodes; per shot-step "
                                 "4 B x m*n history + 4 B x band-frame entries"}[dom],
            "kernel_share_of_step": kt["avg_us"] * kt["launches"] / 1e3 / isteps / (ms / args.steps),
            "pass": "separate instrumented step after the timed region (CUDA events around runs of 8 consecutive "
                    "launches of each step kernel, one run per 16 launches, also inside the graphs; runs that the "
                    "imaging kernel interrupts are dropped); the timed region itself runs without events"}
    line = {"metric": METRIC, "value": value, "unit": "shot-gradients/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded layered model, observed traces modelled on the device)",
            "config": cfg, "gcell_updates_per_s": gcell, "gpu_launches": launches,
            "clocks": clk, "roofline": roof,
            "kernel_ms_per_step": {k: v["avg_us"] * v["launches"] / 1e3 / isteps for k, v in ktimes.items()},
            "kernels": kern}

    if rank == 0 and not args.no_extras:
        # e2e: the public C ABI with host (pinned) buffers, copies inside the timed region
        import ctypes as C
        eps_h = torch.empty(mn, dtype=torch.float64, pin_memory=True).numpy()
        sig_h = torch.empty(mn, dtype=torch.float64, pin_memory=True).numpy()
        eps_h[:] = np.asfortranarray(p.eps0).ravel(order="F")
        sig_h[:] = np.asfortranarray(p.sig0).ravel(order="F")
        dob_h = torch.empty(args.nshots * nr * g.nt, dtype=torch.float64, pin_memory=True).numpy()
        dob_h[:] = np.concatenate([np.asfortranarray(d).ravel(order="F") for d in dobs])
        ge_h = torch.empty(mn, dtype=torch.float64, pin_memory=True).numpy()
        gs_h = torch.empty(mn, dtype=torch.float64, pin_memory=True).numpy()
        mis_h = np.zeros(args.nshots)
        sp = N._ShotPack(p.shots, g.nt)
        gc = N.grid_c(g)
        o = N.OptsC()
        dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))

        def e2e_step():
            st = ctx.lib.gj_w_gradient(ctx.h, C.byref(gc), N.GJ_F32, dp(eps_h), dp(sig_h), sp.arr, sp.n,
                                       dp(dob_h), mode, N.GJ_MISFIT_L2, C.byref(o), dp(ge_h), dp(gs_h),
                                       dp(mis_h), None, None)
            if st != 0:
                raise RuntimeError(ctx.lib.gj_last_error(ctx.h).decode())

        e2e_step()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            e2e_step()
        torch.cuda.synchronize()
        t_e2e = (time.perf_counter() - t0) / args.steps
        line["e2e"] = {"value": args.nshots / t_e2e, "unit": "shot-gradients/s",
                       "h2d_bytes_per_step": int(eps_h.nbytes + sig_h.nbytes + dob_h.nbytes),
                       "d2h_bytes_per_step": int(ge_h.nbytes + gs_h.nbytes + mis_h.nbytes),
                       "ms_per_step": t_e2e * 1e3,
                       "path": "gj_w_gradient (C ABI, host float64 buffers in pinned memory)"}
        # plain per-shot FP64 GPU form on 2 shots, same grid and step count
        o_pl = N.OptsC()
        o_pl.plain = 1
        sub = p.shots[:2]
        r_plain = ctx.w_gradient(g, p.eps0, p.sig0, sub, dobs[:2], mode=mode, precision=N.GJ_F64, opts=o_pl)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r_plain = ctx.w_gradient(g, p.eps0, p.sig0, sub, dobs[:2], mode=mode, precision=N.GJ_F64, opts=o_pl)
        torch.cuda.synchronize()
        t_pl = time.perf_counter() - t0
        r32 = ctx.w_gradient(g, p.eps0, p.sig0, sub, dobs[:2], mode=mode, precision=N.GJ_F32)
        rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
        line["plain_fp64"] = {"value": len(sub) / t_pl, "unit": "shot-gradients/s",
                              "sample": f"{len(sub)} shots, full {g.nt} steps, one half-step per launch, FP64",
                              "speedup_fp32_batched_over_plain_fp64": value / world / (len(sub) / t_pl),
                              "g_eps_rel_l2_fp32_vs_fp64": rel(r32["g_eps"], r_plain["g_eps"]),
                              "g_sig_rel_l2_fp32_vs_fp64": rel(r32["g_sig"], r_plain["g_sig"])}
        # 2.5D DC leg: the full 200-source x 20-ky survey (400 x 100 cells), forward and
        # sensitivity, FP64 CG with FP32 band factors; accuracy against the FP64 direct
        # solve of the oracle on one source
        if not args.no_dc:
            line["dc"] = dc_leg(ctx)
        line["forward"] = _leg(forward_leg, ctx, p)
        line["cfg1"] = _leg(cfg1_leg, ctx)
        line["cfg3"] = cfg3_leg(ctx)
        if not args.no_cfg4:
            line["cfg4"] = cfg4_leg(ctx)
        # CPU baseline (oracle) on the host cores, bounded sample
        threads = min(os.cpu_count() or 1, 32)
        nt_s = max(50, min(args.nt, 150))
        pool = CpuPool(threads)
        pool.sample(p, args.mode, nt_s)  # first round: worker start-up and first-touch memory
        dt_cpu, v_cpu = pool.sample(p, args.mode, nt_s)
        pool.close()
        line["cpu_baseline"] = {"value": v_cpu, "unit": "shot-gradients/s", "cores": threads, "kind": "port",
                                "sample": f"{threads} shots x {nt_s} of {g.nt} steps ({dt_cpu:.1f} s, C++ oracle "
                                          f"FP32 {args.mode} adjoint), scaled to the full step count"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
