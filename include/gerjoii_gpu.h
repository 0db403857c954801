/*
 * gerjoii_gpu.h — C ABI of the B200 (sm_100a) radar full-waveform gradient path
 * and the 2.5D DC-resistivity solves.
 *
 * Every entry point replaces one MATLAB function of the reference
 * (diegozain/gerjoii); the function it replaces is cited beside it as
 * path:line inside that project.  A MEX gateway (mex/gj_mex.c) unpacks the
 * reference's structs and calls these functions, so the reference's L2 layer
 * (w_update_e.m, w_update_s.m, dc_update2_5d.m, ...) keeps its call sites.
 *
 * Conventions
 *  - Arrays are column-major (MATLAB order); the fastest index is depth (i).
 *  - The padded Yee grid has NX = pml_top + air + m + pml rows and
 *    NY = n + 2*pml columns (wdc_geom.m:69-70); Ez nodes are (NX+1) x (NY+1).
 *  - All node indices are 0-based (MATLAB index - 1).  A receiver is a linear
 *    Ez node index i + j*(NX+1), i.e. gerjoii_.w.M - 1 (w_M.m:20).
 *  - Host pointers are double precision; `precision` selects the arithmetic
 *    (GJ_F32 fields and stencils, or GJ_F64).
 *  - Every function returns a gj_status; gj_last_error(ctx) gives the text.
 *  - A context is used by one host thread at a time; several contexts may
 *    share a device.  There is no global mutable state.
 */
#ifndef GERJOII_GPU_H
#define GERJOII_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum gj_status {
  GJ_OK = 0,
  GJ_EINVAL = 1,      /* invalid argument (sizes, indices, null pointers) */
  GJ_ENOMEM = 2,      /* device memory could not be allocated */
  GJ_ENUMERIC = 3,    /* NaN or Inf detected in a result */
  GJ_ETIMEOUT = 4,    /* a bounded device wait expired */
  GJ_ECUDA = 5,       /* CUDA runtime error */
  GJ_EUNSUPPORTED = 6 /* option not supported by this build */
} gj_status;

typedef enum gj_precision { GJ_F32 = 0, GJ_F64 = 1 } gj_precision;

/* REFERENCE: w_grad.m semantics (sigma-flipped forward-type propagation of the
 * time-reversed residual hard-set at the receivers; g_eps from d/dt u, g_sig
 * from u).  EXACT: transpose of the discrete Yee/PML update, i.e. the true
 * gradient of 0.5*sum (d - d_obs)^2 with respect to eps_r and sigma. */
typedef enum gj_adj_mode { GJ_ADJ_REFERENCE = 0, GJ_ADJ_EXACT = 1 } gj_adj_mode;

/* Objective / adjoint source, the reference's obj_FNC (w_bozdag.m:13-54; misfits
 * by w_E.m:7-16 on what w_fwd.m:34-35 stores): L2 on the traces, env_L2 on the
 * envelopes, phase_L2 on the instantaneous phases, env_L22 on the squared
 * envelopes, env_LOG on the log envelopes. */
typedef enum gj_misfit_kind {
  GJ_MISFIT_L2 = 0, GJ_MISFIT_ENV_L2 = 1, GJ_MISFIT_PHASE_L2 = 2, GJ_MISFIT_ENV_L22 = 3, GJ_MISFIT_ENV_LOG = 4
} gj_misfit_kind;

typedef struct gj_ctx gj_ctx;

/* Padded Yee grid (wdc_geom.m:35-125, generalised with pml_top). */
typedef struct gj_w_grid {
  int m, n;      /* model rows (depth) and columns (lateral) */
  int pml;       /* PML cells bottom/left/right (pml_w == pml_d) */
  int pml_top;   /* PML rows on top: == pml (reference layout) or 0 (free top) */
  int air;       /* air rows (eps_r = 1, sigma = 0) above the model; >= 1 for a free top */
  int nt;        /* time steps */
  double dx, dy, dt;
  double eps0, mu0; /* parame_.w.eps_0, parame_.w.mu_0 (param_wdc.m:28-29) */
  int order;        /* PML grading order, 2 in wdc_geom.m:98 */
  double R0;        /* PML reflection, 1e-8 in wdc_geom.m:99 */
} gj_w_grid;

/* One shot (gerjoii_.w.s, gerjoii_.w.wvlet_, gerjoii_.w.M). */
typedef struct gj_w_shot {
  int src_i, src_j;       /* source Ez node, 0-based (gerjoii_.w.s - 1) */
  const double* wavelet;  /* nt samples (w_wavelet.m) */
  int nr;                 /* receivers */
  const long* rec;        /* nr linear Ez node indices, 0-based (gerjoii_.w.M - 1) */
} gj_w_shot;

/* Options for the gradient; zero-initialise for the defaults. */
typedef struct gj_w_opts {
  int ckpt_every;        /* checkpoint interval K in steps; 0 = automatic: keep the whole
                            u history when it fits mem_budget_bytes, else checkpoint */
  size_t mem_budget_bytes; /* 0 = 80% of free device memory */
  int shots_per_launch;  /* shots advanced together per kernel launch; 0 = automatic */
  int no_kahan;          /* 1 = plain FP32 sums for the imaging condition */
  int no_graph;          /* 1 = launch the time loop without CUDA graphs */
  int per_shot;          /* 1 = g_eps/g_sig hold nshots gradients (m*n each), else their sum */
  int plain;             /* 1 = the plain form: one half-step per launch, one shot at a time */
  int no_ring;           /* 1 = register-marching step kernels instead of the warp-task ring
                            kernels (the default for 16-byte vectors: FP32 and FP64) */
  double filt_low;       /* Gaussian band filter of the residual before the adjoint
                            (filt_gauss.m, as w_update_e.m:69-70 applies it to e_2d): band
                            [filt_low, filt_high] in Hz, on when filt_high > filt_low; the
                            misfit stays that of the unfiltered residual */
  double filt_high;
  int filt_steep;        /* exponent of the filter; 0 = 8 (w_update_e.m:70) */
  int condition;         /* 1 = condition every shot's gradients as w_update_e.m:99-137 and
                            w_update_s.m:96-137 do (source taper gaussi.m of width
                            4 c/sqrt(eps_r(source))/cond_fo, k-space low-pass image_gaussian.m,
                            normali.m, zero on NaN), then return their mean over shots
                            (w_update_e_.m:38), or each of them with per_shot */
  double cond_fo;        /* source frequency of the taper width, Hz (regu.fo) */
  double cond_ax, cond_az; /* image_gaussian widths for eps (regu.ax, regu.az); sigma uses twice
                              these (w_update_s.m:105-106) */
} gj_w_opts;

/* ---------------------------------------------------------------- context */
gj_status gj_context_create(gj_ctx** ctx, int device);
gj_status gj_context_destroy(gj_ctx* ctx);
/* Frees the device memory a context keeps between calls (the cached radar plan
 * with its history, checkpoints and graphs, the batch plans with their pool and
 * graph, and the DC band factors and CG vectors, tens of GB for a large survey)
 * and keeps the context usable; the
 * next call plans and allocates again.  No counterpart in the reference
 * (MATLAB's clear / reset between phases of an inversion). */
gj_status gj_context_release(gj_ctx* ctx);
const char* gj_last_error(const gj_ctx* ctx);
const char* gj_version(void);

/* ------------------------------------------------------------ radar (GPR) */

/* Forward model for nshots shots: replaces w_fwd.m:18-24 / w_solve.m:80-124
 * (and w_solve_.m with is == 0 when u_out is NULL).
 *   eps_r, sigma : m x n model (parame_.w.epsilon, parame_.w.sigma)
 *   d_out        : per shot nt x nr traces, shots concatenated (gerjoii_.w.d_2d)
 *   jz_out       : per shot nt samples of Ez at the source (gerjoii_.w.Jy), may be NULL
 *   u_out        : per shot m x n x nt history (gerjoii_.w.u_2d), may be NULL */
gj_status gj_w_forward(gj_ctx* ctx, const gj_w_grid* grid, gj_precision precision,
                       const double* eps_r, const double* sigma, const gj_w_shot* shots,
                       int nshots, double* d_out, double* jz_out, double* u_out);

/* Whole gradient for nshots shots in one call: forward with checkpoints, the
 * residual and misfit (w_fwd.m:34-35 via w_bozdag.m, w_E.m, w_update_e.m:74-76),
 * then the adjoint and imaging condition.  In GJ_ADJ_REFERENCE mode this is
 * w_update_es.m's pair of calls: g_eps = w_grad(d/dt u) (w_update_e.m:83-98)
 * and g_sig = w_grad(u) (w_update_s.m:77).  In GJ_ADJ_EXACT mode g_eps and
 * g_sig are dJ/d(eps_r) and dJ/d(sigma) of J = 0.5*sum (d - d_obs)^2 (or of the
 * envelope misfit).
 *   d_obs   : per shot nt x nr observed traces (parame_.natu.w.d_2d)
 *   g_eps, g_sig : m x n (or nshots x m x n with opts->per_shot)
 *   misfit  : nshots normalised misfits, may be NULL
 *   d_out, e_out : per shot nt x nr modelled traces and adjoint sources, may be NULL */
gj_status gj_w_gradient(gj_ctx* ctx, const gj_w_grid* grid, gj_precision precision,
                        const double* eps_r, const double* sigma, const gj_w_shot* shots,
                        int nshots, const double* d_obs, gj_adj_mode mode,
                        gj_misfit_kind misfit, const gj_w_opts* opts, double* g_eps,
                        double* g_sig, double* misfit_out, double* d_out, double* e_out);

/* One independent problem of gj_w_gradient_batch: its own grid, model,
 * shots, observed traces and outputs (host arrays, as gj_w_gradient). */
typedef struct gj_w_problem {
  gj_w_grid grid;
  const double* eps_r;     /* m x n */
  const double* sigma;     /* m x n */
  const gj_w_shot* shots;
  int nshots;
  const double* d_obs;     /* per shot nt x nr, shots concatenated */
  double* g_eps;           /* m x n, summed over the problem's shots */
  double* g_sig;           /* m x n */
  double* misfit;          /* nshots normalised misfits, may be NULL */
} gj_w_problem;

/* Gradients of many independent problems of uneven sizes in one call: the
 * reference runs such inversions as separate parfor workers and Slurm jobs
 * (w_update_e_.m:32 per shot, one MATLAB process per field line).  The
 * problems run concurrently in memory-budgeted waves (a wave's problems
 * share one device pool; the next wave starts when the previous one ends),
 * and all waves are one CUDA graph launch holding every problem's whole
 * gradient (forward, residual, recompute, exact or reference adjoint,
 * imaging; all its shots per launch); a problem keeps its whole u history
 * when its wave's memory allows, else it checkpoints.  Plans, buffers and the
 * graph are cached in the context
 * while the problems (grids and shots) repeat.  L2 misfit; opts: no_kahan and
 * mem_budget_bytes (the pool budget, 0 = 80% of free memory) apply, the plain,
 * no_ring, filter, conditioning and per_shot options do not (GJ_EUNSUPPORTED).
 *   nwaves : number of waves used, may be NULL */
gj_status gj_w_gradient_batch(gj_ctx* ctx, gj_precision precision, const gj_w_problem* probs, int nprob,
                              gj_adj_mode mode, const gj_w_opts* opts, int* nwaves);

/* Forward runs and misfits only (no history, no adjoint): replaces the
 * objective evaluations of the step-length search, w_objs_e.m:24-65 as called
 * by w_stepparabola_e.m:20-41 for each trial model.  misfit_out: nshots
 * misfits normalised as in w_update_e.m:75-76, of the quantity the misfit kind
 * compares (traces, envelopes, phases). */
gj_status gj_w_misfit(gj_ctx* ctx, const gj_w_grid* grid, gj_precision precision,
                      const double* eps_r, const double* sigma, const gj_w_shot* shots,
                      int nshots, const double* d_obs, gj_misfit_kind misfit, double* misfit_out);

/* Objective values of several trial models for the step-length search:
 * replaces the nparabo calls of w_objs_e.m:24-65 (and w_objs_s.m) that
 * w_stepparabola_e.m:20-27 / w_stepparabola_s.m make, each a forward run of
 * every shot followed by the misfit.
 *   eps_r, sigma : ntrial models, m x n each, concatenated (the perturbed
 *                  parame_.w.epsilon of w_objs_e.m:24-25)
 *   opts         : may be NULL; filt_low < filt_high band-filters both the
 *                  modelled and the observed traces first (filt_gauss.m with
 *                  exponent filt_steep, 0 = 8), as w_objs_e.m:33-36 does with
 *                  regu.f_ and regu.f__; the misfit and its d_o'd_o normaliser
 *                  are then those of the filtered traces
 *   misfit_out   : ntrial x nshots misfits, trial-major
 * With ntrial > 1 all models run as one temporally blocked forward run: each
 * pass is one launch per kernel kind over every (model, shot) pair, each model
 * with its own coefficient set (unless GJ_TB_DEPTH=0 fixes one step per
 * launch, which runs the models one by one). */
gj_status gj_w_misfit_trials(gj_ctx* ctx, const gj_w_grid* grid, gj_precision precision, int ntrial,
                             const double* eps_r, const double* sigma, const gj_w_shot* shots, int nshots,
                             const double* d_obs, gj_misfit_kind misfit, const gj_w_opts* opts,
                             double* misfit_out);

/* Backward half of the forward/backward pair gj_w_forward -> gj_w_backward:
 * the adjoint of the forward map applied to given adjoint sources, the role of
 * [g, a_max] = w_grad(u_w, ...) after w_fwd in the reference (w_grad.m:1,
 * called by w_update_e.m:98 and w_update_s.m:77), for nshots shots at once.
 *   e     : per shot nt x nr adjoint sources, shots concatenated (the residual
 *           e_2d of w_fwd.m:34, or any dJ/dd)
 *   mode  : GJ_ADJ_EXACT gives g = (dd/d eps_r)^T e and (dd/d sigma)^T e, the
 *           PML-coefficient terms of the edge cells included; GJ_ADJ_REFERENCE
 *           gives w_grad.m's g_eps = w_grad(d/dt u), g_sig = w_grad(u)
 *   opts  : as gj_w_gradient (memory plan, per_shot, conditioning, band filter
 *           of e); misfit options do not apply
 * The forward wavefield is recomputed from the model inside the call with the
 * same memory plan as gj_w_gradient (whole history or checkpoints): the exact
 * adjoint needs the forward's PML split fields and strip H fields besides the
 * model-domain u history that gj_w_forward returns.  For w_grad(u) on a
 * caller-supplied u of one shot, see gj_w_grad. */
gj_status gj_w_backward(gj_ctx* ctx, const gj_w_grid* grid, gj_precision precision, const double* eps_r,
                        const double* sigma, const gj_w_shot* shots, int nshots, const double* e,
                        gj_adj_mode mode, const gj_w_opts* opts, double* g_eps, double* g_sig);

/* The adjoint half on its own: replaces [g, a_max] = w_grad(u, ...) (w_grad.m:1-115)
 * for one shot.  u is the m x n x nt history (or its time derivative), e the
 * nt x nr residual.  a_max may be NULL.  Reference semantics only. */
gj_status gj_w_grad(gj_ctx* ctx, const gj_w_grid* grid, gj_precision precision,
                    const double* eps_r, const double* sigma, const gj_w_shot* shot,
                    const double* e, const double* u, double* g, double* a_max);

/* Device-pointer gradient for callers that keep everything in HBM (the torch
 * test harness and the benchmark).  Pointers are device memory of the chosen
 * precision (float or double); d_obs is nshots x nr x nt... laid out per shot
 * as nt x nr.  misfit_out is a host array of nshots doubles, may be NULL.
 * stream is a cudaStream_t (NULL = legacy default stream). */
gj_status gj_w_gradient_dev(gj_ctx* ctx, const gj_w_grid* grid, gj_precision precision,
                            const void* eps_r_dev, const void* sigma_dev,
                            const gj_w_shot* shots, int nshots, const void* d_obs_dev,
                            gj_adj_mode mode, gj_misfit_kind misfit, const gj_w_opts* opts,
                            void* g_eps_dev, void* g_sig_dev, double* misfit_out,
                            void* stream);

/* -------------------------------------------------- 2.5D DC resistivity */

/* Finite-volume grid of dc_fwd2_5d.m: n = finite_.dc.nx lateral nodes and
 * m = finite_.dc.nz depth nodes, both including the Robin padding
 * (wdc_geom.m:76-77, dc_robin.m).  Arrays are n x m with the lateral index
 * fastest; node (l, h) (0-based) is the vectorised unknown l + h*n
 * (coordP.m).  dx and dz are DELTAS(:,:,1) and DELTAS(:,:,2) exactly as
 * do_grid.m computes them (dx is negative for robin = 1 when the model starts
 * at x = 0; the operator uses the value as given). */
typedef struct gj_dc_grid {
  int n, m;     /* nodes incl. Robin padding */
  int robin;    /* Robin padding (parame_.dc.robin): the gradient drops robin
                   columns on each side and robin rows at the bottom */
  int n_ky;     /* wavenumbers per source */
  double dx, dz;
} gj_dc_grid;

/* Number of compact Robin coefficients per (source, ky):
 * [ALPHAS(1,2:m-1) | ALPHAS(2:n-1,m) | ALPHAS(n,2:m-1) | corners(1,1) corners(2,1)
 *  corners(1,2) corners(2,2)] of dc_Lk.m's private alphas (:945-960). */
#define GJ_DC_NALPHA(n, m) (2 * ((m) - 2) + ((n) - 2) + 4)

/* One current dipole and its measurements (gerjoii_.dc.s, .r, dc_M.m). */
typedef struct gj_dc_src {
  long a, b;             /* +I and -I electrode nodes, 0-based, after binning, the
                            parity clean and the Robin shift of dc_electrodes.m */
  double current;        /* I (dc_electrodes.m:54) */
  int nd;                /* measurements */
  const long* mn;        /* nd pairs (M, N) of 0-based nodes: d = u(M) - u(N) (dc_M.m) */
  const double* ky;      /* n_ky wavenumbers (finite_.dc.ky_w_(:,1)) */
  const double* w;       /* n_ky weights (finite_.dc.ky_w_(:,2)) */
  const double* alpha;   /* n_ky x GJ_DC_NALPHA(n, m) Robin coefficients, ky-major */
  const double* d_obs;   /* nd observed data (parame_.natu.dc.d); needed by the gradient */
} gj_dc_src;

typedef struct gj_dc_opts {
  double tol;              /* relative residual of every solve; 0 = 1e-10 */
  int max_iter;            /* CG iterations; 0 = 50 */
  int per_source;          /* 1 = one gradient per source, else their sum */
  int sources_per_batch;   /* 0 = as many as fit mem_budget_bytes */
  size_t mem_budget_bytes; /* 0 = 70% of free device memory */
  int factor_fp32;         /* 1 = FP32 band factor as the preconditioner (half the memory;
                              converges slowly for the smallest ky), else FP64 */
  int precond;             /* 0 = band LDL^T factor of each system (FP64, or FP32 with
                              factor_fp32); 1 = FP32 incomplete Cholesky IC(0) in red-black
                              ordering (no factorisation pass, N floats per system; many
                              more CG iterations); the CG itself is FP64 in both cases */
} gj_dc_opts;

typedef struct gj_dc_stats {
  int max_iterations;      /* largest CG iteration count over all solves */
  double max_rel_residual; /* largest final FP64 relative residual */
} gj_dc_stats;

/* Forward: replaces [gerjoii_, finite_] = dc_fwd2_5d(parame_, finite_, gerjoii_)
 * (dc_fwd2_5d.m:35-63) for nsrc sources at once.
 *   sigma : n x m padded conductivity (parame_.dc.sigma_robin)
 *   d_out : sum(nd) data, sources concatenated (gerjoii_.dc.d)
 *   u_out : nsrc x n x m stacked potentials (gerjoii_.dc.u), may be NULL
 *   stats : may be NULL */
gj_status gj_dc_forward(gj_ctx* ctx, const gj_dc_grid* grid, const double* sigma,
                        const gj_dc_src* srcs, int nsrc, const gj_dc_opts* opts,
                        double* d_out, double* u_out, gj_dc_stats* stats);

/* gj_dc_forward that also returns the per-wavenumber potentials
 * gerjoii_.dc.u_k of dc_fwd2_5d.m:61 (dc_fwd_k.m:43 for every ky).
 *   uk_out : nsrc x n_ky x (n*m), per source the column-major (n*m) x n_ky u_k
 *            (the potential of wavenumber ky_k in column k), may be NULL
 * The other arguments are gj_dc_forward's. */
gj_status gj_dc_forward_k(gj_ctx* ctx, const gj_dc_grid* grid, const double* sigma, const gj_dc_src* srcs,
                          int nsrc, const gj_dc_opts* opts, double* d_out, double* u_out, double* uk_out,
                          gj_dc_stats* stats);

/* Sensitivity: replaces dc_fwd2_5d followed by
 * gerjoii_ = dc_gradient2_5d(parame_, finite_, gerjoii_) (dc_gradient2_5d.m:18-41).
 *   g_out  : (n - 2 robin) x (m - robin) gradient (sum over sources, or nsrc of
 *            them with opts->per_source) (gerjoii_.dc.g)
 *   d_out, e_out : sum(nd) data and residuals d - d_obs, may be NULL
 *   misfit_out   : nsrc values 0.5 e'e, may be NULL */
gj_status gj_dc_gradient(gj_ctx* ctx, const gj_dc_grid* grid, const double* sigma,
                         const gj_dc_src* srcs, int nsrc, const gj_dc_opts* opts,
                         double* g_out, double* d_out, double* e_out, double* misfit_out,
                         gj_dc_stats* stats);

/* Robin coefficients of one source for every wavenumber, written to alpha_out
 * in the layout gj_dc_src.alpha takes (n_ky x GJ_DC_NALPHA(n, m), ky-major):
 * the private alphas of dc_Lk.m:820-960 (called by dc_Lk.m:236-520), which
 * MATLAB code outside dc_Lk.m cannot call.  a_node, b_node are the source
 * electrodes as in gj_dc_src (on the surface row); ky as gj_dc_src.ky.
 * Computed on the host: needs no context and no GPU. */
gj_status gj_dc_alphas(const gj_dc_grid* grid, long a_node, long b_node, const double* ky,
                       double* alpha_out);

/* Scratch limit of gj_w_forward_noalloc, in bytes (32 MiB): enough for a
 * padded grid of about 380 000 Ez nodes (for example 600 x 600). */
#define GJ_W_NOALLOC_SCRATCH_BYTES (32u << 20)

/* Single-shot FP32 forward model that allocates no device memory.  It has no
 * counterpart in the reference.  It is meant for callers that cannot allocate
 * device memory when they call in: a MEX function inside MATLAB, whose GPU
 * memory belongs to MATLAB's own pool, or an application that reserves the
 * whole device up front and treats any later cudaMalloc as an error.
 *   - All pointers except grid and errbuf are device pointers supplied by the
 *     caller: eps_dev, sigma_dev (m x n floats, column-major), wavelet_dev
 *     (nt floats), rec_dev (nr 0-based (NX+1)-linear Ez node indices) and
 *     d_out_dev (nt x nr floats, written).
 *   - Intermediate buffers live in one fixed array of
 *     GJ_W_NOALLOC_SCRATCH_BYTES per device, held by every GPU that loads the
 *     library until the process exits.  Grids that need more are rejected with
 *     GJ_EINVAL and a message in errbuf (may be NULL).
 *   - Every call made outside stream capture looks up the array's device
 *     address (cudaGetSymbolAddress) with the calling thread's current device,
 *     so a context re-created after cudaDeviceReset (MATLAB's
 *     reset(gpuDevice)) gets its own address; a call made while `stream` is
 *     being captured reuses the address of the last uncaptured call on that
 *     device, so make the first call on a device before any stream capture.
 *   - Receivers must be Ez nodes, 0 <= rec < (NX+1)(NY+1).  They are checked
 *     on the device before the time loop and the result read back, which
 *     waits for the work already queued on `stream`; a call with a receiver
 *     outside the grid returns GJ_EINVAL and fills d_out_dev with NaN.
 *   - Calls share the array: work is queued on `stream` (a cudaStream_t, NULL
 *     = legacy default stream), and calls that overlap on the GPU, from any
 *     thread or stream, race on it.  Each call clears the fields it needs. */
gj_status gj_w_forward_noalloc(const gj_w_grid* grid, const float* eps_dev, const float* sigma_dev,
                               int src_i, int src_j, const float* wavelet_dev, int nr,
                               const long* rec_dev, float* d_out_dev, void* stream, char* errbuf,
                               size_t errlen);

/* Number of kernel launches issued by the last call on this context (for the
 * benchmark's launch count).  Graph launches count the kernels they contain. */
long gj_last_launch_count(const gj_ctx* ctx);

/* Per-kernel device timing, accumulated over calls while enabled: CUDA events
 * around runs of 8 consecutive launches of each radar step kernel (one run per
 * 16 launches; a run that another timed kernel interrupts is dropped), around
 * every 16th launch of the other radar kernels (inside captured graphs too)
 * and around every launch of the DC factor and substitution.
 * kind: 0 forward Yee step, 1 reference-adjoint step, 2 exact-adjoint step,
 * 3 receiver I/O, 4 plain kernels, 5 DC band factor, 6 radar imaging,
 * 7 DC band substitution (preconditioner apply), 8 temporally blocked forward
 * pass (one launch advancing up to 4 steps; every 4th pass timed, both tile
 * kernels of the pass inside the bracket).  gj_kernel_time returns the
 * summed milliseconds of the timed launches, their number (ms / sampled is
 * the average launch duration), the number of launches of that kind, and the sum over
 * those launches of the shots each one advanced.  No counterpart in the
 * reference (MATLAB tic/toc around whole phases, w_begin_.m:74-76). */
gj_status gj_set_kernel_timing(gj_ctx* ctx, int on);
gj_status gj_kernel_time(const gj_ctx* ctx, int kind, double* ms, long* sampled, long* launches,
                         long* shot_launches);

#ifdef __cplusplus
}
#endif
#endif /* GERJOII_GPU_H */
