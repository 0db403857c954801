/*
 * gj_mex.c - MATLAB gateway over the C ABI in include/gerjoii_gpu.h.
 *
 * One MEX binary, dispatched on its first argument; the .m files in this folder
 * keep the reference's function signatures (w_solve, w_grad, w_gradient_es,
 * dc_fwd2_5d, dc_gradient2_5d) and unpack the reference's structs into the
 * plain arrays passed here.  All index arguments arrive 1-based (MATLAB) and
 * are converted to the ABI's 0-based convention here.
 *
 * Build (MATLAB, with the CUDA library built by python -m gerjoii_b200.build):
 *   mex -I../include gj_mex.c -L../gerjoii_b200/_lib -lgerjoii_b200
 */
#include <stdlib.h>
#include <string.h>

#include "mex.h"
#include "gerjoii_gpu.h"

static gj_ctx* g_ctx = NULL;

static void cleanup(void) {
  if (g_ctx) gj_context_destroy(g_ctx);
  g_ctx = NULL;
}

static gj_ctx* ctx(void) {
  if (!g_ctx) {
    if (gj_context_create(&g_ctx, 0) != GJ_OK) mexErrMsgIdAndTxt("gerjoii:cuda", "no CUDA device");
    mexAtExit(cleanup);
  }
  return g_ctx;
}

static void check(gj_status st) {
  if (st != GJ_OK) mexErrMsgIdAndTxt("gerjoii:abi", "%s", gj_last_error(g_ctx));
}

static double field(const mxArray* s, const char* name) {
  const mxArray* f = mxGetField(s, 0, name);
  if (!f) mexErrMsgIdAndTxt("gerjoii:arg", "missing field %s", name);
  return mxGetScalar(f);
}

/* grid struct: m n pml pml_top air nt dx dy dt eps0 mu0 (order, R0 optional) */
static gj_w_grid wgrid(const mxArray* s) {
  gj_w_grid g;
  memset(&g, 0, sizeof g);
  g.m = (int)field(s, "m"); g.n = (int)field(s, "n"); g.pml = (int)field(s, "pml");
  g.pml_top = (int)field(s, "pml_top"); g.air = (int)field(s, "air"); g.nt = (int)field(s, "nt");
  g.dx = field(s, "dx"); g.dy = field(s, "dy"); g.dt = field(s, "dt");
  g.eps0 = field(s, "eps0"); g.mu0 = field(s, "mu0");
  g.order = mxGetField(s, 0, "order") ? (int)field(s, "order") : 2;
  g.R0 = mxGetField(s, 0, "R0") ? field(s, "R0") : 1e-8;
  return g;
}

/* shot from s_w = [i j] (1-based), M (1-based linear Ez indices), wavelet */
/* gerjoii_.w.obj_FNC (w_fwd.m:33) -> misfit kind; FREQstp is L2 (w_bozdag.m:13). */
static gj_misfit_kind misfit_kind(const mxArray* a) {
  char s[16];
  if (mxGetString(a, s, sizeof s)) mexErrMsgIdAndTxt("gerjoii:arg", "obj_FNC must be a short string");
  if (!strcmp(s, "L2") || !strcmp(s, "FREQstp")) return GJ_MISFIT_L2;
  if (!strcmp(s, "env_L2")) return GJ_MISFIT_ENV_L2;
  if (!strcmp(s, "phase_L2")) return GJ_MISFIT_PHASE_L2;
  if (!strcmp(s, "env_L22")) return GJ_MISFIT_ENV_L22;
  if (!strcmp(s, "env_LOG")) return GJ_MISFIT_ENV_LOG;
  mexErrMsgIdAndTxt("gerjoii:arg", "unknown obj_FNC '%s'", s);
  return GJ_MISFIT_L2;
}

static gj_w_shot wshot(const mxArray* s_w, const mxArray* M, const mxArray* wav, long** rec_out) {
  gj_w_shot q;
  const double* s = mxGetPr(s_w);
  const double* m = mxGetPr(M);
  const size_t nr = mxGetNumberOfElements(M);
  long* rec = (long*)mxMalloc((nr ? nr : 1) * sizeof(long));
  for (size_t r = 0; r < nr; ++r) rec[r] = (long)m[r] - 1;
  q.src_i = (int)s[0] - 1;
  q.src_j = (int)s[1] - 1;
  q.wavelet = mxGetPr(wav);
  q.nr = (int)nr;
  q.rec = rec;
  *rec_out = rec;
  return q;
}

/* Shots of a batched call: S (ns x 2) source nodes, Mcell{k} receivers, one
   wavelet for all, Dcell{k} nt x nr observed traces packed shot after shot.
   The caller frees recs[k], recs, the shots and dobs with mxFree. */
static gj_w_shot* pack_shots(const mxArray* S, const mxArray* Mcell, const mxArray* wav, const mxArray* Dcell, int nt,
                             long*** recs_out, double** dobs_out, int* ns_out) {
  const int ns = (int)mxGetM(S);
  gj_w_shot* shots = (gj_w_shot*)mxMalloc(ns * sizeof(gj_w_shot));
  long** recs = (long**)mxMalloc(ns * sizeof(long*));
  size_t ntot = 0;
  for (int k = 0; k < ns; ++k) ntot += (size_t)nt * mxGetNumberOfElements(mxGetCell(Mcell, k));
  double* dobs = (double*)mxMalloc((ntot ? ntot : 1) * sizeof(double));
  size_t o = 0;
  for (int k = 0; k < ns; ++k) {
    double sw[2] = {mxGetPr(S)[k], mxGetPr(S)[k + ns]};
    mxArray* swa = mxCreateDoubleMatrix(1, 2, mxREAL);
    memcpy(mxGetPr(swa), sw, sizeof sw);
    shots[k] = wshot(swa, mxGetCell(Mcell, k), wav, &recs[k]);
    mxDestroyArray(swa);
    memcpy(dobs + o, mxGetPr(mxGetCell(Dcell, k)), (size_t)nt * shots[k].nr * sizeof(double));
    o += (size_t)nt * shots[k].nr;
  }
  *recs_out = recs;
  *dobs_out = dobs;
  *ns_out = ns;
  return shots;
}

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  char cmd[64];
  if (nrhs < 1 || mxGetString(prhs[0], cmd, sizeof cmd)) mexErrMsgIdAndTxt("gerjoii:arg", "gj_mex(command, ...)");
  gj_precision prec = GJ_F32;
  if (!strcmp(cmd, "w_solve")) {
    /* [d, u, Jz] = gj_mex('w_solve', eps, sigma, grid, s_w, M, wavelet)   (w_solve.m:80-124) */
    gj_w_grid g = wgrid(prhs[3]);
    long* rec;
    gj_w_shot q = wshot(prhs[4], prhs[5], prhs[6], &rec);
    plhs[0] = mxCreateDoubleMatrix(g.nt, q.nr, mxREAL);
    mwSize du[3] = {(mwSize)g.m, (mwSize)g.n, (mwSize)g.nt};
    double* u = NULL;
    if (nlhs > 1) { plhs[1] = mxCreateNumericArray(3, du, mxDOUBLE_CLASS, mxREAL); u = mxGetPr(plhs[1]); }
    double* jz = NULL;
    if (nlhs > 2) { plhs[2] = mxCreateDoubleMatrix(g.nt, 1, mxREAL); jz = mxGetPr(plhs[2]); }
    check(gj_w_forward(ctx(), &g, prec, mxGetPr(prhs[1]), mxGetPr(prhs[2]), &q, 1, mxGetPr(plhs[0]), jz, u));
    mxFree(rec);
  } else if (!strcmp(cmd, "w_grad")) {
    /* [g, a_max] = gj_mex('w_grad', eps, sigma, grid, s_w, M, e, u)   (w_grad.m:1-115) */
    gj_w_grid g = wgrid(prhs[3]);
    long* rec;
    gj_w_shot q = wshot(prhs[4], prhs[5], prhs[6], &rec); /* wavelet unused by the adjoint */
    plhs[0] = mxCreateDoubleMatrix(g.m, g.n, mxREAL);
    double* am = NULL;
    if (nlhs > 1) { plhs[1] = mxCreateDoubleMatrix(g.m, g.n, mxREAL); am = mxGetPr(plhs[1]); }
    check(gj_w_grad(ctx(), &g, prec, mxGetPr(prhs[1]), mxGetPr(prhs[2]), &q, mxGetPr(prhs[7]), mxGetPr(prhs[8]),
                    mxGetPr(plhs[0]), am));
    mxFree(rec);
  } else if (!strcmp(cmd, "w_gradient")) {
    /* [g_eps, g_sig, E] = gj_mex('w_gradient', eps, sigma, grid, S (ns x 2), Mcell, wavelet, dobs_cell, mode,
                                  obj_FNC)
       (w_update_es.m's w_fwd + w_grad pair for every shot at once; obj_FNC 'L2' by default) */
    gj_w_grid g = wgrid(prhs[3]);
    long** recs;
    double* dobs;
    int ns;
    gj_w_shot* shots = pack_shots(prhs[4], prhs[5], prhs[6], prhs[7], g.nt, &recs, &dobs, &ns);
    const gj_adj_mode mode = nrhs > 8 ? (gj_adj_mode)(int)mxGetScalar(prhs[8]) : GJ_ADJ_REFERENCE;
    const gj_misfit_kind mk = nrhs > 9 ? misfit_kind(prhs[9]) : GJ_MISFIT_L2;
    plhs[0] = mxCreateDoubleMatrix(g.m, g.n, mxREAL);
    plhs[1] = mxCreateDoubleMatrix(g.m, g.n, mxREAL);
    plhs[2] = mxCreateDoubleMatrix(ns, 1, mxREAL);
    check(gj_w_gradient(ctx(), &g, prec, mxGetPr(prhs[1]), mxGetPr(prhs[2]), shots, ns, dobs, mode, mk,
                        NULL, mxGetPr(plhs[0]), mxGetPr(plhs[1]), mxGetPr(plhs[2]), NULL, NULL));
    for (int k = 0; k < ns; ++k) mxFree(recs[k]);
    mxFree(recs); mxFree(shots); mxFree(dobs);
  } else if (!strcmp(cmd, "w_backward")) {
    /* [g_eps, g_sig] = gj_mex('w_backward', eps, sigma, grid, S (ns x 2), Mcell, wavelet, e_cell, mode)
       (the backward half of the pair w_solve -> w_backward: the adjoint of the forward map applied to
        the residuals e_2d of every shot, w_grad.m:1 after w_fwd.m; mode 1 = exact adjoint, the default) */
    gj_w_grid g = wgrid(prhs[3]);
    long** recs;
    double* e;
    int ns;
    gj_w_shot* shots = pack_shots(prhs[4], prhs[5], prhs[6], prhs[7], g.nt, &recs, &e, &ns);
    const gj_adj_mode mode = nrhs > 8 ? (gj_adj_mode)(int)mxGetScalar(prhs[8]) : GJ_ADJ_EXACT;
    plhs[0] = mxCreateDoubleMatrix(g.m, g.n, mxREAL);
    plhs[1] = mxCreateDoubleMatrix(g.m, g.n, mxREAL);
    check(gj_w_backward(ctx(), &g, prec, mxGetPr(prhs[1]), mxGetPr(prhs[2]), shots, ns, e, mode, NULL,
                        mxGetPr(plhs[0]), mxGetPr(plhs[1])));
    for (int k = 0; k < ns; ++k) mxFree(recs[k]);
    mxFree(recs); mxFree(shots); mxFree(e);
  } else if (!strcmp(cmd, "w_misfit")) {
    /* E = gj_mex('w_misfit', eps, sigma, grid, S (ns x 2), Mcell, wavelet, dobs_cell, obj_FNC)
       (the forward-only objective of every shot for a trial model, w_objs_e.m:24-65) */
    gj_w_grid g = wgrid(prhs[3]);
    long** recs;
    double* dobs;
    int ns;
    gj_w_shot* shots = pack_shots(prhs[4], prhs[5], prhs[6], prhs[7], g.nt, &recs, &dobs, &ns);
    const gj_misfit_kind mk = nrhs > 8 ? misfit_kind(prhs[8]) : GJ_MISFIT_L2;
    plhs[0] = mxCreateDoubleMatrix(ns, 1, mxREAL);
    check(gj_w_misfit(ctx(), &g, prec, mxGetPr(prhs[1]), mxGetPr(prhs[2]), shots, ns, dobs, mk, mxGetPr(plhs[0])));
    for (int k = 0; k < ns; ++k) mxFree(recs[k]);
    mxFree(recs); mxFree(shots); mxFree(dobs);
  } else if (!strcmp(cmd, "w_misfit_trials")) {
    /* E = gj_mex('w_misfit_trials', EPS, SIG, grid, S (ns x 2), Mcell, wavelet, dobs_cell, obj_FNC, band)
       (the nparabo trial objectives of one w_stepparabola_e.m search, w_objs_e.m:24-65 for every trial
        model, in one call: EPS and SIG hold the trial models (m x n x ntrial); band = [f_low f_high steep]
        band-filters both trace sets first as w_objs_e.m:33-36 does; E is ns x ntrial) */
    gj_w_grid g = wgrid(prhs[3]);
    long** recs;
    double* dobs;
    int ns;
    gj_w_shot* shots = pack_shots(prhs[4], prhs[5], prhs[6], prhs[7], g.nt, &recs, &dobs, &ns);
    const gj_misfit_kind mk = nrhs > 8 ? misfit_kind(prhs[8]) : GJ_MISFIT_L2;
    const size_t mn = (size_t)g.m * (size_t)g.n;
    const int ntrial = (int)(mxGetNumberOfElements(prhs[1]) / mn);
    if (ntrial < 1 || mxGetNumberOfElements(prhs[2]) != (size_t)ntrial * mn)
      mexErrMsgIdAndTxt("gerjoii:arg", "EPS and SIG must hold the same number of m x n trial models");
    gj_w_opts o;
    memset(&o, 0, sizeof o);
    if (nrhs > 9 && mxGetNumberOfElements(prhs[9]) >= 2) {
      o.filt_low = mxGetPr(prhs[9])[0];
      o.filt_high = mxGetPr(prhs[9])[1];
      if (mxGetNumberOfElements(prhs[9]) >= 3) o.filt_steep = (int)mxGetPr(prhs[9])[2];
    }
    plhs[0] = mxCreateDoubleMatrix(ns, ntrial, mxREAL);
    check(gj_w_misfit_trials(ctx(), &g, prec, ntrial, mxGetPr(prhs[1]), mxGetPr(prhs[2]), shots, ns, dobs, mk, &o,
                             mxGetPr(plhs[0])));
    for (int k = 0; k < ns; ++k) mxFree(recs[k]);
    mxFree(recs); mxFree(shots); mxFree(dobs);
  } else if (!strcmp(cmd, "dc_fwd2_5d") || !strcmp(cmd, "dc_gradient2_5d")) {
    /* [d, u, u_k] = gj_mex('dc_fwd2_5d', sigma_robin, dcgrid, AB (ns x 2, 1-based), I, MNcell, kyw_cell,
                            alpha_cell)   (u_k: (n*m) x n_ky x ns, gerjoii_.dc.u_k of dc_fwd2_5d.m:61)
       (alpha_cell = [] has the library compute dc_Lk.m's alphas, gj_dc_alphas)
       [g, d, e] = gj_mex('dc_gradient2_5d', ..., dobs_cell)   (dc_fwd2_5d.m, dc_gradient2_5d.m) */
    const int grad = !strcmp(cmd, "dc_gradient2_5d");
    gj_dc_grid g;
    g.n = (int)mxGetM(prhs[1]); g.m = (int)mxGetN(prhs[1]);
    g.robin = (int)field(prhs[2], "robin"); g.dx = field(prhs[2], "dx"); g.dz = field(prhs[2], "dz");
    const mxArray* AB = prhs[3];
    const int ns = (int)mxGetM(AB);
    gj_dc_src* srcs = (gj_dc_src*)mxMalloc(ns * sizeof(gj_dc_src));
    long** mns = (long**)mxMalloc(ns * sizeof(long*));
    double** als = (double**)mxMalloc(ns * sizeof(double*));
    for (int k = 0; k < ns; ++k) als[k] = NULL;
    size_t nd = 0;
    for (int k = 0; k < ns; ++k) {
      const mxArray* MN = mxGetCell(prhs[5], k);
      const mxArray* kyw = mxGetCell(prhs[6], k);
      const int ndk = (int)mxGetM(MN);
      g.n_ky = (int)mxGetM(kyw);
      mns[k] = (long*)mxMalloc((ndk ? 2 * ndk : 1) * sizeof(long));
      for (int j = 0; j < ndk; ++j) {
        mns[k][2 * j] = (long)mxGetPr(MN)[j] - 1;
        mns[k][2 * j + 1] = (long)mxGetPr(MN)[j + ndk] - 1;
      }
      srcs[k].a = (long)mxGetPr(AB)[k] - 1;
      srcs[k].b = (long)mxGetPr(AB)[k + ns] - 1;
      srcs[k].current = mxGetPr(prhs[4])[mxGetNumberOfElements(prhs[4]) > 1 ? k : 0];
      srcs[k].nd = ndk;
      srcs[k].mn = mns[k];
      srcs[k].ky = mxGetPr(kyw);
      srcs[k].w = mxGetPr(kyw) + g.n_ky;
      if (mxGetNumberOfElements(prhs[7]) > 0) {
        srcs[k].alpha = mxGetPr(mxGetCell(prhs[7], k)); /* GJ_DC_NALPHA x n_ky, column per ky */
      } else {  /* [] : the library computes dc_Lk.m's alphas for this source */
        als[k] = (double*)mxMalloc((size_t)g.n_ky * GJ_DC_NALPHA(g.n, g.m) * sizeof(double));
        check(gj_dc_alphas(&g, srcs[k].a, srcs[k].b, srcs[k].ky, als[k]));
        srcs[k].alpha = als[k];
      }
      srcs[k].d_obs = grad ? mxGetPr(mxGetCell(prhs[8], k)) : NULL;
      nd += ndk;
    }
    if (!grad) {
      plhs[0] = mxCreateDoubleMatrix(nd, 1, mxREAL);
      double* u = NULL;
      double* uk = NULL;
      if (nlhs > 1) {  /* stacked potentials, n*m per source */
        plhs[1] = mxCreateDoubleMatrix((size_t)g.n * g.m, ns, mxREAL);
        u = mxGetPr(plhs[1]);
      }
      if (nlhs > 2) {  /* per-wavenumber potentials, (n*m) x n_ky per source */
        mwSize dk[3] = {(mwSize)g.n * g.m, (mwSize)g.n_ky, (mwSize)ns};
        plhs[2] = mxCreateNumericArray(3, dk, mxDOUBLE_CLASS, mxREAL);
        uk = mxGetPr(plhs[2]);
      }
      check(gj_dc_forward_k(ctx(), &g, mxGetPr(prhs[1]), srcs, ns, NULL, mxGetPr(plhs[0]), u, uk, NULL));
    } else {
      plhs[0] = mxCreateDoubleMatrix(g.n - 2 * g.robin, g.m - g.robin, mxREAL);
      plhs[1] = mxCreateDoubleMatrix(nd, 1, mxREAL);
      plhs[2] = mxCreateDoubleMatrix(nd, 1, mxREAL);
      check(gj_dc_gradient(ctx(), &g, mxGetPr(prhs[1]), srcs, ns, NULL, mxGetPr(plhs[0]), mxGetPr(plhs[1]),
                           mxGetPr(plhs[2]), NULL, NULL));
    }
    for (int k = 0; k < ns; ++k) {
      mxFree(mns[k]);
      if (als[k]) mxFree(als[k]);
    }
    mxFree(mns); mxFree(als); mxFree(srcs);
  } else {
    mexErrMsgIdAndTxt("gerjoii:arg", "unknown command %s", cmd);
  }
}
