// extern "C" entry points declared in include/gerjoii_gpu.h.
#include <new>

#include "gj_internal.h"

struct gj_ctx {
  gj::Ctx c;
};

static gj_status guard_ctx(gj_ctx* ctx) {
  if (!ctx) return GJ_EINVAL;
  ctx->c.err.code = GJ_OK;
  ctx->c.err.msg.clear();
  ctx->c.launches = 0;
  cudaError_t e = cudaSetDevice(ctx->c.device);
  if (e != cudaSuccess) return ctx->c.err.set(GJ_ECUDA, "cudaSetDevice(%d): %s", ctx->c.device, cudaGetErrorString(e));
  return GJ_OK;
}

extern "C" {

const char* gj_version(void) { return "gerjoii_b200 0.1 (sm_100a)"; }

gj_status gj_context_create(gj_ctx** ctx, int device) {
  if (!ctx) return GJ_EINVAL;
  *ctx = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return GJ_ECUDA;
  }
  if (device < 0 || device >= n) return GJ_EINVAL;
  gj_ctx* c = new (std::nothrow) gj_ctx();
  if (!c) return GJ_ENOMEM;
  c->c.device = device;
  if (cudaSetDevice(device) != cudaSuccess) {
    delete c;
    return GJ_ECUDA;
  }
  *ctx = c;
  return GJ_OK;
}

gj_status gj_context_destroy(gj_ctx* ctx) {
  if (!ctx) return GJ_OK;
  cudaSetDevice(ctx->c.device);
  delete ctx;
  return GJ_OK;
}

gj_status gj_context_release(gj_ctx* ctx) {
  GJ_TRY(guard_ctx(ctx));
  cudaDeviceSynchronize();
  ctx->c.wsolver.reset();
  ctx->c.wkey.clear();
  ctx->c.wbatch.reset();
  ctx->c.dc_fac.release();
  ctx->c.dc_vec.release();
  return GJ_OK;
}

const char* gj_last_error(const gj_ctx* ctx) { return ctx ? ctx->c.err.msg.c_str() : "null context"; }

long gj_last_launch_count(const gj_ctx* ctx) { return ctx ? ctx->c.launches : 0; }

gj_status gj_set_kernel_timing(gj_ctx* ctx, int on) {
  if (!ctx) return GJ_EINVAL;
  ctx->c.timer.on = on != 0;
  ctx->c.timer.reset();
  return GJ_OK;
}

gj_status gj_kernel_time(const gj_ctx* ctx, int kind, double* ms, long* sampled, long* launches,
                         long* shot_launches) {
  if (!ctx || kind < 0 || kind >= gj::KK_NKINDS) return GJ_EINVAL;
  const gj::KernelTimer& t = ctx->c.timer;
  if (ms) *ms = t.ms[kind];
  if (sampled) *sampled = t.sampled[kind];
  if (launches) *launches = t.launches[kind];
  if (shot_launches) *shot_launches = t.shot_launches[kind];
  return GJ_OK;
}

gj_status gj_w_forward(gj_ctx* ctx, const gj_w_grid* grid, gj_precision precision, const double* eps_r,
                       const double* sigma, const gj_w_shot* shots, int nshots, double* d_out, double* jz_out,
                       double* u_out) {
  GJ_TRY(guard_ctx(ctx));
  if (!grid) return ctx->c.err.set(GJ_EINVAL, "null grid");
  return gj::w_forward(ctx->c, *grid, precision, eps_r, sigma, shots, nshots, d_out, jz_out, u_out);
}

gj_status gj_w_gradient(gj_ctx* ctx, const gj_w_grid* grid, gj_precision precision, const double* eps_r,
                        const double* sigma, const gj_w_shot* shots, int nshots, const double* d_obs,
                        gj_adj_mode mode, gj_misfit_kind misfit, const gj_w_opts* opts, double* g_eps,
                        double* g_sig, double* misfit_out, double* d_out, double* e_out) {
  GJ_TRY(guard_ctx(ctx));
  if (!grid) return ctx->c.err.set(GJ_EINVAL, "null grid");
  gj_w_opts o{};
  if (opts) o = *opts;
  return gj::w_gradient(ctx->c, *grid, precision, eps_r, sigma, false, shots, nshots, d_obs, false, mode, misfit,
                        o, g_eps, g_sig, false, misfit_out, d_out, e_out, 0);
}

gj_status gj_w_gradient_batch(gj_ctx* ctx, gj_precision precision, const gj_w_problem* probs, int nprob,
                              gj_adj_mode mode, const gj_w_opts* opts, int* nwaves) {
  GJ_TRY(guard_ctx(ctx));
  gj_w_opts o{};
  if (opts) o = *opts;
  return gj::w_gradient_batch(ctx->c, precision, probs, nprob, mode, o, nwaves);
}

gj_status gj_w_backward(gj_ctx* ctx, const gj_w_grid* grid, gj_precision precision, const double* eps_r,
                        const double* sigma, const gj_w_shot* shots, int nshots, const double* e, gj_adj_mode mode,
                        const gj_w_opts* opts, double* g_eps, double* g_sig) {
  GJ_TRY(guard_ctx(ctx));
  if (!grid) return ctx->c.err.set(GJ_EINVAL, "null grid");
  gj_w_opts o{};
  if (opts) o = *opts;
  return gj::w_gradient(ctx->c, *grid, precision, eps_r, sigma, false, shots, nshots, e, false, mode, GJ_MISFIT_L2,
                        o, g_eps, g_sig, false, nullptr, nullptr, nullptr, 0, true);
}

gj_status gj_w_misfit(gj_ctx* ctx, const gj_w_grid* grid, gj_precision precision, const double* eps_r,
                      const double* sigma, const gj_w_shot* shots, int nshots, const double* d_obs,
                      gj_misfit_kind misfit, double* misfit_out) {
  GJ_TRY(guard_ctx(ctx));
  if (!grid) return ctx->c.err.set(GJ_EINVAL, "null grid");
  return gj::w_misfit(ctx->c, *grid, precision, eps_r, sigma, shots, nshots, d_obs, misfit, misfit_out);
}

gj_status gj_w_misfit_trials(gj_ctx* ctx, const gj_w_grid* grid, gj_precision precision, int ntrial,
                             const double* eps_r, const double* sigma, const gj_w_shot* shots, int nshots,
                             const double* d_obs, gj_misfit_kind misfit, const gj_w_opts* opts, double* misfit_out) {
  GJ_TRY(guard_ctx(ctx));
  if (!grid) return ctx->c.err.set(GJ_EINVAL, "null grid");
  return gj::w_misfit(ctx->c, *grid, precision, eps_r, sigma, shots, nshots, d_obs, misfit, misfit_out, ntrial, opts);
}

gj_status gj_w_gradient_dev(gj_ctx* ctx, const gj_w_grid* grid, gj_precision precision, const void* eps_r_dev,
                            const void* sigma_dev, const gj_w_shot* shots, int nshots, const void* d_obs_dev,
                            gj_adj_mode mode, gj_misfit_kind misfit, const gj_w_opts* opts, void* g_eps_dev,
                            void* g_sig_dev, double* misfit_out, void* stream) {
  GJ_TRY(guard_ctx(ctx));
  if (!grid) return ctx->c.err.set(GJ_EINVAL, "null grid");
  gj_w_opts o{};
  if (opts) o = *opts;
  return gj::w_gradient(ctx->c, *grid, precision, eps_r_dev, sigma_dev, true, shots, nshots, d_obs_dev, true, mode,
                        misfit, o, g_eps_dev, g_sig_dev, true, misfit_out, nullptr, nullptr,
                        static_cast<cudaStream_t>(stream));
}

gj_status gj_w_grad(gj_ctx* ctx, const gj_w_grid* grid, gj_precision precision, const double* eps_r,
                    const double* sigma, const gj_w_shot* shot, const double* e, const double* u, double* g,
                    double* a_max) {
  GJ_TRY(guard_ctx(ctx));
  if (!grid || !shot) return ctx->c.err.set(GJ_EINVAL, "null grid or shot");
  return gj::w_grad_only(ctx->c, *grid, precision, eps_r, sigma, *shot, e, u, g, a_max);
}

gj_status gj_dc_forward(gj_ctx* ctx, const gj_dc_grid* grid, const double* sigma, const gj_dc_src* srcs, int nsrc,
                        const gj_dc_opts* opts, double* d_out, double* u_out, gj_dc_stats* stats) {
  GJ_TRY(guard_ctx(ctx));
  if (!grid) return ctx->c.err.set(GJ_EINVAL, "null grid");
  gj_dc_opts o{};
  if (opts) o = *opts;
  return gj::dc_run(ctx->c, *grid, sigma, srcs, nsrc, false, o, d_out, nullptr, u_out, nullptr, nullptr, stats);
}

gj_status gj_dc_forward_k(gj_ctx* ctx, const gj_dc_grid* grid, const double* sigma, const gj_dc_src* srcs,
                          int nsrc, const gj_dc_opts* opts, double* d_out, double* u_out, double* uk_out,
                          gj_dc_stats* stats) {
  GJ_TRY(guard_ctx(ctx));
  if (!grid) return ctx->c.err.set(GJ_EINVAL, "null grid");
  gj_dc_opts o{};
  if (opts) o = *opts;
  return gj::dc_run(ctx->c, *grid, sigma, srcs, nsrc, false, o, d_out, nullptr, u_out, nullptr, nullptr, stats,
                    uk_out);
}

gj_status gj_dc_gradient(gj_ctx* ctx, const gj_dc_grid* grid, const double* sigma, const gj_dc_src* srcs, int nsrc,
                         const gj_dc_opts* opts, double* g_out, double* d_out, double* e_out, double* misfit_out,
                         gj_dc_stats* stats) {
  GJ_TRY(guard_ctx(ctx));
  if (!grid || !g_out) return ctx->c.err.set(GJ_EINVAL, "null grid or gradient output");
  gj_dc_opts o{};
  if (opts) o = *opts;
  return gj::dc_run(ctx->c, *grid, sigma, srcs, nsrc, true, o, d_out, e_out, nullptr, g_out, misfit_out, stats);
}

}  // extern "C"
