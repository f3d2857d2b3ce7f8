// The caller-side steps around a propagator solve, on the device: the
// twisted-basis rotation of the source and of the sink (get_qprop,
// projects/ib/prop.cpp:41-112, without its photon and free-theory branches)
// and the reconstruction of the twisted doublet (reconstruct_tm_doublet,
// dirac_operators/tmQ/reconstruct_tm_doublet.cpp:13-26, whose body is a
// CRASH("reimplement") stub there; its commented body defines it).
//
// The rotation is safe_dirac_prod_spincolor with P- (r = 0) or P+ (r = 1)
// (tau3 = {-1, +1}, new_types/dirac.hpp:38-41): the diagonal Dirac matrices
// (1 -+ i g5)/sqrt2 = diag(1-+i, 1-+i, 1+-i, 1+-i)/sqrt2 of new_types/dirac.cpp:60-61.
#include "tms_internal.cuh"

using namespace tms;
using namespace tms_int;

namespace
{
  // out = P(r) in, V lx AoS sites (in == out allowed: P is diagonal)
  __global__ void rotate_kernel(long long n, int r, double rad2, const double* in, double* out)
  {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; // one complex component
    if (i >= n) return;
    const int spin = (int)((i / 3) % 4);
    // P+ : (rad2, +rad2) on spins 0,1 and (rad2, -rad2) on spins 2,3; P- the opposite
    const double s = ((r == 1) == (spin < 2)) ? rad2 : -rad2;
    const double a = in[2 * i], b = in[2 * i + 1];
    out[2 * i] = a * rad2 - b * s;
    out[2 * i + 1] = a * s + b * rad2;
  }

  // outplus = outminus - 2 i mu in
  __global__ void doublet_kernel(long long n, double mu, const double* in, const double* outminus, double* outplus)
  {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double a = in[2 * i], b = in[2 * i + 1];
    const double m = -2 * mu;
    outplus[2 * i] = outminus[2 * i] - b * m;
    outplus[2 * i + 1] = outminus[2 * i + 1] + a * m;
  }

  tms_status ensure_lxbuf(tms_ctx* ctx, int k)
  {
    if (!ctx->lxbuf[k]) CU(cudaMalloc(&ctx->lxbuf[k], (size_t)ctx->g.V * 24 * sizeof(double)));
    return TMS_OK;
  }

  cudaMemcpyKind kind_in(const tms_ctx* ctx) { return ctx->ptr_mode == TMS_PTR_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice; }
  cudaMemcpyKind kind_out(const tms_ctx* ctx) { return ctx->ptr_mode == TMS_PTR_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice; }

  void rotate(tms_ctx* ctx, int r, const double* in, double* out)
  {
    const long long n = ctx->g.V * 12;
    ++ctx->launches;
    rotate_kernel<<<div_up(n, 256), 256, 0, ctx->stream>>>(n, r, 1. / sqrt(2.), in, out);
  }

  // run `solve` with device pointers, restoring the caller's pointer mode
  template <class F>
  tms_status with_device_pointers(tms_ctx* ctx, F&& solve)
  {
    const int mode = ctx->ptr_mode;
    ctx->ptr_mode = TMS_PTR_DEVICE;
    const tms_status s = solve();
    ctx->ptr_mode = mode;
    return s;
  }
}

extern "C" {

tms_status tms_rotate_twisted(tms_ctx* ctx, int r, const double* in_lx, double* out_lx)
{
  TRY(check_conf(ctx));
  if ((r != 0 && r != 1) || !in_lx || !out_lx) return fail(ctx, TMS_ERR_BAD_ARG, "r must be 0 or 1");
  TRY(ensure_lxbuf(ctx, 0));
  const size_t bytes = (size_t)ctx->g.V * 24 * sizeof(double);
  CU(cudaMemcpyAsync(ctx->lxbuf[0], in_lx, bytes, kind_in(ctx), ctx->stream));
  rotate(ctx, r, ctx->lxbuf[0], ctx->lxbuf[0]);
  CU(cudaGetLastError());
  CU(cudaMemcpyAsync(out_lx, ctx->lxbuf[0], bytes, kind_out(ctx), ctx->stream));
  return finish(ctx);
}

tms_status tms_get_qprop(tms_ctx* ctx, int r, int rotate_source, double kappa, int has_anis, double anis, double cSW,
                         double mu, int niter, double residue, int precision, const double* src_lx, double* out_lx,
                         tms_stats* stats)
{
  TRY(check_conf(ctx));
  if ((r != 0 && r != 1) || !src_lx || !out_lx) return fail(ctx, TMS_ERR_BAD_ARG, "r must be 0 or 1");
  TRY(ensure_lxbuf(ctx, 0));
  TRY(ensure_lxbuf(ctx, 1));
  const size_t bytes = (size_t)ctx->g.V * 24 * sizeof(double);
  CU(cudaMemcpyAsync(ctx->lxbuf[0], src_lx, bytes, kind_in(ctx), ctx->stream));
  if (rotate_source) rotate(ctx, r, ctx->lxbuf[0], ctx->lxbuf[0]);
  CU(cudaGetLastError());
  const tms_status st = with_device_pointers(ctx, [&]() {
    return cSW != 0.0 ? tms_cg_tmclov_eoprec(ctx, ctx->lxbuf[1], ctx->lxbuf[0], kappa, has_anis, anis, cSW, mu, niter,
                                             residue, precision, stats)
                      : tms_cg_eoprec(ctx, ctx->lxbuf[1], ctx->lxbuf[0], kappa, has_anis, anis, mu, niter, residue,
                                      precision, stats);
  });
  if (st != TMS_OK && st != TMS_ERR_NOT_CONVERGED) return st;
  rotate(ctx, r, ctx->lxbuf[1], ctx->lxbuf[1]);
  CU(cudaGetLastError());
  CU(cudaMemcpyAsync(out_lx, ctx->lxbuf[1], bytes, kind_out(ctx), ctx->stream));
  TRY(finish(ctx));
  return st;
}

tms_status tms_reconstruct_tm_doublet(tms_ctx* ctx, double kappa, int has_anis, double anis, double mu,
                                      const double* in_lx, double* outminus_lx, double* outplus_lx)
{
  TRY(check_conf(ctx));
  if (!in_lx || !outminus_lx || !outplus_lx) return TMS_ERR_BAD_ARG;
  TRY(ensure_lxbuf(ctx, 0));
  TRY(ensure_lxbuf(ctx, 1));
  const size_t bytes = (size_t)ctx->g.V * 24 * sizeof(double);
  CU(cudaMemcpyAsync(ctx->lxbuf[0], in_lx, bytes, kind_in(ctx), ctx->stream));
  // outminus = Q(tau3[1] mu) in
  TRY(with_device_pointers(ctx, [&]() {
    return tms_apply_tmQ(ctx, kappa, has_anis, anis, +mu, ctx->lxbuf[0], ctx->lxbuf[1]);
  }));
  CU(cudaMemcpyAsync(outminus_lx, ctx->lxbuf[1], bytes, kind_out(ctx), ctx->stream));
  const long long n = ctx->g.V * 12;
  ++ctx->launches;
  doublet_kernel<<<div_up(n, 256), 256, 0, ctx->stream>>>(n, mu, ctx->lxbuf[0], ctx->lxbuf[1], ctx->lxbuf[0]);
  CU(cudaGetLastError());
  CU(cudaMemcpyAsync(outplus_lx, ctx->lxbuf[0], bytes, kind_out(ctx), ctx->stream));
  return finish(ctx);
}

} // extern "C"
