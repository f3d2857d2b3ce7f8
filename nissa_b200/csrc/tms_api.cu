// C ABI of the B200 twisted-mass solver: contexts, resident gauge
// configuration, geometry tables, operators and instrumentation.  The solvers
// are in tms_cg.cu.
#include "tms_internal.cuh"

using namespace tms_int;

namespace
{
  template <int P, int LF>
  tms_status bench_hop_t(tms_ctx* ctx, const LinkT<LF>& U, int variant, int nrep, int flush, double* ms,
                         double link_bytes, double spinor_bytes, double* bytes)
  {
    Field in, out, x;
    TRY(alloc_field(ctx, in, P));
    TRY(alloc_field(ctx, out, P));
    TRY(alloc_field(ctx, x, P));
    struct G
    {
      Field *a, *b, *c;
      ~G()
      {
        for (Field* f : {a, b, c})
          {
            if (f->d) cudaFree(f->d);
            if (f->n) cudaFree(f->n);
          }
      }
    } guard{&in, &out, &x};
    // deterministic non-trivial input: the ones vector scaled
    const int n = (int)ctx->g.Vh;
    axpby_kernel<P, P, P><<<div_up(n, BLAS_THREADS), BLAS_THREADS, 0, ctx->stream>>>(n, 0.0, view<P>(in), 0.0,
                                                                                     view<P>(in), view<P>(in));
    void* scratch = nullptr;
    const size_t sbytes = size_t(512) << 20;
    if (flush) CU(cudaMalloc(&scratch, sbytes));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double total = 0;
    // one untimed launch first: the first launch of a kernel also loads its code
    for (int r = -1; r < nrep; r++)
      {
        if (flush) cudaMemsetAsync(scratch, r & 0xff, sbytes, ctx->stream);
        cudaEventRecord(e0, ctx->stream);
        if (variant == 0)
          {
            EpiPlain<P> e{{view<P>(out), view<P>(out)}};
            launch_hop<P, LF>(ctx, ctx->stream, 0, 1, in, in, U, ctx->prm, e);
          }
        else if (variant == 1)
          {
            EpiInvDiag<P> e{{view<P>(out), view<P>(out)}, ctx->prm, 1.0};
            launch_hop<P, LF>(ctx, ctx->stream, 0, 1, in, in, U, ctx->prm, e);
          }
        else
          {
            EpiKern<P, true> e{{view<P>(out), view<P>(out)}, {view<P>(x), view<P>(x)}, ctx->prm, 1.0};
            launch_hop<P, LF>(ctx, ctx->stream, 1, 1, in, in, U, ctx->prm, e);
          }
        cudaEventRecord(e1, ctx->stream);
        cudaEventSynchronize(e1);
        float t = 0;
        cudaEventElapsedTime(&t, e0, e1);
        if (r >= 0) total += t;
      }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (scratch) cudaFree(scratch);
    CU(cudaGetLastError());
    *ms = total / nrep;
    *bytes = (double)ctx->g.Vh * (8 * link_bytes + 2 * spinor_bytes + (variant == 2 ? spinor_bytes : 0));
    return TMS_OK;
  }
}

// =================================================================== C ABI

extern "C" {

tms_status tms_create4(tms_ctx** out, int T, int LX, int LY, int LZ, double bc_t, int device)
{
  if (!out) return TMS_ERR_BAD_ARG;
  *out = nullptr;
  if (T <= 0 || LX <= 0 || LY <= 0 || LZ <= 0 || (T | LX | LY | LZ) & 1) return TMS_ERR_BAD_ARG;
  const int64_t V = (int64_t)T * LX * LY * LZ;
  if (V >= (int64_t(1) << 31)) return TMS_ERR_BAD_ARG;
  tms_ctx* ctx = new tms_ctx;
  ctx->g.T = T;
  ctx->g.LX = LX;
  ctx->g.LY = LY;
  ctx->g.LZ = LZ;
  ctx->g.V = V;
  ctx->g.Vh = V / 2;
  ctx->g.stride = round_up(V / 2, 64);
  ctx->g.bc_t = bc_t;
  ctx->device = device;
  auto cleanup = [&](tms_status s) {
    tms_destroy(ctx);
    return s;
  };
  if (cudaSetDevice(device) != cudaSuccess) return cleanup(TMS_ERR_CUDA);
  if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) return cleanup(TMS_ERR_CUDA);
  ctx->red_cap = div_up(V, 16) + 1024; // block partials: a launch of at least 16 sites per block
  if (cudaMalloc(&ctx->lx_of_eo, sizeof(int) * V) != cudaSuccess ||
      cudaMalloc(&ctx->prm, sizeof(OpParams) * 2) != cudaSuccess ||
      cudaMalloc(&ctx->st, sizeof(CgState)) != cudaSuccess ||
      cudaMalloc(&ctx->red_partial, sizeof(double) * ctx->red_cap) != cudaSuccess ||
      cudaMalloc(&ctx->red_counter, sizeof(unsigned)) != cudaSuccess ||
      cudaMalloc(&ctx->red_result, sizeof(double)) != cudaSuccess ||
      cudaMalloc(&ctx->tma_timeouts, sizeof(unsigned)) != cudaSuccess ||
      cudaHostAlloc(&ctx->st_h, sizeof(CgState), cudaHostAllocMapped) != cudaSuccess ||
      cudaMalloc(&ctx->cgm, sizeof(CgmState)) != cudaSuccess ||
      cudaMallocHost(&ctx->cgm_h, sizeof(CgmState)) != cudaSuccess ||
      cudaHostAlloc(&ctx->red_h, sizeof(double), cudaHostAllocMapped) != cudaSuccess ||
      cudaHostAlloc(&ctx->hring, kHostRing, cudaHostAllocMapped) != cudaSuccess)
    return cleanup(TMS_ERR_OOM);
  if (cudaHostGetDevicePointer(reinterpret_cast<void**>(&ctx->st_hd), ctx->st_h, 0) != cudaSuccess ||
      cudaHostGetDevicePointer(reinterpret_cast<void**>(&ctx->red_hd), ctx->red_h, 0) != cudaSuccess ||
      cudaHostGetDevicePointer(reinterpret_cast<void**>(&ctx->hring_d), ctx->hring, 0) != cudaSuccess)
    return cleanup(TMS_ERR_CUDA);
  cudaMemset(ctx->red_counter, 0, sizeof(unsigned));
  cudaMemset(ctx->tma_timeouts, 0, sizeof(unsigned));
  cudaMemset(ctx->st, 0, sizeof(CgState));
  cudaEventCreate(&ctx->ev0);
  cudaEventCreate(&ctx->ev1);
  ++ctx->launches;
  lx_of_eo_kernel<<<div_up(V, 256), 256, 0, ctx->stream>>>(ctx->g, ctx->lx_of_eo);
  if (cudaStreamSynchronize(ctx->stream) != cudaSuccess || cudaGetLastError() != cudaSuccess)
    return cleanup(TMS_ERR_CUDA);
  *out = ctx;
  return TMS_OK;
}

tms_status tms_create(tms_ctx** out, int T, int L, double bc_t, int device)
{
  return tms_create4(out, T, L, L, L, bc_t, device);
}

tms_status tms_destroy(tms_ctx* ctx)
{
  if (!ctx) return TMS_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->cstream) cudaStreamSynchronize(ctx->cstream);
  for (auto& gr : ctx->graph)
    if (gr) cudaGraphExecDestroy(gr);
  auto fr = [](void* p) {
    if (p) cudaFree(p);
  };
  for (auto& f : ctx->f64) { fr(f.d); fr(f.n); }
  for (auto& f : ctx->lo) { fr(f.d); fr(f.n); }
  for (auto& f : ctx->ex) { fr(f.d); fr(f.n); }
  if (ctx->bw && ctx->bw_free) ctx->bw_free(ctx->bw);
  for (auto& f : ctx->lx64) { fr(f.d); fr(f.n); }
  for (auto& f : ctx->lxlo) { fr(f.d); fr(f.n); }
  fr(ctx->lxxlo.d);
  fr(ctx->lxxlo.n);
  fr(ctx->cgm_x);
  fr(ctx->cgm_ps);
  fr(ctx->cgm);
  if (ctx->cgm_h) cudaFreeHost(ctx->cgm_h);
  fr(ctx->xlo32.d);
  fr(ctx->xlo32.n);
  fr(ctx->lx_of_eo);
  fr(ctx->U64);
  fr(ctx->lxbuf[0]);
  fr(ctx->lxbuf[1]);
  fr(ctx->cl64);
  fr(ctx->cl32);
  fr(ctx->icl64);
  fr(ctx->icl32);
  fr(ctx->U32r);
  fr(ctx->U32f);
  fr(ctx->U16r);
  fr(ctx->U16h);
  fr(ctx->prm);
  fr(ctx->st);
  fr(ctx->red_partial);
  fr(ctx->red_counter);
  fr(ctx->tma_timeouts);
  fr(ctx->slab_ghost);
  fr(ctx->red_result);
  fr(ctx->stage);
  for (double*& b : ctx->colbuf) fr(b);
  for (cudaEvent_t& e : ctx->colev)
    if (e) cudaEventDestroy(e);
  if (ctx->cstream) cudaStreamDestroy(ctx->cstream);
  if (ctx->st_h) cudaFreeHost(ctx->st_h);
  if (ctx->red_h) cudaFreeHost(ctx->red_h);
  if (ctx->hring) cudaFreeHost(ctx->hring);
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return TMS_OK;
}

const char* tms_last_error(const tms_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

tms_status tms_set_pointer_mode(tms_ctx* ctx, int mode)
{
  if (!ctx || (mode != TMS_PTR_HOST && mode != TMS_PTR_DEVICE)) return TMS_ERR_BAD_ARG;
  ctx->ptr_mode = mode;
  return TMS_OK;
}

int64_t tms_volume(const tms_ctx* ctx) { return ctx ? ctx->g.V : 0; }

tms_status tms_geometry_tables(tms_ctx* ctx, int32_t* parity, int32_t* eo_of_lx, int32_t* lx_of_eo, int32_t* neighup,
                               int32_t* neighdw)
{
  if (!ctx) return TMS_ERR_BAD_ARG;
  CU(cudaSetDevice(ctx->device));
  const int64_t V = ctx->g.V;
  int* d = nullptr;
  CU(cudaMalloc(&d, sizeof(int) * V * 11));
  ++ctx->launches;
  geometry_tables_kernel<<<div_up(V, 256), 256, 0, ctx->stream>>>(ctx->g, d, d + V, d + 2 * V, d + 3 * V, d + 7 * V);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  int32_t* outs[5] = {parity, eo_of_lx, lx_of_eo, neighup, neighdw};
  const int64_t off[5] = {0, V, 2 * V, 3 * V, 7 * V}, len[5] = {V, V, V, 4 * V, 4 * V};
  for (int k = 0; k < 5 && e == cudaSuccess; k++)
    if (outs[k]) e = cudaMemcpy(outs[k], d + off[k], sizeof(int) * len[k], cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return fail(ctx, TMS_ERR_CUDA, "geometry tables: %s", cudaGetErrorString(e));
  return TMS_OK;
}

tms_status tms_conf_upload(tms_ctx* ctx, const double* conf, int layout, int flags)
{
  if (!ctx || !conf || (layout != TMS_LAYOUT_LX && layout != TMS_LAYOUT_EO)) return TMS_ERR_BAD_ARG;
  CU(cudaSetDevice(ctx->device));
  const int64_t V = ctx->g.V, Vh = ctx->g.Vh;
  const size_t bytes = (size_t)V * 72 * sizeof(double);
  if (!ctx->U64) CU(cudaMalloc(&ctx->U64, (size_t)V * 36 * sizeof(double2)));
  if (!ctx->U32r) CU(cudaMalloc(&ctx->U32r, (size_t)V * 12 * sizeof(float4)));
  if (!ctx->U32f) CU(cudaMalloc(&ctx->U32f, (size_t)V * 36 * sizeof(float2)));
  if (!ctx->U16r) CU(cudaMalloc(&ctx->U16r, LinkT<LINK_I16_12>::bytes(ctx->g.Vh)));
  if (!ctx->U16h) CU(cudaMalloc(&ctx->U16h, LinkT<LINK_H16_12>::bytes(ctx->g.Vh)));
  const double* src = conf;
  if (ctx->ptr_mode == TMS_PTR_HOST)
    {
      TRY(ensure_stage(ctx, bytes));
      CU(cudaMemcpyAsync(ctx->stage, conf, bytes, cudaMemcpyHostToDevice, ctx->stream));
      src = ctx->stage;
    }
  const int unfold = (flags & TMS_CONF_BC_INCLUDED) ? 1 : 0;
  ++ctx->launches;
  conf_to_soa_kernel<<<div_up(V, 128), 128, 0, ctx->stream>>>(ctx->g, src, layout, unfold, ctx->lx_of_eo, ctx->U64);
  CU(cudaGetLastError());
  const int64_t nl = 8 * Vh;
  ++ctx->launches;
  conf_lowprec_kernel<<<div_up(nl, 256), 256, 0, ctx->stream>>>(nl, (int)Vh, ctx->U64, ctx->U32r, ctx->U32f, ctx->U16r, ctx->U16h,
                                                                 reducer(ctx));
  CU(cudaGetLastError());
  const double dev = read_result(ctx);
  CU(cudaGetLastError());
  ctx->su3 = (dev < 1e-10);
  ctx->su3_dev = dev;
  ctx->conf_loaded = true;
  ctx->clov_ok = ctx->icl_ok = false; // a clover term belongs to the conf it was computed from
  return TMS_OK;
}

int tms_conf_is_su3(const tms_ctx* ctx) { return (ctx && ctx->su3) ? 1 : 0; }

tms_status tms_hop_eo(tms_ctx* ctx, int par_out, const double* in, double* out, int has_anis, double anis)
{
  TRY(check_conf(ctx));
  if (par_out != 0 && par_out != 1) return fail(ctx, TMS_ERR_BAD_ARG, "parity must be 0 or 1");
  TRY(set_params(ctx, 1.0, 0.0, has_anis, anis));
  Field &a = ctx->f64[6], &b = ctx->f64[7];
  TRY(spinor_in(ctx, in, nullptr, ctx->g.Vh, a));
  TRY(alloc_field(ctx, b, PREC_F64));
  EpiPlain<PREC_F64> e{{view<PREC_F64>(b), view<PREC_F64>(b)}};
  launch_hop<PREC_F64, LINK_F64_18>(ctx, ctx->stream, par_out, 1, a, a, links64(ctx), ctx->prm, e);
  CU(cudaGetLastError());
  TRY(spinor_out(ctx, b, nullptr, ctx->g.Vh, out, true));
  return finish(ctx);
}

static tms_status diag_common(tms_ctx* ctx, double kappa, double mu, const double* in, double* out, int inverse)
{
  if (!ctx) return TMS_ERR_BAD_ARG;
  CU(cudaSetDevice(ctx->device));
  TRY(set_params(ctx, kappa, mu, 0, 1.0));
  Field &a = ctx->f64[6], &b = ctx->f64[7];
  TRY(spinor_in(ctx, in, nullptr, ctx->g.Vh, a));
  TRY(alloc_field(ctx, b, PREC_F64));
  const int n = (int)ctx->g.Vh;
  ++ctx->launches;
  diag_kernel<PREC_F64><<<div_up(n, 256), 256, 0, ctx->stream>>>(n, view<PREC_F64>(a), view<PREC_F64>(b), ctx->prm,
                                                                   1.0, inverse);
  CU(cudaGetLastError());
  TRY(spinor_out(ctx, b, nullptr, ctx->g.Vh, out, true));
  return finish(ctx);
}

tms_status tms_tmDee(tms_ctx* ctx, double kappa, double mu, const double* in, double* out)
{
  return diag_common(ctx, kappa, mu, in, out, 0);
}

tms_status tms_inv_tmDee(tms_ctx* ctx, double kappa, double mu, const double* in, double* out)
{
  return diag_common(ctx, kappa, mu, in, out, 1);
}

tms_status tms_kern_eoprec(tms_ctx* ctx, double kappa, int has_anis, double anis, double mu, const double* in,
                           double* out)
{
  TRY(check_conf(ctx));
  TRY(set_params(ctx, kappa, mu, has_anis, anis));
  Field &a = ctx->f64[6], &b = ctx->f64[7], &te = ctx->f64[5];
  TRY(spinor_in(ctx, in, nullptr, ctx->g.Vh, a));
  TRY(alloc_field(ctx, b, PREC_F64));
  TRY(alloc_field(ctx, te, PREC_F64));
  kern_op<PREC_F64>(ctx, links64(ctx), a, te, b, +1.0, ctx->prm);
  CU(cudaGetLastError());
  TRY(spinor_out(ctx, b, nullptr, ctx->g.Vh, out, true));
  return finish(ctx);
}

tms_status tms_kern_eoprec_square(tms_ctx* ctx, double kappa, int has_anis, double anis, double mu, const double* in,
                                  double* out)
{
  TRY(check_conf(ctx));
  TRY(set_params(ctx, kappa, mu, has_anis, anis));
  Field &a = ctx->f64[6], &b = ctx->f64[7], &te = ctx->f64[5], &t1 = ctx->f64[4];
  TRY(spinor_in(ctx, in, nullptr, ctx->g.Vh, a));
  TRY(alloc_field(ctx, b, PREC_F64));
  TRY(alloc_field(ctx, te, PREC_F64));
  TRY(alloc_field(ctx, t1, PREC_F64));
  kern_op<PREC_F64>(ctx, links64(ctx), a, te, t1, -1.0, ctx->prm);
  kern_op<PREC_F64>(ctx, links64(ctx), t1, te, b, +1.0, ctx->prm);
  CU(cudaGetLastError());
  TRY(spinor_out(ctx, b, nullptr, ctx->g.Vh, out, true));
  return finish(ctx);
}

// full-lattice operators: lx spinors are split into the two parities of
// fields 6 (even) / 7 (odd) -> outputs in 4 (even) / 5 (odd)
static tms_status tmQ_common(tms_ctx* ctx, double kappa, int has_anis, double anis, double mu, const double* in,
                             double* out, bool square)
{
  TRY(check_conf(ctx));
  TRY(set_params(ctx, kappa, mu, has_anis, anis));
  Field* f = ctx->f64;
  for (int i = 1; i <= 7; i++) TRY(alloc_field(ctx, f[i], PREC_F64));
  const int64_t Vh = ctx->g.Vh;
  // in: split lx -> (e, o)
  const double* src = in;
  const size_t bytes = (size_t)ctx->g.V * 24 * sizeof(double);
  if (ctx->ptr_mode == TMS_PTR_HOST)
    {
      TRY(ensure_stage(ctx, bytes));
      CU(cudaMemcpyAsync(ctx->stage, in, bytes, cudaMemcpyHostToDevice, ctx->stream));
      src = ctx->stage;
    }
  const int n = (int)Vh;
  ++ctx->launches;
  aos_to_soa_kernel<PREC_F64><<<div_up(n, 256), 256, 0, ctx->stream>>>(n, src, ctx->lx_of_eo, view<PREC_F64>(f[6]));
  ++ctx->launches;
  aos_to_soa_kernel<PREC_F64><<<div_up(n, 256), 256, 0, ctx->stream>>>(n, src, ctx->lx_of_eo + Vh,
                                                                       view<PREC_F64>(f[7]));
  auto U = links64(ctx);
  auto V = [&](int i) { return view<PREC_F64>(f[i]); };
  if (!square)
    {
      EpiTmQ<PREC_F64, false> e{{V(4), V(5)}, {V(6), V(7)}, ctx->prm, +1.0};
      launch_hop<PREC_F64, LINK_F64_18>(ctx, ctx->stream, 0, 2, f[6], f[7], U, ctx->prm, e);
    }
  else
    {
      // temp = Q(+mu) in ; out = Q(-mu) temp
      EpiTmQ<PREC_F64, false> e1{{V(2), V(3)}, {V(6), V(7)}, ctx->prm, +1.0};
      launch_hop<PREC_F64, LINK_F64_18>(ctx, ctx->stream, 0, 2, f[6], f[7], U, ctx->prm, e1);
      EpiTmQ<PREC_F64, false> e2{{V(4), V(5)}, {V(2), V(3)}, ctx->prm, -1.0};
      launch_hop<PREC_F64, LINK_F64_18>(ctx, ctx->stream, 0, 2, f[2], f[3], U, ctx->prm, e2);
    }
  CU(cudaGetLastError());
  TRY(spinor_out(ctx, f[4], ctx->lx_of_eo, ctx->g.V, out, false));
  // second parity goes to the same staging/destination buffer
  double* d = (ctx->ptr_mode == TMS_PTR_HOST) ? ctx->stage : out;
  ++ctx->launches;
  soa_to_aos_kernel<PREC_F64><<<div_up(n, 256), 256, 0, ctx->stream>>>(n, V(5), ctx->lx_of_eo + Vh, d);
  CU(cudaGetLastError());
  if (ctx->ptr_mode == TMS_PTR_HOST)
    CU(cudaMemcpyAsync(out, ctx->stage, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  return finish(ctx);
}

tms_status tms_apply_tmQ(tms_ctx* ctx, double kappa, int has_anis, double anis, double mu, const double* in,
                         double* out)
{
  return tmQ_common(ctx, kappa, has_anis, anis, mu, in, out, false);
}

tms_status tms_apply_tmQ2(tms_ctx* ctx, double kappa, int has_anis, double anis, double mu, const double* in,
                          double* out)
{
  return tmQ_common(ctx, kappa, has_anis, anis, mu, in, out, true);
}

uint64_t tms_launch_count(const tms_ctx* ctx) { return ctx ? ctx->launches : 0; }

int64_t tms_hop_stage_timeouts(tms_ctx* ctx)
{
  if (!ctx) return -1;
  unsigned v = 0;
  if (cudaStreamSynchronize(ctx->stream) != cudaSuccess ||
      cudaMemcpy(&v, ctx->tma_timeouts, sizeof v, cudaMemcpyDeviceToHost) != cudaSuccess)
    return -1;
  return (int64_t)v;
}

tms_status tms_set_tuning(tms_ctx* ctx, const char* key, double value)
{
  if (!ctx || !key) return TMS_ERR_BAD_ARG;
  const std::string k = key;
  auto drop_all = [&]() {
    cudaStreamSynchronize(ctx->stream);
    for (auto& g : ctx->graph)
      if (g)
        {
          cudaGraphExecDestroy(g);
          g = nullptr;
        }
  };
  if (k == "hop_cfg_double" || k == "hop_cfg_single" || k == "hop_cfg_half")
    {
      const int v = (int)value;
      const int p = (k == "hop_cfg_double") ? PREC_F64 : (k == "hop_cfg_single") ? PREC_F32 : PREC_F16;
      const int ncfg = (p == PREC_F64) ? HOP_CFGS : HOP_CFGS_ALL;
      if (v < 0 || v >= ncfg || v != value) return fail(ctx, TMS_ERR_BAD_ARG, "%s: 0..%d", key, ncfg - 1);
      if (ctx->hop_cfg[p] != v) drop_all();
      ctx->hop_cfg[p] = v;
      return TMS_OK;
    }
  if (k == "half_arith")
    {
      if (value != 0.0 && value != 1.0) return fail(ctx, TMS_ERR_BAD_ARG, "half_arith: 0 (FP32 arithmetic) or 1");
      if (ctx->half_arith != (int)value) drop_all();
      ctx->half_arith = (int)value;
      return TMS_OK;
    }
  if (k == "tma_rows")
    {
      const int v = (int)value;
      if (v != value || (v != 0 && !tma_rows_ok(ctx->g, v)))
        return fail(ctx, TMS_ERR_BAD_ARG,
                    "tma_rows: 0 or a divisor R of LY with R*LZ/2 <= %d and R == LY or R + 2 <= LY (LZ a multiple "
                    "of 8)", HOP_TMA_THREADS);
      if (ctx->tma_rows != v) drop_all();
      ctx->tma_rows = v;
      return TMS_OK;
    }
  if (k == "graph_iters")
    {
      const int v = (int)value;
      if (v < 1 || v > 64 || v != value) return fail(ctx, TMS_ERR_BAD_ARG, "graph_iters: 1..64");
      if (ctx->graph_iters != v) drop_all();
      ctx->graph_iters = v;
      return TMS_OK;
    }
  if (k == "cgm_refine_batched")
    {
      if (value != 0.0 && value != 1.0) return fail(ctx, TMS_ERR_BAD_ARG, "cgm_refine_batched: 0 or 1");
      ctx->cgm_refine_batched = (int)value;
      return TMS_OK;
    }
  if (k == "cgm_floor_single")
    {
      if (!(value >= 1e-20 && value < 1.0)) return fail(ctx, TMS_ERR_BAD_ARG, "cgm_floor_single: in [1e-20, 1)");
      ctx->cgm_floor32 = value;
      return TMS_OK;
    }
  if (k == "stream_priority")
    {
      // the context's stream is recreated with this priority (CUDA's convention:
      // lower numbers run first); captured graphs run at the priority of the stream
      int least = 0, greatest = 0;
      CU(cudaDeviceGetStreamPriorityRange(&least, &greatest));
      const int v = (int)value;
      if ((double)v != value || v > least || v < greatest)
        return fail(ctx, TMS_ERR_BAD_ARG, "stream_priority: an integer in [%d, %d]", greatest, least);
      CU(cudaStreamSynchronize(ctx->stream));
      cudaStream_t s = nullptr;
      CU(cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, v));
      cudaStreamDestroy(ctx->stream);
      ctx->stream = s;
      return TMS_OK;
    }
  if (k == "pdl")
    {
      if (value != 0.0 && value != 1.0) return fail(ctx, TMS_ERR_BAD_ARG, "pdl: 0 or 1");
      if (ctx->pdl != (int)value) drop_all();
      ctx->pdl = (int)value;
      return TMS_OK;
    }
  if (k == "batch_graph_iters")
    {
      const int v = (int)value;
      if (v < 0 || v > 64 || v != value) return fail(ctx, TMS_ERR_BAD_ARG, "batch_graph_iters: 0 (automatic)..64");
      ctx->batch_iters = v; // sessions recapture their graph at the next step
      return TMS_OK;
    }
  if (k == "mrhs_per_thread")
    {
      const int v = (int)value;
      if (v != 0 && v != 1 && v != 2 && v != 4 || v != value)
        return fail(ctx, TMS_ERR_BAD_ARG, "mrhs_per_thread: 0 (1, pipelined), 1, 2 or 4");
      if (ctx->mrhs_r != v && ctx->bw && ctx->bw_free)
        {
          cudaStreamSynchronize(ctx->stream);
          ctx->bw_free(ctx->bw); // its graphs were captured with the old shape
          ctx->bw = nullptr;
        }
      ctx->mrhs_r = v;
      return TMS_OK;
    }
  if (k == "links_single")
    {
      if (value != 0.0 && value != 1.0) return fail(ctx, TMS_ERR_BAD_ARG, "links_single: 0 (FP32) or 1 (16-bit)");
      if (ctx->single_links16 != (int)value) drop_all();
      ctx->single_links16 = (int)value;
      return TMS_OK;
    }
  if (k == "links_reliable")
    {
      if (value != 0.0 && value != 1.0) return fail(ctx, TMS_ERR_BAD_ARG, "links_reliable: 0 (18 reals) or 1 (12)");
      ctx->reliable_links12 = (int)value;
      return TMS_OK;
    }
  if (k == "reliable_delta_single" || k == "reliable_delta_half")
    {
      if (!(value > 0.0 && value < 1.0)) return fail(ctx, TMS_ERR_BAD_ARG, "%s: in (0, 1)", key);
      (k == "reliable_delta_single" ? ctx->delta_single : ctx->delta_half) = value;
      return TMS_OK;
    }
  return fail(ctx, TMS_ERR_BAD_ARG, "unknown tuning key %s", key);
}

tms_status tms_get_tuning(tms_ctx* ctx, const char* key, double* value)
{
  if (!ctx || !key || !value) return TMS_ERR_BAD_ARG;
  const std::string k = key;
  if (k == "hop_cfg_double") *value = ctx->hop_cfg[PREC_F64];
  else if (k == "hop_cfg_single") *value = ctx->hop_cfg[PREC_F32];
  else if (k == "hop_cfg_half") *value = ctx->hop_cfg[PREC_F16];
  else if (k == "tma_rows") *value = ctx->tma_rows;
  else if (k == "half_arith") *value = ctx->half_arith;
  else if (k == "graph_iters") *value = ctx->graph_iters;
  else if (k == "batch_graph_iters") *value = ctx->batch_iters;
  else if (k == "mrhs_per_thread") *value = ctx->mrhs_r;
  else if (k == "links_single") *value = ctx->single_links16;
  else if (k == "links_reliable") *value = ctx->reliable_links12;
  else if (k == "reliable_delta_single") *value = ctx->delta_single;
  else if (k == "reliable_delta_half") *value = ctx->delta_half;
  else if (k == "pdl") *value = ctx->pdl;
  else if (k == "cgm_floor_single") *value = ctx->cgm_floor32;
  else if (k == "cgm_refine_batched") *value = ctx->cgm_refine_batched;
  else if (k == "stream_priority")
    {
      int prio = 0;
      CU(cudaStreamGetPriority(ctx->stream, &prio));
      *value = prio;
    }
  else return fail(ctx, TMS_ERR_BAD_ARG, "unknown tuning key %s", key);
  return TMS_OK;
}

tms_status tms_bench_hop(tms_ctx* ctx, int precision, int variant, int nrep, int flush, double* ms_per_launch,
                         double* bytes_per_launch)
{
  TRY(check_conf(ctx));
  if (nrep <= 0 || variant < 0 || variant > 2 || !ms_per_launch || !bytes_per_launch)
    return fail(ctx, TMS_ERR_BAD_ARG, "bad bench arguments");
  TRY(set_params(ctx, 0.16, 0.01, 0, 1.0));
  if (precision == TMS_PREC_DOUBLE)
    return bench_hop_t<PREC_F64>(ctx, links64(ctx), variant, nrep, flush, ms_per_launch, 144.0, 192.0,
                                 bytes_per_launch);
  if (precision == TMS_PREC_MIXED_SINGLE && ctx->su3 && ctx->single_links16)
    return bench_hop_t<PREC_F32>(ctx, links16r(ctx), variant, nrep, flush, ms_per_launch, 24.0, 96.0,
                                 bytes_per_launch);
  if (precision == TMS_PREC_MIXED_SINGLE)
    return ctx->su3 ? bench_hop_t<PREC_F32>(ctx, links32r(ctx), variant, nrep, flush, ms_per_launch, 48.0, 96.0,
                                            bytes_per_launch)
                    : bench_hop_t<PREC_F32>(ctx, links32f(ctx), variant, nrep, flush, ms_per_launch, 72.0, 96.0,
                                            bytes_per_launch);
  if (precision == TMS_PREC_MIXED_HALF && ctx->su3 && ctx->half_arith)
    return bench_hop_t<PREC_F16>(ctx, links16h(ctx), variant, nrep, flush, ms_per_launch, 24.0, 52.0,
                                 bytes_per_launch);
  if (precision == TMS_PREC_MIXED_HALF)
    return ctx->su3 ? bench_hop_t<PREC_F16>(ctx, links16r(ctx), variant, nrep, flush, ms_per_launch, 24.0, 52.0,
                                            bytes_per_launch)
                    : bench_hop_t<PREC_F16>(ctx, links32f(ctx), variant, nrep, flush, ms_per_launch, 72.0, 52.0,
                                            bytes_per_launch);
  return fail(ctx, TMS_ERR_BAD_ARG, "unknown precision %d", precision);
}

} // extern "C"
