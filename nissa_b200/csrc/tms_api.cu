// C ABI of the B200 twisted-mass solver: contexts, resident gauge
// configuration, operators and the e/o CG solvers (FP64 and mixed precision
// with FP64 reliable updates), each CG iteration replayed as a CUDA graph.
#include "tmsolve.h"
#include "tms_kernels.cuh"

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

using namespace tms;

namespace
{
  inline int div_up(int64_t a, int b) { return (int)((a + b - 1) / b); }
  inline int round_up(int64_t a, int b) { return (int)(((a + b - 1) / b) * b); }

  // device spinor buffer of one precision, e/o sized (stride >= Vh)
  struct Field
  {
    int prec = -1;
    void* d = nullptr;
    float* n = nullptr;
    int stride = 0;
    size_t bytes = 0;
  };

  template <int P>
  SpinorT<P> view(const Field& f)
  {
    SpinorT<P> s;
    s.d = reinterpret_cast<decltype(s.d)>(f.d);
    s.n = f.n;
    s.stride = f.stride;
    return s;
  }
}

struct tms_ctx
{
  Lattice g{};
  int device = 0;
  int ptr_mode = TMS_PTR_HOST;
  cudaStream_t stream = nullptr;
  std::string err;

  // geometry
  int* lx_of_eo = nullptr; // [2][Vh] device

  // gauge configuration
  bool conf_loaded = false, su3 = false;
  double2* U64 = nullptr;
  float4* U32r = nullptr; // 12-real
  float2* U32f = nullptr; // 18-real

  // scalars and reduction scratch
  OpParams* prm = nullptr;       // [2]: operator params (slot 0 solver, slot 1 free use)
  CgState* st = nullptr;         // device solver state
  CgState* st_h = nullptr;       // pinned host mirror
  double* red_partial = nullptr;
  unsigned* red_counter = nullptr;
  double* red_result = nullptr;
  double* red_h = nullptr;       // pinned
  int red_cap = 0;

  // staging for AoS conversions (device AoS doubles), grows on demand
  double* stage = nullptr;
  size_t stage_bytes = 0;

  // work fields (allocated on first use)
  Field f64[8];   // 0:b 1:x 2:r 3:p 4:t1 5:te(even) 6:s 7:tmp
  Field lo[6];    // inner precision: 0:x 1:r 2:p 3:t1 4:te 5:spare
  int lo_prec = -1;
  Field xlo32;    // FP32 accumulator of x for the half-precision inner solver
  Field ex[4];    // full solves: eta_e, eta_o, psi_e, psi_o

  // CUDA graphs of one CG iteration block, per precision (0: FP64, 1: FP32, 2: FP16)
  cudaGraphExec_t graph[3] = {nullptr, nullptr, nullptr};
  int graph_iters = 8;
  uint64_t graph_nodes[3] = {0, 0, 0};

  // kernels launched by this context (graph replays count their nodes)
  uint64_t launches = 0;

  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

namespace
{
  tms_status fail(tms_ctx* c, tms_status s, const char* fmt, ...)
  {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (c) c->err = buf;
    return s;
  }

#define CU(call)                                                                                                 \
  do                                                                                                             \
    {                                                                                                            \
      cudaError_t e_ = (call);                                                                                   \
      if (e_ != cudaSuccess)                                                                                     \
        return fail(ctx, e_ == cudaErrorMemoryAllocation ? TMS_ERR_OOM : TMS_ERR_CUDA, "%s: %s (%s:%d)", #call,  \
                    cudaGetErrorString(e_), __FILE__, __LINE__);                                                 \
    }                                                                                                            \
  while (0)

#define TRY(...)                                                                                                 \
  do                                                                                                             \
    {                                                                                                            \
      tms_status s_ = (__VA_ARGS__);                                                                             \
      if (s_ != TMS_OK) return s_;                                                                               \
    }                                                                                                            \
  while (0)

  tms_status alloc_field(tms_ctx* ctx, Field& f, int prec)
  {
    if (f.d && f.prec == prec) return TMS_OK;
    if (f.d)
      {
        cudaFree(f.d);
        f.d = nullptr;
        if (f.n) cudaFree(f.n);
        f.n = nullptr;
      }
    f.prec = prec;
    f.stride = ctx->g.stride;
    const size_t per = (prec == PREC_F64) ? 192 : (prec == PREC_F32) ? 96 : 48;
    f.bytes = per * (size_t)f.stride;
    CU(cudaMalloc(&f.d, f.bytes));
    CU(cudaMemsetAsync(f.d, 0, f.bytes, ctx->stream));
    if (prec == PREC_F16)
      {
        CU(cudaMalloc(&f.n, sizeof(float) * (size_t)f.stride));
        CU(cudaMemsetAsync(f.n, 0, sizeof(float) * (size_t)f.stride, ctx->stream));
      }
    return TMS_OK;
  }

  tms_status ensure_stage(tms_ctx* ctx, size_t bytes)
  {
    if (ctx->stage_bytes >= bytes) return TMS_OK;
    if (ctx->stage) cudaFree(ctx->stage);
    ctx->stage = nullptr;
    ctx->stage_bytes = 0;
    CU(cudaMalloc(&ctx->stage, bytes));
    ctx->stage_bytes = bytes;
    return TMS_OK;
  }

  Reducer reducer(tms_ctx* c) { return Reducer{c->red_partial, c->red_counter, c->red_result}; }

  tms_status set_params(tms_ctx* ctx, double kappa, double mu, int has_anis, double anis, int slot = 0)
  {
    if (!(kappa > 0.0) || !std::isfinite(kappa) || !std::isfinite(mu))
      return fail(ctx, TMS_ERR_BAD_ARG, "invalid kappa %g / mu %g", kappa, mu);
    OpParams h{kappa, mu, has_anis ? anis : 1.0};
    CU(cudaMemcpyAsync(ctx->prm + slot, &h, sizeof h, cudaMemcpyHostToDevice, ctx->stream));
    return TMS_OK;
  }

  // ------------------------------------------------------------ hop launch
  template <int P, int LF, class Epi, class Fin = NoFin>
  void launch_hop(tms_ctx* c, cudaStream_t s, int par_out, int npar, const Field& in_e, const Field& in_o,
                  const LinkT<LF>& U, const OpParams* prm, const Epi& epi, const Fin& fin = Fin{},
                  const int* stop = nullptr)
  {
    const int nsite = (int)(npar * c->g.Vh);
    ++c->launches;
    hop_kernel<P, LF, Epi, Fin><<<div_up(nsite, HOP_THREADS), HOP_THREADS, 0, s>>>(
      c->g, par_out, npar, view<P>(in_e), view<P>(in_o), U, prm, epi, reducer(c), fin, stop);
  }

  LinkT<LINK_F64_18> links64(tms_ctx* c) { return LinkT<LINK_F64_18>{c->U64, (int)c->g.Vh}; }
  LinkT<LINK_F32_12> links32r(tms_ctx* c) { return LinkT<LINK_F32_12>{c->U32r, (int)c->g.Vh}; }
  LinkT<LINK_F32_18> links32f(tms_ctx* c) { return LinkT<LINK_F32_18>{c->U32f, (int)c->g.Vh}; }

  // --------------------------------------------------------- conf kernels
  __global__ void conf_to_soa_kernel(Lattice g, const double* __restrict__ src, int layout, int unfold,
                                     const int* __restrict__ lx_of_eo, double2* __restrict__ U)
  {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= g.V) return;
    const int p = idx >= g.Vh, ieo = idx - (p ? (int)g.Vh : 0);
    const int lx = lx_of_eo[idx];
    const size_t row = (layout == TMS_LAYOUT_LX) ? (size_t)lx : (size_t)idx;
    const int t = lx / (g.LX * g.LY * g.LZ);
    const double2* a = reinterpret_cast<const double2*>(src + row * 72);
    for (int mu = 0; mu < 4; mu++)
      {
        const double sg = (unfold && mu == 0 && t == g.T - 1) ? g.bc_t : 1.0;
        for (int k = 0; k < 9; k++)
          {
            const double2 w = a[mu * 9 + k];
            U[((size_t)(p * 4 + mu) * 9 + k) * g.Vh + ieo] = make_double2(w.x * sg, w.y * sg);
          }
      }
  }

  // FP32 copies and the special-unitarity check (max deviation over links)
  __global__ void conf_lowprec_kernel(int64_t nlinks_per_parmu, int Vh, const double2* __restrict__ U,
                                      float4* __restrict__ Ur, float2* __restrict__ Uf, Reducer red)
  {
    const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; // over 8*Vh (par,mu,site)
    double dev = 0.0;
    if (idx < nlinks_per_parmu)
      {
        const int pm = (int)(idx / Vh), site = (int)(idx - (int64_t)pm * Vh);
        C<double> u[9];
        for (int k = 0; k < 9; k++)
          {
            const double2 w = U[((size_t)pm * 9 + k) * Vh + site];
            u[k] = {w.x, w.y};
            Uf[((size_t)pm * 9 + k) * Vh + site] = make_float2((float)w.x, (float)w.y);
          }
        Ur[((size_t)pm * 3 + 0) * Vh + site] = make_float4((float)u[0].re, (float)u[0].im, (float)u[1].re, (float)u[1].im);
        Ur[((size_t)pm * 3 + 1) * Vh + site] = make_float4((float)u[2].re, (float)u[2].im, (float)u[3].re, (float)u[3].im);
        Ur[((size_t)pm * 3 + 2) * Vh + site] = make_float4((float)u[4].re, (float)u[4].im, (float)u[5].re, (float)u[5].im);
        // deviation of row 2 from conj(row0 x row1), plus row-0/1 unitarity
        const C<double> c0 = cconj(csub(cmul(u[1], u[5]), cmul(u[2], u[4])));
        const C<double> c1 = cconj(csub(cmul(u[2], u[3]), cmul(u[0], u[5])));
        const C<double> c2 = cconj(csub(cmul(u[0], u[4]), cmul(u[1], u[3])));
        dev = fmax(dev, fabs(c0.re - u[6].re) + fabs(c0.im - u[6].im));
        dev = fmax(dev, fabs(c1.re - u[7].re) + fabs(c1.im - u[7].im));
        dev = fmax(dev, fabs(c2.re - u[8].re) + fabs(c2.im - u[8].im));
        double n0 = 0, n1 = 0;
        C<double> d01 = {0, 0};
        for (int k = 0; k < 3; k++)
          {
            n0 += u[k].re * u[k].re + u[k].im * u[k].im;
            n1 += u[3 + k].re * u[3 + k].re + u[3 + k].im * u[3 + k].im;
            d01 = cadd(d01, cjmul(u[k], u[3 + k]));
          }
        dev = fmax(dev, fabs(n0 - 1.0));
        dev = fmax(dev, fabs(n1 - 1.0));
        dev = fmax(dev, fabs(d01.re) + fabs(d01.im));
      }
    // max-reduction through the generic sum reducer: reduce exp-free via a
    // per-block max written as partial; the last block takes the max
    __shared__ double sh[8];
    __shared__ bool last;
    for (int o = 16; o > 0; o >>= 1) dev = fmax(dev, __shfl_xor_sync(0xffffffffu, dev, o));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) sh[warp] = dev;
    __syncthreads();
    if (threadIdx.x == 0)
      {
        double m = 0;
        for (int w = 0; w < (int)(blockDim.x / 32); w++) m = fmax(m, sh[w]);
        red.partial[blockIdx.x] = m;
        __threadfence();
        last = (atomicAdd(red.counter, 1u) == gridDim.x - 1);
      }
    __syncthreads();
    if (last && threadIdx.x == 0)
      {
        __threadfence();
        double m = 0;
        for (int b = 0; b < (int)gridDim.x; b++) m = fmax(m, ((volatile double*)red.partial)[b]);
        *red.result = m;
        *red.counter = 0u;
      }
  }

  __global__ void lx_of_eo_kernel(Lattice g, int* __restrict__ out)
  {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= g.V) return;
    const int p = idx >= g.Vh, ieo = idx - (p ? (int)g.Vh : 0);
    out[idx] = eo_site(g, p, ieo).lx;
  }

  template <int MU, bool UP>
  __device__ int nbr(const Lattice& g, const Site& s)
  {
    bool w;
    return UP ? nbr_up<MU>(g, s, w) : nbr_dw<MU>(g, s, w);
  }

  __global__ void geometry_tables_kernel(Lattice g, int* parity, int* eo_of_lx, int* lx_of_eo, int* nup, int* ndw)
  {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= g.V) return;
    const int p = idx >= g.Vh, ieo = idx - (p ? (int)g.Vh : 0);
    const Site s = eo_site(g, p, ieo);
    parity[s.lx] = p;
    eo_of_lx[s.lx] = ieo;
    lx_of_eo[idx] = s.lx;
    nup[idx * 4 + 0] = nbr<0, true>(g, s);
    nup[idx * 4 + 1] = nbr<1, true>(g, s);
    nup[idx * 4 + 2] = nbr<2, true>(g, s);
    nup[idx * 4 + 3] = nbr<3, true>(g, s);
    ndw[idx * 4 + 0] = nbr<0, false>(g, s);
    ndw[idx * 4 + 1] = nbr<1, false>(g, s);
    ndw[idx * 4 + 2] = nbr<2, false>(g, s);
    ndw[idx * 4 + 3] = nbr<3, false>(g, s);
  }

  // out = (1/2k + i sgn mu g5)^(+-1) in
  template <int P>
  __global__ void diag_kernel(int n, SpinorT<P> in, SpinorT<P> out, const OpParams* prm, double sgn, int inverse)
  {
    using R = typename SpinorT<P>::R;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const C<R> z = inverse ? zinvdiag<R>(*prm, sgn) : zdiag<R>(*prm, sgn);
    C<R> v[12];
    in.load(i, v);
#pragma unroll
    for (int c = 0; c < 12; c++) v[c] = diag_apply(v[c], z, c);
    out.store(i, v);
  }

  // ------------------------------------------------------ spinor transfer
  // bring an e/o spinor (Vh x 24 doubles, host or device) into a FP64 field
  tms_status spinor_in(tms_ctx* ctx, const double* src, const int* site_map, int64_t nrows, Field& f)
  {
    TRY(alloc_field(ctx, f, PREC_F64));
    const double* d = src;
    const size_t bytes = (size_t)nrows * 24 * sizeof(double);
    if (ctx->ptr_mode == TMS_PTR_HOST)
      {
        TRY(ensure_stage(ctx, bytes));
        CU(cudaMemcpyAsync(ctx->stage, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
        d = ctx->stage;
      }
    const int n = (int)ctx->g.Vh;
    ++ctx->launches;
    aos_to_soa_kernel<PREC_F64><<<div_up(n, 256), 256, 0, ctx->stream>>>(n, d, site_map, view<PREC_F64>(f));
    CU(cudaGetLastError());
    return TMS_OK;
  }

  // write a FP64 field out as Vh rows (optionally scattered through site_map) of 24 doubles
  tms_status spinor_out(tms_ctx* ctx, const Field& f, const int* site_map, int64_t nrows, double* dst, bool flush)
  {
    const size_t bytes = (size_t)nrows * 24 * sizeof(double);
    double* d = dst;
    if (ctx->ptr_mode == TMS_PTR_HOST)
      {
        TRY(ensure_stage(ctx, bytes));
        d = ctx->stage;
      }
    const int n = (int)ctx->g.Vh;
    ++ctx->launches;
    soa_to_aos_kernel<PREC_F64><<<div_up(n, 256), 256, 0, ctx->stream>>>(n, view<PREC_F64>(f), site_map, d);
    CU(cudaGetLastError());
    if (ctx->ptr_mode == TMS_PTR_HOST && flush)
      {
        CU(cudaMemcpyAsync(dst, ctx->stage, bytes, cudaMemcpyDeviceToHost, ctx->stream));
        CU(cudaStreamSynchronize(ctx->stream));
      }
    return TMS_OK;
  }

  tms_status finish(tms_ctx* ctx)
  {
    CU(cudaGetLastError());
    CU(cudaStreamSynchronize(ctx->stream));
    return TMS_OK;
  }

  tms_status check_conf(tms_ctx* ctx)
  {
    if (!ctx) return TMS_ERR_BAD_ARG;
    if (!ctx->conf_loaded) return fail(ctx, TMS_ERR_NO_CONF, "no gauge configuration uploaded");
    CU(cudaSetDevice(ctx->device));
    return TMS_OK;
  }

  double read_result(tms_ctx* ctx)
  {
    cudaMemcpyAsync(ctx->red_h, ctx->red_result, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
    cudaStreamSynchronize(ctx->stream);
    return *ctx->red_h;
  }

  template <int P>
  tms_status norm2(tms_ctx* ctx, const Field& a, double* out)
  {
    const int n = (int)ctx->g.Vh;
    ++ctx->launches;
    norm_kernel<P, false><<<div_up(n, BLAS_THREADS), BLAS_THREADS, 0, ctx->stream>>>(n, view<P>(a), view<P>(a),
                                                                                      reducer(ctx));
    CU(cudaGetLastError());
    *out = read_result(ctx);
    return TMS_OK;
  }

  // ------------------------------------------------------ K operators FP64
  // out = K(sgn mu) in  (odd -> odd), te is the even temporary
  template <int P, int LF>
  void kern_op(tms_ctx* c, const LinkT<LF>& U, const Field& in, const Field& te, const Field& out, double sgn,
               const OpParams* prm)
  {
    EpiInvDiag<P> ea{{view<P>(te), view<P>(te)}, prm, sgn};
    launch_hop<P, LF>(c, c->stream, 0, 1, in, in, U, prm, ea);
    EpiKern<P, false> eb{{view<P>(out), view<P>(out)}, {view<P>(in), view<P>(in)}, prm, sgn};
    launch_hop<P, LF>(c, c->stream, 1, 1, te, te, U, prm, eb);
  }

  // true residual r = b - K(+mu)K(-mu) x in FP64; returns |r|^2
  tms_status true_residual(tms_ctx* ctx, const Field& b, const Field& x, const Field& r, double* rr)
  {
    Field &t1 = ctx->f64[4], &te = ctx->f64[5], &s = ctx->f64[6];
    auto U = links64(ctx);
    kern_op<PREC_F64>(ctx, U, x, te, t1, -1.0, ctx->prm);
    kern_op<PREC_F64>(ctx, U, t1, te, s, +1.0, ctx->prm);
    const int n = (int)ctx->g.Vh;
    ++ctx->launches;
    residual_kernel<<<div_up(n, BLAS_THREADS), BLAS_THREADS, 0, ctx->stream>>>(
      n, view<PREC_F64>(b), view<PREC_F64>(s), view<PREC_F64>(r), reducer(ctx));
    CU(cudaGetLastError());
    *rr = read_result(ctx);
    return TMS_OK;
  }

  // record `iters` CG iterations in precision P (x in precision PX) on the stream
  template <int P, int PX, int LF>
  void record_cg_iterations(tms_ctx* c, cudaStream_t s, const LinkT<LF>& U, Field* v, const Field& x, int iters)
  {
    // v: 0 unused, 1 r, 2 p, 3 t1, 4 te
    const Field &r = v[1], &p = v[2], &t1 = v[3], &te = v[4];
    const int* stop = &c->st->stop;
    const OpParams* prm = c->prm;
    for (int it = 0; it < iters; it++)
      {
        EpiInvDiag<P> a1{{view<P>(te), view<P>(te)}, prm, -1.0};
        launch_hop<P, LF>(c, s, 0, 1, p, p, U, prm, a1, NoFin{}, stop);
        EpiKern<P, true> b1{{view<P>(t1), view<P>(t1)}, {view<P>(p), view<P>(p)}, prm, -1.0};
        launch_hop<P, LF>(c, s, 1, 1, te, te, U, prm, b1, FinAlpha{c->st}, stop);
        EpiInvDiag<P> a2{{view<P>(te), view<P>(te)}, prm, +1.0};
        launch_hop<P, LF>(c, s, 0, 1, t1, t1, U, prm, a2, NoFin{}, stop);
        EpiKernCgUpdate<P, PX> b2{view<P>(t1), view<P>(r), view<P>(p), view<PX>(x), prm, c->st, +1.0};
        launch_hop<P, LF>(c, s, 1, 1, te, te, U, prm, b2, FinBeta{c->st}, stop);
        const int n = (int)c->g.Vh;
        ++c->launches;
        xpay_kernel<P><<<div_up(n, BLAS_THREADS), BLAS_THREADS, 0, s>>>(n, view<P>(r), view<P>(p), c->st, stop);
      }
  }

  template <int P, int PX, int LF>
  tms_status build_graph(tms_ctx* ctx, int slot, const LinkT<LF>& U, Field* v, const Field& x)
  {
    if (ctx->graph[slot]) return TMS_OK;
    cudaStream_t cs;
    CU(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaGraph_t graph;
    CU(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    const uint64_t before = ctx->launches;
    record_cg_iterations<P, PX, LF>(ctx, cs, U, v, x, ctx->graph_iters);
    ctx->graph_nodes[slot] = ctx->launches - before;
    ctx->launches = before;
    cudaError_t e = cudaStreamEndCapture(cs, &graph);
    cudaStreamDestroy(cs);
    if (e != cudaSuccess) return fail(ctx, TMS_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&ctx->graph[slot], graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return fail(ctx, TMS_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
    return TMS_OK;
  }

  tms_status push_state(tms_ctx* ctx)
  {
    CU(cudaMemcpyAsync(ctx->st, ctx->st_h, sizeof(CgState), cudaMemcpyHostToDevice, ctx->stream));
    return TMS_OK;
  }
  tms_status pull_state(tms_ctx* ctx)
  {
    CU(cudaMemcpyAsync(ctx->st_h, ctx->st, sizeof(CgState), cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    return TMS_OK;
  }

  template <int PD, int PS>
  void convert(tms_ctx* c, const Field& src, const Field& dst, double a = 1.0)
  {
    const int n = (int)c->g.Vh;
    ++c->launches;
    axpby_kernel<PD, PS, PS><<<div_up(n, BLAS_THREADS), BLAS_THREADS, 0, c->stream>>>(n, a, view<PS>(src), 0.0,
                                                                                       view<PS>(src), view<PD>(dst));
  }

  // ------------------------------------------------------------- CG, FP64
  // b = f64[0] (odd source), x = f64[1] (initial guess / solution).  Implements
  // cg_invert (cg_invert_template_threaded.hpp:17-150) with the operator of
  // inv_tmDkern_eoprec_square_eos_cg_64 (cg_64_invert_tmD_eoprec.hpp:11-40).
  tms_status cg_double(tms_ctx* ctx, int niter, double residue, bool have_guess, tms_stats* stats)
  {
    Field* f = ctx->f64;
    for (int i = 1; i <= 6; i++) TRY(alloc_field(ctx, f[i], PREC_F64));
    double b2;
    TRY(norm2<PREC_F64>(ctx, f[0], &b2));
    if (b2 == 0.0 || std::isnan(b2)) return fail(ctx, TMS_ERR_INVALID_SOURCE, "invalid norm: %g", b2);
    double rr;
    if (have_guess) TRY(true_residual(ctx, f[0], f[1], f[2], &rr));
    else
      {
        CU(cudaMemsetAsync(f[1].d, 0, f[1].bytes, ctx->stream));
        CU(cudaMemcpyAsync(f[2].d, f[0].d, f[0].bytes, cudaMemcpyDeviceToDevice, ctx->stream));
        rr = b2;
      }
    CU(cudaMemcpyAsync(f[3].d, f[2].d, f[2].bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    CgState& S = *ctx->st_h;
    memset(&S, 0, sizeof S);
    S.rr = rr;
    S.b2 = b2;
    S.target = residue * b2;
    S.rel_trigger = -1.0;
    S.niter_max = niter;
    S.stop = (rr < S.target) ? STOP_CONVERGED : STOP_RUN;
    TRY(push_state(ctx));
    auto U = links64(ctx);
    Field v[5] = {Field{}, f[2], f[3], f[4], f[5]};
    TRY(build_graph<PREC_F64, PREC_F64>(ctx, 0, U, v, f[1]));
    CU(cudaEventRecord(ctx->ev0, ctx->stream));
    while (S.stop == STOP_RUN)
      {
        CU(cudaGraphLaunch(ctx->graph[0], ctx->stream));
        ctx->launches += ctx->graph_nodes[0];
        TRY(pull_state(ctx));
      }
    CU(cudaEventRecord(ctx->ev1, ctx->stream));
    double tr;
    TRY(true_residual(ctx, f[0], f[1], f[6], &tr));
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    tms_status st = TMS_OK;
    if (S.stop == STOP_BREAKDOWN) st = fail(ctx, TMS_ERR_NAN, "nanned (iteration %d)", S.iter);
    else if (S.stop == STOP_MAXITER) st = fail(ctx, TMS_ERR_NOT_CONVERGED, "exit without converging");
    if (stats)
      {
        stats->status = st;
        stats->iterations = S.iter;
        stats->reliable_updates = 0;
        stats->iterated_rel_res2 = S.rr / b2;
        stats->true_rel_res2 = tr / b2;
        stats->seconds = ms * 1e-3;
      }
    return st;
  }

  // ------------------------------------------------- CG, mixed precision
  // FP32 (or FP16-spinor) inner CG with FP64 reliable updates: the solution is
  // accumulated in FP64 and the residual recomputed with the FP64 operator
  // whenever the iterated residual has dropped by delta since the last update
  // (the outer defect-correction loop of cg_128_invert_template_threaded.cpp:36-109,
  // here with the Krylov direction kept across updates).
  template <int P, int LF>
  tms_status cg_mixed(tms_ctx* ctx, const LinkT<LF>& U, int slot, int niter, double residue, bool have_guess,
                      tms_stats* stats)
  {
    constexpr int PX = (P == PREC_F16) ? PREC_F32 : P; // x accumulates in FP32 at least
    Field* f = ctx->f64;
    for (int i = 1; i <= 6; i++) TRY(alloc_field(ctx, f[i], PREC_F64));
    if (ctx->lo_prec != P)
      {
        // the inner-precision fields move: graphs captured on the old ones are void
        CU(cudaStreamSynchronize(ctx->stream));
        for (int g = 1; g < 3; g++)
          if (ctx->graph[g])
            {
              cudaGraphExecDestroy(ctx->graph[g]);
              ctx->graph[g] = nullptr;
            }
        for (auto& l : ctx->lo) TRY(alloc_field(ctx, l, P));
        ctx->lo_prec = P;
      }
    TRY(alloc_field(ctx, ctx->xlo32, PX));
    Field* lo = ctx->lo;
    Field& xlo = ctx->xlo32;
    const double delta = (P == PREC_F16) ? 0.1 : 0.05; // reliable-update trigger (residual reduction)
    double b2;
    TRY(norm2<PREC_F64>(ctx, f[0], &b2));
    if (b2 == 0.0 || std::isnan(b2)) return fail(ctx, TMS_ERR_INVALID_SOURCE, "invalid norm: %g", b2);
    double rr;
    if (have_guess) TRY(true_residual(ctx, f[0], f[1], f[2], &rr));
    else
      {
        CU(cudaMemsetAsync(f[1].d, 0, f[1].bytes, ctx->stream));
        CU(cudaMemcpyAsync(f[2].d, f[0].d, f[0].bytes, cudaMemcpyDeviceToDevice, ctx->stream));
        rr = b2;
      }
    const double target = residue * b2;
    CgState& S = *ctx->st_h;
    memset(&S, 0, sizeof S);
    int reliable = 0;
    float ms = 0;
    tms_status st = TMS_OK;
    if (rr >= target)
      {
        convert<P, PREC_F64>(ctx, f[2], lo[1]); // r_lo = r
        convert<P, PREC_F64>(ctx, f[2], lo[2]); // p_lo = r
        CU(cudaMemsetAsync(xlo.d, 0, xlo.bytes, ctx->stream));
        S.rr = rr;
        S.b2 = b2;
        S.target = target;
        S.rel_trigger = delta * delta * rr;
        S.niter_max = niter;
        S.stop = STOP_RUN;
        TRY(push_state(ctx));
        Field v[5] = {Field{}, lo[1], lo[2], lo[3], lo[4]};
        TRY(build_graph<P, PX>(ctx, slot, U, v, xlo));
        CU(cudaEventRecord(ctx->ev0, ctx->stream));
        for (;;)
          {
            CU(cudaGraphLaunch(ctx->graph[slot], ctx->stream));
            ctx->launches += ctx->graph_nodes[slot];
            TRY(pull_state(ctx));
            if (S.stop == STOP_RUN) continue;
            if (S.stop == STOP_BREAKDOWN)
              {
                st = fail(ctx, TMS_ERR_NAN, "nanned (iteration %d)", S.iter);
                break;
              }
            // reliable update: x += x_lo (FP64), r = b - A x (FP64)
            const int n = (int)ctx->g.Vh;
            ++ctx->launches;
            axpby_kernel<PREC_F64, PREC_F64, PX><<<div_up(n, BLAS_THREADS), BLAS_THREADS, 0, ctx->stream>>>(
              n, 1.0, view<PREC_F64>(f[1]), 1.0, view<PX>(xlo), view<PREC_F64>(f[1]));
            CU(cudaMemsetAsync(xlo.d, 0, xlo.bytes, ctx->stream));
            if (xlo.n) CU(cudaMemsetAsync(xlo.n, 0, sizeof(float) * xlo.stride, ctx->stream));
            double rt;
            TRY(true_residual(ctx, f[0], f[1], f[2], &rt));
            reliable++;
            if (rt < target) break;
            if (S.stop == STOP_MAXITER || S.iter >= niter)
              {
                st = fail(ctx, TMS_ERR_NOT_CONVERGED, "exit without converging");
                break;
              }
            // restart the recurrence from the true residual, keeping the direction
            convert<P, PREC_F64>(ctx, f[2], lo[1]);
            const double beta = rt / S.rr_prev;
            S.beta = beta;
            S.rr = rt;
            S.rel_trigger = delta * delta * rt;
            S.stop = STOP_RUN;
            TRY(push_state(ctx));
            ++ctx->launches;
            xpay_kernel<P><<<div_up(n, BLAS_THREADS), BLAS_THREADS, 0, ctx->stream>>>(n, view<P>(lo[1]),
                                                                                       view<P>(lo[2]), ctx->st,
                                                                                       nullptr);
            CU(cudaGetLastError());
          }
        CU(cudaEventRecord(ctx->ev1, ctx->stream));
        CU(cudaEventSynchronize(ctx->ev1));
        cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
      }
    double tr;
    TRY(true_residual(ctx, f[0], f[1], f[6], &tr));
    if (stats)
      {
        stats->status = st;
        stats->iterations = S.iter;
        stats->reliable_updates = reliable;
        stats->iterated_rel_res2 = S.rr / b2;
        stats->true_rel_res2 = tr / b2;
        stats->seconds = ms * 1e-3;
      }
    return st;
  }

  tms_status cg_dispatch(tms_ctx* ctx, int precision, int niter, double residue, bool have_guess, tms_stats* stats)
  {
    if (precision == TMS_PREC_DOUBLE) return cg_double(ctx, niter, residue, have_guess, stats);
    if (precision == TMS_PREC_MIXED_SINGLE)
      return ctx->su3 ? cg_mixed<PREC_F32>(ctx, links32r(ctx), 1, niter, residue, have_guess, stats)
                      : cg_mixed<PREC_F32>(ctx, links32f(ctx), 1, niter, residue, have_guess, stats);
    if (precision == TMS_PREC_MIXED_HALF)
      return ctx->su3 ? cg_mixed<PREC_F16>(ctx, links32r(ctx), 2, niter, residue, have_guess, stats)
                      : cg_mixed<PREC_F16>(ctx, links32f(ctx), 2, niter, residue, have_guess, stats);
    return fail(ctx, TMS_ERR_BAD_ARG, "unknown precision %d", precision);
  }
}

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
    for (int r = 0; r < nrep; r++)
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
        total += t;
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
  ctx->red_cap = div_up(V, 64) + 1024;
  if (cudaMalloc(&ctx->lx_of_eo, sizeof(int) * V) != cudaSuccess ||
      cudaMalloc(&ctx->prm, sizeof(OpParams) * 2) != cudaSuccess ||
      cudaMalloc(&ctx->st, sizeof(CgState)) != cudaSuccess ||
      cudaMalloc(&ctx->red_partial, sizeof(double) * ctx->red_cap) != cudaSuccess ||
      cudaMalloc(&ctx->red_counter, sizeof(unsigned)) != cudaSuccess ||
      cudaMalloc(&ctx->red_result, sizeof(double)) != cudaSuccess ||
      cudaMallocHost(&ctx->st_h, sizeof(CgState)) != cudaSuccess ||
      cudaMallocHost(&ctx->red_h, sizeof(double)) != cudaSuccess)
    return cleanup(TMS_ERR_OOM);
  cudaMemset(ctx->red_counter, 0, sizeof(unsigned));
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
  for (auto& gr : ctx->graph)
    if (gr) cudaGraphExecDestroy(gr);
  auto fr = [](void* p) {
    if (p) cudaFree(p);
  };
  for (auto& f : ctx->f64) { fr(f.d); fr(f.n); }
  for (auto& f : ctx->lo) { fr(f.d); fr(f.n); }
  for (auto& f : ctx->ex) { fr(f.d); fr(f.n); }
  fr(ctx->xlo32.d);
  fr(ctx->xlo32.n);
  fr(ctx->lx_of_eo);
  fr(ctx->U64);
  fr(ctx->U32r);
  fr(ctx->U32f);
  fr(ctx->prm);
  fr(ctx->st);
  fr(ctx->red_partial);
  fr(ctx->red_counter);
  fr(ctx->red_result);
  fr(ctx->stage);
  if (ctx->st_h) cudaFreeHost(ctx->st_h);
  if (ctx->red_h) cudaFreeHost(ctx->red_h);
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
  conf_lowprec_kernel<<<div_up(nl, 256), 256, 0, ctx->stream>>>(nl, (int)Vh, ctx->U64, ctx->U32r, ctx->U32f,
                                                                 reducer(ctx));
  CU(cudaGetLastError());
  const double dev = read_result(ctx);
  CU(cudaGetLastError());
  ctx->su3 = (dev < 1e-10);
  ctx->conf_loaded = true;
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

tms_status tms_cg_eoprec_square(tms_ctx* ctx, double* sol, const double* guess, const double* src, double kappa,
                                int has_anis, double anis, double mu, int niter, double residue, int precision,
                                tms_stats* stats)
{
  TRY(check_conf(ctx));
  if (!sol || !src || niter <= 0 || !(residue > 0)) return fail(ctx, TMS_ERR_BAD_ARG, "bad solver arguments");
  TRY(set_params(ctx, kappa, mu, has_anis, anis));
  Field* f = ctx->f64;
  TRY(spinor_in(ctx, src, nullptr, ctx->g.Vh, f[0]));
  if (guess) TRY(spinor_in(ctx, guess, nullptr, ctx->g.Vh, f[1]));
  const tms_status st = cg_dispatch(ctx, precision, niter, residue, guess != nullptr, stats);
  if (st == TMS_OK || st == TMS_ERR_NOT_CONVERGED) TRY(spinor_out(ctx, f[1], nullptr, ctx->g.Vh, sol, true));
  TRY(finish(ctx));
  return st;
}

tms_status tms_cg_eoprec(tms_ctx* ctx, double* sol_lx, const double* src_lx, double kappa, int has_anis, double anis,
                         double mu, int niter, double residue, int precision, tms_stats* stats)
{
  TRY(check_conf(ctx));
  if (!sol_lx || !src_lx || niter <= 0 || !(residue > 0)) return fail(ctx, TMS_ERR_BAD_ARG, "bad solver arguments");
  TRY(set_params(ctx, kappa, mu, has_anis, anis));
  Field* f = ctx->f64;
  for (int i = 0; i <= 7; i++) TRY(alloc_field(ctx, f[i], PREC_F64));
  Field *eta = ctx->ex, *psi = ctx->ex + 2; // [0] even, [1] odd
  for (auto& e : ctx->ex) TRY(alloc_field(ctx, e, PREC_F64));
  const int64_t Vh = ctx->g.Vh;
  const int n = (int)Vh;
  const size_t bytes = (size_t)ctx->g.V * 24 * sizeof(double);
  auto V = [&](const Field& x) { return view<PREC_F64>(x); };
  auto U = links64(ctx);
  // split_lx_vector_into_eo_parts(source)
  const double* src = src_lx;
  if (ctx->ptr_mode == TMS_PTR_HOST)
    {
      TRY(ensure_stage(ctx, bytes));
      CU(cudaMemcpyAsync(ctx->stage, src_lx, bytes, cudaMemcpyHostToDevice, ctx->stream));
      src = ctx->stage;
    }
  ++ctx->launches;
  aos_to_soa_kernel<PREC_F64><<<div_up(n, 256), 256, 0, ctx->stream>>>(n, src, ctx->lx_of_eo, V(eta[0]));
  ++ctx->launches;
  aos_to_soa_kernel<PREC_F64><<<div_up(n, 256), 256, 0, ctx->stream>>>(n, src, ctx->lx_of_eo + Vh, V(eta[1]));
  // Eq. (8a): te = D_ee^-1 eta_e ; Eq. (8b): varphi = g5 (eta_o + hop(te)/2) -> f0
  ++ctx->launches;
  diag_kernel<PREC_F64><<<div_up(n, 256), 256, 0, ctx->stream>>>(n, V(eta[0]), V(f[5]), ctx->prm, 1.0, 1);
  EpiSrcPrep<PREC_F64> sp{{V(f[0]), V(f[0])}, {V(eta[1]), V(eta[1])}};
  launch_hop<PREC_F64, LINK_F64_18>(ctx, ctx->stream, 1, 1, f[5], f[5], U, ctx->prm, sp);
  CU(cudaGetLastError());
  // Eq. (9)
  const tms_status st = cg_dispatch(ctx, precision, niter, residue, false, stats);
  if (st != TMS_OK && st != TMS_ERR_NOT_CONVERGED) return st;
  // Eq. (10): psi_o = K(-mu) x ; Eq. (11): psi_e = D_ee^-1 (eta_e + hop(psi_o)/2)
  kern_op<PREC_F64>(ctx, U, f[1], f[5], psi[1], -1.0, ctx->prm);
  EpiReco<PREC_F64> rc{{V(psi[0]), V(psi[0])}, {V(eta[0]), V(eta[0])}, ctx->prm, 1.0};
  launch_hop<PREC_F64, LINK_F64_18>(ctx, ctx->stream, 0, 1, psi[1], psi[1], U, ctx->prm, rc);
  CU(cudaGetLastError());
  // paste_eo_parts_into_lx_vector
  double* d = (ctx->ptr_mode == TMS_PTR_HOST) ? ctx->stage : sol_lx;
  ++ctx->launches;
  soa_to_aos_kernel<PREC_F64><<<div_up(n, 256), 256, 0, ctx->stream>>>(n, V(psi[0]), ctx->lx_of_eo, d);
  ++ctx->launches;
  soa_to_aos_kernel<PREC_F64><<<div_up(n, 256), 256, 0, ctx->stream>>>(n, V(psi[1]), ctx->lx_of_eo + Vh, d);
  CU(cudaGetLastError());
  if (ctx->ptr_mode == TMS_PTR_HOST) CU(cudaMemcpyAsync(sol_lx, ctx->stage, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  // lx residual check (cg_invert_tmD_eoprec.cpp:192-212): |g5 Q sol - src|^2 / |src|^2
  if (stats)
    {
      EpiTmQ<PREC_F64, false> e{{V(f[2]), V(f[3])}, {V(psi[0]), V(psi[1])}, ctx->prm, +1.0};
      launch_hop<PREC_F64, LINK_F64_18>(ctx, ctx->stream, 0, 2, psi[0], psi[1], U, ctx->prm, e);
      double num = 0, den = 0;
      for (int par = 0; par < 2; par++)
        {
          ++ctx->launches;
          g5_residual_kernel<<<div_up(n, BLAS_THREADS), BLAS_THREADS, 0, ctx->stream>>>(n, V(f[2 + par]), V(eta[par]),
                                                                                       reducer(ctx));
          CU(cudaGetLastError());
          num += read_result(ctx);
          double e2;
          TRY(norm2<PREC_F64>(ctx, eta[par], &e2));
          den += e2;
        }
      stats->lx_rel_res2 = num / den;
    }
  TRY(finish(ctx));
  return st;
}

uint64_t tms_launch_count(const tms_ctx* ctx) { return ctx ? ctx->launches : 0; }

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
  if (precision == TMS_PREC_MIXED_SINGLE)
    return ctx->su3 ? bench_hop_t<PREC_F32>(ctx, links32r(ctx), variant, nrep, flush, ms_per_launch, 48.0, 96.0,
                                            bytes_per_launch)
                    : bench_hop_t<PREC_F32>(ctx, links32f(ctx), variant, nrep, flush, ms_per_launch, 72.0, 96.0,
                                            bytes_per_launch);
  if (precision == TMS_PREC_MIXED_HALF)
    return ctx->su3 ? bench_hop_t<PREC_F16>(ctx, links32r(ctx), variant, nrep, flush, ms_per_launch, 48.0, 52.0,
                                            bytes_per_launch)
                    : bench_hop_t<PREC_F16>(ctx, links32f(ctx), variant, nrep, flush, ms_per_launch, 72.0, 52.0,
                                            bytes_per_launch);
  return fail(ctx, TMS_ERR_BAD_ARG, "unknown precision %d", precision);
}

} // extern "C"
