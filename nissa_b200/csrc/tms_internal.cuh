// Internal state and helpers of the C ABI shared by its translation units:
// the context (tms_ctx), device fields, error handling, parameter upload,
// kernel launch helpers and the boundary (AoS <-> SoA) transfers.
#pragma once
#include "tmsolve.h"
#include "tms_kernels.cuh"
#include "tms_pipe.cuh"
#include "tms_hop_sp.cuh"
#include "tms_hop_tma.cuh"
#include "tms_clover.cuh"

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

using namespace tms;

namespace tms_int
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

using tms_int::Field;

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
  char* U16r = nullptr; // 12-real, 16-bit fixed point (LinkT<LINK_I16_12> blocks)
  char* U16h = nullptr; // 12-real, FP16 values (LinkT<LINK_H16_12>), for the FP16-arithmetic hop

  // scalars and reduction scratch
  OpParams* prm = nullptr;       // [2]: operator params (slot 0 solver, slot 1 free use)
  CgState* st = nullptr;         // device solver state
  CgState* st_h = nullptr;       // pinned host mirror
  double* red_partial = nullptr;
  unsigned* red_counter = nullptr;
  double* red_result = nullptr;
  unsigned* tma_timeouts = nullptr; // timed-out tile waits of the staged hop (launch shape 7); stays 0

  // time-slab context (tms_create_slab): slices [slab_t0, slab_t0 + T) of a lattice of slab_T slices
  bool slab = false;
  int slab_T = 0, slab_t0 = 0;
  double slab_bc_fwd = 1.0, slab_bc_bwd = 1.0; // signs of the faces crossing t = T-1 -> 0
  void* slab_ghost = nullptr;                  // device copies of the two received faces
  double* red_h = nullptr;       // pinned
  int red_cap = 0;
  // Scalars cross between host and device through mapped page-locked memory
  // and a one-block copy kernel on the stream, not through the copy engines,
  // which may be busy with the column copies of the copy stream: st_h and
  // red_h are mapped (device addresses st_hd, red_hd); host->device scalars
  // are staged in the ring hring (device address hring_d).
  CgState* st_hd = nullptr;
  double* red_hd = nullptr;
  unsigned char* hring = nullptr;
  unsigned char* hring_d = nullptr;
  size_t hring_off = 0;

  // staging for AoS conversions (device AoS doubles), grows on demand
  double* stage = nullptr;
  size_t stage_bytes = 0;

  // work fields (allocated on first use)
  Field f64[8];   // 0:b 1:x 2:r 3:p 4:t1 5:te(even) 6:s 7:tmp
  Field lo[6];    // inner precision: 0:x 1:r 2:p 3:t1 4:te 5:spare
  int lo_prec = -1;
  Field xlo32;    // FP32 accumulator of x for the half-precision inner solver
  Field ex[4];    // full solves: eta_e, eta_o, psi_e, psi_o

  // full-lattice fields (both parities, plane stride 2*g.stride, parity p at offset p*g.stride)
  Field lx64[8];  // 0:b 1:x 2:r 3:p 4:t 5:s 6,7:tmp
  Field lxlo[5];  // inner precision: 1:r 2:p 3:t
  int lxlo_prec = -1;
  Field lxxlo;    // FP32 accumulator of x (full lattice)

  // multi-shift CGM: state and the per-shift solutions / directions
  CgmState* cgm = nullptr;
  CgmState* cgm_h = nullptr;
  void* cgm_x = nullptr;
  void* cgm_ps = nullptr;
  int cgm_prec = -1, cgm_nshift = 0;

  // lx spinor buffers on the device for the propagator entry points (tms_prop.cu)
  double* lxbuf[2] = {nullptr, nullptr};

  // twisted clover (tms_clover_term): the clover term of both parities and
  // the twisted inverse on even sites for (icl_kappa, icl_mu)
  bool clov_ok = false, icl_ok = false;
  double clov_csw = 0.0, icl_kappa = 0.0, icl_mu = 0.0;
  double2* cl64 = nullptr;  // [par][36][Vh]
  float2* cl32 = nullptr;
  double2* icl64 = nullptr; // [2 chiralities][6][6][Vh], even sites
  float2* icl32 = nullptr;

  // CUDA graphs of one iteration block: 0-2 e/o CG (FP64, FP32, FP16),
  // 3-5 full-lattice CG (FP64, FP32, FP16), 6-7 CGM (FP64, FP32),
  // 8-10 e/o twisted-clover CG (FP64, FP32, FP16)
  static constexpr int kGraphs = 11;
  cudaGraphExec_t graph[kGraphs] = {};
  int graph_iters = 8;
  int batch_iters = 0;  // CG iterations per batch-session graph block (0: by batch size)
  uint64_t graph_nodes[kGraphs] = {};

  // tuning (tms_set_tuning): hopping-kernel launch shape per precision, the
  // reliable-update trigger of the mixed solvers
  int hop_cfg[3] = {0, 1, 6};
  int tma_rows = 0; // lattice rows per tile of the staged hop (launch shape 7): 0 the most that fit
  double delta_single = 1e-3, delta_half = 0.005;
  int single_links16 = 1; // FP32-spinor inner solver on 16-bit fixed-point links (1) or FP32 12-real links (0)
  int half_arith = 0; // FP16-spinor e/o solver: FP32 arithmetic (0) or the FP16-arithmetic pipelined hop (1)
  int reliable_links12 = 1; // FP64 residuals of the mixed solvers on 12-real FP64 links (when SU(3) to rounding)
  double su3_dev = 1.0;     // largest deviation of the resident links from SU(3) (unitarity, row 2)
  int mrhs_r = 1; // right-hand sides per thread in the batched hopping kernel (1, 2, 4; FP64 at most 2)
  int pdl = 1;    // launch the CG iteration kernels with programmatic dependent launch
  double cgm_floor32 = 1e-12; // squared residue at which the FP32 multi-shift phase hands over to refinement
  int cgm_refine_batched = 0; // mixed multi-shift: shifts corrected one after the other (0) or as batched solves (1)

  // batched-solver workspace (owned by tms_batch.cu)
  void* bw = nullptr;
  void (*bw_free)(void*) = nullptr;

  // kernels launched by this context (graph replays count their nodes)
  uint64_t launches = 0;

  cudaEvent_t ev0 = nullptr, ev1 = nullptr;

  // pipelined host-buffer column solves: a copy stream, two source and two
  // solution staging buffers, and the events that order them
  cudaStream_t cstream = nullptr;
  double* colbuf[4] = {nullptr, nullptr, nullptr, nullptr}; // in 0, in 1, out 0, out 1
  size_t colbuf_bytes = 0;
  cudaEvent_t colev[8] = {}; // in ready 0/1, in free 0/1, out ready 0/1, out free 0/1
};

namespace tms_int
{
  inline tms_status fail(tms_ctx* c, tms_status s, const char* fmt, ...)
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

  inline tms_status alloc_field(tms_ctx* ctx, Field& f, int prec, int stride = 0)
  {
    if (stride == 0) stride = ctx->g.stride;
    if (f.d && f.prec == prec && f.stride == stride) return TMS_OK;
    if (f.d)
      {
        cudaFree(f.d);
        f.d = nullptr;
        if (f.n) cudaFree(f.n);
        f.n = nullptr;
      }
    f.prec = prec;
    f.stride = stride;
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

  inline tms_status ensure_stage(tms_ctx* ctx, size_t bytes)
  {
    if (ctx->stage_bytes >= bytes) return TMS_OK;
    if (ctx->stage) cudaFree(ctx->stage);
    ctx->stage = nullptr;
    ctx->stage_bytes = 0;
    CU(cudaMalloc(&ctx->stage, bytes));
    ctx->stage_bytes = bytes;
    return TMS_OK;
  }

  inline Reducer reducer(tms_ctx* c) { return Reducer{c->red_partial, c->red_counter, c->red_result}; }

  constexpr size_t kHostRing = 64 << 10;

  // dst[0..nwords) = src[..]; either side may be mapped host memory
  static __global__ void word_copy_kernel(const unsigned* __restrict__ src, unsigned* __restrict__ dst, int nwords)
  {
    for (int i = threadIdx.x; i < nwords; i += blockDim.x) dst[i] = src[i];
    __threadfence_system();
  }

  // host scalars -> device memory, in stream order (staged in the mapped ring;
  // the ring is reused only after the stream has drained)
  inline tms_status put_small(tms_ctx* ctx, void* dst, const void* src, size_t bytes)
  {
    const size_t need = (bytes + 15) & ~size_t(15);
    if (bytes % 4 || need > kHostRing) return fail(ctx, TMS_ERR_BAD_ARG, "put_small: %zu bytes", bytes);
    if (ctx->hring_off + need > kHostRing)
      {
        CU(cudaStreamSynchronize(ctx->stream));
        ctx->hring_off = 0;
      }
    memcpy(ctx->hring + ctx->hring_off, src, bytes);
    ++ctx->launches;
    word_copy_kernel<<<1, 64, 0, ctx->stream>>>(reinterpret_cast<const unsigned*>(ctx->hring_d + ctx->hring_off),
                                                static_cast<unsigned*>(dst), (int)(bytes / 4));
    ctx->hring_off += need;
    CU(cudaGetLastError());
    return TMS_OK;
  }

  inline tms_status set_params(tms_ctx* ctx, double kappa, double mu, int has_anis, double anis, int slot = 0)
  {
    if (!(kappa > 0.0) || !std::isfinite(kappa) || !std::isfinite(mu))
      return fail(ctx, TMS_ERR_BAD_ARG, "invalid kappa %g / mu %g", kappa, mu);
    OpParams h{kappa, mu, has_anis ? anis : 1.0};
    return put_small(ctx, ctx->prm + slot, &h, sizeof h);
  }

  // ------------------------------------------------------------ hop launch
  // a launch with programmatic stream serialisation (when enabled): the kernel
  // may start while its predecessor drains; it waits in pdl_enter()
  template <typename... KArgs, typename... Args>
  inline void launch_pdl(tms_ctx* c, void (*k)(KArgs...), int grid, int block, size_t smem, cudaStream_t s,
                         Args... args)
  {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3((unsigned)block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = c->pdl ? 1 : 0;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, k, static_cast<KArgs>(args)...);
  }

  template <int P, int LF, class Epi, class Fin = NoFin>
  void launch_hop_v(tms_ctx* c, cudaStream_t s, int par_out, int npar, const SpinorT<P>& in_e,
                    const SpinorT<P>& in_o, const LinkT<LF>& U, const OpParams* prm, const Epi& epi,
                    const Fin& fin = Fin{}, const int* stop = nullptr)
  {
    const int nsite = (int)(npar * c->g.Vh);
    ++c->launches;
    if constexpr (LF == LINK_H16_12)
      {
        // FP16 arithmetic: the pipelined one-site kernel only
        constexpr int DIST = 2, MINB = 5;
        constexpr int smem = SppFmt<P, LF>::template smem<DIST>();
        auto k = hop_spp_kernel<P, LF, Epi, Fin, DIST, MINB>;
        static const cudaError_t attr = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        (void)attr;
        launch_pdl(c, k, div_up(nsite, SPP_THREADS), SPP_THREADS, smem, s, c->g, par_out, npar, in_e, in_o, U, prm, epi,
                   reducer(c), fin, stop);
        return;
      }
    else
      {
    if constexpr (P != PREC_F64)
          {
            if (c->hop_cfg[P] == 5)
              {
                launch_pdl(c, hop_sp_kernel<P, LF, Epi, Fin>, div_up(nsite, HOP_SP_THREADS), HOP_SP_THREADS, 0, s, c->g,
                           par_out, npar, in_e, in_o, U, prm, epi, reducer(c), fin, stop);
                return;
              }
            if (c->hop_cfg[P] == 6)
              {
                // two directions ahead: three slots of 76 B (FP16) per thread keep 5 blocks per SM
                // with ~90 KB of L1 left for the neighbours' reuse (three ahead left ~30 KB: 4 % slower)
                constexpr int DIST = 2;
                constexpr int MINB = (P == PREC_F16) ? 5 : 3;
                constexpr int smem = SppFmt<P, LF>::template smem<DIST>();
                auto k = hop_spp_kernel<P, LF, Epi, Fin, DIST, MINB>;
                static const cudaError_t attr = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
                (void)attr;
                launch_pdl(c, k, div_up(nsite, SPP_THREADS), SPP_THREADS, smem, s, c->g, par_out, npar, in_e, in_o, U, prm,
                           epi, reducer(c), fin, stop);
                return;
              }
            if constexpr (LF == LINK_I16_12 || LF == LINK_F32_12)
              if (c->hop_cfg[P] == 7)
                {
                  const TmaGeom G = tma_geom(c->g, c->tma_timeouts, c->tma_rows);
                  const int ntiles = G.ns ? (int)(npar * c->g.Vh / G.ns) : 0;
                  if (G.ns && ntiles <= c->red_cap)
                    {
                      const size_t smem = tma_smem_bytes<P, LF>(G.nc, G.ns);
                      auto k = hop_tma_kernel<P, LF, Epi, Fin>;
                      // the largest tile: at most HOP_TMA_THREADS sites and two halo rows of at most 64 sites
                      static const cudaError_t a1 = cudaFuncSetAttribute(
                        k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                        (int)tma_smem_bytes<P, LF>(HOP_TMA_THREADS + 128, HOP_TMA_THREADS));
                      static const cudaError_t a2 = cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
                      (void)a1;
                      (void)a2;
                      launch_pdl(c, k, ntiles, HOP_TMA_THREADS, smem, s, c->g, G, par_out, npar, in_e, in_o, U, prm, epi,
                                 reducer(c), fin, stop);
                      return;
                    }
                }
          }
        if constexpr (P != PREC_F64)
          if ((c->hop_cfg[P] == 3 || c->hop_cfg[P] == 4) && c->g.T % 4 == 0)
            {
              const int n2 = nsite / 2;
              if (c->hop_cfg[P] == 4)
                launch_pdl(c, hop2_kernel<P, LF, Epi, Fin>, div_up(n2, HOP2_THREADS), HOP2_THREADS, 0, s, c->g, par_out,
                           npar, in_e, in_o, U, prm, epi, reducer(c), fin, stop);
              else
                {
                  constexpr int smem = PipeFmt<P, LF>::SMEM;
                  static const cudaError_t attr = cudaFuncSetAttribute(
                    hop_pipe_kernel<P, LF, Epi, Fin>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
                  (void)attr;
                  launch_pdl(c, hop_pipe_kernel<P, LF, Epi, Fin>, div_up(n2, PIPE_THREADS), PIPE_THREADS, smem, s, c->g,
                             par_out, npar, in_e, in_o, U, prm, epi, reducer(c), fin, stop);
                }
              return;
            }
        switch (c->hop_cfg[P])
          {
          case 1:
            launch_pdl(c, hop_kernel<P, LF, Epi, Fin, 1>, div_up(nsite, HopCfg<P, 1>::NT), HopCfg<P, 1>::NT, 0, s, c->g,
                       par_out, npar, in_e, in_o, U, prm, epi, reducer(c), fin, stop);
            break;
          case 2:
            launch_pdl(c, hop_kernel<P, LF, Epi, Fin, 2>, div_up(nsite, HopCfg<P, 2>::NT), HopCfg<P, 2>::NT, 0, s, c->g,
                       par_out, npar, in_e, in_o, U, prm, epi, reducer(c), fin, stop);
            break;
          default:
            launch_pdl(c, hop_kernel<P, LF, Epi, Fin, 0>, div_up(nsite, HopCfg<P, 0>::NT), HopCfg<P, 0>::NT, 0, s, c->g,
                       par_out, npar, in_e, in_o, U, prm, epi, reducer(c), fin, stop);
          }
      }
  }

  template <int P, int LF, class Epi, class Fin = NoFin>
  void launch_hop(tms_ctx* c, cudaStream_t s, int par_out, int npar, const Field& in_e, const Field& in_o,
                  const LinkT<LF>& U, const OpParams* prm, const Epi& epi, const Fin& fin = Fin{},
                  const int* stop = nullptr)
  {
    launch_hop_v<P, LF>(c, s, par_out, npar, view<P>(in_e), view<P>(in_o), U, prm, epi, fin, stop);
  }

  inline LinkT<LINK_F64_18> links64(tms_ctx* c) { return LinkT<LINK_F64_18>{c->U64, (int)c->g.Vh}; }
  inline LinkT<LINK_F64_12> links64r(tms_ctx* c) { return LinkT<LINK_F64_12>{c->U64, (int)c->g.Vh}; }
  // the FP64 residual recomputations of the mixed solvers may read the links as
  // 12 reals when the conf is SU(3) to FP64 rounding
  inline bool reliable_links12(const tms_ctx* c) { return c->reliable_links12 && c->su3_dev < 1e-13; }
  inline LinkT<LINK_F32_12> links32r(tms_ctx* c) { return LinkT<LINK_F32_12>{c->U32r, (int)c->g.Vh}; }
  inline LinkT<LINK_F32_18> links32f(tms_ctx* c) { return LinkT<LINK_F32_18>{c->U32f, (int)c->g.Vh}; }
  inline LinkT<LINK_I16_12> links16r(tms_ctx* c) { return LinkT<LINK_I16_12>{c->U16r, (int)c->g.Vh}; }
  inline LinkT<LINK_H16_12> links16h(tms_ctx* c) { return LinkT<LINK_H16_12>{c->U16h, (int)c->g.Vh}; }

  // --------------------------------------------------------- conf kernels
  static __global__ void conf_to_soa_kernel(Lattice g, const double* __restrict__ src, int layout, int unfold,
                                     const int* __restrict__ lx_of_eo, double2* __restrict__ U)
  {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= g.V) return;
    const int p = idx >= g.Vh, ieo = idx - (p ? (int)g.Vh : 0);
    const int lx = lx_of_eo[idx];
    const size_t row = (layout == TMS_LAYOUT_LX) ? (size_t)lx : (size_t)idx;
    const int t = lx / (g.LX * g.LY * g.LZ);
    const double* a = src + row * 72; // 8-byte accesses: the caller's buffer need not be 16-byte aligned
    for (int mu = 0; mu < 4; mu++)
      {
        const double sg = (unfold && mu == 0 && t == g.T - 1) ? g.bc_t : 1.0;
        for (int k = 0; k < 9; k++)
          {
            const double wx = a[2 * (mu * 9 + k)], wy = a[2 * (mu * 9 + k) + 1];
            U[((size_t)(p * 4 + mu) * 9 + k) * g.Vh + ieo] = make_double2(wx * sg, wy * sg);
          }
      }
  }

  // FP32 copies and the special-unitarity check (max deviation over links)
  static __global__ void conf_lowprec_kernel(int64_t nlinks_per_parmu, int Vh, const double2* __restrict__ U,
                                      float4* __restrict__ Ur, float2* __restrict__ Uf, char* __restrict__ Us,
                                      char* __restrict__ Uh,
                                      Reducer red)
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
        auto q = [](double x) { return (short)__double2int_rn(fmin(1.0, fmax(-1.0, x)) * 32767.0); };
        {
          // LinkT<LINK_I16_12>: shorts 0-7 as a 16-byte word, 8-11 as an 8-byte word
          const short4 a0 = make_short4(q(u[0].re), q(u[0].im), q(u[1].re), q(u[1].im));
          const short4 a1 = make_short4(q(u[2].re), q(u[2].im), q(u[3].re), q(u[3].im));
          const short4 a2 = make_short4(q(u[4].re), q(u[4].im), q(u[5].re), q(u[5].im));
          uint4 w;
          memcpy(&w.x, &a0, 8);
          memcpy(&w.z, &a1, 8);
          reinterpret_cast<uint4*>(Us)[(size_t)pm * Vh + site] = w;
          reinterpret_cast<short4*>(Us + (size_t)128 * Vh)[(size_t)pm * Vh + site] = a2;
          // LinkT<LINK_H16_12>: the same 12 reals as FP16 values, same planes
          __half2 hv[6];
#pragma unroll
          for (int k = 0; k < 6; k++) hv[k] = __floats2half2_rn((float)u[k].re, (float)u[k].im);
          uint4 wh;
          uint2 wh2;
          memcpy(&wh, hv, 16);
          memcpy(&wh2, hv + 4, 8);
          reinterpret_cast<uint4*>(Uh)[(size_t)pm * Vh + site] = wh;
          reinterpret_cast<uint2*>(Uh + (size_t)128 * Vh)[(size_t)pm * Vh + site] = wh2;
        }
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

  static __global__ void lx_of_eo_kernel(Lattice g, int* __restrict__ out)
  {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= g.V) return;
    const int p = idx >= g.Vh, ieo = idx - (p ? (int)g.Vh : 0);
    out[idx] = eo_site(g, p, ieo).lx;
  }

  template <int MU, bool UP>
  __device__ inline int nbr(const Lattice& g, const Site& s)
  {
    bool w;
    return UP ? nbr_up<MU>(g, s, w) : nbr_dw<MU>(g, s, w);
  }

  static __global__ void geometry_tables_kernel(Lattice g, int* parity, int* eo_of_lx, int* lx_of_eo, int* nup, int* ndw)
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
  inline tms_status spinor_in(tms_ctx* ctx, const double* src, const int* site_map, int64_t nrows, Field& f)
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
  inline tms_status spinor_out(tms_ctx* ctx, const Field& f, const int* site_map, int64_t nrows, double* dst, bool flush)
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

  inline tms_status finish(tms_ctx* ctx)
  {
    CU(cudaGetLastError());
    CU(cudaStreamSynchronize(ctx->stream));
    return TMS_OK;
  }

  inline tms_status check_conf(tms_ctx* ctx)
  {
    if (!ctx) return TMS_ERR_BAD_ARG;
    if (!ctx->conf_loaded) return fail(ctx, TMS_ERR_NO_CONF, "no gauge configuration uploaded");
    CU(cudaSetDevice(ctx->device));
    return TMS_OK;
  }

  inline double read_result(tms_ctx* ctx)
  {
    ++ctx->launches;
    word_copy_kernel<<<1, 64, 0, ctx->stream>>>(reinterpret_cast<const unsigned*>(ctx->red_result),
                                                reinterpret_cast<unsigned*>(ctx->red_hd), 2);
    cudaStreamSynchronize(ctx->stream);
    return *static_cast<volatile double*>(ctx->red_h);
  }

  // the parity-p half of a full-lattice field
  template <int P>
  SpinorT<P> view_par(const Field& f, int p)
  {
    SpinorT<P> s = view<P>(f);
    const size_t off = (size_t)p * (size_t)(f.stride / 2);
    s.d += off;
    if (s.n) s.n += off;
    return s;
  }

  // lx AoS spinor (V rows of 24 doubles, host or device) <-> full-lattice FP64 field
  inline tms_status lx_in(tms_ctx* ctx, const double* src, Field& full)
  {
    TRY(alloc_field(ctx, full, PREC_F64, 2 * ctx->g.stride));
    const int64_t Vh = ctx->g.Vh;
    const int n = (int)Vh;
    const double* d = src;
    if (ctx->ptr_mode == TMS_PTR_HOST)
      {
        const size_t bytes = (size_t)ctx->g.V * 24 * sizeof(double);
        TRY(ensure_stage(ctx, bytes));
        CU(cudaMemcpyAsync(ctx->stage, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
        d = ctx->stage;
      }
    for (int p = 0; p < 2; p++)
      {
        ++ctx->launches;
        aos_to_soa_kernel<PREC_F64><<<div_up(n, 256), 256, 0, ctx->stream>>>(n, d, ctx->lx_of_eo + p * Vh,
                                                                             view_par<PREC_F64>(full, p));
      }
    CU(cudaGetLastError());
    return TMS_OK;
  }

  inline tms_status lx_out(tms_ctx* ctx, const Field& full, double* dst)
  {
    const int64_t Vh = ctx->g.Vh;
    const int n = (int)Vh;
    const size_t bytes = (size_t)ctx->g.V * 24 * sizeof(double);
    double* d = dst;
    if (ctx->ptr_mode == TMS_PTR_HOST)
      {
        TRY(ensure_stage(ctx, bytes));
        d = ctx->stage;
      }
    for (int p = 0; p < 2; p++)
      {
        ++ctx->launches;
        soa_to_aos_kernel<PREC_F64><<<div_up(n, 256), 256, 0, ctx->stream>>>(n, view_par<PREC_F64>(full, p),
                                                                             ctx->lx_of_eo + p * Vh, d);
      }
    CU(cudaGetLastError());
    if (ctx->ptr_mode == TMS_PTR_HOST)
      {
        CU(cudaMemcpyAsync(dst, ctx->stage, bytes, cudaMemcpyDeviceToHost, ctx->stream));
        CU(cudaStreamSynchronize(ctx->stream));
      }
    return TMS_OK;
  }

  template <int P>
  tms_status norm2(tms_ctx* ctx, const Field& a, double* out, int nsites = 0)
  {
    const int n = nsites ? nsites : (int)ctx->g.Vh;
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


  // ------------------------------------------------- twisted clover helpers
  inline ClovT<PREC_F64> clov64(tms_ctx* c) { return ClovT<PREC_F64>{c->cl64, c->icl64, (int)c->g.Vh}; }
  inline ClovT<PREC_F32> clov32(tms_ctx* c) { return ClovT<PREC_F32>{c->cl32, c->icl32, (int)c->g.Vh}; }
  inline ClovT<PREC_F16> clov16(tms_ctx* c) { return ClovT<PREC_F16>{c->cl32, c->icl32, (int)c->g.Vh}; }
  template <int P> ClovT<P> clov(tms_ctx* c);
  template <> inline ClovT<PREC_F64> clov<PREC_F64>(tms_ctx* c) { return clov64(c); }
  template <> inline ClovT<PREC_F32> clov<PREC_F32>(tms_ctx* c) { return clov32(c); }
  template <> inline ClovT<PREC_F16> clov<PREC_F16>(tms_ctx* c) { return clov16(c); }

  inline tms_status check_clover(tms_ctx* ctx)
  {
    TRY(check_conf(ctx));
    if (!ctx->clov_ok) return fail(ctx, TMS_ERR_NO_CONF, "no clover term: call tms_clover_term after the conf upload");
    return TMS_OK;
  }

  // the twisted inverse on even sites for (kappa, mu), recomputed when they change (tms_clover.cu)
  tms_status ensure_clover_inverse(tms_ctx* ctx, double kappa, double mu);
  // out = T_ee^-1(dag) in on even sites, FP64 (tms_clover.cu)
  void inv_clov_apply(tms_ctx* c, const Field& in, const Field& out, int dag);

  // out = K_clov(dag) in  (odd -> odd), te is the even temporary
  template <int P, int LF>
  void clov_kern_op(tms_ctx* c, const LinkT<LF>& U, const ClovT<P>& cl, const Field& in, const Field& te,
                    const Field& out, int dag, const OpParams* prm)
  {
    EpiInvClov<P> ea{{view<P>(te), view<P>(te)}, cl, dag};
    launch_hop<P, LF>(c, c->stream, 0, 1, in, in, U, prm, ea);
    EpiClovKern<P, false> eb{{view<P>(out), view<P>(out)}, {view<P>(in), view<P>(in)}, cl, prm, dag};
    launch_hop<P, LF>(c, c->stream, 1, 1, te, te, U, prm, eb);
  }

  // Q_clov on the full lattice, FP64: (in_e, in_o) -> (out_e, out_o)
  inline void tmclovQ_op(tms_ctx* c, const Field& in_e, const Field& in_o, const Field& out_e, const Field& out_o,
                         const OpParams* prm)
  {
    EpiTmClovQ<PREC_F64> e{{view<PREC_F64>(out_e), view<PREC_F64>(out_o)},
                           {view<PREC_F64>(in_e), view<PREC_F64>(in_o)}, clov64(c), prm};
    launch_hop<PREC_F64, LINK_F64_18>(c, c->stream, 0, 2, in_e, in_o, links64(c), prm, e);
  }

  static_assert(sizeof(CgState) % 4 == 0 && sizeof(OpParams) % 4 == 0, "scalar transfers copy 32-bit words");
  inline tms_status push_state(tms_ctx* ctx) { return put_small(ctx, ctx->st, ctx->st_h, sizeof(CgState)); }
  inline tms_status pull_state(tms_ctx* ctx)
  {
    ++ctx->launches;
    word_copy_kernel<<<1, 64, 0, ctx->stream>>>(reinterpret_cast<const unsigned*>(ctx->st),
                                                reinterpret_cast<unsigned*>(ctx->st_hd), (int)(sizeof(CgState) / 4));
    CU(cudaGetLastError());
    CU(cudaStreamSynchronize(ctx->stream));
    return TMS_OK;
  }

  template <int PD, int PS>
  void convert(tms_ctx* c, const Field& src, const Field& dst, double a = 1.0, int nsites = 0)
  {
    const int n = nsites ? nsites : (int)c->g.Vh;
    ++c->launches;
    axpby_kernel<PD, PS, PS><<<div_up(n, BLAS_THREADS), BLAS_THREADS, 0, c->stream>>>(n, a, view<PS>(src), 0.0,
                                                                                       view<PS>(src), view<PD>(dst));
  }


}

