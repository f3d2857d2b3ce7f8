// Batched e/o solves: k right-hand sides, each with its own kappa and twisted
// mass, solved together so that every hop of the CG reads the links once for
// all of them (the reference solves them one inv_tmD_cg_eoprec call at a time),
// and batch sessions that admit new right-hand sides as others finish.
#include "tms_internal.cuh"
#include "tms_batch.cuh"

#include <algorithm>
#include <chrono>

using namespace tms_int;

namespace
{
  // k fields of one precision, one after the other
  struct BField
  {
    int prec = -1, stride = 0, nrhs = 0;
    void* d = nullptr;
    float* n = nullptr;
    size_t bytes = 0;
  };

  size_t planes_bytes(int prec) { return prec == PREC_F64 ? 192 : prec == PREC_F32 ? 96 : 48; }

  template <int P>
  SpinorBatch<P> bview(const BField& f)
  {
    SpinorBatch<P> b;
    b.f.d = reinterpret_cast<decltype(b.f.d)>(f.d);
    b.f.n = f.n;
    b.f.stride = f.stride;
    b.rhs_elems = planes_bytes(P) * (size_t)f.stride / sizeof(*b.f.d);
    b.rhs_norms = (size_t)f.stride;
    return b;
  }

  // one right-hand side of a batch field as a plain field (for single-RHS kernels)
  Field one(const BField& f, int k)
  {
    Field o;
    o.prec = f.prec;
    o.stride = f.stride;
    o.bytes = planes_bytes(f.prec) * (size_t)f.stride;
    o.d = (unsigned char*)f.d + o.bytes * k;
    o.n = f.n ? f.n + (size_t)f.stride * k : nullptr;
    return o;
  }

  struct BatchWork
  {
    int cap = 0;          // right-hand sides the buffers hold
    int lo_prec = -1;
    BField hi[7];         // FP64: 0 b, 1 x, 2 r, 3 t1, 4 te, 5 s, 6 spare
    BField lo[5];         // inner: 0 second direction (paired x updates), 1 r, 2 p, 3 t1, 4 te
    BField xlo;           // inner x accumulator (FP32 for FP16 inner)
    CgState *st = nullptr, *st_h = nullptr, *mask = nullptr, *mask_h = nullptr;
    BatchParams *bp = nullptr, *bp_h = nullptr;
    BatchReducer red{};
    double* res_h = nullptr;
    int grid = 0;
    cudaGraphExec_t graph[3] = {};
    uint64_t nodes[3] = {};
    int graph_nrhs[3] = {};
    int graph_iters[3] = {};
    bool open = false;    // a batch session owns the buffers
  };

  void free_bfield(BField& f)
  {
    if (f.d) cudaFree(f.d);
    if (f.n) cudaFree(f.n);
    f = BField{};
  }

  void free_work(void* p)
  {
    BatchWork* w = static_cast<BatchWork*>(p);
    if (!w) return;
    for (auto& g : w->graph)
      if (g) cudaGraphExecDestroy(g);
    for (auto& f : w->hi) free_bfield(f);
    for (auto& f : w->lo) free_bfield(f);
    free_bfield(w->xlo);
    cudaFree(w->st);
    cudaFree(w->mask);
    cudaFree(w->bp);
    cudaFree(w->red.partial);
    cudaFree(w->red.counter);
    cudaFree(w->red.result);
    cudaFreeHost(w->st_h);
    cudaFreeHost(w->mask_h);
    cudaFreeHost(w->bp_h);
    cudaFreeHost(w->res_h);
    delete w;
  }

  tms_status alloc_bfield(tms_ctx* ctx, BField& f, int prec, int nrhs)
  {
    if (f.d && f.prec == prec && f.nrhs >= nrhs) return TMS_OK;
    free_bfield(f);
    f.prec = prec;
    f.stride = ctx->g.stride;
    f.nrhs = nrhs;
    f.bytes = planes_bytes(prec) * (size_t)f.stride * nrhs;
    CU(cudaMalloc(&f.d, f.bytes));
    CU(cudaMemsetAsync(f.d, 0, f.bytes, ctx->stream));
    if (prec == PREC_F16)
      {
        CU(cudaMalloc(&f.n, sizeof(float) * (size_t)f.stride * nrhs));
        CU(cudaMemsetAsync(f.n, 0, sizeof(float) * (size_t)f.stride * nrhs, ctx->stream));
      }
    return TMS_OK;
  }

  tms_status work(tms_ctx* ctx, BatchWork** out)
  {
    if (!ctx->bw)
      {
        BatchWork* w = new BatchWork;
        ctx->bw = w;
        ctx->bw_free = free_work;
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        w->grid = std::max(1, div_up(ctx->g.Vh, 32 * MRHS_WARPS)); // one 32-site chunk per warp
        CU(cudaMalloc(&w->st, sizeof(CgState) * MRHS_MAX));
        CU(cudaMalloc(&w->mask, sizeof(CgState) * MRHS_MAX));
        CU(cudaMalloc(&w->bp, sizeof(BatchParams)));
        // rows long enough for the hop kernels' grid and the BLAS grid (blas_grid <= 592)
        CU(cudaMalloc(&w->red.partial, sizeof(double) * MRHS_MAX * (size_t)std::max(w->grid, 592)));
        CU(cudaMalloc(&w->red.counter, sizeof(unsigned) * MRHS_MAX));
        CU(cudaMalloc(&w->red.result, sizeof(double) * MRHS_MAX));
        CU(cudaMemset(w->red.counter, 0, sizeof(unsigned) * MRHS_MAX));
        CU(cudaMallocHost(&w->st_h, sizeof(CgState) * MRHS_MAX));
        CU(cudaMallocHost(&w->mask_h, sizeof(CgState) * MRHS_MAX));
        CU(cudaMallocHost(&w->bp_h, sizeof(BatchParams)));
        CU(cudaMallocHost(&w->res_h, sizeof(double) * MRHS_MAX));
      }
    *out = static_cast<BatchWork*>(ctx->bw);
    return TMS_OK;
  }

  int blas_grid(tms_ctx* ctx) { return std::max(1, std::min(div_up(ctx->g.Vh, 256), 592)); }

  // right-hand sides per warp (R): the autotuned mrhs_r, capped by the batch
  template <int P, int LF, class Epi, class Fin>
  void launch_mrhs(tms_ctx* c, BatchWork* w, cudaStream_t s, int par_out, int nrhs, const BField& in,
                   const LinkT<LF>& U, const Epi& epi, const Fin& fin, const CgState* st)
  {
    ++c->launches;
    int r = c->mrhs_r;
    if (P == PREC_F64 && r > 2) r = 2; // FP64 accumulators: 48 registers per right-hand side
    while (r > 1 && r > nrhs) r >>= 1;
    const int threads = MRHS_WARPS * 32;
    if constexpr (P != PREC_F64)
      if (r == 0)
        {
          // one right-hand side per thread, gathers pipelined through shared memory
          constexpr int smem = SppFmt<P, LF>::template smem<MrhsPipe<P>::DIST>();
          auto k = hop_mrhs_kernel<P, LF, Epi, Fin, 1, true>;
          static const cudaError_t attr = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
          (void)attr;
          k<<<w->grid, threads, smem, s>>>(c->g, par_out, nrhs, bview<P>(in), U, w->bp, epi, w->red, fin, st);
          return;
        }
    if (r < 1) r = 1;
#define TMS_MRHS(RR)                                                                                             \
  hop_mrhs_kernel<P, LF, Epi, Fin, RR><<<w->grid, threads, 0, s>>>(c->g, par_out, nrhs, bview<P>(in), U, w->bp, epi, \
                                                                   w->red, fin, st)
    switch (r)
      {
      case 4: TMS_MRHS(4); break;
      case 2: TMS_MRHS(2); break;
      default: TMS_MRHS(1);
      }
#undef TMS_MRHS
  }

  // s = K(+mu_k)K(-mu_k) x_k, r_k = b_k - s_k and |r_k|^2 in FP64 for the right-hand sides the mask lets through
  tms_status true_residual_b(tms_ctx* ctx, BatchWork* w, int nrhs, const BField& x, double* rr)
  {
    auto U = links64(ctx);
    const CgState* m = w->mask;
    EpiBInvDiag<PREC_F64> a1{bview<PREC_F64>(w->hi[4]), -1.0};
    launch_mrhs<PREC_F64>(ctx, w, ctx->stream, 0, nrhs, x, U, a1, NoFinB{}, m);
    EpiBKern<PREC_F64, false> b1{bview<PREC_F64>(w->hi[3]), bview<PREC_F64>(x), -1.0};
    launch_mrhs<PREC_F64>(ctx, w, ctx->stream, 1, nrhs, w->hi[4], U, b1, NoFinB{}, m);
    EpiBInvDiag<PREC_F64> a2{bview<PREC_F64>(w->hi[4]), +1.0};
    launch_mrhs<PREC_F64>(ctx, w, ctx->stream, 0, nrhs, w->hi[3], U, a2, NoFinB{}, m);
    EpiBKern<PREC_F64, false> b2{bview<PREC_F64>(w->hi[5]), bview<PREC_F64>(w->hi[3]), +1.0};
    launch_mrhs<PREC_F64>(ctx, w, ctx->stream, 1, nrhs, w->hi[4], U, b2, NoFinB{}, m);
    ++ctx->launches;
    residual_mrhs_kernel<<<dim3(blas_grid(ctx), nrhs), 256, 0, ctx->stream>>>(
      (int)ctx->g.Vh, nrhs, bview<PREC_F64>(w->hi[0]), bview<PREC_F64>(w->hi[5]), bview<PREC_F64>(w->hi[2]), w->red, m);
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(w->res_h, w->red.result, sizeof(double) * nrhs, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    for (int k = 0; k < nrhs; k++) rr[k] = w->res_h[k];
    return TMS_OK;
  }




}

namespace
{
  template <int P, int LF>
  tms_status bench_mrhs_t(tms_ctx* ctx, BatchWork* w, const LinkT<LF>& U, int nrhs, int nrep, int flush, double* ms,
                          double link_bytes, double spinor_bytes, double* bytes)
  {
    TRY(alloc_bfield(ctx, w->lo[1], P, nrhs));
    TRY(alloc_bfield(ctx, w->lo[2], P, nrhs));
    BatchParams& bp = *w->bp_h;
    bp.anis = 1.0;
    for (int k = 0; k < nrhs; k++)
      {
        bp.kappa[k] = 0.16;
        bp.mu[k] = 0.01;
      }
    CU(cudaMemcpyAsync(w->bp, w->bp_h, sizeof(BatchParams), cudaMemcpyHostToDevice, ctx->stream));
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
        EpiBInvDiag<P> a{bview<P>(w->lo[2]), 1.0};
        launch_mrhs<P>(ctx, w, ctx->stream, 0, nrhs, w->lo[1], U, a, NoFinB{}, nullptr);
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
    *bytes = (double)ctx->g.Vh * (8 * link_bytes + 2 * spinor_bytes * nrhs);
    return TMS_OK;
  }
}

extern "C" tms_status tms_bench_hop_batched(tms_ctx* ctx, int precision, int nrhs, int nrep, int flush,
                                            double* ms_per_launch, double* bytes_per_launch)
{
  TRY(check_conf(ctx));
  if (nrhs <= 0 || nrhs > MRHS_MAX || nrep <= 0 || !ms_per_launch || !bytes_per_launch)
    return fail(ctx, TMS_ERR_BAD_ARG, "bad bench arguments");
  BatchWork* w;
  TRY(work(ctx, &w));
  if (precision == TMS_PREC_DOUBLE)
    return bench_mrhs_t<PREC_F64>(ctx, w, links64(ctx), nrhs, nrep, flush, ms_per_launch, 144.0, 192.0,
                                  bytes_per_launch);
  if (precision == TMS_PREC_MIXED_SINGLE)
    return ctx->su3 ? bench_mrhs_t<PREC_F32>(ctx, w, links32r(ctx), nrhs, nrep, flush, ms_per_launch, 48.0, 96.0,
                                             bytes_per_launch)
                    : bench_mrhs_t<PREC_F32>(ctx, w, links32f(ctx), nrhs, nrep, flush, ms_per_launch, 72.0, 96.0,
                                             bytes_per_launch);
  if (precision == TMS_PREC_MIXED_HALF)
    return ctx->su3 ? bench_mrhs_t<PREC_F16>(ctx, w, links16r(ctx), nrhs, nrep, flush, ms_per_launch, 24.0, 52.0,
                                             bytes_per_launch)
                    : bench_mrhs_t<PREC_F16>(ctx, w, links32f(ctx), nrhs, nrep, flush, ms_per_launch, 72.0, 52.0,
                                             bytes_per_launch);
  return fail(ctx, TMS_ERR_BAD_ARG, "unknown precision %d", precision);
}

// ===================================================== batch sessions
// A session keeps nslots right-hand sides of one lattice in flight: a
// right-hand side is submitted into a free slot (its source prepared by
// Eq. 8), every step runs one CUDA-graph block of lock-step CG iterations
// for all running slots (and the FP64 reliable updates of the slots that ask
// for one), and a converged slot is collected (Eq. 10-11) and freed for the
// next right-hand side while the others keep iterating.

constexpr int SLOT_FREE = 0, SLOT_RUNNING = 1, SLOT_FINISHED = 2;
constexpr int STOP_IDLE = 5; // CgState.stop of a slot that is not iterating

struct tms_batch
{
  tms_ctx* ctx = nullptr;
  BatchWork* w = nullptr;
  int nslots = 0, prec = 0, has_anis = 0;
  double anis = 1.0;
  std::vector<int> state;
  std::vector<double> b2, tres;
  std::vector<int> reliable, niter;
  std::vector<tms_status> status;
  std::vector<std::chrono::steady_clock::time_point> t0;
  std::vector<double> secs;
};

namespace
{
  tms_status open_fields(tms_batch* b)
  {
    tms_ctx* ctx = b->ctx;
    BatchWork* w = b->w;
    const int n = b->nslots;
    for (int i = 0; i <= 6; i++) TRY(alloc_bfield(ctx, w->hi[i], PREC_F64, n));
    const int P = b->prec == TMS_PREC_DOUBLE ? PREC_F64 : b->prec == TMS_PREC_MIXED_SINGLE ? PREC_F32 : PREC_F16;
    const int PX = (P == PREC_F16) ? PREC_F32 : P;
    if (w->lo_prec != P || w->lo[1].nrhs < n || w->xlo.prec != PX)
      for (auto& g : w->graph)
        if (g)
          {
            CU(cudaStreamSynchronize(ctx->stream));
            cudaGraphExecDestroy(g);
            g = nullptr;
          }
    for (int i = (P == PREC_F64) ? 1 : 0; i <= 4; i++) TRY(alloc_bfield(ctx, w->lo[i], P, n));
    TRY(alloc_bfield(ctx, w->xlo, PX, n));
    w->lo_prec = P;
    return TMS_OK;
  }

  // capture one block of lock-step iterations over all nslots slots
  // CG iterations per session graph block: a right-hand side that stops for a
  // reliable update (or converges) waits for the end of its block, so large
  // batches, whose iterations are long, use short blocks; small ones amortise
  // the host round trip over up to graph_iters iterations
  int batch_block_iters(const tms_ctx* ctx, int nrhs)
  {
    if (ctx->batch_iters > 0) return ctx->batch_iters;
    const double work = (double)ctx->g.Vh * nrhs;          // site right-hand sides per iteration
    const int it = (int)((double)(8 << 20) / work);
    return it < 1 ? 1 : it > ctx->graph_iters ? ctx->graph_iters : it;
  }

  template <int P, int LF>
  tms_status session_graph(tms_batch* b, const LinkT<LF>& U)
  {
    constexpr int PX = (P == PREC_F16) ? PREC_F32 : P;
    tms_ctx* ctx = b->ctx;
    BatchWork* w = b->w;
    const int slot = P, nrhs = b->nslots, n = (int)ctx->g.Vh;
    // mixed precision: x updated every other iteration (two directions, lo[2]
    // and lo[0]), so a block has an even number of iterations
    constexpr bool paired = (P != PREC_F64);
    const int iters0 = batch_block_iters(ctx, nrhs);
    const int iters = paired ? iters0 + (iters0 & 1) : iters0;
    if (w->graph[slot] && w->graph_nrhs[slot] == nrhs && w->graph_iters[slot] == iters) return TMS_OK;
    if (w->graph[slot])
      {
        CU(cudaStreamSynchronize(ctx->stream));
        cudaGraphExecDestroy(w->graph[slot]);
        w->graph[slot] = nullptr;
      }
    const dim3 bg(blas_grid(ctx), nrhs);
    cudaStream_t cs;
    CU(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaGraph_t graph;
    CU(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    const uint64_t before = ctx->launches;
    for (int it = 0; it < iters; it++)
      {
        const bool odd = paired && (it & 1);
        const BField& p = odd ? w->lo[0] : w->lo[2];               // this iteration's direction
        const BField& pn = (paired && !odd) ? w->lo[0] : w->lo[2]; // the next one
        EpiBInvDiag<P> a1{bview<P>(w->lo[4]), -1.0};
        launch_mrhs<P>(ctx, w, cs, 0, nrhs, p, U, a1, NoFinB{}, w->st);
        EpiBKern<P, true> b1{bview<P>(w->lo[3]), bview<P>(p), -1.0};
        launch_mrhs<P>(ctx, w, cs, 1, nrhs, w->lo[4], U, b1, FinAlphaB{w->st}, w->st);
        EpiBInvDiag<P> a2{bview<P>(w->lo[4]), +1.0};
        launch_mrhs<P>(ctx, w, cs, 0, nrhs, w->lo[3], U, a2, NoFinB{}, w->st);
        if (!paired)
          {
            EpiBKernCgUpdate<P, PX, 1> b2e{bview<P>(w->lo[3]), bview<P>(w->lo[1]), bview<P>(p), bview<PX>(w->xlo),
                                           w->st, +1.0};
            launch_mrhs<P>(ctx, w, cs, 1, nrhs, w->lo[4], U, b2e, FinBetaB{w->st}, w->st);
          }
        else if (!odd)
          {
            EpiBKernCgUpdate<P, PX, 0> b2e{bview<P>(w->lo[3]), bview<P>(w->lo[1]), bview<P>(p), bview<PX>(w->xlo),
                                           w->st, +1.0};
            launch_mrhs<P>(ctx, w, cs, 1, nrhs, w->lo[4], U, b2e, FinBetaB{w->st}, w->st);
          }
        else
          {
            EpiBKernCgUpdate<P, PX, 2> b2e{bview<P>(w->lo[3]), bview<P>(w->lo[1]), bview<P>(p), bview<PX>(w->xlo),
                                           w->st,              +1.0,               bview<P>(w->lo[2])};
            launch_mrhs<P>(ctx, w, cs, 1, nrhs, w->lo[4], U, b2e, FinBetaB{w->st}, w->st);
          }
        ++ctx->launches;
        if (paired)
          xpay_to_mrhs_kernel<P><<<bg, 256, 0, cs>>>(n, nrhs, bview<P>(w->lo[1]), bview<P>(p), bview<P>(p),
                                                      bview<P>(pn), 0, w->st, nullptr);
        else
          xpay_mrhs_kernel<P><<<bg, 256, 0, cs>>>(n, nrhs, bview<P>(w->lo[1]), bview<P>(w->lo[2]), w->st, nullptr);
      }
    w->nodes[slot] = ctx->launches - before;
    ctx->launches = before;
    cudaError_t e = cudaStreamEndCapture(cs, &graph);
    cudaStreamDestroy(cs);
    if (e != cudaSuccess) return fail(ctx, TMS_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&w->graph[slot], graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return fail(ctx, TMS_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
    w->graph_nrhs[slot] = nrhs;
    w->graph_iters[slot] = iters;
    return TMS_OK;
  }

  template <int P>
  tms_status session_submit(tms_batch* b, int k, double residue, int niter)
  {
    constexpr int PX = (P == PREC_F16) ? PREC_F32 : P;
    tms_ctx* ctx = b->ctx;
    BatchWork* w = b->w;
    const int n = (int)ctx->g.Vh;
    // varphi (the CG source) is in hi[0][k]: |b|^2
    double b2;
    TRY(norm2<PREC_F64>(ctx, one(w->hi[0], k), &b2));
    if (b2 == 0.0 || std::isnan(b2)) return fail(ctx, TMS_ERR_INVALID_SOURCE, "invalid norm: %g", b2);
    const Field x = one(w->hi[1], k), r = one(w->hi[2], k), v = one(w->hi[0], k);
    CU(cudaMemsetAsync(x.d, 0, x.bytes, ctx->stream));
    CU(cudaMemcpyAsync(r.d, v.d, v.bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    convert<P, PREC_F64>(ctx, v, one(w->lo[1], k));
    convert<P, PREC_F64>(ctx, v, one(w->lo[2], k));
    const Field xl = one(w->xlo, k);
    CU(cudaMemsetAsync(xl.d, 0, xl.bytes, ctx->stream));
    (void)n;
    (void)sizeof(PX);
    const bool mixed = (P != PREC_F64);
    const double delta = (P == PREC_F16) ? ctx->delta_half : ctx->delta_single;
    CgState& S = w->st_h[k];
    memset(&S, 0, sizeof S);
    S.rr = b2;
    S.b2 = b2;
    S.target = residue * b2;
    S.rel_trigger = mixed ? delta * delta * b2 : -1.0;
    S.niter_max = niter;
    S.stop = STOP_RUN;
    CU(cudaMemcpyAsync(w->st + k, &S, sizeof(CgState), cudaMemcpyHostToDevice, ctx->stream));
    CU(cudaMemcpyAsync(w->bp, w->bp_h, sizeof(BatchParams), cudaMemcpyHostToDevice, ctx->stream));
    b->b2[k] = b2;
    b->tres[k] = 0.0;
    b->reliable[k] = 0;
    b->niter[k] = niter;
    b->status[k] = TMS_OK;
    return TMS_OK;
  }

  // one graph block for all running slots, then the slots that stopped are
  // finished (FP64) or updated in FP64 and either finished or restarted (mixed)
  template <int P, int LF>
  tms_status session_step(tms_batch* b, const LinkT<LF>& U, int* finished)
  {
    constexpr int PX = (P == PREC_F16) ? PREC_F32 : P;
    tms_ctx* ctx = b->ctx;
    BatchWork* w = b->w;
    const int nrhs = b->nslots, n = (int)ctx->g.Vh, slot = P;
    const bool mixed = (P != PREC_F64);
    const double delta = (P == PREC_F16) ? ctx->delta_half : ctx->delta_single;
    const dim3 bg(blas_grid(ctx), nrhs);
    CgState* S = w->st_h;
    TRY(session_graph<P>(b, U));
    std::vector<int> iter0(nrhs);
    for (int k = 0; k < nrhs; k++) iter0[k] = S[k].iter;
    CU(cudaGraphLaunch(w->graph[slot], ctx->stream));
    ctx->launches += w->nodes[slot];
    CU(cudaMemcpyAsync(S, w->st, sizeof(CgState) * nrhs, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    std::vector<int> fin(nrhs, 0);
    bool any = false;
    for (int k = 0; k < nrhs; k++)
      {
        w->mask_h[k].stop = 1;
        if (b->state[k] != SLOT_RUNNING || S[k].stop == STOP_RUN) continue;
        if (S[k].stop == STOP_BREAKDOWN)
          {
            b->status[k] = TMS_ERR_NAN;
            fin[k] = 1;
            continue;
          }
        w->mask_h[k].stop = 0; // final residual (FP64) or reliable update (mixed)
        any = true;
      }
    if (any)
      {
        CU(cudaMemcpyAsync(w->mask, w->mask_h, sizeof(CgState) * nrhs, cudaMemcpyHostToDevice, ctx->stream));
        std::vector<double> rr(nrhs, 0.0);
        if (!mixed)
          {
            // the FP64 iteration accumulated x in the inner field
            ++ctx->launches;
            axpby_mrhs_kernel<PREC_F64, PX, PX><<<bg, 256, 0, ctx->stream>>>(
              n, nrhs, 1.0, bview<PX>(w->xlo), 0.0, bview<PX>(w->xlo), bview<PREC_F64>(w->hi[1]), w->mask);
            TRY(true_residual_b(ctx, w, nrhs, w->hi[1], rr.data()));
            for (int k = 0; k < nrhs; k++)
              if (!w->mask_h[k].stop)
                {
                  b->tres[k] = rr[k];
                  b->status[k] = (S[k].stop == STOP_MAXITER) ? TMS_ERR_NOT_CONVERGED : TMS_OK;
                  fin[k] = 1;
                }
          }
        else
          {
            // paired x updates: a block cut after an odd number of iterations
            // leaves the last step alpha p (direction in lo[2]) out of x_lo; after
            // an even number the direction to restart from is in lo[0] (dir 1)
            for (int k = 0; k < nrhs; k++)
              if (!w->mask_h[k].stop) S[k].dir = ((S[k].iter - iter0[k]) & 1) ? 0 : 1;
            CU(cudaMemcpyAsync(w->st, S, sizeof(CgState) * nrhs, cudaMemcpyHostToDevice, ctx->stream));
            ++ctx->launches;
            xflush_mrhs_kernel<PX, P><<<bg, 256, 0, ctx->stream>>>(n, nrhs, bview<PX>(w->xlo), bview<P>(w->lo[2]),
                                                                    w->st, w->mask);
            // x += x_lo ; x_lo = 0 ; r = b - A x   (FP64, masked)
            ctx->launches += 2;
            axpby_mrhs_kernel<PREC_F64, PREC_F64, PX><<<bg, 256, 0, ctx->stream>>>(
              n, nrhs, 1.0, bview<PREC_F64>(w->hi[1]), 1.0, bview<PX>(w->xlo), bview<PREC_F64>(w->hi[1]), w->mask);
            axpby_mrhs_kernel<PX, PX, PX><<<bg, 256, 0, ctx->stream>>>(n, nrhs, 0.0, bview<PX>(w->xlo), 0.0,
                                                                       bview<PX>(w->xlo), bview<PX>(w->xlo), w->mask);
            TRY(true_residual_b(ctx, w, nrhs, w->hi[1], rr.data()));
            bool restart = false;
            for (int k = 0; k < nrhs; k++)
              {
                if (w->mask_h[k].stop) continue;
                b->reliable[k]++;
                b->tres[k] = rr[k];
                if (rr[k] < S[k].target || S[k].stop == STOP_MAXITER || S[k].iter >= b->niter[k])
                  {
                    b->status[k] = (rr[k] < S[k].target) ? TMS_OK : TMS_ERR_NOT_CONVERGED;
                    fin[k] = 1;
                    w->mask_h[k].stop = 1;
                    continue;
                  }
                S[k].beta = rr[k] / S[k].rr_prev;
                S[k].rr = rr[k];
                S[k].rel_trigger = delta * delta * rr[k];
                S[k].stop = STOP_RUN;
                restart = true;
              }
            if (restart)
              {
                CU(cudaMemcpyAsync(w->mask, w->mask_h, sizeof(CgState) * nrhs, cudaMemcpyHostToDevice, ctx->stream));
                // r_lo = r ; p_lo = r_lo + beta p_lo   (masked)
                ++ctx->launches;
                axpby_mrhs_kernel<P, PREC_F64, PREC_F64><<<bg, 256, 0, ctx->stream>>>(
                  n, nrhs, 1.0, bview<PREC_F64>(w->hi[2]), 0.0, bview<PREC_F64>(w->hi[2]), bview<P>(w->lo[1]),
                  w->mask);
                CU(cudaMemcpyAsync(w->st, S, sizeof(CgState) * nrhs, cudaMemcpyHostToDevice, ctx->stream));
                ++ctx->launches;
                xpay_to_mrhs_kernel<P><<<bg, 256, 0, ctx->stream>>>(n, nrhs, bview<P>(w->lo[1]), bview<P>(w->lo[2]),
                                                                    bview<P>(w->lo[0]), bview<P>(w->lo[2]), 1, w->st,
                                                                    w->mask);
              }
          }
      }
    const auto now = std::chrono::steady_clock::now();
    bool changed = false;
    for (int k = 0; k < nrhs; k++)
      {
        finished[k] = fin[k];
        if (!fin[k]) continue;
        S[k].stop = STOP_IDLE;
        b->state[k] = SLOT_FINISHED;
        b->secs[k] = std::chrono::duration<double>(now - b->t0[k]).count();
        changed = true;
      }
    if (changed || any) CU(cudaMemcpyAsync(w->st, S, sizeof(CgState) * nrhs, cudaMemcpyHostToDevice, ctx->stream));
    CU(cudaGetLastError());
    CU(cudaStreamSynchronize(ctx->stream));
    return TMS_OK;
  }
}

extern "C" {

tms_status tms_batch_open(tms_ctx* ctx, int nslots, int precision, int has_anis, double anis, tms_batch** out)
{
  if (!out) return TMS_ERR_BAD_ARG;
  *out = nullptr;
  TRY(check_conf(ctx));
  if (nslots <= 0 || nslots > MRHS_MAX) return fail(ctx, TMS_ERR_BAD_ARG, "nslots: 1..%d", MRHS_MAX);
  if (precision != TMS_PREC_DOUBLE && precision != TMS_PREC_MIXED_SINGLE && precision != TMS_PREC_MIXED_HALF)
    return fail(ctx, TMS_ERR_BAD_ARG, "unknown precision %d", precision);
  BatchWork* w;
  TRY(work(ctx, &w));
  if (w->open) return fail(ctx, TMS_ERR_BAD_ARG, "a batch session is already open on this context");
  tms_batch* b = new tms_batch;
  b->ctx = ctx;
  b->w = w;
  b->nslots = nslots;
  b->prec = precision;
  b->has_anis = has_anis;
  b->anis = has_anis ? anis : 1.0;
  b->state.assign(nslots, SLOT_FREE);
  b->b2.assign(nslots, 0.0);
  b->tres.assign(nslots, 0.0);
  b->reliable.assign(nslots, 0);
  b->niter.assign(nslots, 0);
  b->status.assign(nslots, TMS_OK);
  b->t0.assign(nslots, std::chrono::steady_clock::now());
  b->secs.assign(nslots, 0.0);
  const tms_status st = open_fields(b);
  if (st != TMS_OK)
    {
      delete b;
      return st;
    }
  for (int k = 0; k < nslots; k++)
    {
      memset(&w->st_h[k], 0, sizeof(CgState));
      w->st_h[k].stop = STOP_IDLE;
      w->bp_h->kappa[k] = 0.125;
      w->bp_h->mu[k] = 0.0;
    }
  w->bp_h->anis = b->anis;
  CU(cudaMemcpyAsync(w->st, w->st_h, sizeof(CgState) * nslots, cudaMemcpyHostToDevice, ctx->stream));
  CU(cudaMemcpyAsync(w->bp, w->bp_h, sizeof(BatchParams), cudaMemcpyHostToDevice, ctx->stream));
  CU(cudaStreamSynchronize(ctx->stream));
  w->open = true;
  *out = b;
  return TMS_OK;
}

tms_status tms_batch_submit(tms_batch* b, int slot, const double* src_lx, double kappa, double mu, int niter,
                            double residue)
{
  if (!b) return TMS_ERR_BAD_ARG;
  tms_ctx* ctx = b->ctx;
  TRY(check_conf(ctx));
  if (slot < 0 || slot >= b->nslots || b->state[slot] != SLOT_FREE)
    return fail(ctx, TMS_ERR_BAD_ARG, "slot %d is not free", slot);
  if (!src_lx || niter <= 0 || !(residue > 0) || !(kappa > 0) || !std::isfinite(mu))
    return fail(ctx, TMS_ERR_BAD_ARG, "bad right-hand side arguments");
  BatchWork* w = b->w;
  w->bp_h->kappa[slot] = kappa;
  w->bp_h->mu[slot] = mu;
  // Eq. (8): varphi -> hi[0][slot], eta_e -> hi[6][slot] (single-RHS FP64 kernels)
  TRY(set_params(ctx, kappa, mu, b->has_anis, b->anis));
  Field* f = ctx->f64;
  for (int i = 0; i <= 7; i++) TRY(alloc_field(ctx, f[i], PREC_F64));
  for (auto& e : ctx->ex) TRY(alloc_field(ctx, e, PREC_F64));
  const int64_t Vh = ctx->g.Vh;
  const int n = (int)Vh;
  const size_t bytes = (size_t)ctx->g.V * 24 * sizeof(double);
  const double* src = src_lx;
  if (ctx->ptr_mode == TMS_PTR_HOST)
    {
      TRY(ensure_stage(ctx, bytes));
      CU(cudaMemcpyAsync(ctx->stage, src_lx, bytes, cudaMemcpyHostToDevice, ctx->stream));
      src = ctx->stage;
    }
  auto V = [](const Field& x) { return view<PREC_F64>(x); };
  const Field ek = one(w->hi[6], slot), vk = one(w->hi[0], slot);
  ctx->launches += 3;
  aos_to_soa_kernel<PREC_F64><<<div_up(n, 256), 256, 0, ctx->stream>>>(n, src, ctx->lx_of_eo, V(ek));
  aos_to_soa_kernel<PREC_F64><<<div_up(n, 256), 256, 0, ctx->stream>>>(n, src, ctx->lx_of_eo + Vh, V(ctx->ex[1]));
  diag_kernel<PREC_F64><<<div_up(n, 256), 256, 0, ctx->stream>>>(n, V(ek), V(f[5]), ctx->prm, 1.0, 1);
  EpiSrcPrep<PREC_F64> sp{{V(vk), V(vk)}, {V(ctx->ex[1]), V(ctx->ex[1])}};
  launch_hop<PREC_F64, LINK_F64_18>(ctx, ctx->stream, 1, 1, f[5], f[5], links64(ctx), ctx->prm, sp);
  CU(cudaGetLastError());
  tms_status st;
  if (b->prec == TMS_PREC_DOUBLE) st = session_submit<PREC_F64>(b, slot, residue, niter);
  else if (b->prec == TMS_PREC_MIXED_SINGLE) st = session_submit<PREC_F32>(b, slot, residue, niter);
  else st = session_submit<PREC_F16>(b, slot, residue, niter);
  if (st != TMS_OK) return st;
  CU(cudaStreamSynchronize(ctx->stream));
  b->state[slot] = SLOT_RUNNING;
  b->t0[slot] = std::chrono::steady_clock::now();
  return TMS_OK;
}

tms_status tms_batch_step(tms_batch* b, int* finished, int* nfinished)
{
  if (!b || !finished) return TMS_ERR_BAD_ARG;
  tms_ctx* ctx = b->ctx;
  TRY(check_conf(ctx));
  int running = 0;
  for (int k = 0; k < b->nslots; k++)
    {
      finished[k] = 0;
      running += (b->state[k] == SLOT_RUNNING);
    }
  if (nfinished) *nfinished = 0;
  if (!running) return TMS_OK;
  tms_status st;
  if (b->prec == TMS_PREC_DOUBLE) st = session_step<PREC_F64>(b, links64(ctx), finished);
  else if (b->prec == TMS_PREC_MIXED_SINGLE)
    st = ctx->su3 ? session_step<PREC_F32>(b, links32r(ctx), finished)
                  : session_step<PREC_F32>(b, links32f(ctx), finished);
  else
    st = ctx->su3 ? session_step<PREC_F16>(b, links16r(ctx), finished)
                  : session_step<PREC_F16>(b, links32f(ctx), finished);
  if (st != TMS_OK) return st;
  if (nfinished)
    for (int k = 0; k < b->nslots; k++) *nfinished += finished[k];
  return TMS_OK;
}

tms_status tms_batch_collect(tms_batch* b, int slot, double* sol_lx, tms_stats* stats)
{
  if (!b) return TMS_ERR_BAD_ARG;
  tms_ctx* ctx = b->ctx;
  TRY(check_conf(ctx));
  if (slot < 0 || slot >= b->nslots || b->state[slot] != SLOT_FINISHED)
    return fail(ctx, TMS_ERR_BAD_ARG, "slot %d has no finished solution", slot);
  if (!sol_lx) return fail(ctx, TMS_ERR_BAD_ARG, "null solution buffer");
  BatchWork* w = b->w;
  const double kappa = w->bp_h->kappa[slot], mu = w->bp_h->mu[slot];
  TRY(set_params(ctx, kappa, mu, b->has_anis, b->anis));
  Field* f = ctx->f64;
  Field* psi = ctx->ex + 2;
  const int64_t Vh = ctx->g.Vh;
  const int n = (int)Vh;
  const size_t bytes = (size_t)ctx->g.V * 24 * sizeof(double);
  auto U = links64(ctx);
  auto V = [](const Field& x) { return view<PREC_F64>(x); };
  // Eq. (10)-(11) and paste
  const Field xk = one(w->hi[1], slot), ek = one(w->hi[6], slot);
  kern_op<PREC_F64>(ctx, U, xk, f[5], psi[1], -1.0, ctx->prm);
  EpiReco<PREC_F64> rc{{V(psi[0]), V(psi[0])}, {V(ek), V(ek)}, ctx->prm, 1.0};
  launch_hop<PREC_F64, LINK_F64_18>(ctx, ctx->stream, 0, 1, psi[1], psi[1], U, ctx->prm, rc);
  double* d = (ctx->ptr_mode == TMS_PTR_HOST) ? ctx->stage : sol_lx;
  if (ctx->ptr_mode == TMS_PTR_HOST) TRY(ensure_stage(ctx, bytes));
  d = (ctx->ptr_mode == TMS_PTR_HOST) ? ctx->stage : sol_lx;
  ctx->launches += 2;
  soa_to_aos_kernel<PREC_F64><<<div_up(n, 256), 256, 0, ctx->stream>>>(n, V(psi[0]), ctx->lx_of_eo, d);
  soa_to_aos_kernel<PREC_F64><<<div_up(n, 256), 256, 0, ctx->stream>>>(n, V(psi[1]), ctx->lx_of_eo + Vh, d);
  CU(cudaGetLastError());
  if (ctx->ptr_mode == TMS_PTR_HOST) CU(cudaMemcpyAsync(sol_lx, ctx->stage, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  TRY(finish(ctx));
  const CgState& S = w->st_h[slot];
  if (stats)
    {
      stats->status = b->status[slot];
      stats->iterations = S.iter;
      stats->reliable_updates = b->reliable[slot];
      stats->iterated_rel_res2 = S.rr / b->b2[slot];
      stats->true_rel_res2 = b->tres[slot] / b->b2[slot];
      stats->lx_rel_res2 = 0.0;
      stats->seconds = b->secs[slot];
    }
  b->state[slot] = SLOT_FREE;
  return b->status[slot];
}

tms_status tms_batch_close(tms_batch* b)
{
  if (!b) return TMS_OK;
  b->w->open = false;
  delete b;
  return TMS_OK;
}

tms_status tms_cg_eoprec_batched(tms_ctx* ctx, int nrhs, double* const* sols_lx, const double* const* srcs_lx,
                                 double kappa, int has_anis, double anis, const double* mus, int niter,
                                 const double* residues, int precision, tms_stats* stats)
{
  TRY(check_conf(ctx));
  if (nrhs <= 0 || nrhs > MRHS_MAX || !sols_lx || !srcs_lx || !mus || !residues || niter <= 0)
    return fail(ctx, TMS_ERR_BAD_ARG, "bad batched arguments (1 <= nrhs <= %d)", MRHS_MAX);
  for (int k = 0; k < nrhs; k++)
    if (!sols_lx[k] || !srcs_lx[k] || !(residues[k] > 0) || !std::isfinite(mus[k]))
      return fail(ctx, TMS_ERR_BAD_ARG, "bad right-hand side %d", k);
  tms_batch* b = nullptr;
  TRY(tms_batch_open(ctx, nrhs, precision, has_anis, anis, &b));
  struct Closer
  {
    tms_batch* b;
    ~Closer() { tms_batch_close(b); }
  } closer{b};
  for (int k = 0; k < nrhs; k++)
    {
      const tms_status s = tms_batch_submit(b, k, srcs_lx[k], kappa, mus[k], niter, residues[k]);
      if (s != TMS_OK) return s;
    }
  std::vector<int> fin(nrhs);
  int left = nrhs;
  tms_status worst = TMS_OK;
  while (left > 0)
    {
      int nf = 0;
      TRY(tms_batch_step(b, fin.data(), &nf));
      for (int k = 0; k < nrhs; k++)
        if (fin[k])
          {
            const tms_status s = tms_batch_collect(b, k, sols_lx[k], stats ? stats + k : nullptr);
            if (s != TMS_OK && s != TMS_ERR_NOT_CONVERGED && s != TMS_ERR_NAN) return s;
            if (s != TMS_OK && worst == TMS_OK) worst = s;
            left--;
          }
    }
  if (worst == TMS_ERR_NAN) return fail(ctx, worst, "nanned");
  if (worst == TMS_ERR_NOT_CONVERGED) return fail(ctx, worst, "exit without converging");
  return TMS_OK;
}

} // extern "C"
