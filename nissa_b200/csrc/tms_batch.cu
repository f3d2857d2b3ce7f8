// Batched e/o solves: k right-hand sides with one kappa and a twisted mass
// each, solved together so that every hop of the CG reads the links once for
// all of them (the reference solves them one inv_tmD_cg_eoprec call at a time).
#include "tms_internal.cuh"
#include "tms_batch.cuh"

#include <algorithm>

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
    BField lo[5];         // inner: 1 r, 2 p, 3 t1, 4 te
    BField xlo;           // inner x accumulator (FP32 for FP16 inner)
    CgState *st = nullptr, *st_h = nullptr, *mask = nullptr, *mask_h = nullptr;
    BatchParams *bp = nullptr, *bp_h = nullptr;
    BatchReducer red{};
    double* res_h = nullptr;
    int grid = 0;
    cudaGraphExec_t graph[3] = {};
    uint64_t nodes[3] = {};
    int graph_nrhs[3] = {};
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

  tms_status push_mask(tms_ctx* ctx, BatchWork* w, int nrhs)
  {
    CU(cudaMemcpyAsync(w->mask, w->mask_h, sizeof(CgState) * nrhs, cudaMemcpyHostToDevice, ctx->stream));
    return TMS_OK;
  }

  // Lock-step CG on K(+mu_k)K(-mu_k) for nrhs odd sources hi[0], solutions in
  // hi[1].  Inner precision P (FP64: plain CG as in cg_invert; FP32/FP16: FP64
  // reliable updates of the right-hand sides that ask for one).
  template <int P, int LF>
  tms_status cg_batch(tms_ctx* ctx, BatchWork* w, const LinkT<LF>& U, int nrhs, int niter, const double* residue,
                      tms_stats* stats)
  {
    constexpr int PX = (P == PREC_F16) ? PREC_F32 : P;
    const int slot = P;
    const int n = (int)ctx->g.Vh;
    const bool mixed = (P != PREC_F64);
    for (int i = 1; i <= 5; i++) TRY(alloc_bfield(ctx, w->hi[i], PREC_F64, nrhs));
    if (w->lo_prec != P || w->lo[1].nrhs < nrhs)
      for (auto& g : w->graph)
        if (g)
          {
            CU(cudaStreamSynchronize(ctx->stream));
            cudaGraphExecDestroy(g);
            g = nullptr;
          }
    for (int i = 1; i <= 4; i++) TRY(alloc_bfield(ctx, w->lo[i], P, nrhs));
    TRY(alloc_bfield(ctx, w->xlo, PX, nrhs));
    w->lo_prec = P;
    const double delta = (P == PREC_F16) ? ctx->delta_half : ctx->delta_single;
    const dim3 bg(blas_grid(ctx), nrhs);

    // |b_k|^2: the residual of x = 0 against b
    CU(cudaMemsetAsync(w->hi[1].d, 0, w->hi[1].bytes, ctx->stream));
    for (int k = 0; k < nrhs; k++) w->mask_h[k].stop = 0;
    TRY(push_mask(ctx, w, nrhs));
    std::vector<double> b2(nrhs), rr(nrhs);
    TRY(true_residual_b(ctx, w, nrhs, w->hi[1], b2.data()));
    for (int k = 0; k < nrhs; k++)
      if (b2[k] == 0.0 || std::isnan(b2[k]))
        return fail(ctx, TMS_ERR_INVALID_SOURCE, "invalid norm of right-hand side %d: %g", k, b2[k]);
    // r = b (in hi[2] already), r_lo = r, p_lo = r, x_lo = 0
    ++ctx->launches;
    axpby_mrhs_kernel<P, PREC_F64, PREC_F64><<<bg, 256, 0, ctx->stream>>>(
      n, nrhs, 1.0, bview<PREC_F64>(w->hi[2]), 0.0, bview<PREC_F64>(w->hi[2]), bview<P>(w->lo[1]), nullptr);
    ++ctx->launches;
    axpby_mrhs_kernel<P, PREC_F64, PREC_F64><<<bg, 256, 0, ctx->stream>>>(
      n, nrhs, 1.0, bview<PREC_F64>(w->hi[2]), 0.0, bview<PREC_F64>(w->hi[2]), bview<P>(w->lo[2]), nullptr);
    CU(cudaMemsetAsync(w->xlo.d, 0, w->xlo.bytes, ctx->stream));
    std::vector<int> done(nrhs, 0), reliable(nrhs, 0);
    std::vector<double> tres(nrhs, 0.0);
    std::vector<tms_status> status(nrhs, TMS_OK);
    CgState* S = w->st_h;
    for (int k = 0; k < nrhs; k++)
      {
        memset(&S[k], 0, sizeof(CgState));
        S[k].rr = b2[k];
        S[k].b2 = b2[k];
        S[k].target = residue[k] * b2[k];
        S[k].rel_trigger = mixed ? delta * delta * b2[k] : -1.0;
        S[k].niter_max = niter;
      }
    CU(cudaMemcpyAsync(w->st, S, sizeof(CgState) * nrhs, cudaMemcpyHostToDevice, ctx->stream));
    // graph of graph_iters lock-step iterations for this nrhs
    if (w->graph[slot] && w->graph_nrhs[slot] != nrhs)
      {
        CU(cudaStreamSynchronize(ctx->stream));
        cudaGraphExecDestroy(w->graph[slot]);
        w->graph[slot] = nullptr;
      }
    if (!w->graph[slot])
      {
        cudaStream_t cs;
        CU(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        cudaGraph_t graph;
        CU(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
        const uint64_t before = ctx->launches;
        for (int it = 0; it < ctx->graph_iters; it++)
          {
            EpiBInvDiag<P> a1{bview<P>(w->lo[4]), -1.0};
            launch_mrhs<P>(ctx, w, cs, 0, nrhs, w->lo[2], U, a1, NoFinB{}, w->st);
            EpiBKern<P, true> b1{bview<P>(w->lo[3]), bview<P>(w->lo[2]), -1.0};
            launch_mrhs<P>(ctx, w, cs, 1, nrhs, w->lo[4], U, b1, FinAlphaB{w->st}, w->st);
            EpiBInvDiag<P> a2{bview<P>(w->lo[4]), +1.0};
            launch_mrhs<P>(ctx, w, cs, 0, nrhs, w->lo[3], U, a2, NoFinB{}, w->st);
            EpiBKernCgUpdate<P, PX> b2e{bview<P>(w->lo[3]), bview<P>(w->lo[1]), bview<P>(w->lo[2]), bview<PX>(w->xlo),
                                        w->st, +1.0};
            launch_mrhs<P>(ctx, w, cs, 1, nrhs, w->lo[4], U, b2e, FinBetaB{w->st}, w->st);
            ++ctx->launches;
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
      }
    CU(cudaEventRecord(ctx->ev0, ctx->stream));
    int ndone = 0;
    while (ndone < nrhs)
      {
        CU(cudaGraphLaunch(w->graph[slot], ctx->stream));
        ctx->launches += w->nodes[slot];
        CU(cudaMemcpyAsync(S, w->st, sizeof(CgState) * nrhs, cudaMemcpyDeviceToHost, ctx->stream));
        CU(cudaStreamSynchronize(ctx->stream));
        // right-hand sides that stopped: finish them, or update and restart them
        bool any = false;
        for (int k = 0; k < nrhs; k++)
          {
            w->mask_h[k].stop = 1;
            if (done[k] || S[k].stop == STOP_RUN) continue;
            if (S[k].stop == STOP_BREAKDOWN)
              {
                status[k] = TMS_ERR_NAN;
                done[k] = 1;
                ndone++;
                continue;
              }
            if (!mixed)
              {
                status[k] = (S[k].stop == STOP_MAXITER) ? TMS_ERR_NOT_CONVERGED : TMS_OK;
                done[k] = 1;
                ndone++;
                continue;
              }
            w->mask_h[k].stop = 0; // take part in the reliable update
            any = true;
          }
        if (!mixed)
          {
            // keep the finished ones out of the graph's kernels
            continue;
          }
        if (!any) continue;
        TRY(push_mask(ctx, w, nrhs));
        // x += x_lo ; x_lo = 0 (for the masked right-hand sides)
        ++ctx->launches;
        axpby_mrhs_kernel<PREC_F64, PREC_F64, PX><<<bg, 256, 0, ctx->stream>>>(
          n, nrhs, 1.0, bview<PREC_F64>(w->hi[1]), 1.0, bview<PX>(w->xlo), bview<PREC_F64>(w->hi[1]), w->mask);
        ++ctx->launches;
        axpby_mrhs_kernel<PX, PX, PX><<<bg, 256, 0, ctx->stream>>>(n, nrhs, 0.0, bview<PX>(w->xlo), 0.0,
                                                                   bview<PX>(w->xlo), bview<PX>(w->xlo), w->mask);
        TRY(true_residual_b(ctx, w, nrhs, w->hi[1], rr.data()));
        bool restart = false;
        for (int k = 0; k < nrhs; k++)
          {
            if (w->mask_h[k].stop) continue;
            reliable[k]++;
            tres[k] = rr[k];
            if (rr[k] < S[k].target || S[k].stop == STOP_MAXITER || S[k].iter >= niter)
              {
                status[k] = (rr[k] < S[k].target) ? TMS_OK : TMS_ERR_NOT_CONVERGED;
                done[k] = 1;
                ndone++;
                S[k].stop = 5; // finished: the graph's kernels skip it
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
            TRY(push_mask(ctx, w, nrhs));
            // r_lo = r ; p_lo = r_lo + beta p_lo  (masked)
            ++ctx->launches;
            axpby_mrhs_kernel<P, PREC_F64, PREC_F64><<<bg, 256, 0, ctx->stream>>>(
              n, nrhs, 1.0, bview<PREC_F64>(w->hi[2]), 0.0, bview<PREC_F64>(w->hi[2]), bview<P>(w->lo[1]), w->mask);
          }
        CU(cudaMemcpyAsync(w->st, S, sizeof(CgState) * nrhs, cudaMemcpyHostToDevice, ctx->stream));
        if (restart)
          {
            ++ctx->launches;
            xpay_mrhs_kernel<P><<<bg, 256, 0, ctx->stream>>>(n, nrhs, bview<P>(w->lo[1]), bview<P>(w->lo[2]), w->st,
                                                             w->mask);
          }
        CU(cudaGetLastError());
      }
    CU(cudaEventRecord(ctx->ev1, ctx->stream));
    CU(cudaEventSynchronize(ctx->ev1));
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    if (!mixed)
      {
        // the FP64 iteration accumulated x in the inner field
        ++ctx->launches;
        axpby_mrhs_kernel<PREC_F64, PX, PX><<<bg, 256, 0, ctx->stream>>>(n, nrhs, 1.0, bview<PX>(w->xlo), 0.0,
                                                                         bview<PX>(w->xlo), bview<PREC_F64>(w->hi[1]),
                                                                         nullptr);
        for (int k = 0; k < nrhs; k++) w->mask_h[k].stop = 0;
        TRY(push_mask(ctx, w, nrhs));
        TRY(true_residual_b(ctx, w, nrhs, w->hi[1], tres.data()));
      }
    tms_status worst = TMS_OK;
    for (int k = 0; k < nrhs; k++)
      {
        if (stats)
          {
            stats[k].status = status[k];
            stats[k].iterations = S[k].iter;
            stats[k].reliable_updates = reliable[k];
            stats[k].iterated_rel_res2 = S[k].rr / b2[k];
            stats[k].true_rel_res2 = tres[k] / b2[k];
            stats[k].seconds = ms * 1e-3;
          }
        if (status[k] != TMS_OK && worst == TMS_OK) worst = status[k];
      }
    if (worst == TMS_ERR_NAN) return fail(ctx, worst, "nanned");
    if (worst == TMS_ERR_NOT_CONVERGED) return fail(ctx, worst, "exit without converging");
    return TMS_OK;
  }
}

extern "C" tms_status tms_cg_eoprec_batched(tms_ctx* ctx, int nrhs, double* const* sols_lx,
                                             const double* const* srcs_lx, double kappa, int has_anis, double anis,
                                             const double* mus, int niter, const double* residues, int precision,
                                             tms_stats* stats)
{
  TRY(check_conf(ctx));
  if (nrhs <= 0 || nrhs > MRHS_MAX || !sols_lx || !srcs_lx || !mus || !residues || niter <= 0)
    return fail(ctx, TMS_ERR_BAD_ARG, "bad batched arguments (1 <= nrhs <= %d)", MRHS_MAX);
  for (int k = 0; k < nrhs; k++)
    if (!sols_lx[k] || !srcs_lx[k] || !(residues[k] > 0) || !std::isfinite(mus[k]))
      return fail(ctx, TMS_ERR_BAD_ARG, "bad right-hand side %d", k);
  if (precision != TMS_PREC_DOUBLE && precision != TMS_PREC_MIXED_SINGLE && precision != TMS_PREC_MIXED_HALF)
    return fail(ctx, TMS_ERR_BAD_ARG, "unknown precision %d", precision);
  BatchWork* w;
  TRY(work(ctx, &w));
  TRY(alloc_bfield(ctx, w->hi[0], PREC_F64, nrhs));
  TRY(alloc_bfield(ctx, w->hi[6], PREC_F64, nrhs)); // eta_e per right-hand side
  Field* f = ctx->f64;
  for (int i = 0; i <= 7; i++) TRY(alloc_field(ctx, f[i], PREC_F64));
  Field *eta = ctx->ex, *psi = ctx->ex + 2;
  for (auto& e : ctx->ex) TRY(alloc_field(ctx, e, PREC_F64));
  BatchParams& bp = *w->bp_h;
  bp.kappa = kappa;
  bp.anis = has_anis ? anis : 1.0;
  for (int k = 0; k < nrhs; k++) bp.mu[k] = mus[k];
  CU(cudaMemcpyAsync(w->bp, w->bp_h, sizeof(BatchParams), cudaMemcpyHostToDevice, ctx->stream));
  const int64_t Vh = ctx->g.Vh;
  const int n = (int)Vh;
  const size_t bytes = (size_t)ctx->g.V * 24 * sizeof(double);
  auto U = links64(ctx);
  auto V = [](const Field& x) { return view<PREC_F64>(x); };
  // Eq. (8) per right-hand side (single-RHS FP64 kernels): varphi_k -> hi[0][k], eta_e,k -> hi[6][k]
  for (int k = 0; k < nrhs; k++)
    {
      TRY(set_params(ctx, kappa, mus[k], has_anis, anis));
      const double* src = srcs_lx[k];
      if (ctx->ptr_mode == TMS_PTR_HOST)
        {
          TRY(ensure_stage(ctx, bytes));
          CU(cudaMemcpyAsync(ctx->stage, srcs_lx[k], bytes, cudaMemcpyHostToDevice, ctx->stream));
          src = ctx->stage;
        }
      const Field ek = one(w->hi[6], k), vk = one(w->hi[0], k);
      ctx->launches += 4;
      aos_to_soa_kernel<PREC_F64><<<div_up(n, 256), 256, 0, ctx->stream>>>(n, src, ctx->lx_of_eo, V(ek));
      aos_to_soa_kernel<PREC_F64><<<div_up(n, 256), 256, 0, ctx->stream>>>(n, src, ctx->lx_of_eo + Vh, V(eta[1]));
      diag_kernel<PREC_F64><<<div_up(n, 256), 256, 0, ctx->stream>>>(n, V(ek), V(f[5]), ctx->prm, 1.0, 1);
      EpiSrcPrep<PREC_F64> sp{{V(vk), V(vk)}, {V(eta[1]), V(eta[1])}};
      launch_hop<PREC_F64, LINK_F64_18>(ctx, ctx->stream, 1, 1, f[5], f[5], U, ctx->prm, sp);
      CU(cudaGetLastError());
    }
  // Eq. (9), all right-hand sides at once
  tms_status st;
  if (precision == TMS_PREC_DOUBLE) st = cg_batch<PREC_F64>(ctx, w, links64(ctx), nrhs, niter, residues, stats);
  else if (precision == TMS_PREC_MIXED_SINGLE)
    st = ctx->su3 ? cg_batch<PREC_F32>(ctx, w, links32r(ctx), nrhs, niter, residues, stats)
                  : cg_batch<PREC_F32>(ctx, w, links32f(ctx), nrhs, niter, residues, stats);
  else
    st = ctx->su3 ? cg_batch<PREC_F16>(ctx, w, links16r(ctx), nrhs, niter, residues, stats)
                  : cg_batch<PREC_F16>(ctx, w, links32f(ctx), nrhs, niter, residues, stats);
  if (st != TMS_OK && st != TMS_ERR_NOT_CONVERGED) return st;
  // Eq. (10)-(11) and paste, per right-hand side
  for (int k = 0; k < nrhs; k++)
    {
      TRY(set_params(ctx, kappa, mus[k], has_anis, anis));
      const Field xk = one(w->hi[1], k), ek = one(w->hi[6], k);
      kern_op<PREC_F64>(ctx, U, xk, f[5], psi[1], -1.0, ctx->prm);
      EpiReco<PREC_F64> rc{{V(psi[0]), V(psi[0])}, {V(ek), V(ek)}, ctx->prm, 1.0};
      launch_hop<PREC_F64, LINK_F64_18>(ctx, ctx->stream, 0, 1, psi[1], psi[1], U, ctx->prm, rc);
      double* d = (ctx->ptr_mode == TMS_PTR_HOST) ? ctx->stage : sols_lx[k];
      ctx->launches += 2;
      soa_to_aos_kernel<PREC_F64><<<div_up(n, 256), 256, 0, ctx->stream>>>(n, V(psi[0]), ctx->lx_of_eo, d);
      soa_to_aos_kernel<PREC_F64><<<div_up(n, 256), 256, 0, ctx->stream>>>(n, V(psi[1]), ctx->lx_of_eo + Vh, d);
      CU(cudaGetLastError());
      if (ctx->ptr_mode == TMS_PTR_HOST)
        CU(cudaMemcpyAsync(sols_lx[k], ctx->stage, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    }
  TRY(finish(ctx));
  return st;
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
    bp.kappa = 0.16;
    bp.anis = 1.0;
    for (int k = 0; k < nrhs; k++) bp.mu[k] = 0.01;
    CU(cudaMemcpyAsync(w->bp, w->bp_h, sizeof(BatchParams), cudaMemcpyHostToDevice, ctx->stream));
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
        EpiBInvDiag<P> a{bview<P>(w->lo[2]), 1.0};
        launch_mrhs<P>(ctx, w, ctx->stream, 0, nrhs, w->lo[1], U, a, NoFinB{}, nullptr);
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
