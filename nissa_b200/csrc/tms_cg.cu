// C ABI of the solvers: the e/o CG of K(+mu)K(-mu) (FP64, and FP32 / FP16
// inner with FP64 reliable updates), the full solve of Eq. (8)-(11), the
// full-lattice CG of Q(+m)Q(-m) and the multi-shift CGM of the tm Q^2
// operator.  Each CG/CGM iteration block is replayed as a CUDA graph.
#include "tms_internal.cuh"
#include <type_traits>

#include <algorithm>

using namespace tms_int;

namespace
{
  // ================================================================ operators
  // A CG "operator policy" fixes the matrix, the fields it works on and the
  // number of sites of its vectors.
  //   EoOp: K(+mu)K(-mu) on odd sites (inv_tmDkern_eoprec_square_eos_cg)
  //   LxOp: Q(+mu)Q(-mu) on the full lattice (inv_tmQ2_cg, and the per-shift
  //         refinement of the multi-shift solver)
  // hi fields (FP64): 0 b, 1 x, 2 r, 3 p, 4-6 temporaries; lo fields (inner
  // precision): 1 r, 2 p, 3-4 temporaries.

  struct EoOp
  {
    static constexpr int slot0 = 0;
    static constexpr int nlo = 6;
    static int stride(tms_ctx* c) { return c->g.stride; }
    static int nsites(tms_ctx* c) { return (int)c->g.Vh; }
    static Field* hi(tms_ctx* c) { return c->f64; }
    static Field* lo(tms_ctx* c) { return c->lo; }
    static int& lo_prec(tms_ctx* c) { return c->lo_prec; }
    static Field& xlo(tms_ctx* c) { return c->xlo32; }

    // r = b - K(+mu)K(-mu) x in FP64; returns |r|^2 (uses hi 4, 5, 6).  For the
    // mixed solvers (`mixed`) the links may be read as 12 reals.
    static tms_status true_residual(tms_ctx* ctx, const Field& b, const Field& x, const Field& r, double* rr,
                                    bool mixed = false)
    {
      Field &t1 = ctx->f64[4], &te = ctx->f64[5], &s = ctx->f64[6];
      if (mixed)
        {
          // the mixed solvers' recomputation: K(+mu) fused with r = b - s and |r|^2
          auto res = [&](const auto& U) {
            kern_op<PREC_F64>(ctx, U, x, te, t1, -1.0, ctx->prm);
            EpiInvDiag<PREC_F64> a{{view<PREC_F64>(te), view<PREC_F64>(te)}, ctx->prm, +1.0};
            launch_hop<PREC_F64>(ctx, ctx->stream, 0, 1, t1, t1, U, ctx->prm, a);
            EpiKernResidual<PREC_F64> e{view<PREC_F64>(r), view<PREC_F64>(t1), view<PREC_F64>(b), ctx->prm, +1.0};
            launch_hop<PREC_F64>(ctx, ctx->stream, 1, 1, te, te, U, ctx->prm, e);
          };
          if (reliable_links12(ctx)) res(links64r(ctx));
          else res(links64(ctx));
          CU(cudaGetLastError());
          *rr = read_result(ctx);
          return TMS_OK;
        }
      auto U = links64(ctx);
      kern_op<PREC_F64>(ctx, U, x, te, t1, -1.0, ctx->prm);
      kern_op<PREC_F64>(ctx, U, t1, te, s, +1.0, ctx->prm);
      const int n = nsites(ctx);
      ++ctx->launches;
      residual_kernel<<<div_up(n, BLAS_THREADS), BLAS_THREADS, 0, ctx->stream>>>(
        n, view<PREC_F64>(b), view<PREC_F64>(s), view<PREC_F64>(r), reducer(ctx));
      CU(cudaGetLastError());
      *rr = read_result(ctx);
      return TMS_OK;
    }

    // the paired x update (record with paired = true) keeps the second direction here
    static constexpr bool kPaired = true;
    static Field& p2(tms_ctx* c) { return c->lo[5]; }

    // `iters` CG iterations in precision P (x in PX): v 1 r, 2 p, 3 t1, 4 te.
    // paired (iters even): iteration 2k reads its direction from p and writes
    // the next into p2, iteration 2k+1 reads p2, writes p and adds both
    // iterations' steps to x; a replay starts and ends with the direction in p.
    template <int P, int PX, int LF>
    static void record(tms_ctx* c, cudaStream_t s, const LinkT<LF>& U, Field* v, const Field& x, int iters,
                       bool paired = false)
    {
      const Field &r = v[1], &t1 = v[3], &te = v[4];
      const int* stop = &c->st->stop;
      const OpParams* prm = c->prm;
      const int n = nsites(c);
      for (int it = 0; it < iters; it++)
        {
          const bool odd = paired && (it & 1);
          const Field& p = odd ? p2(c) : v[2];         // this iteration's direction
          const Field& pn = (paired && !odd) ? p2(c) : v[2]; // the next one
          EpiInvDiag<P> a1{{view<P>(te), view<P>(te)}, prm, -1.0};
          launch_hop<P, LF>(c, s, 0, 1, p, p, U, prm, a1, NoFin{}, stop);
          EpiKern<P, true> b1{{view<P>(t1), view<P>(t1)}, {view<P>(p), view<P>(p)}, prm, -1.0};
          launch_hop<P, LF>(c, s, 1, 1, te, te, U, prm, b1, FinAlpha{c->st}, stop);
          EpiInvDiag<P> a2{{view<P>(te), view<P>(te)}, prm, +1.0};
          launch_hop<P, LF>(c, s, 0, 1, t1, t1, U, prm, a2, NoFin{}, stop);
          if (!paired)
            {
              EpiKernCgUpdate<P, PX, 1> b2{view<P>(t1), view<P>(r), view<P>(p), view<PX>(x), prm, c->st, +1.0};
              launch_hop<P, LF>(c, s, 1, 1, te, te, U, prm, b2, FinBeta{c->st}, stop);
            }
          else if (!odd)
            {
              EpiKernCgUpdate<P, PX, 0> b2{view<P>(t1), view<P>(r), view<P>(p), view<PX>(x), prm, c->st, +1.0};
              launch_hop<P, LF>(c, s, 1, 1, te, te, U, prm, b2, FinBeta{c->st}, stop);
            }
          else
            {
              EpiKernCgUpdate<P, PX, 2> b2{view<P>(t1), view<P>(r),   view<P>(p),       view<PX>(x),
                                           prm,          c->st,         +1.0,             view<P>(v[2])};
              launch_hop<P, LF>(c, s, 1, 1, te, te, U, prm, b2, FinBeta{c->st}, stop);
            }
          ++c->launches;
          if (paired)
            launch_pdl(c, xpay_to_kernel<P>, div_up(n, BLAS_THREADS), BLAS_THREADS, 0, s, n, view<P>(r), view<P>(p),
                       view<P>(pn), (const CgState*)c->st, stop);
          else
            launch_pdl(c, xpay_kernel<P>, div_up(n, BLAS_THREADS), BLAS_THREADS, 0, s, n, view<P>(r), view<P>(p),
                       (const CgState*)c->st, stop);
        }
    }
  };

  struct LxOp
  {
    static constexpr int slot0 = 3;
    static constexpr bool kPaired = false;
    static constexpr int nlo = 5;
    static int stride(tms_ctx* c) { return 2 * c->g.stride; }
    static int nsites(tms_ctx* c) { return 2 * c->g.stride; }
    static Field* hi(tms_ctx* c) { return c->lx64; }
    static Field* lo(tms_ctx* c) { return c->lxlo; }
    static int& lo_prec(tms_ctx* c) { return c->lxlo_prec; }
    static Field& xlo(tms_ctx* c) { return c->lxxlo; }

    template <int P>
    static void qop(tms_ctx* c, cudaStream_t s, const Field& in, const Field& out, double sgn, const OpParams* prm)
    {
      EpiTmQ<P, false> e{{view_par<P>(out, 0), view_par<P>(out, 1)}, {view_par<P>(in, 0), view_par<P>(in, 1)}, prm,
                         sgn};
      launch_hop_v<P, LINK_F64_18>(c, s, 0, 2, view_par<P>(in, 0), view_par<P>(in, 1), links64(c), prm, e);
    }

    // r = b - Q(+mu)Q(-mu) x in FP64; returns |r|^2 (uses hi 4, 5); 18-real links always
    static tms_status true_residual(tms_ctx* ctx, const Field& b, const Field& x, const Field& r, double* rr,
                                    bool = false)
    {
      Field &t = ctx->lx64[4], &s = ctx->lx64[5];
      qop<PREC_F64>(ctx, ctx->stream, x, t, -1.0, ctx->prm);
      qop<PREC_F64>(ctx, ctx->stream, t, s, +1.0, ctx->prm);
      const int n = nsites(ctx);
      ++ctx->launches;
      residual_kernel<<<div_up(n, BLAS_THREADS), BLAS_THREADS, 0, ctx->stream>>>(
        n, view<PREC_F64>(b), view<PREC_F64>(s), view<PREC_F64>(r), reducer(ctx));
      CU(cudaGetLastError());
      *rr = read_result(ctx);
      return TMS_OK;
    }

    // `iters` CG iterations: t = Q(-mu) p reducing |t|^2 ; s = Q(+mu) t fused
    // with the x and r updates ; p = r + beta p.   v 1 r, 2 p, 3 t
    template <int P, int PX, int LF>
    static void record(tms_ctx* c, cudaStream_t s, const LinkT<LF>& U, Field* v, const Field& x, int iters,
                       bool = false)
    {
      const Field &r = v[1], &p = v[2], &t = v[3];
      const int* stop = &c->st->stop;
      const OpParams* prm = c->prm;
      auto V = [](const Field& f, int par) { return view_par<P>(f, par); };
      for (int it = 0; it < iters; it++)
        {
          EpiTmQ<P, true> a{{V(t, 0), V(t, 1)}, {V(p, 0), V(p, 1)}, prm, -1.0};
          launch_hop_v<P, LF>(c, s, 0, 2, V(p, 0), V(p, 1), U, prm, a, FinAlpha{c->st}, stop);
          EpiTmQCgUpdate<P, PX> b{{V(t, 0), V(t, 1)},
                                  {V(r, 0), V(r, 1)},
                                  {V(p, 0), V(p, 1)},
                                  {view_par<PX>(x, 0), view_par<PX>(x, 1)},
                                  prm,
                                  c->st,
                                  +1.0};
          launch_hop_v<P, LF>(c, s, 0, 2, V(t, 0), V(t, 1), U, prm, b, FinBeta{c->st}, stop);
          const int n = nsites(c);
          ++c->launches;
          launch_pdl(c, xpay_kernel<P>, div_up(n, BLAS_THREADS), BLAS_THREADS, 0, s, n, view<P>(r), view<P>(p),
                     (const CgState*)c->st, stop);
        }
    }
  };

  // ClovOp: K_clov(dag=false) K_clov(dag=true) on odd sites
  // (inv_tmclovDkern_eoprec_square_eos_cg), on the e/o fields of EoOp
  struct ClovOp
  {
    static constexpr int slot0 = 8;
    static constexpr bool kPaired = true;
    static Field& p2(tms_ctx* c) { return c->lo[5]; }
    static constexpr int nlo = 6;
    static int stride(tms_ctx* c) { return c->g.stride; }
    static int nsites(tms_ctx* c) { return (int)c->g.Vh; }
    static Field* hi(tms_ctx* c) { return c->f64; }
    static Field* lo(tms_ctx* c) { return c->lo; }
    static int& lo_prec(tms_ctx* c) { return c->lo_prec; }
    static Field& xlo(tms_ctx* c) { return c->xlo32; }

    // r = b - K(false)K(true) x in FP64; returns |r|^2 (uses hi 4, 5, 6).  For the
    // mixed solvers (`mixed`) the links may be read as 12 reals.
    static tms_status true_residual(tms_ctx* ctx, const Field& b, const Field& x, const Field& r, double* rr,
                                    bool mixed = false)
    {
      Field &t1 = ctx->f64[4], &te = ctx->f64[5], &s = ctx->f64[6];
      if (mixed && reliable_links12(ctx))
        {
          auto U = links64r(ctx);
          clov_kern_op<PREC_F64>(ctx, U, clov64(ctx), x, te, t1, 1, ctx->prm);
          clov_kern_op<PREC_F64>(ctx, U, clov64(ctx), t1, te, s, 0, ctx->prm);
        }
      else
        {
          auto U = links64(ctx);
          clov_kern_op<PREC_F64>(ctx, U, clov64(ctx), x, te, t1, 1, ctx->prm);
          clov_kern_op<PREC_F64>(ctx, U, clov64(ctx), t1, te, s, 0, ctx->prm);
        }
      const int n = nsites(ctx);
      ++ctx->launches;
      residual_kernel<<<div_up(n, BLAS_THREADS), BLAS_THREADS, 0, ctx->stream>>>(
        n, view<PREC_F64>(b), view<PREC_F64>(s), view<PREC_F64>(r), reducer(ctx));
      CU(cudaGetLastError());
      *rr = read_result(ctx);
      return TMS_OK;
    }

    // `iters` CG iterations in precision P (x in PX): v 1 r, 2 p, 3 t1, 4 te.
    // (p, K(false)K(true) p) = |K(true) p|^2 is reduced in the second launch.
    // paired: the two directions and every-other-iteration x update of EoOp.
    template <int P, int PX, int LF>
    static void record(tms_ctx* c, cudaStream_t s, const LinkT<LF>& U, Field* v, const Field& x, int iters,
                       bool paired = false)
    {
      const Field &r = v[1], &t1 = v[3], &te = v[4];
      const int* stop = &c->st->stop;
      const OpParams* prm = c->prm;
      const ClovT<P> cl = clov<P>(c);
      const int n = nsites(c);
      for (int it = 0; it < iters; it++)
        {
          const bool odd = paired && (it & 1);
          const Field& p = odd ? p2(c) : v[2];
          const Field& pn = (paired && !odd) ? p2(c) : v[2];
          EpiInvClov<P> a1{{view<P>(te), view<P>(te)}, cl, 1};
          launch_hop<P, LF>(c, s, 0, 1, p, p, U, prm, a1, NoFin{}, stop);
          EpiClovKern<P, true> b1{{view<P>(t1), view<P>(t1)}, {view<P>(p), view<P>(p)}, cl, prm, 1};
          launch_hop<P, LF>(c, s, 1, 1, te, te, U, prm, b1, FinAlpha{c->st}, stop);
          EpiInvClov<P> a2{{view<P>(te), view<P>(te)}, cl, 0};
          launch_hop<P, LF>(c, s, 0, 1, t1, t1, U, prm, a2, NoFin{}, stop);
          if (!paired)
            {
              EpiClovKernCgUpdate<P, PX, 1> b2{view<P>(t1), view<P>(r), view<P>(p), view<PX>(x), cl, prm, c->st};
              launch_hop<P, LF>(c, s, 1, 1, te, te, U, prm, b2, FinBeta{c->st}, stop);
            }
          else if (!odd)
            {
              EpiClovKernCgUpdate<P, PX, 0> b2{view<P>(t1), view<P>(r), view<P>(p), view<PX>(x), cl, prm, c->st};
              launch_hop<P, LF>(c, s, 1, 1, te, te, U, prm, b2, FinBeta{c->st}, stop);
            }
          else
            {
              EpiClovKernCgUpdate<P, PX, 2> b2{view<P>(t1), view<P>(r), view<P>(p),  view<PX>(x),
                                               cl,           prm,         c->st,        view<P>(v[2])};
              launch_hop<P, LF>(c, s, 1, 1, te, te, U, prm, b2, FinBeta{c->st}, stop);
            }
          ++c->launches;
          if (paired)
            launch_pdl(c, xpay_to_kernel<P>, div_up(n, BLAS_THREADS), BLAS_THREADS, 0, s, n, view<P>(r), view<P>(p),
                       view<P>(pn), (const CgState*)c->st, stop);
          else
            launch_pdl(c, xpay_kernel<P>, div_up(n, BLAS_THREADS), BLAS_THREADS, 0, s, n, view<P>(r), view<P>(p),
                       (const CgState*)c->st, stop);
        }
    }
  };

  // capture a block of iterations once per (slot, fields); replayed every launch
  template <class Rec>
  tms_status capture(tms_ctx* ctx, int slot, const Rec& rec)
  {
    if (ctx->graph[slot]) return TMS_OK;
    cudaStream_t cs;
    CU(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaGraph_t graph;
    CU(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    const uint64_t before = ctx->launches;
    rec(cs);
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

  tms_status drop_graph(tms_ctx* ctx, int slot)
  {
    if (ctx->graph[slot])
      {
        CU(cudaStreamSynchronize(ctx->stream));
        cudaGraphExecDestroy(ctx->graph[slot]);
        ctx->graph[slot] = nullptr;
      }
    return TMS_OK;
  }

  tms_status launch_graph(tms_ctx* ctx, int slot)
  {
    CU(cudaGraphLaunch(ctx->graph[slot], ctx->stream));
    ctx->launches += ctx->graph_nodes[slot];
    return TMS_OK;
  }

  void fill_stats(tms_stats* stats, tms_status st, int iters, int reliable, double it_res, double true_res, float ms)
  {
    if (!stats) return;
    stats->status = st;
    stats->iterations = iters;
    stats->reliable_updates = reliable;
    stats->iterated_rel_res2 = it_res;
    stats->true_rel_res2 = true_res;
    stats->seconds = ms * 1e-3;
  }

  // ------------------------------------------------------------- CG, FP64
  // b = hi[0], x = hi[1] (initial guess / solution).  cg_invert
  // (cg_invert_template_threaded.hpp:17-150) with the operator of the policy.
  template <class Op>
  tms_status cg_double(tms_ctx* ctx, int niter, double residue, bool have_guess, tms_stats* stats)
  {
    Field* f = Op::hi(ctx);
    const int n = Op::nsites(ctx);
    for (int i = 1; i <= 6; i++) TRY(alloc_field(ctx, f[i], PREC_F64, Op::stride(ctx)));
    double b2;
    TRY(norm2<PREC_F64>(ctx, f[0], &b2, n));
    if (b2 == 0.0 || std::isnan(b2)) return fail(ctx, TMS_ERR_INVALID_SOURCE, "invalid norm: %g", b2);
    double rr;
    if (have_guess) TRY(Op::true_residual(ctx, f[0], f[1], f[2], &rr));
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
    const int slot = Op::slot0;
    TRY(capture(ctx, slot, [&](cudaStream_t cs) {
      Op::template record<PREC_F64, PREC_F64>(ctx, cs, U, v, f[1], ctx->graph_iters);
    }));
    CU(cudaEventRecord(ctx->ev0, ctx->stream));
    while (S.stop == STOP_RUN)
      {
        TRY(launch_graph(ctx, slot));
        TRY(pull_state(ctx));
      }
    CU(cudaEventRecord(ctx->ev1, ctx->stream));
    double tr;
    TRY(Op::true_residual(ctx, f[0], f[1], f[6], &tr));
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    tms_status st = TMS_OK;
    if (S.stop == STOP_BREAKDOWN) st = fail(ctx, TMS_ERR_NAN, "nanned (iteration %d)", S.iter);
    else if (S.stop == STOP_MAXITER) st = fail(ctx, TMS_ERR_NOT_CONVERGED, "exit without converging");
    fill_stats(stats, st, S.iter, 0, S.rr / b2, tr / b2, ms);
    return st;
  }

  // ------------------------------------------------- CG, mixed precision
  // FP32 (or FP16-spinor) inner CG with FP64 reliable updates: the solution is
  // accumulated in FP64 and the residual recomputed with the FP64 operator
  // whenever the iterated residual has dropped by delta since the last update
  // (the outer defect-correction loop of cg_128_invert_template_threaded.cpp:36-109,
  // here with the Krylov direction kept across updates).
  template <class Op, int P, int LF>
  tms_status cg_mixed(tms_ctx* ctx, const LinkT<LF>& U, int niter, double residue, bool have_guess,
                      tms_stats* stats)
  {
    constexpr int PX = (P == PREC_F16) ? PREC_F32 : P; // x accumulates in FP32 at least
    const int slot = Op::slot0 + (P == PREC_F16 ? 2 : 1);
    const int n = Op::nsites(ctx);
    Field* f = Op::hi(ctx);
    for (int i = 1; i <= 6; i++) TRY(alloc_field(ctx, f[i], PREC_F64, Op::stride(ctx)));
    Field* lo = Op::lo(ctx);
    if (Op::lo_prec(ctx) != P)
      {
        // the inner-precision fields move: graphs captured on the old ones are void
        // (the FP32 multi-shift graph uses the full-lattice inner fields too)
        TRY(drop_graph(ctx, Op::slot0 + 1));
        TRY(drop_graph(ctx, Op::slot0 + 2));
        if (Op::slot0 == LxOp::slot0) TRY(drop_graph(ctx, 7));
        // the twisted-mass and twisted-clover e/o solvers share the inner fields
        if (Op::slot0 == EoOp::slot0 || Op::slot0 == ClovOp::slot0)
          for (int k : {EoOp::slot0 + 1, EoOp::slot0 + 2, ClovOp::slot0 + 1, ClovOp::slot0 + 2}) TRY(drop_graph(ctx, k));
        for (int i = 0; i < Op::nlo; i++) TRY(alloc_field(ctx, lo[i], P, Op::stride(ctx)));
        Op::lo_prec(ctx) = P;
      }
    Field& xlo = Op::xlo(ctx);
    TRY(alloc_field(ctx, xlo, PX, Op::stride(ctx)));
    const double delta = (P == PREC_F16) ? ctx->delta_half : ctx->delta_single; // reliable-update trigger
    double b2;
    TRY(norm2<PREC_F64>(ctx, f[0], &b2, n));
    if (b2 == 0.0 || std::isnan(b2)) return fail(ctx, TMS_ERR_INVALID_SOURCE, "invalid norm: %g", b2);
    double rr;
    if (have_guess) TRY(Op::true_residual(ctx, f[0], f[1], f[2], &rr, true));
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
    double last_rt = have_guess ? rr : -1.0; // true residual of the current x, if known
    if (rr >= target)
      {
        convert<P, PREC_F64>(ctx, f[2], lo[1], 1.0, n); // r_lo = r
        convert<P, PREC_F64>(ctx, f[2], lo[2], 1.0, n); // p_lo = r
        CU(cudaMemsetAsync(xlo.d, 0, xlo.bytes, ctx->stream));
        S.rr = rr;
        S.b2 = b2;
        S.target = target;
        S.rel_trigger = delta * delta * rr;
        S.niter_max = niter;
        S.stop = STOP_RUN;
        TRY(push_state(ctx));
        Field v[5] = {Field{}, lo[1], lo[2], lo[3], lo[4]};
        // x updated every other iteration (e/o operator, even replay length)
        const bool paired = Op::kPaired && ctx->graph_iters % 2 == 0;
        TRY(capture(ctx, slot, [&](cudaStream_t cs) {
          Op::template record<P, PX>(ctx, cs, U, v, xlo, ctx->graph_iters, paired);
        }));
        CU(cudaEventRecord(ctx->ev0, ctx->stream));
        for (;;)
          {
            const int iter0 = S.iter;
            TRY(launch_graph(ctx, slot));
            TRY(pull_state(ctx));
            if (S.stop == STOP_RUN) continue;
            if (S.stop == STOP_BREAKDOWN)
              {
                st = fail(ctx, TMS_ERR_NAN, "nanned (iteration %d)", S.iter);
                break;
              }
            // a replay cut after an odd number of paired iterations leaves the last
            // step (alpha p, direction in p) out of x; after an even number the
            // direction to keep is in p2
            bool dir_in_p2 = false;
            if constexpr (Op::kPaired)
              if (paired)
                {
                  if ((S.iter - iter0) & 1)
                    {
                      ++ctx->launches;
                      axpby_kernel<PX, PX, P><<<div_up(n, BLAS_THREADS), BLAS_THREADS, 0, ctx->stream>>>(
                        n, 1.0, view<PX>(xlo), S.alpha, view<P>(lo[2]), view<PX>(xlo));
                      CU(cudaGetLastError());
                    }
                  else
                    dir_in_p2 = true;
                }
            // reliable update: x += x_lo (FP64), r = b - A x (FP64)
            ++ctx->launches;
            axpby_kernel<PREC_F64, PREC_F64, PX><<<div_up(n, BLAS_THREADS), BLAS_THREADS, 0, ctx->stream>>>(
              n, 1.0, view<PREC_F64>(f[1]), 1.0, view<PX>(xlo), view<PREC_F64>(f[1]));
            CU(cudaMemsetAsync(xlo.d, 0, xlo.bytes, ctx->stream));
            if (xlo.n) CU(cudaMemsetAsync(xlo.n, 0, sizeof(float) * xlo.stride, ctx->stream));
            double rt;
            TRY(Op::true_residual(ctx, f[0], f[1], f[2], &rt, true));
            reliable++;
            last_rt = rt; // the true residual of the current x
            if (rt < target) break;
            if (S.stop == STOP_MAXITER || S.iter >= niter)
              {
                st = fail(ctx, TMS_ERR_NOT_CONVERGED, "exit without converging");
                break;
              }
            // restart the recurrence from the true residual, keeping the direction
            convert<P, PREC_F64>(ctx, f[2], lo[1], 1.0, n);
            S.beta = rt / S.rr_prev;
            S.rr = rt;
            S.rel_trigger = delta * delta * rt;
            S.stop = STOP_RUN;
            TRY(push_state(ctx));
            ++ctx->launches;
            if constexpr (Op::kPaired)
              if (dir_in_p2)
                {
                  xpay_to_kernel<P><<<div_up(n, BLAS_THREADS), BLAS_THREADS, 0, ctx->stream>>>(
                    n, view<P>(lo[1]), view<P>(Op::p2(ctx)), view<P>(lo[2]), ctx->st, nullptr);
                  CU(cudaGetLastError());
                  continue;
                }
            xpay_kernel<P><<<div_up(n, BLAS_THREADS), BLAS_THREADS, 0, ctx->stream>>>(n, view<P>(lo[1]),
                                                                                       view<P>(lo[2]), ctx->st,
                                                                                       nullptr);
            CU(cudaGetLastError());
          }
        CU(cudaEventRecord(ctx->ev1, ctx->stream));
        CU(cudaEventSynchronize(ctx->ev1));
        cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
      }
    // the last reliable update left x with its FP64 true residual; otherwise recompute it
    double tr = last_rt;
    if (tr < 0.0) TRY(Op::true_residual(ctx, f[0], f[1], f[6], &tr, true));
    fill_stats(stats, st, S.iter, reliable, S.rr / b2, tr / b2, ms);
    return st;
  }

  template <class Op>
  tms_status cg_dispatch(tms_ctx* ctx, int precision, int niter, double residue, bool have_guess, tms_stats* stats)
  {
    if (precision == TMS_PREC_DOUBLE) return cg_double<Op>(ctx, niter, residue, have_guess, stats);
    if (precision == TMS_PREC_MIXED_SINGLE)
      {
        if (!ctx->su3) return cg_mixed<Op, PREC_F32>(ctx, links32f(ctx), niter, residue, have_guess, stats);
        return ctx->single_links16 ? cg_mixed<Op, PREC_F32>(ctx, links16r(ctx), niter, residue, have_guess, stats)
                                   : cg_mixed<Op, PREC_F32>(ctx, links32r(ctx), niter, residue, have_guess, stats);
      }
    if (precision == TMS_PREC_MIXED_HALF)
      {
        // the e/o twisted-mass solver may run its hops in FP16 arithmetic (tuning "half_arith")
        if constexpr (std::is_same<Op, EoOp>::value)
          if (ctx->su3 && ctx->half_arith)
            return cg_mixed<Op, PREC_F16>(ctx, links16h(ctx), niter, residue, have_guess, stats);
        return ctx->su3 ? cg_mixed<Op, PREC_F16>(ctx, links16r(ctx), niter, residue, have_guess, stats)
                        : cg_mixed<Op, PREC_F16>(ctx, links32f(ctx), niter, residue, have_guess, stats);
      }
    return fail(ctx, TMS_ERR_BAD_ARG, "unknown precision %d", precision);
  }

  // ------------------------------------------------------ multi-shift CGM
  // cgm_invert (cgm_invert_template_threaded.hpp:11-295) on Q_W^2 = Q(0)Q(0),
  // shifts sigma_i = m_i^2, for the source in lx64[0].  Vectors in precision P;
  // solutions left in ctx->cgm_x.  Returns the solver status, *iters the
  // iteration count (the reference's final_iter).
  size_t per_site_bytes(int prec) { return prec == PREC_F64 ? 192 : prec == PREC_F32 ? 96 : 52; }

  template <int P, int LF>
  tms_status cgm_run(tms_ctx* ctx, const LinkT<LF>& U, int nshift, const double* sigma, const double* target,
                     int niter, double b2, int* iters, float* ms)
  {
    const int slot = (P == PREC_F64) ? 6 : 7;
    const int stride = 2 * ctx->g.stride, n = stride;
    const size_t fbytes = per_site_bytes(P) * (size_t)stride;
    if (ctx->cgm_prec != P || ctx->cgm_nshift < nshift)
      {
        TRY(drop_graph(ctx, 6));
        TRY(drop_graph(ctx, 7));
        if (ctx->cgm_x) cudaFree(ctx->cgm_x);
        if (ctx->cgm_ps) cudaFree(ctx->cgm_ps);
        ctx->cgm_x = ctx->cgm_ps = nullptr;
        ctx->cgm_prec = -1;
        CU(cudaMalloc(&ctx->cgm_x, fbytes * nshift));
        CU(cudaMalloc(&ctx->cgm_ps, fbytes * nshift));
        ctx->cgm_prec = P;
        ctx->cgm_nshift = nshift;
      }
    // inner vectors: r, p, t in precision P (FP64: hi 2-4, otherwise lo 1-3)
    if (P == PREC_F64)
      {
        for (int i = 2; i <= 4; i++) TRY(alloc_field(ctx, ctx->lx64[i], PREC_F64, stride));
      }
    else if (ctx->lxlo_prec != P)
      {
        TRY(drop_graph(ctx, LxOp::slot0 + 1));
        TRY(drop_graph(ctx, LxOp::slot0 + 2));
        for (int i = 0; i < LxOp::nlo; i++) TRY(alloc_field(ctx, ctx->lxlo[i], P, stride));
        ctx->lxlo_prec = P;
      }
    const bool hi = (P == PREC_F64);
    const Field& r = hi ? ctx->lx64[2] : ctx->lxlo[1];
    const Field& p = hi ? ctx->lx64[3] : ctx->lxlo[2];
    const Field& t = hi ? ctx->lx64[4] : ctx->lxlo[3];
    // solution / direction views of shift k
    auto shift_field = [&](void* base, int k) {
      Field f;
      f.prec = P;
      f.d = (unsigned char*)base + fbytes * k;
      f.n = nullptr;
      f.stride = stride;
      f.bytes = fbytes;
      return f;
    };
    // r = p = b ; ps_i = b ; x_i = 0
    convert<P, PREC_F64>(ctx, ctx->lx64[0], r, 1.0, n);
    convert<P, PREC_F64>(ctx, ctx->lx64[0], p, 1.0, n);
    for (int k = 0; k < nshift; k++) convert<P, PREC_F64>(ctx, ctx->lx64[0], shift_field(ctx->cgm_ps, k), 1.0, n);
    CU(cudaMemsetAsync(ctx->cgm_x, 0, fbytes * nshift, ctx->stream));
    CgmState& S = *ctx->cgm_h;
    memset(&S, 0, sizeof S);
    S.rr = b2;
    S.b2 = b2;
    S.betaa = 1.0;
    S.alpha = 0.0;
    S.nshift = nshift;
    S.nrun = nshift;
    S.niter_max = niter;
    for (int k = 0; k < nshift; k++)
      {
        S.sigma[k] = sigma[k];
        S.target[k] = target[k];
        S.zps[k] = S.zas[k] = 1.0;
        S.alphas[k] = 0.0;
        S.run[k] = 1;
      }
    CU(cudaMemcpyAsync(ctx->cgm, &S, sizeof S, cudaMemcpyHostToDevice, ctx->stream));
    const OpParams* prm = ctx->prm + 1; // the CGM operator: mu = 0
    const size_t shift_elems = fbytes / (P == PREC_F64 ? sizeof(double2) : P == PREC_F32 ? sizeof(float4) : sizeof(uint4));
    TRY(capture(ctx, slot, [&](cudaStream_t cs) {
      auto V = [](const Field& f, int par) { return view_par<P>(f, par); };
      const int* stop = &ctx->cgm->stop;
      for (int it = 0; it < ctx->graph_iters; it++)
        {
          ++ctx->launches;
          cgm_begin_kernel<<<1, 1, 0, cs>>>(ctx->cgm);
          EpiTmQ<P, true> a{{V(t, 0), V(t, 1)}, {V(p, 0), V(p, 1)}, prm, +1.0};
          launch_hop_v<P, LF>(ctx, cs, 0, 2, V(p, 0), V(p, 1), U, prm, a, FinCgm1{ctx->cgm}, stop);
          EpiCgm2<P> b{{V(t, 0), V(t, 1)}, {V(r, 0), V(r, 1)}, prm, ctx->cgm};
          launch_hop_v<P, LF>(ctx, cs, 0, 2, V(t, 0), V(t, 1), U, prm, b, FinCgm2{ctx->cgm}, stop);
          ++ctx->launches;
          cgm_update_kernel<P><<<div_up(n, 256), 256, 0, cs>>>(n, view<P>(r), view<P>(p),
                                                               view<P>(shift_field(ctx->cgm_x, 0)),
                                                               view<P>(shift_field(ctx->cgm_ps, 0)), shift_elems,
                                                               ctx->cgm);
        }
    }));
    CU(cudaEventRecord(ctx->ev0, ctx->stream));
    do
      {
        TRY(launch_graph(ctx, slot));
        CU(cudaMemcpyAsync(ctx->cgm_h, ctx->cgm, sizeof(CgmState), cudaMemcpyDeviceToHost, ctx->stream));
        CU(cudaStreamSynchronize(ctx->stream));
      }
    while (S.stop == STOP_RUN);
    CU(cudaEventRecord(ctx->ev1, ctx->stream));
    CU(cudaEventSynchronize(ctx->ev1));
    cudaEventElapsedTime(ms, ctx->ev0, ctx->ev1);
    *iters = S.iter;
    if (S.stop == STOP_BREAKDOWN) return fail(ctx, TMS_ERR_NAN, "nanned (cgm iteration %d)", S.iter);
    if (S.stop == STOP_MAXITER) return fail(ctx, TMS_ERR_NOT_CONVERGED, "exit without converging");
    return TMS_OK;
  }

  // x (FP64 full field) = solution of shift k of the last CGM
  template <int P>
  void cgm_solution(tms_ctx* ctx, int k, const Field& x)
  {
    const int stride = 2 * ctx->g.stride;
    Field f;
    f.prec = P;
    f.d = (unsigned char*)ctx->cgm_x + per_site_bytes(P) * (size_t)stride * k;
    f.stride = stride;
    convert<PREC_F64, P>(ctx, f, x, 1.0, stride);
  }
}

extern "C" {

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
  const tms_status st = cg_dispatch<EoOp>(ctx, precision, niter, residue, guess != nullptr, stats);
  if (st == TMS_OK || st == TMS_ERR_NOT_CONVERGED) TRY(spinor_out(ctx, f[1], nullptr, ctx->g.Vh, sol, true));
  TRY(finish(ctx));
  return st;
}

} // extern "C"

namespace
{
  // Eq. (8)-(11) of inv_tmD_cg_eoprec_native (cg_invert_tmD_eoprec.cpp:102-150) on
  // device fields: the source's parities in ex[0] (even) and ex[1] (odd), the
  // solution's in ex[2], ex[3].  The operator parameters must be set.
  // (the FP64 steps around a mixed-precision solve read the links as 12 reals
  // when the conf is SU(3) to rounding; the FP64 solve reads all 18)
  template <int LF>
  tms_status eo_full_solve_t(tms_ctx* ctx, const LinkT<LF>& U, int niter, double residue, int precision,
                             tms_stats* stats, const double* guess_Koo)
  {
    Field* f = ctx->f64;
    for (int i = 0; i <= 7; i++) TRY(alloc_field(ctx, f[i], PREC_F64));
    Field *eta = ctx->ex, *psi = ctx->ex + 2; // [0] even, [1] odd
    const int n = (int)ctx->g.Vh;
    auto V = [&](const Field& x) { return view<PREC_F64>(x); };
    // Eq. (8a): te = D_ee^-1 eta_e ; Eq. (8b): varphi = g5 (eta_o + hop(te)/2) -> f0
    ++ctx->launches;
    diag_kernel<PREC_F64><<<div_up(n, 256), 256, 0, ctx->stream>>>(n, V(eta[0]), V(f[5]), ctx->prm, 1.0, 1);
    EpiSrcPrep<PREC_F64> sp{{V(f[0]), V(f[0])}, {V(eta[1]), V(eta[1])}};
    launch_hop<PREC_F64, LF>(ctx, ctx->stream, 1, 1, f[5], f[5], U, ctx->prm, sp);
    CU(cudaGetLastError());
    // Eq. (9), from the caller's odd-site guess when given
    if (guess_Koo) TRY(spinor_in(ctx, guess_Koo, nullptr, ctx->g.Vh, f[1]));
    const tms_status st = cg_dispatch<EoOp>(ctx, precision, niter, residue, guess_Koo != nullptr, stats);
    if (st != TMS_OK && st != TMS_ERR_NOT_CONVERGED) return st;
    // Eq. (10): psi_o = K(-mu) x ; Eq. (11): psi_e = D_ee^-1 (eta_e + hop(psi_o)/2)
    kern_op<PREC_F64>(ctx, U, f[1], f[5], psi[1], -1.0, ctx->prm);
    EpiReco<PREC_F64> rc{{V(psi[0]), V(psi[0])}, {V(eta[0]), V(eta[0])}, ctx->prm, 1.0};
    launch_hop<PREC_F64, LF>(ctx, ctx->stream, 0, 1, psi[1], psi[1], U, ctx->prm, rc);
    CU(cudaGetLastError());
    return st;
  }

  tms_status eo_full_solve(tms_ctx* ctx, int niter, double residue, int precision, tms_stats* stats,
                           const double* guess_Koo = nullptr)
  {
    if (precision != TMS_PREC_DOUBLE && reliable_links12(ctx))
      return eo_full_solve_t(ctx, links64r(ctx), niter, residue, precision, stats, guess_Koo);
    return eo_full_solve_t(ctx, links64(ctx), niter, residue, precision, stats, guess_Koo);
  }
}

namespace
{
  // inv_tmD_cg_eoprec between AoS lx spinors in device memory (the operator
  // parameters set): split the source into its parities, Eq. (8)-(11), paste
  // the solution's parities, then the reference's lx residual check.  When
  // given, `src_read` is recorded on the stream once the source has been read
  // and `dst_ready` once the solution is written.
  tms_status cg_eoprec_lx(tms_ctx* ctx, double* dst, const double* src, int niter, double residue, int precision,
                          tms_stats* stats, cudaEvent_t src_read, cudaEvent_t dst_ready,
                          const double* guess_Koo = nullptr)
  {
    Field* f = ctx->f64;
    for (int i = 0; i <= 7; i++) TRY(alloc_field(ctx, f[i], PREC_F64));
    Field *eta = ctx->ex, *psi = ctx->ex + 2; // [0] even, [1] odd
    for (auto& e : ctx->ex) TRY(alloc_field(ctx, e, PREC_F64));
    const int n = (int)ctx->g.Vh;
    const int lxblocks = div_up(ctx->g.V, LXCOPY_THREADS);
    auto V = [&](const Field& x) { return view<PREC_F64>(x); };
    // split_lx_vector_into_eo_parts(source)
    ++ctx->launches;
    lx_split_kernel<PREC_F64><<<lxblocks, LXCOPY_THREADS, 0, ctx->stream>>>(ctx->g, src, V(eta[0]), V(eta[1]));
    CU(cudaGetLastError());
    if (src_read) CU(cudaEventRecord(src_read, ctx->stream));
    const tms_status st = eo_full_solve(ctx, niter, residue, precision, stats, guess_Koo);
    if (st != TMS_OK && st != TMS_ERR_NOT_CONVERGED) return st;
    // paste_eo_parts_into_lx_vector
    ++ctx->launches;
    lx_paste_kernel<PREC_F64><<<lxblocks, LXCOPY_THREADS, 0, ctx->stream>>>(ctx->g, V(psi[0]), V(psi[1]), dst);
    CU(cudaGetLastError());
    if (dst_ready) CU(cudaEventRecord(dst_ready, ctx->stream));
    // lx residual check (cg_invert_tmD_eoprec.cpp:192-212): |g5 Q sol - src|^2 / |src|^2
    if (stats)
      {
        EpiTmQ<PREC_F64, false> e{{V(f[2]), V(f[3])}, {V(psi[0]), V(psi[1])}, ctx->prm, +1.0};
        launch_hop<PREC_F64, LINK_F64_18>(ctx, ctx->stream, 0, 2, psi[0], psi[1], links64(ctx), ctx->prm, e);
        double num = 0, den = 0;
        for (int par = 0; par < 2; par++)
          {
            ++ctx->launches;
            g5_residual_kernel<<<div_up(n, BLAS_THREADS), BLAS_THREADS, 0, ctx->stream>>>(n, V(f[2 + par]),
                                                                                         V(eta[par]), reducer(ctx));
            CU(cudaGetLastError());
            num += read_result(ctx);
            double e2;
            TRY(norm2<PREC_F64>(ctx, eta[par], &e2));
            den += e2;
          }
        stats->lx_rel_res2 = num / den;
      }
    return st;
  }

  // the copy stream, the staging buffers and the events of pipelined column solves
  tms_status ensure_columns(tms_ctx* ctx, size_t bytes)
  {
    if (!ctx->cstream) CU(cudaStreamCreateWithFlags(&ctx->cstream, cudaStreamNonBlocking));
    for (cudaEvent_t& e : ctx->colev)
      if (!e) CU(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    if (ctx->colbuf_bytes >= bytes) return TMS_OK;
    for (double*& b : ctx->colbuf)
      {
        if (b) cudaFree(b);
        b = nullptr;
      }
    ctx->colbuf_bytes = 0;
    for (double*& b : ctx->colbuf) CU(cudaMalloc(&b, bytes));
    ctx->colbuf_bytes = bytes;
    return TMS_OK;
  }

  // Column k's source is copied in while column k-1 is solved, and its solution
  // copied out while column k+1 is solved: two staging buffers each way on a
  // copy stream, ordered against the solver's stream by events.
  tms_status columns_host(tms_ctx* ctx, int ncols, double* const* sols, const double* const* srcs, int niter,
                          double residue, int precision, tms_stats* stats, size_t bytes)
  {
    cudaEvent_t* in_ready = ctx->colev;
    cudaEvent_t* in_free = ctx->colev + 2;
    cudaEvent_t* out_ready = ctx->colev + 4;
    cudaEvent_t* out_free = ctx->colev + 6;
    double** in = ctx->colbuf;
    double** out = ctx->colbuf + 2;
    cudaStream_t cs = ctx->cstream;
    CU(cudaMemcpyAsync(in[0], srcs[0], bytes, cudaMemcpyHostToDevice, cs));
    CU(cudaEventRecord(in_ready[0], cs));
    tms_status worst = TMS_OK;
    for (int k = 0; k < ncols; k++)
      {
        const int b = k & 1;
        if (k + 1 < ncols)
          {
            const int nb = (k + 1) & 1;
            if (k >= 1) CU(cudaStreamWaitEvent(cs, in_free[nb], 0)); // column k-1 has read it
            CU(cudaMemcpyAsync(in[nb], srcs[k + 1], bytes, cudaMemcpyHostToDevice, cs));
            CU(cudaEventRecord(in_ready[nb], cs));
          }
        CU(cudaStreamWaitEvent(ctx->stream, in_ready[b], 0));
        if (k >= 2) CU(cudaStreamWaitEvent(ctx->stream, out_free[b], 0)); // column k-2 has been copied out
        const tms_status st = cg_eoprec_lx(ctx, out[b], in[b], niter, residue, precision, stats ? stats + k : nullptr,
                                           in_free[b], out_ready[b]);
        if (st != TMS_OK && st != TMS_ERR_NOT_CONVERGED) return st;
        if (st != TMS_OK) worst = st;
        CU(cudaStreamWaitEvent(cs, out_ready[b], 0));
        CU(cudaMemcpyAsync(sols[k], out[b], bytes, cudaMemcpyDeviceToHost, cs));
        CU(cudaEventRecord(out_free[b], cs));
      }
    return worst;
  }
}

namespace
{
  // the reference's chiral gamma5 on lx AoS spinors (spins 2, 3 negated), in place
  __global__ void aos_g5_kernel(int64_t nsites, double* __restrict__ a)
  {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nsites * 12) return;
    const int64_t site = i / 12, k = i % 12;
    a[site * 24 + 12 + k] = -a[site * 24 + 12 + k];
  }

  // y += x over n doubles
  __global__ void aos_axpy_kernel(int64_t n, const double* __restrict__ x, double* __restrict__ y)
  {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] += x[i];
  }

  struct DevArrays
  {
    std::vector<double*> p;
    ~DevArrays()
    {
      for (double* q : p)
        if (q) cudaFree(q);
    }
  };

  // Mixed multi-shift: every shift's FP32 multi-shift solution brought to its
  // target by defect correction through the e/o solver, all shifts at once:
  // (Q_W^2 + m^2)^-1 = Q(-m)^-1 Q(+m)^-1 and Q(mu)^-1 = D(mu)^-1 g5, so one
  // round is e_k = D(-m_k)^-1 g5 D(+m_k)^-1 g5 r_k for all unconverged shifts
  // as two batched e/o solves (one right-hand side per shift, per-shift mu),
  // then x_k += e_k and the FP64 true residual r_k = b - (Q_W^2 + m_k^2) x_k.
  // Each e/o solve goes to a tenth of the shift's remaining squared factor.
  tms_status cgm_refine_batched(tms_ctx* ctx, double kappa, int has_anis, double anis, const double* masses, int nmass,
                                int niter, const double* residues, int precision, double b2, tms_status st0,
                                int iters, float ms, double* const* sols, tms_stats* stats)
  {
    Field* f = ctx->lx64;
    const int64_t V = ctx->g.V;
    const size_t bytes = (size_t)V * 24 * sizeof(double);
    DevArrays X, Rg, Y, E;
    for (DevArrays* a : {&X, &Rg, &Y, &E})
      {
        a->p.assign(nmass, nullptr);
        for (int k = 0; k < nmass; k++) CU(cudaMalloc(&a->p[k], bytes));
      }
    const int saved_mode = ctx->ptr_mode;
    struct ModeGuard
    {
      tms_ctx* c;
      int m;
      ~ModeGuard() { c->ptr_mode = m; }
    } guard{ctx, saved_mode};
    ctx->ptr_mode = TMS_PTR_DEVICE;
    const int blk = 256;
    const unsigned g5grid = (unsigned)div_up(V * 12, (int64_t)blk), axgrid = (unsigned)div_up(V * 24, (int64_t)blk);
    std::vector<double> rt(nmass);
    std::vector<tms_stats> sk(nmass);
    // the multi-shift solutions, their true residues and g5 r
    for (int k = 0; k < nmass; k++)
      {
        cgm_solution<PREC_F32>(ctx, k, f[1]);
        TRY(set_params(ctx, kappa, masses[k], has_anis, anis));
        TRY(LxOp::true_residual(ctx, f[0], f[1], f[2], &rt[k]));
        fill_stats(&sk[k], st0, iters, 0, ctx->cgm_h->res[k], rt[k] / b2, ms);
        TRY(lx_out(ctx, f[1], X.p[k]));
        TRY(lx_out(ctx, f[2], Rg.p[k]));
        ++ctx->launches;
        aos_g5_kernel<<<g5grid, blk, 0, ctx->stream>>>(V, Rg.p[k]);
      }
    CU(cudaGetLastError());
    tms_status worst = TMS_OK;
    for (int round = 0; round < 4; round++)
      {
        std::vector<int> act;
        for (int k = 0; k < nmass; k++)
          if (rt[k] >= residues[k] * b2) act.push_back(k);
        if (act.empty()) break;
        const int na = (int)act.size();
        std::vector<double*> src(na), sol(na);
        std::vector<double> mu(na), rel(na);
        std::vector<tms_stats> es(na);
        for (int a = 0; a < na; a++)
          {
            const int k = act[a];
            rel[a] = std::min(1e-2, std::max(1e-22, 1e-1 * residues[k] * b2 / rt[k]));
          }
        for (int pass = 0; pass < 2; pass++)
          {
            for (int a = 0; a < na; a++)
              {
                const int k = act[a];
                src[a] = pass ? Y.p[k] : Rg.p[k];
                sol[a] = pass ? E.p[k] : Y.p[k];
                mu[a] = pass ? -masses[k] : masses[k];
              }
            const tms_status s = tms_cg_eoprec_batched(ctx, na, sol.data(), src.data(), kappa, has_anis, anis,
                                                       mu.data(), niter, rel.data(), precision, es.data());
            if (s != TMS_OK && s != TMS_ERR_NOT_CONVERGED) return s;
            if (s != TMS_OK) worst = s;
            for (int a = 0; a < na; a++)
              {
                sk[act[a]].iterations += es[a].iterations;
                sk[act[a]].seconds += es[a].seconds;
                ++ctx->launches;
                if (pass == 0) aos_g5_kernel<<<g5grid, blk, 0, ctx->stream>>>(V, Y.p[act[a]]);
                else aos_axpy_kernel<<<axgrid, blk, 0, ctx->stream>>>(V * 24, E.p[act[a]], X.p[act[a]]);
              }
            CU(cudaGetLastError());
          }
        for (int a = 0; a < na; a++)
          {
            const int k = act[a];
            TRY(lx_in(ctx, X.p[k], f[1]));
            TRY(set_params(ctx, kappa, masses[k], has_anis, anis));
            TRY(LxOp::true_residual(ctx, f[0], f[1], f[2], &rt[k]));
            TRY(lx_out(ctx, f[2], Rg.p[k]));
            ++ctx->launches;
            aos_g5_kernel<<<g5grid, blk, 0, ctx->stream>>>(V, Rg.p[k]);
            sk[k].reliable_updates++;
          }
        CU(cudaGetLastError());
      }
    ctx->ptr_mode = saved_mode;
    for (int k = 0; k < nmass; k++)
      {
        const tms_status sk_st = (rt[k] >= residues[k] * b2) ? TMS_ERR_NOT_CONVERGED : (worst == TMS_ERR_NOT_CONVERGED ? TMS_OK : worst);
        sk[k].true_rel_res2 = rt[k] / b2;
        sk[k].iterated_rel_res2 = rt[k] / b2;
        sk[k].status = sk_st;
        if (sk_st != TMS_OK) worst = TMS_ERR_NOT_CONVERGED;
        if (stats) stats[k] = sk[k];
        if (saved_mode == TMS_PTR_HOST)
          {
            CU(cudaMemcpyAsync(sols[k], X.p[k], bytes, cudaMemcpyDeviceToHost, ctx->stream));
            CU(cudaStreamSynchronize(ctx->stream));
          }
        else
          CU(cudaMemcpyAsync(sols[k], X.p[k], bytes, cudaMemcpyDeviceToDevice, ctx->stream));
      }
    CU(cudaStreamSynchronize(ctx->stream));
    return worst;
  }
}

extern "C" {

tms_status tms_cg_eoprec(tms_ctx* ctx, double* sol_lx, const double* src_lx, double kappa, int has_anis, double anis,
                         double mu, int niter, double residue, int precision, tms_stats* stats)
{
  return tms_cg_eoprec_guess(ctx, sol_lx, nullptr, src_lx, kappa, has_anis, anis, mu, niter, residue, precision,
                             stats);
}

tms_status tms_cg_eoprec_guess(tms_ctx* ctx, double* sol_lx, const double* guess_Koo, const double* src_lx,
                               double kappa, int has_anis, double anis, double mu, int niter, double residue,
                               int precision, tms_stats* stats)
{
  TRY(check_conf(ctx));
  if (!sol_lx || !src_lx || niter <= 0 || !(residue > 0)) return fail(ctx, TMS_ERR_BAD_ARG, "bad solver arguments");
  TRY(set_params(ctx, kappa, mu, has_anis, anis));
  const size_t bytes = (size_t)ctx->g.V * 24 * sizeof(double);
  const double* src = src_lx;
  double* dst = sol_lx;
  if (ctx->ptr_mode == TMS_PTR_HOST)
    {
      TRY(ensure_stage(ctx, bytes));
      CU(cudaMemcpyAsync(ctx->stage, src_lx, bytes, cudaMemcpyHostToDevice, ctx->stream));
      src = dst = ctx->stage; // the source is split before the solution is pasted
    }
  const tms_status st = cg_eoprec_lx(ctx, dst, src, niter, residue, precision, stats, nullptr, nullptr, guess_Koo);
  if (st != TMS_OK && st != TMS_ERR_NOT_CONVERGED) return st;
  if (ctx->ptr_mode == TMS_PTR_HOST) CU(cudaMemcpyAsync(sol_lx, ctx->stage, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  TRY(finish(ctx));
  return st;
}

tms_status tms_cg_eoprec_columns(tms_ctx* ctx, int ncols, double* const* sols_lx, const double* const* srcs_lx,
                                 double kappa, int has_anis, double anis, double mu, int niter, double residue,
                                 int precision, tms_stats* stats)
{
  TRY(check_conf(ctx));
  if (ncols <= 0 || !sols_lx || !srcs_lx || niter <= 0 || !(residue > 0))
    return fail(ctx, TMS_ERR_BAD_ARG, "bad solver arguments");
  for (int k = 0; k < ncols; k++)
    if (!sols_lx[k] || !srcs_lx[k]) return fail(ctx, TMS_ERR_BAD_ARG, "column %d: null pointer", k);
  TRY(set_params(ctx, kappa, mu, has_anis, anis));
  tms_status st = TMS_OK;
  if (ctx->ptr_mode == TMS_PTR_DEVICE)
    {
      for (int k = 0; k < ncols; k++)
        {
          const tms_status s = cg_eoprec_lx(ctx, sols_lx[k], srcs_lx[k], niter, residue, precision,
                                            stats ? stats + k : nullptr, nullptr, nullptr);
          if (s != TMS_OK && s != TMS_ERR_NOT_CONVERGED) return s;
          if (s != TMS_OK) st = s;
        }
      TRY(finish(ctx));
      return st;
    }
  const size_t bytes = (size_t)ctx->g.V * 24 * sizeof(double);
  TRY(ensure_columns(ctx, bytes));
  st = columns_host(ctx, ncols, sols_lx, srcs_lx, niter, residue, precision, stats, bytes);
  // no copy into or out of the caller's buffers outlives the call, whatever the outcome
  const cudaError_t e = cudaStreamSynchronize(ctx->cstream);
  if (st != TMS_OK && st != TMS_ERR_NOT_CONVERGED) return st;
  if (e != cudaSuccess) return fail(ctx, TMS_ERR_CUDA, "column copies: %s", cudaGetErrorString(e));
  TRY(finish(ctx));
  return st;
}


// ------------------------------------------------------------ twisted clover
tms_status tms_cg_tmclov_eoprec_square(tms_ctx* ctx, double* sol, const double* guess, const double* src, double kappa,
                                       int has_anis, double anis, double mu, int niter, double residue, int precision,
                                       tms_stats* stats)
{
  TRY(check_clover(ctx));
  if (!sol || !src || niter <= 0 || !(residue > 0)) return fail(ctx, TMS_ERR_BAD_ARG, "bad solver arguments");
  TRY(set_params(ctx, kappa, mu, has_anis, anis));
  TRY(ensure_clover_inverse(ctx, kappa, mu));
  Field* f = ctx->f64;
  TRY(spinor_in(ctx, src, nullptr, ctx->g.Vh, f[0]));
  if (guess) TRY(spinor_in(ctx, guess, nullptr, ctx->g.Vh, f[1]));
  const tms_status st = cg_dispatch<ClovOp>(ctx, precision, niter, residue, guess != nullptr, stats);
  if (st == TMS_OK || st == TMS_ERR_NOT_CONVERGED) TRY(spinor_out(ctx, f[1], nullptr, ctx->g.Vh, sol, true));
  TRY(finish(ctx));
  return st;
}

tms_status tms_cg_tmclov_eoprec(tms_ctx* ctx, double* sol_lx, const double* src_lx, double kappa, int has_anis,
                                double anis, double cSW, double mu, int niter, double residue, int precision,
                                tms_stats* stats)
{
  TRY(check_conf(ctx));
  if (!sol_lx || !src_lx || niter <= 0 || !(residue > 0)) return fail(ctx, TMS_ERR_BAD_ARG, "bad solver arguments");
  // clover_term(Cl, cSW, conf) and invert_twisted_clover_term(invCl, mu, kappa, Cl) of the call
  // (cg_invert_tmclovD_eoprec.cpp:72-76), kept across calls with the same conf and parameters
  if (!ctx->clov_ok || ctx->clov_csw != cSW) TRY(tms_clover_term(ctx, cSW));
  TRY(set_params(ctx, kappa, mu, has_anis, anis));
  TRY(ensure_clover_inverse(ctx, kappa, mu));
  Field* f = ctx->f64;
  for (int i = 0; i <= 7; i++) TRY(alloc_field(ctx, f[i], PREC_F64));
  Field *eta = ctx->ex, *psi = ctx->ex + 2; // [0] even, [1] odd
  for (auto& e : ctx->ex) TRY(alloc_field(ctx, e, PREC_F64));
  const int64_t Vh = ctx->g.Vh;
  const int n = (int)Vh;
  const size_t bytes = (size_t)ctx->g.V * 24 * sizeof(double);
  auto V = [&](const Field& x) { return view<PREC_F64>(x); };
  auto U = links64(ctx);
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
  // Eq. (8a): te = T_ee^-1 eta_e ; Eq. (8b): varphi = g5 (eta_o + hop(te)/2) -> f0  (:84-90)
  inv_clov_apply(ctx, eta[0], f[5], 0);
  EpiSrcPrep<PREC_F64> sp{{V(f[0]), V(f[0])}, {V(eta[1]), V(eta[1])}};
  launch_hop<PREC_F64, LINK_F64_18>(ctx, ctx->stream, 1, 1, f[5], f[5], U, ctx->prm, sp);
  CU(cudaGetLastError());
  // Eq. (9)
  const tms_status st = cg_dispatch<ClovOp>(ctx, precision, niter, residue, false, stats);
  if (st != TMS_OK && st != TMS_ERR_NOT_CONVERGED) return st;
  // Eq. (10): psi_o = K(dag) x ; Eq. (11): psi_e = T_ee^-1 (eta_e + hop(psi_o)/2)  (:97-107)
  clov_kern_op<PREC_F64>(ctx, U, clov64(ctx), f[1], f[5], psi[1], 1, ctx->prm);
  EpiClovReco<PREC_F64> rc{{V(psi[0]), V(psi[0])}, {V(eta[0]), V(eta[0])}, clov64(ctx)};
  launch_hop<PREC_F64, LINK_F64_18>(ctx, ctx->stream, 0, 1, psi[1], psi[1], U, ctx->prm, rc);
  CU(cudaGetLastError());
  double* d = (ctx->ptr_mode == TMS_PTR_HOST) ? ctx->stage : sol_lx;
  ++ctx->launches;
  soa_to_aos_kernel<PREC_F64><<<div_up(n, 256), 256, 0, ctx->stream>>>(n, V(psi[0]), ctx->lx_of_eo, d);
  ++ctx->launches;
  soa_to_aos_kernel<PREC_F64><<<div_up(n, 256), 256, 0, ctx->stream>>>(n, V(psi[1]), ctx->lx_of_eo + Vh, d);
  CU(cudaGetLastError());
  if (ctx->ptr_mode == TMS_PTR_HOST) CU(cudaMemcpyAsync(sol_lx, ctx->stage, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  // the residual check of inv_tmclovD_cg_eoprec (:140-175): |g5 Q_clov sol - src|^2 / |src|^2
  if (stats)
    {
      tmclovQ_op(ctx, psi[0], psi[1], f[2], f[3], ctx->prm);
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

tms_status tms_cg_tmQ2(tms_ctx* ctx, double* sol_lx, const double* guess_lx, const double* src_lx, double kappa,
                       int has_anis, double anis, double m, int niter, double residue, int precision,
                       tms_stats* stats)
{
  TRY(check_conf(ctx));
  if (!sol_lx || !src_lx || niter <= 0 || !(residue > 0)) return fail(ctx, TMS_ERR_BAD_ARG, "bad solver arguments");
  TRY(set_params(ctx, kappa, m, has_anis, anis));
  Field* f = ctx->lx64;
  TRY(lx_in(ctx, src_lx, f[0]));
  if (guess_lx) TRY(lx_in(ctx, guess_lx, f[1]));
  const tms_status st = cg_dispatch<LxOp>(ctx, precision, niter, residue, guess_lx != nullptr, stats);
  if (st == TMS_OK || st == TMS_ERR_NOT_CONVERGED) TRY(lx_out(ctx, f[1], sol_lx));
  TRY(finish(ctx));
  return st;
}

tms_status tms_cgm_tmQ2(tms_ctx* ctx, double* const* sols, const double* src_lx, double kappa, int has_anis,
                        double anis, const double* masses, int nmass, int niter, const double* residues,
                        int precision, tms_stats* stats)
{
  TRY(check_conf(ctx));
  if (!sols || !src_lx || !masses || !residues || nmass <= 0 || nmass > CGM_MAX_SHIFTS || niter <= 0)
    return fail(ctx, TMS_ERR_BAD_ARG, "bad multi-shift arguments (1 <= nmass <= %d)", CGM_MAX_SHIFTS);
  if (precision != TMS_PREC_DOUBLE && precision != TMS_PREC_MIXED_SINGLE && precision != TMS_PREC_MIXED_HALF)
    return fail(ctx, TMS_ERR_BAD_ARG, "unknown precision %d", precision);
  for (int k = 0; k < nmass; k++)
    if (!sols[k] || !(residues[k] > 0) || !std::isfinite(masses[k]))
      return fail(ctx, TMS_ERR_BAD_ARG, "bad shift %d", k);
  TRY(set_params(ctx, kappa, 0.0, has_anis, anis, 1)); // the CGM operator Q(0)^2
  Field* f = ctx->lx64;
  const int stride = 2 * ctx->g.stride;
  for (int i = 1; i <= 6; i++) TRY(alloc_field(ctx, f[i], PREC_F64, stride));
  TRY(lx_in(ctx, src_lx, f[0]));
  double b2;
  TRY(norm2<PREC_F64>(ctx, f[0], &b2, stride));
  if (b2 == 0.0 || std::isnan(b2)) return fail(ctx, TMS_ERR_INVALID_SOURCE, "invalid norm: %g", b2);
  double sigma[CGM_MAX_SHIFTS], target[CGM_MAX_SHIFTS];
  // the FP32 multi-shift solve stops at the squared relative residue
  // cgm_floor_single at most; each shift is then brought to its target by the
  // mixed-precision CG from that guess
  const double floor32 = ctx->cgm_floor32;
  for (int k = 0; k < nmass; k++)
    {
      sigma[k] = masses[k] * masses[k];
      target[k] = (precision == TMS_PREC_DOUBLE) ? residues[k] : std::max(residues[k], floor32);
    }
  int iters = 0;
  float ms = 0;
  tms_status st;
  if (precision == TMS_PREC_DOUBLE)
    st = cgm_run<PREC_F64>(ctx, links64(ctx), nmass, sigma, target, niter, b2, &iters, &ms);
  else
    st = ctx->su3 ? cgm_run<PREC_F32>(ctx, links32r(ctx), nmass, sigma, target, niter, b2, &iters, &ms)
                  : cgm_run<PREC_F32>(ctx, links32f(ctx), nmass, sigma, target, niter, b2, &iters, &ms);
  if (st != TMS_OK && st != TMS_ERR_NOT_CONVERGED) return st;
  if (precision != TMS_PREC_DOUBLE && ctx->cgm_refine_batched)
    {
      // all shifts' corrections as batched e/o solves (tuning "cgm_refine_batched")
      tms_status worst = st;
      const tms_status s2 = cgm_refine_batched(ctx, kappa, has_anis, anis, masses, nmass, niter, residues, precision,
                                               b2, st, iters, ms, sols, stats);
      if (s2 != TMS_OK && s2 != TMS_ERR_NOT_CONVERGED) return s2;
      if (s2 != TMS_OK) worst = s2;
      TRY(finish(ctx));
      if (worst != TMS_OK) return fail(ctx, worst, "exit without converging");
      return TMS_OK;
    }
  tms_status worst = st;
  for (int k = 0; k < nmass; k++)
    {
      if (precision == TMS_PREC_DOUBLE) cgm_solution<PREC_F64>(ctx, k, f[1]);
      else cgm_solution<PREC_F32>(ctx, k, f[1]);
      // final true residue of the shift (cgm_invert_template_threaded.hpp:266-279)
      TRY(set_params(ctx, kappa, masses[k], has_anis, anis));
      double rt;
      TRY(LxOp::true_residual(ctx, f[0], f[1], f[2], &rt));
      tms_stats sk{};
      fill_stats(&sk, st, iters, 0, ctx->cgm_h->res[k], rt / b2, ms);
      if (precision != TMS_PREC_DOUBLE && rt >= residues[k] * b2)
        {
          // defect correction through the e/o solver, FP64 residuals in between:
          // (Q_W^2 + m^2)^-1 = Q(-m)^-1 Q(+m)^-1 and Q(mu)^-1 = D(mu)^-1 g5, so
          // e = D(-m)^-1 g5 D(+m)^-1 g5 r ; x += e ; r = b - (Q_W^2 + m^2) x
          Field* ex = ctx->ex;
          for (auto& e : ctx->ex) TRY(alloc_field(ctx, e, PREC_F64));
          const int n = (int)ctx->g.Vh;
          tms_status s2 = TMS_OK;
          int corrections = 0;
          while (rt >= residues[k] * b2 && corrections < 4)
            {
              // each e/o solve to a tenth of the remaining factor (squared residues):
              // one correction per shift at 32^3x64 with the true residual a third
              // of its target (a hundredth took 4 % longer; 0.3 needed a second one)
              const double rel = std::min(1e-2, std::max(1e-22, 1e-1 * residues[k] * b2 / rt));
              for (int p = 0; p < 2; p++)
                {
                  ++ctx->launches;
                  g5_copy_kernel<<<div_up(n, BLAS_THREADS), BLAS_THREADS, 0, ctx->stream>>>(
                    n, view_par<PREC_F64>(f[2], p), view<PREC_F64>(ex[p]));
                }
              for (int pass = 0; pass < 2; pass++)
                {
                  const double sg = pass ? -1.0 : +1.0;
                  TRY(set_params(ctx, kappa, sg * masses[k], has_anis, anis));
                  tms_stats es{};
                  s2 = eo_full_solve(ctx, niter, rel, precision, &es);
                  if (s2 != TMS_OK && s2 != TMS_ERR_NOT_CONVERGED) return s2;
                  sk.iterations += es.iterations;
                  sk.seconds += es.seconds;
                  for (int p = 0; p < 2; p++)
                    {
                      ++ctx->launches;
                      if (sg > 0)
                        g5_copy_kernel<<<div_up(n, BLAS_THREADS), BLAS_THREADS, 0, ctx->stream>>>(
                          n, view<PREC_F64>(ex[2 + p]), view<PREC_F64>(ex[p]));
                      else
                        axpby_kernel<PREC_F64, PREC_F64, PREC_F64><<<div_up(n, BLAS_THREADS), BLAS_THREADS, 0,
                                                                     ctx->stream>>>(
                          n, 1.0, view_par<PREC_F64>(f[1], p), 1.0, view<PREC_F64>(ex[2 + p]),
                          view_par<PREC_F64>(f[1], p));
                    }
                }
              CU(cudaGetLastError());
              TRY(set_params(ctx, kappa, masses[k], has_anis, anis));
              TRY(LxOp::true_residual(ctx, f[0], f[1], f[2], &rt));
              corrections++;
            }
          if (s2 == TMS_OK && rt >= residues[k] * b2) s2 = TMS_ERR_NOT_CONVERGED;
          if (s2 != TMS_OK) worst = s2;
          sk.reliable_updates = corrections;
          sk.true_rel_res2 = rt / b2;
          sk.iterated_rel_res2 = rt / b2;
          sk.status = s2;
        }
      if (stats) stats[k] = sk;
      TRY(lx_out(ctx, f[1], sols[k]));
    }
  TRY(finish(ctx));
  if (worst != TMS_OK) return fail(ctx, worst, "exit without converging");
  return TMS_OK;
}

} // extern "C"
