// Multi-RHS kernels: k right-hand sides, each with its own twisted mass and
// its own CG scalars, share one pass over the gauge links.
//
// A warp takes 32 consecutive sites and, one group after the other, the
// right-hand sides in groups of R (R per thread, in registers), so each link
// is loaded once per group and applied to R spinors; each right-hand side's
// spinors are read as contiguous 128-bit segments.
//
// Reductions are per right-hand side: a block accumulates each right-hand
// side's warp sums in shared memory, writes one partial per block, and the
// warp that takes the last ticket of that right-hand side sums the row in a
// fixed order and finalises its scalars (no warp ever waits).
#pragma once

#include "tms_kernels.cuh"
#include "tms_hop_sp.cuh"

namespace tms
{
  constexpr int MRHS_MAX = 64;

  // k fields of one precision laid out one after the other
  template <int P>
  struct SpinorBatch
  {
    SpinorT<P> f;       // right-hand side 0
    size_t rhs_elems;   // element offset between right-hand sides (d)
    size_t rhs_norms;   // float offset between right-hand sides (n, FP16 only)
    __device__ __forceinline__ SpinorT<P> rhs(int r) const
    {
      SpinorT<P> s = f;
      s.d += (size_t)r * rhs_elems;
      if (s.n) s.n += (size_t)r * rhs_norms;
      return s;
    }
  };

  // per right-hand side hopping parameter and twisted mass (the hop itself
  // does not depend on them: only the diagonal terms do)
  struct BatchParams
  {
    double anis;
    double kappa[MRHS_MAX];
    double mu[MRHS_MAX];
  };

  struct BatchReducer
  {
    double* partial;    // [rhs][gridDim.x]
    unsigned* counter;  // [rhs]
    double* result;     // [rhs]
  };

  // finish the reduction of right-hand side `rhs`: lane 0 holds this block's
  // partial; the warp holding the last ticket of that right-hand side sums the
  // row in a fixed order and calls fin(rhs, total)
  template <class Fin>
  __device__ __forceinline__ void warp_rhs_finish(double v, int rhs, const BatchReducer& red, const Fin& fin)
  {
    const int lane = threadIdx.x & 31;
    unsigned last = 0;
    if (lane == 0)
      {
        red.partial[(size_t)rhs * gridDim.x + blockIdx.x] = v;
        __threadfence();
        last = (atomicAdd(red.counter + rhs, 1u) == gridDim.x - 1);
      }
    last = __shfl_sync(0xffffffffu, last, 0);
    if (!last) return;
    __threadfence();
    double s = 0.0;
    const double* row = red.partial + (size_t)rhs * gridDim.x;
#pragma unroll 8
    for (int i = lane; i < (int)gridDim.x; i += 32) s += __ldcg(row + i); // past L1, several in flight
    s = warp_sum(s);
    if (lane == 0)
      {
        red.result[rhs] = s;
        red.counter[rhs] = 0u;
        fin(rhs, s);
      }
  }

  struct NoFinB
  {
    __device__ void operator()(int, double) const {}
  };

  // per right-hand side: alpha = rr / |K(-mu) p|^2
  struct FinAlphaB
  {
    CgState* st;
    __device__ void operator()(int r, double pAp) const { FinAlpha{st + r}(pAp); }
  };
  struct FinBetaB
  {
    CgState* st;
    __device__ void operator()(int r, double rr) const { FinBeta{st + r}(rr); }
  };

  // ------------------------------------------------------------ epilogues
  template <int P>
  struct EpiBInvDiag
  {
    static constexpr bool kReduce = false;
    SpinorBatch<P> out;
    double sgn;
    __device__ __forceinline__ double operator()(int r, int ieo, const BatchParams& bp,
                                                 C<typename SpinorT<P>::R> acc[12]) const
    {
      using R = typename SpinorT<P>::R;
      const OpParams o{bp.kappa[r], bp.mu[r], bp.anis};
      const C<R> z = zinvdiag<R>(o, sgn);
#pragma unroll
      for (int c = 0; c < 12; c++) acc[c] = diag_apply(acc[c], z, c);
      out.rhs(r).store(ieo, acc);
      return 0.0;
    }
  };

  template <int P, bool RED>
  struct EpiBKern
  {
    static constexpr bool kReduce = RED;
    SpinorBatch<P> out, x;
    double sgn;
    __device__ __forceinline__ double operator()(int r, int ieo, const BatchParams& bp,
                                                 C<typename SpinorT<P>::R> acc[12]) const
    {
      using R = typename SpinorT<P>::R;
      const OpParams o{bp.kappa[r], bp.mu[r], bp.anis};
      const C<R> z = zdiag<R>(o, sgn);
      C<R> xv[12];
      x.rhs(r).load(ieo, xv);
      double n2 = 0.0;
#pragma unroll
      for (int c = 0; c < 12; c++)
        {
          const C<R> d = diag_apply(xv[c], z, c);
          const C<R> q = cscale(acc[c], R(0.25));
          acc[c] = (c < 6) ? csub(d, q) : csub(q, d);
          if (RED) n2 += (double)acc[c].re * acc[c].re + (double)acc[c].im * acc[c].im;
        }
      out.rhs(r).store(ieo, acc);
      return n2;
    }
  };

  // s = K(+mu) t1 ; x += alpha p ; r -= alpha s ; reduce |r|^2 (per right-hand side)
  template <int P, int PX, int XM = 1>
  struct EpiBKernCgUpdate
  {
    static constexpr bool kReduce = true;
    SpinorBatch<P> t1, r, p;
    SpinorBatch<PX> x;
    const CgState* st;
    double sgn;
    SpinorBatch<P> pp; // XM == 2: the previous direction
    __device__ __forceinline__ double operator()(int k, int ieo, const BatchParams& bp,
                                                 C<typename SpinorT<P>::R> acc[12]) const
    {
      using R = typename SpinorT<P>::R;
      using RX = typename SpinorT<PX>::R;
      const OpParams o{bp.kappa[k], bp.mu[k], bp.anis};
      const C<R> z = zdiag<R>(o, sgn);
      const double a = st[k].alpha;
      const R alpha = R(a);
      C<R> v[12];
      t1.rhs(k).load(ieo, v);
#pragma unroll
      for (int c = 0; c < 12; c++)
        {
          const C<R> d = diag_apply(v[c], z, c);
          const C<R> q = cscale(acc[c], R(0.25));
          acc[c] = (c < 6) ? csub(d, q) : csub(q, d);
        }
      const SpinorT<P> rk = r.rhs(k);
      rk.load(ieo, v);
      double n2 = 0.0;
#pragma unroll
      for (int c = 0; c < 12; c++)
        {
          v[c] = csub(v[c], cscale(acc[c], alpha));
          n2 += (double)v[c].re * v[c].re + (double)v[c].im * v[c].im;
        }
      rk.store(ieo, v);
      if (XM == 0) return n2;
      const SpinorT<PX> xk = x.rhs(k);
      C<RX> xv[12];
      xk.load(ieo, xv);
      if (XM == 2)
        {
          pp.rhs(k).load(ieo, v);
          const RX ap = RX(st[k].alpha_prev);
#pragma unroll
          for (int c = 0; c < 12; c++)
            {
              xv[c].re += ap * RX(v[c].re);
              xv[c].im += ap * RX(v[c].im);
            }
        }
      p.rhs(k).load(ieo, v);
#pragma unroll
      for (int c = 0; c < 12; c++)
        {
          xv[c].re += RX(a) * RX(v[c].re);
          xv[c].im += RX(a) * RX(v[c].im);
        }
      xk.store(ieo, xv);
      return n2;
    }
  };

  // ---------------------------------------------------------- hop kernel
  // One parity (par_out) for nrhs right-hand sides, register-blocked: a
  // thread computes one site for R right-hand sides at once, so each link is
  // loaded (and rebuilt) once into registers and applied to the R neighbour
  // spinors (in FP32 arithmetic with the spin rows in packed lanes).  A warp takes 32 consecutive sites and the groups of R
  // right-hand sides one after the other (the links of its sites stay in L1
  // across groups).
  // A right-hand side whose state says stop is skipped.  Per right-hand side
  // sums are reduced with warp shuffles, kept per warp in shared memory and
  // combined in a fixed order: deterministic.
  constexpr int MRHS_WARPS = 4;

  template <int MU, bool FWD, int P, int LF, int R>
  __device__ __forceinline__ void hop_dir_multi(const Lattice& g, const Site& s, int p, int ieo,
                                                const SpinorBatch<P>& in, int rhs0, unsigned on, const LinkT<LF>& U,
                                                typename SpinorT<P>::R anis, C<typename SpinorT<P>::R> acc[R][12])
  {
    using Re = typename SpinorT<P>::R;
    const Re fmu = (MU > 0) ? anis : Re(1);
    bool w;
    const int n = FWD ? nbr_up<MU>(g, s, w) : nbr_dw<MU>(g, s, w);
    C<Re> L[9];
    Re ls;
    U.template load_scaled<false>(FWD ? p : 1 - p, MU, FWD ? ieo : n, L, ls);
    const Re f = (w ? fmu * Re(g.bc_t) : fmu) * ls;
#pragma unroll
    for (int j = 0; j < R; j++)
      if (on & (1u << j))
        {
          C<Re> sp[12], h0[3], h1[3], u0[3], u1[3];
          Re ss;
          in.rhs(rhs0 + j).load_raw(n, sp, ss);
          project<MU, FWD>(sp, h0, h1);
          link_mul<FWD>(L, h0, u0, f * ss);
          link_mul<FWD>(L, h1, u1, f * ss);
          reconstruct<MU, FWD>(acc[j], u0, u1);
        }
  }

  // The FP16-spinor form: the link of a direction is loaded and rebuilt once,
  // then applied to the R right-hand sides with the two spin rows of each half
  // spinor in the lanes of packed FP32 instructions (sp_dir_compute); 16-bit
  // links keep row 2 in raw^2 units, scaled on the packed pairs.
  template <int MU, bool FWD, int P, int LF, int R>
  __device__ __forceinline__ void hop_dir_multi_sp(const Lattice& g, const Site& s, int p, int ieo,
                                                   const SpinorBatch<P>& in, int rhs0, unsigned on,
                                                   const LinkT<LF>& U, float anis, C<P2> A01[R][3], C<P2> A23[R][3])
  {
    constexpr bool K2 = (LF == LINK_I16_12);
    const float fmu = (MU > 0) ? anis : 1.0f;
    bool w;
    const int n = FWD ? nbr_up<MU>(g, s, w) : nbr_dw<MU>(g, s, w);
    C<float> L[9];
    float ls;
    if constexpr (K2)
      {
        U.template load_rows<false>(FWD ? p : 1 - p, MU, FWD ? ieo : n, L);
        row2_unscaled(L);
        ls = LinkT<LF>::kUnit;
      }
    else
      U.template load_scaled<false>(FWD ? p : 1 - p, MU, FWD ? ieo : n, L, ls);
    const float f = (w ? fmu * float(g.bc_t) : fmu) * ls;
#pragma unroll
    for (int j = 0; j < R; j++)
      if (on & (1u << j))
        {
          C<float> sp[12];
          float ss;
          in.rhs(rhs0 + j).load_raw(n, sp, ss);
          sp_dir_compute<MU, FWD, K2>(sp, L, f * ss, A01[j], A23[j], LinkT<LF>::kUnit);
        }
  }

  // resident blocks the register budget is capped for: more right-hand sides
  // per thread need more accumulator registers
  template <int P, int R>
  struct MrhsMinBlocks
  {
    static constexpr int value = (P == PREC_F64) ? (R == 1 ? 3 : 2) : (R == 1 ? 5 : R == 2 ? 4 : 2);
  };

  // PIPE (FP32 arithmetic, R = 1): each right-hand side's gathers streamed
  // through the thread's shared-memory slots by cp.async, DIST directions ahead
  // (spp_hop_site); the block's dynamic shared memory is SppFmt::smem<DIST>()
  template <int P>
  struct MrhsPipe
  {
    static constexpr int DIST = 2;
  };

  template <int P, int LF, class Epi, class Fin, int R, bool PIPE = false>
  __global__ void __launch_bounds__(MRHS_WARPS * 32, PIPE ? (P == PREC_F16 ? 5 : 3) : MrhsMinBlocks<P, R>::value)
    hop_mrhs_kernel(Lattice g, int par_out, int nrhs, SpinorBatch<P> in, LinkT<LF> U, const BatchParams* __restrict__ bp,
                    Epi epi, BatchReducer red, Fin fin, const CgState* __restrict__ st)
  {
    using Re = typename SpinorT<P>::R;
    extern __shared__ __align__(16) char mrhs_smem[];
    __shared__ double sh[Epi::kReduce ? MRHS_WARPS * MRHS_MAX : 1];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int ngroups = (nrhs + R - 1) / R;
    if (Epi::kReduce)
      {
        for (int i = threadIdx.x; i < MRHS_WARPS * MRHS_MAX; i += blockDim.x) sh[i] = 0.0;
        __syncthreads();
      }
    const Re anis = Re(bp->anis);
    const int nchunks = (int)((g.Vh + 31) / 32);
    const int c = blockIdx.x * MRHS_WARPS + w;
    if (c < nchunks)
      {
        const int ieo = c * 32 + lane;
        for (int gr = 0; gr < ngroups; gr++)
          {
            const int rhs0 = gr * R;
            unsigned on = 0;
#pragma unroll
            for (int j = 0; j < R; j++)
              if (rhs0 + j < nrhs && !(st && st[rhs0 + j].stop)) on |= 1u << j;
            if (!on) continue; // warp-uniform
            double part[R];
#pragma unroll
            for (int j = 0; j < R; j++) part[j] = 0.0;
            if (ieo < g.Vh)
              {
                const Site s = eo_site(g, par_out, ieo);
                if constexpr (PIPE && P != PREC_F64 && R == 1)
                  {
                    // (the epilogue's operands are read from global memory here: staging them in
                    // the free pipeline slots, as the single-RHS kernel does, made the whole batched
                    // solve 7.7 % slower, although each launch timed alone was faster)
                    C<float> acc[12];
                    spp_hop_site<P, LF, MrhsPipe<P>::DIST>(mrhs_smem, g, par_out, ieo, in.rhs(rhs0), U, float(anis),
                                                           acc);
                    part[0] = epi(rhs0, ieo, *bp, acc);
                  }
                else if constexpr (P != PREC_F16)
                  {
                    // FP64, and FP32 spinors (whose float4 words do not pair the spin rows: the
                    // packed form needs moves there and measured slower)
                    C<Re> acc[R][12];
#pragma unroll
                    for (int j = 0; j < R; j++)
#pragma unroll
                      for (int k = 0; k < 12; k++) acc[j][k] = {Re(0), Re(0)};
                    hop_dir_multi<0, true, P, LF, R>(g, s, par_out, ieo, in, rhs0, on, U, anis, acc);
                    hop_dir_multi<0, false, P, LF, R>(g, s, par_out, ieo, in, rhs0, on, U, anis, acc);
                    hop_dir_multi<1, true, P, LF, R>(g, s, par_out, ieo, in, rhs0, on, U, anis, acc);
                    hop_dir_multi<1, false, P, LF, R>(g, s, par_out, ieo, in, rhs0, on, U, anis, acc);
                    hop_dir_multi<2, true, P, LF, R>(g, s, par_out, ieo, in, rhs0, on, U, anis, acc);
                    hop_dir_multi<2, false, P, LF, R>(g, s, par_out, ieo, in, rhs0, on, U, anis, acc);
                    hop_dir_multi<3, true, P, LF, R>(g, s, par_out, ieo, in, rhs0, on, U, anis, acc);
                    hop_dir_multi<3, false, P, LF, R>(g, s, par_out, ieo, in, rhs0, on, U, anis, acc);
#pragma unroll
                    for (int j = 0; j < R; j++)
                      if (on & (1u << j)) part[j] = epi(rhs0 + j, ieo, *bp, acc[j]);
                  }
                else
                  {
                    C<P2> A01[R][3], A23[R][3];
#pragma unroll
                    for (int j = 0; j < R; j++)
#pragma unroll
                      for (int c = 0; c < 3; c++)
                        {
                          A01[j][c] = {p2(0.f, 0.f), p2(0.f, 0.f)};
                          A23[j][c] = {p2(0.f, 0.f), p2(0.f, 0.f)};
                        }
                    hop_dir_multi_sp<0, true, P, LF, R>(g, s, par_out, ieo, in, rhs0, on, U, anis, A01, A23);
                    hop_dir_multi_sp<0, false, P, LF, R>(g, s, par_out, ieo, in, rhs0, on, U, anis, A01, A23);
                    hop_dir_multi_sp<1, true, P, LF, R>(g, s, par_out, ieo, in, rhs0, on, U, anis, A01, A23);
                    hop_dir_multi_sp<1, false, P, LF, R>(g, s, par_out, ieo, in, rhs0, on, U, anis, A01, A23);
                    hop_dir_multi_sp<2, true, P, LF, R>(g, s, par_out, ieo, in, rhs0, on, U, anis, A01, A23);
                    hop_dir_multi_sp<2, false, P, LF, R>(g, s, par_out, ieo, in, rhs0, on, U, anis, A01, A23);
                    hop_dir_multi_sp<3, true, P, LF, R>(g, s, par_out, ieo, in, rhs0, on, U, anis, A01, A23);
                    hop_dir_multi_sp<3, false, P, LF, R>(g, s, par_out, ieo, in, rhs0, on, U, anis, A01, A23);
#pragma unroll
                    for (int j = 0; j < R; j++)
                      if (on & (1u << j))
                        {
                          C<float> acc[12];
#pragma unroll
                          for (int c = 0; c < 3; c++)
                            {
                              acc[c] = {A01[j][c].re.v.x, A01[j][c].im.v.x};
                              acc[3 + c] = {A01[j][c].re.v.y, A01[j][c].im.v.y};
                              acc[6 + c] = {A23[j][c].re.v.x, A23[j][c].im.v.x};
                              acc[9 + c] = {A23[j][c].re.v.y, A23[j][c].im.v.y};
                            }
                          part[j] = epi(rhs0 + j, ieo, *bp, acc);
                        }
                  }
              }
            if (Epi::kReduce)
#pragma unroll
              for (int j = 0; j < R; j++)
                if (on & (1u << j))
                  {
                    const double v = warp_sum(part[j]);
                    if (lane == 0) sh[w * MRHS_MAX + rhs0 + j] += v;
                  }
          }
      }
    if (Epi::kReduce)
      {
        __syncthreads();
        // warp w finishes right-hand sides w, w + MRHS_WARPS, ...
        for (int rhs = w; rhs < nrhs; rhs += MRHS_WARPS)
          {
            if (st && st[rhs].stop) continue;
            double v = 0.0;
            if (lane == 0)
#pragma unroll
              for (int ww = 0; ww < MRHS_WARPS; ww++) v += sh[ww * MRHS_MAX + rhs];
            warp_rhs_finish(v, rhs, red, fin);
          }
      }
  }

  // r = b - s and |r|^2 per right-hand side (FP64); grid (blocks, nrhs)
  static __global__ void __launch_bounds__(256)
    residual_mrhs_kernel(int n, int nrhs, SpinorBatch<PREC_F64> b, SpinorBatch<PREC_F64> s, SpinorBatch<PREC_F64> r,
                         BatchReducer red, const CgState* __restrict__ mask)
  {
    __shared__ double sh[8];
    const int k = blockIdx.y;
    if (k >= nrhs || (mask && mask[k].stop)) return; // whole block
    const SpinorT<PREC_F64> bk = b.rhs(k), sk = s.rhs(k), rk = r.rhs(k);
    double acc = 0.0;
    for (int i = blockIdx.x * 256 + threadIdx.x; i < n; i += gridDim.x * 256)
      {
        C<double> u[12], v[12];
        bk.load(i, u);
        sk.load(i, v);
#pragma unroll
        for (int c = 0; c < 12; c++)
          {
            u[c] = csub(u[c], v[c]);
            acc += u[c].re * u[c].re + u[c].im * u[c].im;
          }
        rk.store(i, u);
      }
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32)
      {
        double v = (threadIdx.x < 8) ? sh[threadIdx.x] : 0.0;
        v = warp_sum(v);
        warp_rhs_finish(v, k, red, NoFinB{});
      }
  }

  // out = a x + b y per right-hand side (any precisions), masked
  template <int PO, int PX, int PY>
  __global__ void __launch_bounds__(256)
    axpby_mrhs_kernel(int n, int nrhs, double a, SpinorBatch<PX> x, double b, SpinorBatch<PY> y, SpinorBatch<PO> out,
                      const CgState* __restrict__ mask)
  {
    using RO = typename SpinorT<PO>::R;
    const int k = blockIdx.y;
    if (k >= nrhs || (mask && mask[k].stop)) return;
    const SpinorT<PX> xk = x.rhs(k);
    const SpinorT<PY> yk = y.rhs(k);
    const SpinorT<PO> ok = out.rhs(k);
    for (int i = blockIdx.x * 256 + threadIdx.x; i < n; i += gridDim.x * 256)
      {
        C<typename SpinorT<PX>::R> u[12];
        C<typename SpinorT<PY>::R> v[12];
        C<RO> w[12];
        xk.load(i, u);
        if (b != 0.0) yk.load(i, v);
#pragma unroll
        for (int c = 0; c < 12; c++)
          {
            double re = a * (double)u[c].re, im = a * (double)u[c].im;
            if (b != 0.0)
              {
                re += b * (double)v[c].re;
                im += b * (double)v[c].im;
              }
            w[c] = {RO(re), RO(im)};
          }
        ok.store(i, w);
      }
  }

  // pout = r + beta pin per right-hand side; with sel, right-hand side k reads
  // pin2 instead of pin when st[k].dir is set (the paired CG's restart)
  template <int P>
  __global__ void __launch_bounds__(256)
    xpay_to_mrhs_kernel(int n, int nrhs, SpinorBatch<P> r, SpinorBatch<P> pin, SpinorBatch<P> pin2,
                        SpinorBatch<P> pout, int sel, const CgState* __restrict__ st,
                        const CgState* __restrict__ mask)
  {
    using R = typename SpinorT<P>::R;
    const int k = blockIdx.y;
    if (k >= nrhs || (mask ? mask[k].stop : st[k].stop)) return;
    const R beta = R(st[k].beta);
    const SpinorT<P> rk = r.rhs(k), ik = (sel && st[k].dir) ? pin2.rhs(k) : pin.rhs(k), ok = pout.rhs(k);
    for (int i = blockIdx.x * 256 + threadIdx.x; i < n; i += gridDim.x * 256)
      {
        C<R> a[12], b[12];
        rk.load(i, a);
        ik.load(i, b);
#pragma unroll
        for (int c = 0; c < 12; c++) b[c] = cadd(a[c], cscale(b[c], beta));
        ok.store(i, b);
      }
  }

  // the paired CG's pending step: x += alpha p for the right-hand sides
  // (unmasked) whose block was cut after an odd number of iterations (dir 0)
  template <int PX, int P>
  __global__ void __launch_bounds__(256)
    xflush_mrhs_kernel(int n, int nrhs, SpinorBatch<PX> x, SpinorBatch<P> p, const CgState* __restrict__ st,
                       const CgState* __restrict__ mask)
  {
    using RX = typename SpinorT<PX>::R;
    const int k = blockIdx.y;
    if (k >= nrhs || mask[k].stop || st[k].dir) return;
    const RX a = RX(st[k].alpha);
    const SpinorT<PX> xk = x.rhs(k);
    const SpinorT<P> pk = p.rhs(k);
    for (int i = blockIdx.x * 256 + threadIdx.x; i < n; i += gridDim.x * 256)
      {
        C<RX> u[12];
        C<typename SpinorT<P>::R> v[12];
        xk.load(i, u);
        pk.load(i, v);
#pragma unroll
        for (int c = 0; c < 12; c++)
          {
            u[c].re += a * RX(v[c].re);
            u[c].im += a * RX(v[c].im);
          }
        xk.store(i, u);
      }
  }

  // p = r + beta p per right-hand side
  template <int P>
  __global__ void __launch_bounds__(256)
    xpay_mrhs_kernel(int n, int nrhs, SpinorBatch<P> r, SpinorBatch<P> p, const CgState* __restrict__ st,
                     const CgState* __restrict__ mask)
  {
    using R = typename SpinorT<P>::R;
    const int k = blockIdx.y;
    if (k >= nrhs || (mask ? mask[k].stop : st[k].stop)) return;
    const R beta = R(st[k].beta);
    const SpinorT<P> rk = r.rhs(k), pk = p.rhs(k);
    for (int i = blockIdx.x * 256 + threadIdx.x; i < n; i += gridDim.x * 256)
      {
        C<R> a[12], b[12];
        rk.load(i, a);
        pk.load(i, b);
#pragma unroll
        for (int c = 0; c < 12; c++) b[c] = cadd(a[c], cscale(b[c], beta));
        pk.store(i, b);
      }
  }
}
