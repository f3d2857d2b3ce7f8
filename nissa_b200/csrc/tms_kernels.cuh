// Hopping stencil with fused epilogues, fused CG linear algebra and
// deterministic FP64 reductions.
//
// One thread computes one output site.  The stencil body gathers the eight
// neighbours directly from the structure-of-arrays planes: along z and y the
// neighbours of a warp are contiguous, along x and t they are a whole row /
// time slice away, which for the volumes served here sits in the 126 MB L2,
// so each input spinor and link crosses HBM about once per launch.  The
// antiperiodic time boundary is a sign applied in the kernel when a hop
// crosses t = T-1 -> 0 (links are stored periodic).
//
// Every kernel whose result feeds a global scalar (alpha, beta, |r|^2) reduces
// per block in FP64 with warp shuffles, and the last block to finish sums the
// block partials in a fixed order: the result does not depend on scheduling
// and no block ever waits for another.
#pragma once

#include "tms_common.cuh"

namespace tms
{
  constexpr int HOP_THREADS = 128;

  // -------------------------------------------------- FP64 block reduction
  __device__ __forceinline__ double warp_sum(double v)
  {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
  }

  // Reduce v over the grid.  The last block to finish calls fin(total) from
  // thread 0.  Must be reached by every thread of every block.
  template <int NT, class Fin>
  __device__ __forceinline__ void grid_reduce(double v, const Reducer& red, const Fin& fin)
  {
    __shared__ double sh[NT / 32];
    __shared__ bool amLast;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v = warp_sum(v);
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    if (warp == 0)
      {
        double w = (lane < NT / 32) ? sh[lane] : 0.0;
        w = warp_sum(w);
        if (lane == 0)
          {
            red.partial[blockIdx.x] = w;
            __threadfence();
            const unsigned ticket = atomicAdd(red.counter, 1u);
            amLast = (ticket == gridDim.x - 1);
          }
      }
    __syncthreads();
    if (amLast)
      {
        __threadfence();
        // the partials of the other blocks are in L2 (__threadfence before each
        // ticket): load them past L1, several in flight, in a fixed order per thread
        double s = 0.0;
#pragma unroll 8
        for (int i = threadIdx.x; i < (int)gridDim.x; i += NT) s += __ldcg(red.partial + i);
        s = warp_sum(s);
        if (lane == 0) sh[warp] = s;
        __syncthreads();
        if (threadIdx.x == 0)
          {
            double t = 0.0;
#pragma unroll
            for (int w = 0; w < NT / 32; w++) t += sh[w];
            *red.result = t;
            *red.counter = 0u;
            fin(t);
          }
      }
  }

  struct NoFin
  {
    __device__ void operator()(double) const {}
  };

  // pick the accessor of parity p by value (keeps it in registers, no local-memory array)
  template <class T>
  __device__ __forceinline__ T pick(const T& a0, const T& a1, int p)
  {
    T r;
    r.d = p ? a1.d : a0.d;
    r.n = p ? a1.n : a0.n;
    r.stride = a0.stride;
    return r;
  }

  // Epilogue operand loads go through a loader, ld(k, field, site, v): operand
  // k of the output site.  The plain one reads global memory; the pipelined
  // hops pass one that reads the operands they staged in shared memory while
  // the last directions were computed (the first EpiStaged<E>::n operands,
  // whose fields the epilogue names with staged()).
  struct LoadGlobal
  {
    template <int P>
    __device__ __forceinline__ void operator()(int, const SpinorT<P>& f, int site, C<typename SpinorT<P>::R> v[12]) const
    {
      f.load(site, v);
    }
  };
  template <class E, class = void>
  struct EpiStaged
  {
    static constexpr int n = 0;
  };
  template <class E>
  struct EpiStaged<E, decltype((void)E::kStaged)>
  {
    static constexpr int n = E::kStaged;
  };

  // ------------------------------------------------------- stencil body
  // Accumulates the -2*hopping term sum_mu [(1-g_mu) U_x,mu in(x+mu) + (1+g_mu) U^+_x-mu,mu in(x-mu)]
  // in the reference's chiral basis; projection and reconstruction tables follow
  // dirac_operator_tmD_eoprec_portable.hpp:56-166.
  template <int MU, bool FWD, typename R>
  __device__ __forceinline__ void project(const C<R> s[12], C<R> h0[3], C<R> h1[3])
  {
#pragma unroll
    for (int c = 0; c < 3; c++)
      {
        const C<R> s0 = s[c], s1 = s[3 + c], s2 = s[6 + c], s3 = s[9 + c];
        if (FWD)
          {
            if (MU == 0) { h0[c] = cadd(s0, s2); h1[c] = cadd(s1, s3); }
            if (MU == 1) { h0[c] = ciadd(s0, s3); h1[c] = ciadd(s1, s2); }
            if (MU == 2) { h0[c] = cadd(s0, s3); h1[c] = csub(s1, s2); }
            if (MU == 3) { h0[c] = ciadd(s0, s2); h1[c] = cisub(s1, s3); }
          }
        else
          {
            if (MU == 0) { h0[c] = csub(s0, s2); h1[c] = csub(s1, s3); }
            if (MU == 1) { h0[c] = cisub(s0, s3); h1[c] = cisub(s1, s2); }
            if (MU == 2) { h0[c] = csub(s0, s3); h1[c] = cadd(s1, s2); }
            if (MU == 3) { h0[c] = cisub(s0, s2); h1[c] = ciadd(s1, s3); }
          }
      }
  }

  template <int MU, bool FWD, typename R>
  __device__ __forceinline__ void reconstruct(C<R> acc[12], const C<R> u0[3], const C<R> u1[3])
  {
#pragma unroll
    for (int c = 0; c < 3; c++)
      {
        acc[c] = cadd(acc[c], u0[c]);
        acc[3 + c] = cadd(acc[3 + c], u1[c]);
        if (FWD)
          {
            if (MU == 0) { acc[6 + c] = cadd(acc[6 + c], u0[c]); acc[9 + c] = cadd(acc[9 + c], u1[c]); }
            if (MU == 1) { acc[6 + c] = cisub(acc[6 + c], u1[c]); acc[9 + c] = cisub(acc[9 + c], u0[c]); }
            if (MU == 2) { acc[6 + c] = csub(acc[6 + c], u1[c]); acc[9 + c] = cadd(acc[9 + c], u0[c]); }
            if (MU == 3) { acc[6 + c] = cisub(acc[6 + c], u0[c]); acc[9 + c] = ciadd(acc[9 + c], u1[c]); }
          }
        else
          {
            if (MU == 0) { acc[6 + c] = csub(acc[6 + c], u0[c]); acc[9 + c] = csub(acc[9 + c], u1[c]); }
            if (MU == 1) { acc[6 + c] = ciadd(acc[6 + c], u1[c]); acc[9 + c] = ciadd(acc[9 + c], u0[c]); }
            if (MU == 2) { acc[6 + c] = cadd(acc[6 + c], u1[c]); acc[9 + c] = csub(acc[9 + c], u0[c]); }
            if (MU == 3) { acc[6 + c] = ciadd(acc[6 + c], u0[c]); acc[9 + c] = cisub(acc[9 + c], u1[c]); }
          }
      }
  }

  // u = U h (FWD) or U^+ h (backward), times a real factor
  template <bool FWD, typename R>
  __device__ __forceinline__ void link_mul(const C<R> U[9], const C<R> h[3], C<R> u[3], R f)
  {
#pragma unroll
    for (int i = 0; i < 3; i++)
      {
        C<R> a;
        if (FWD)
          {
            a = cmul(U[3 * i], h[0]);
            a = cadd(a, cmul(U[3 * i + 1], h[1]));
            a = cadd(a, cmul(U[3 * i + 2], h[2]));
          }
        else
          {
            a = cjmul(U[i], h[0]);
            a = cadd(a, cjmul(U[3 + i], h[1]));
            a = cadd(a, cjmul(U[6 + i], h[2]));
          }
        u[i] = cscale(a, f);
      }
  }

  // One direction of the stencil.  The factors of the hop (anisotropy, the
  // time-boundary sign, the FP16 per-site scale of the neighbour, the 16-bit
  // link scale) are folded into one multiplication of the two link products.
  template <int MU, int P, int LF>
  __device__ __forceinline__ void hop_dir(const Lattice& g, const Site& s, int p, int ieo, const SpinorT<P>& in,
                                          const LinkT<LF>& U, typename SpinorT<P>::R anis,
                                          C<typename SpinorT<P>::R> acc[12])
  {
    using R = typename SpinorT<P>::R;
    const R fmu = (MU > 0) ? anis : R(1);
    {
      bool w;
      const int n = nbr_up<MU>(g, s, w);
      C<R> sp[12], h0[3], h1[3], u0[3], u1[3], L[9];
      R ss, ls;
      in.load_raw(n, sp, ss);
      project<MU, true>(sp, h0, h1);
      U.load_scaled(p, MU, ieo, L, ls);
      const R f = (w ? fmu * R(g.bc_t) : fmu) * ss * ls;
      link_mul<true>(L, h0, u0, f);
      link_mul<true>(L, h1, u1, f);
      reconstruct<MU, true>(acc, u0, u1);
    }
    {
      bool w;
      const int n = nbr_dw<MU>(g, s, w);
      C<R> sp[12], h0[3], h1[3], u0[3], u1[3], L[9];
      R ss, ls;
      in.load_raw(n, sp, ss);
      project<MU, false>(sp, h0, h1);
      U.load_scaled(1 - p, MU, n, L, ls);
      const R f = (w ? fmu * R(g.bc_t) : fmu) * ss * ls;
      link_mul<false>(L, h0, u0, f);
      link_mul<false>(L, h1, u1, f);
      reconstruct<MU, false>(acc, u0, u1);
    }
  }

  template <int P, int LF>
  __device__ __forceinline__ void hop_site(const Lattice& g, int p, int ieo, const SpinorT<P>& in, const LinkT<LF>& U,
                                           typename SpinorT<P>::R anis, C<typename SpinorT<P>::R> acc[12])
  {
    using R = typename SpinorT<P>::R;
#pragma unroll
    for (int c = 0; c < 12; c++) acc[c] = {R(0), R(0)};
    const Site s = eo_site(g, p, ieo);
    hop_dir<0, P, LF>(g, s, p, ieo, in, U, anis, acc);
    hop_dir<1, P, LF>(g, s, p, ieo, in, U, anis, acc);
    hop_dir<2, P, LF>(g, s, p, ieo, in, U, anis, acc);
    hop_dir<3, P, LF>(g, s, p, ieo, in, U, anis, acc);
  }

  // ------------------------------------------------------------ epilogues
  // Each epilogue consumes the accumulated hop of one site (parity p, index
  // ieo) and returns its contribution to the kernel's reduction (if any).

  // (FP32 arithmetic: the factors in FP32, from correctly rounded reciprocals,
  // instead of FP64 divisions in every thread)
  template <typename R>
  __device__ __forceinline__ C<R> zdiag(const OpParams& o, double sgn)
  {
    if constexpr (sizeof(R) == 4) return {__frcp_rn(2.0f * float(o.kappa)), float(sgn * o.mu)};
    else return {R(1.0 / (2.0 * o.kappa)), R(sgn * o.mu)};
  }
  template <typename R>
  __device__ __forceinline__ C<R> zinvdiag(const OpParams& o, double sgn)
  {
    if constexpr (sizeof(R) == 4)
      {
        const float a = __frcp_rn(2.0f * float(o.kappa)), b = float(sgn * o.mu);
        const float inv = __frcp_rn(fmaf(a, a, b * b));
        return {a * inv, -b * inv};
      }
    else
      {
        const double a = 1.0 / (2.0 * o.kappa), b = sgn * o.mu, nrm = a * a + b * b;
        return {R(+a / nrm), R(-b / nrm)};
      }
  }
  // (z on spins 0,1; conj(z) on spins 2,3): tmDee_or_oo_eos, ..._portable.hpp:171-195
  template <typename R>
  __device__ __forceinline__ C<R> diag_apply(C<R> v, C<R> z, int c)
  {
    return (c < 6) ? cmul(v, z) : cmul(v, cconj(z));
  }

  // out = hop (tmn2Deo_or_tmn2Doe_eos)
  template <int P>
  struct EpiPlain
  {
    static constexpr bool kReduce = false;
    SpinorT<P> out[2];
    __device__ __forceinline__ double operator()(int p, int ieo, C<typename SpinorT<P>::R> acc[12]) const
    {
      pick(out[0], out[1], p).store(ieo, acc);
      return 0.0;
    }
  };

  // out = (1/2k + i s mu g5)^-1 hop  (inv_tmDee_or_oo_eos applied to the hop)
  template <int P>
  struct EpiInvDiag
  {
    static constexpr bool kReduce = false;
    SpinorT<P> out[2];
    const OpParams* prm;
    double sgn;
    __device__ __forceinline__ double operator()(int p, int ieo, C<typename SpinorT<P>::R> acc[12]) const
    {
      using R = typename SpinorT<P>::R;
      const C<R> z = zinvdiag<R>(*prm, sgn);
#pragma unroll
      for (int c = 0; c < 12; c++) acc[c] = diag_apply(acc[c], z, c);
      pick(out[0], out[1], p).store(ieo, acc);
      return 0.0;
    }
  };

  // out = g5 ( (1/2k + i s mu g5) x - hop/4 ), the Schur operator K_oo
  // (tmDkern_eoprec_eos with ..._put_together_and_include_gamma5,
  // dirac_operator_tmD_eoprec_portable.cpp:18-51).  Optionally reduces |out|^2.
  template <int P, bool RED>
  struct EpiKern
  {
    static constexpr bool kReduce = RED;
    static constexpr int kStaged = (P == PREC_F16) ? 1 : 0; // x
    SpinorT<P> out[2];
    SpinorT<P> x[2];
    const OpParams* prm;
    double sgn;
    __device__ __forceinline__ SpinorT<P> staged(int p, int) const { return pick(x[0], x[1], p); }
    __device__ __forceinline__ double operator()(int p, int ieo, C<typename SpinorT<P>::R> acc[12]) const
    {
      return run(p, ieo, acc, LoadGlobal{});
    }
    template <class LD>
    __device__ __forceinline__ double run(int p, int ieo, C<typename SpinorT<P>::R> acc[12], const LD& ld) const
    {
      using R = typename SpinorT<P>::R;
      const C<R> z = zdiag<R>(*prm, sgn);
      C<R> xv[12];
      ld(0, pick(x[0], x[1], p), ieo, xv);
      double n2 = 0.0;
#pragma unroll
      for (int c = 0; c < 12; c++)
        {
          const C<R> d = diag_apply(xv[c], z, c);
          const C<R> q = cscale(acc[c], R(0.25));
          acc[c] = (c < 6) ? csub(d, q) : csub(q, d);
          if (RED) n2 += (double)acc[c].re * acc[c].re + (double)acc[c].im * acc[c].im;
        }
      pick(out[0], out[1], p).store(ieo, acc);
      return n2;
    }
  };

  // r = b - K x in the second half of K (the residual recomputation of the
  // mixed solvers fused into the stencil): out = b - g5 ((1/2k + i s mu g5) x - hop/4),
  // reducing |r|^2
  template <int P>
  struct EpiKernResidual
  {
    static constexpr bool kReduce = true;
    SpinorT<P> out; // r
    SpinorT<P> x;   // the operand of this K at the output site
    SpinorT<P> b;
    const OpParams* prm;
    double sgn;
    __device__ __forceinline__ double operator()(int, int ieo, C<typename SpinorT<P>::R> acc[12]) const
    {
      using R = typename SpinorT<P>::R;
      const C<R> z = zdiag<R>(*prm, sgn);
      C<R> xv[12], bv[12];
      x.load(ieo, xv);
      b.load(ieo, bv);
      double n2 = 0.0;
#pragma unroll
      for (int c = 0; c < 12; c++)
        {
          const C<R> d = diag_apply(xv[c], z, c);
          const C<R> q = cscale(acc[c], R(0.25));
          acc[c] = csub(bv[c], (c < 6) ? csub(d, q) : csub(q, d));
          n2 += (double)acc[c].re * acc[c].re + (double)acc[c].im * acc[c].im;
        }
      out.store(ieo, acc);
      return n2;
    }
  };

  // varphi = g5 (eta_o + hop/2): Eq. (8b), cg_invert_tmD_eoprec.cpp:37-58
  template <int P>
  struct EpiSrcPrep
  {
    static constexpr bool kReduce = false;
    SpinorT<P> out[2];
    SpinorT<P> eta[2];
    __device__ __forceinline__ double operator()(int p, int ieo, C<typename SpinorT<P>::R> acc[12]) const
    {
      using R = typename SpinorT<P>::R;
      C<R> e[12];
      pick(eta[0], eta[1], p).load(ieo, e);
#pragma unroll
      for (int c = 0; c < 12; c++)
        {
          const C<R> h = cscale(acc[c], R(0.5));
          acc[c] = (c < 6) ? cadd(e[c], h) : csub(cscale(e[c], R(-1)), h);
        }
      pick(out[0], out[1], p).store(ieo, acc);
      return 0.0;
    }
  };

  // psi_e = (1/2k + i mu g5)^-1 (eta_e + hop/2): Eq. (11), cg_invert_tmD_eoprec.cpp:81-99 and :144-145
  template <int P>
  struct EpiReco
  {
    static constexpr bool kReduce = false;
    SpinorT<P> out[2];
    SpinorT<P> eta[2];
    const OpParams* prm;
    double sgn;
    __device__ __forceinline__ double operator()(int p, int ieo, C<typename SpinorT<P>::R> acc[12]) const
    {
      using R = typename SpinorT<P>::R;
      const C<R> z = zinvdiag<R>(*prm, sgn);
      C<R> e[12];
      pick(eta[0], eta[1], p).load(ieo, e);
#pragma unroll
      for (int c = 0; c < 12; c++) acc[c] = diag_apply(cadd(e[c], cscale(acc[c], R(0.5))), z, c);
      pick(out[0], out[1], p).store(ieo, acc);
      return 0.0;
    }
  };

  // Full-lattice Q = g5 D_tm in the twisted basis (apply_tmQ,
  // dirac_operator_tmQ_portable.cpp:160-174): spins 0,1: -hop/2 + kcf in + i m in;
  // spins 2,3: +hop/2 - kcf in + i m in.  Optionally reduces |out|^2.
  template <int P, bool RED>
  struct EpiTmQ
  {
    static constexpr bool kReduce = RED;
    SpinorT<P> out[2];
    SpinorT<P> x[2];
    const OpParams* prm;
    double sgn;
    __device__ __forceinline__ double operator()(int p, int ieo, C<typename SpinorT<P>::R> acc[12]) const
    {
      using R = typename SpinorT<P>::R;
      const R kcf = R(1.0 / (2.0 * prm->kappa)), m = R(sgn * prm->mu);
      C<R> xv[12];
      pick(x[0], x[1], p).load(ieo, xv);
      double n2 = 0.0;
#pragma unroll
      for (int c = 0; c < 12; c++)
        {
          const C<R> im = {-m * xv[c].im, m * xv[c].re};
          const C<R> h = cscale(acc[c], R(0.5));
          const C<R> k = cscale(xv[c], kcf);
          acc[c] = (c < 6) ? cadd(csub(k, h), im) : cadd(csub(h, k), im);
          if (RED) n2 += (double)acc[c].re * acc[c].re + (double)acc[c].im * acc[c].im;
        }
      pick(out[0], out[1], p).store(ieo, acc);
      return n2;
    }
  };

  // ------------------------------------------------------ solver state
  struct CgState
  {
    double rr;         // current iterated |r|^2
    double rr_prev;    // |r|^2 of the previous iteration
    double pAp;        // (p, A p)
    double alpha;      // step length
    double alpha_prev; // step length of the previous iteration (paired x updates)
    double beta;       // direction update
    double target;     // stop when rr < target (residue * |b|^2)
    double rel_trigger;// reliable update when rr < rel_trigger
    double b2;         // |b|^2
    int iter;          // iterations done
    int niter_max;
    int stop;          // 0 running, 1 converged, 2 max iterations, 3 reliable update due, 4 breakdown
    int dir;           // paired batched CG: which buffer holds the direction after a cut (set by the host)
  };

  enum StopCode { STOP_RUN = 0, STOP_CONVERGED = 1, STOP_MAXITER = 2, STOP_RELIABLE = 3, STOP_BREAKDOWN = 4 };

  // alpha = rr / (p, A p)
  struct FinAlpha
  {
    CgState* st;
    __device__ void operator()(double pAp) const
    {
      st->pAp = pAp;
      if (!(pAp > 0.0) || isnan(pAp))
        {
          st->stop = STOP_BREAKDOWN;
          return;
        }
      st->alpha_prev = st->alpha;
      st->alpha = st->rr / pAp;
    }
  };

  // new |r|^2: beta, iteration count and the stopping tests of
  // cg_invert_template_threaded.hpp:104-129
  struct FinBeta
  {
    CgState* st;
    __device__ void operator()(double rr) const
    {
      st->rr_prev = st->rr;
      st->rr = rr;
      st->beta = rr / st->rr_prev;
      st->iter += 1;
      if (isnan(rr) || isnan(st->beta)) st->stop = STOP_BREAKDOWN;
      else if (rr < st->target) st->stop = STOP_CONVERGED;
      else if (st->iter >= st->niter_max) st->stop = STOP_MAXITER;
      else if (rr < st->rel_trigger) st->stop = STOP_RELIABLE;
    }
  };

  // Second half of K(+mu)K(-mu) fused with the CG update:
  //   s = K(+mu) t1 ;  x += alpha p ;  r -= alpha s ;  reduce |r|^2
  // (cg_invert_template_threaded.hpp:82-107).  x may be kept in a wider
  // precision (PX) than the iterated vectors (P).  XM selects the x update:
  // 1 x += alpha p; 0 none; 2 x += alpha_prev pp + alpha p, where pp is the
  // previous iteration's direction (x updated every other iteration: the
  // paired form reads and writes x half as often).
  template <int P, int PX, int XM = 1>
  struct EpiKernCgUpdate
  {
    static constexpr bool kReduce = true;
    static constexpr int kStaged = (P == PREC_F16) ? 2 : 0; // t1, r
    SpinorT<P> t1;    // the input of K(+mu) at the output site
    SpinorT<P> r, p;
    SpinorT<PX> x;
    const OpParams* prm;
    const CgState* st;
    double sgn;
    SpinorT<P> pp;    // XM == 2: the previous direction
    __device__ __forceinline__ SpinorT<P> staged(int, int k) const { return k ? r : t1; }
    __device__ __forceinline__ double operator()(int par, int ieo, C<typename SpinorT<P>::R> acc[12]) const
    {
      return run(par, ieo, acc, LoadGlobal{});
    }
    template <class LD>
    __device__ __forceinline__ double run(int par, int ieo, C<typename SpinorT<P>::R> acc[12], const LD& ld) const
    {
      using R = typename SpinorT<P>::R;
      using RX = typename SpinorT<PX>::R;
      const C<R> z = zdiag<R>(*prm, sgn);
      const R alpha = R(st->alpha);
      C<R> v[12];
      ld(0, t1, ieo, v);
#pragma unroll
      for (int c = 0; c < 12; c++)
        {
          const C<R> d = diag_apply(v[c], z, c);
          const C<R> q = cscale(acc[c], R(0.25));
          acc[c] = (c < 6) ? csub(d, q) : csub(q, d); // s
        }
      ld(1, r, ieo, v);
      double n2 = 0.0;
#pragma unroll
      for (int c = 0; c < 12; c++)
        {
          v[c] = csub(v[c], cscale(acc[c], alpha));
          n2 += (double)v[c].re * v[c].re + (double)v[c].im * v[c].im;
        }
      r.store(ieo, v);
      if (XM == 0) return n2;
      C<RX> xv[12];
      x.load(ieo, xv);
      if (XM == 2)
        {
          pp.load(ieo, v);
          const RX ap = RX(st->alpha_prev);
#pragma unroll
          for (int c = 0; c < 12; c++)
            {
              xv[c].re += ap * RX(v[c].re);
              xv[c].im += ap * RX(v[c].im);
            }
        }
      p.load(ieo, v);
      const RX ax = RX(st->alpha);
#pragma unroll
      for (int c = 0; c < 12; c++)
        {
          xv[c].re += ax * RX(v[c].re);
          xv[c].im += ax * RX(v[c].im);
        }
      x.store(ieo, xv);
      return n2;
    }
  };

  // Second half of Q(+mu)Q(-mu) on the full lattice fused with the CG update
  // (both parities in one launch):  s = Q(+mu) t ;  x += alpha p ;
  // r -= alpha s ; reduce |r|^2.  The first half is EpiTmQ<P, true>, whose
  // |Q(-mu) p|^2 = (p, Q(+mu)Q(-mu) p) gives alpha (Q(-mu)^+ = Q(+mu)).
  template <int P, int PX>
  struct EpiTmQCgUpdate
  {
    static constexpr bool kReduce = true;
    SpinorT<P> t[2], r[2], p[2];
    SpinorT<PX> x[2];
    const OpParams* prm;
    const CgState* st;
    double sgn;
    __device__ __forceinline__ double operator()(int par, int ieo, C<typename SpinorT<P>::R> acc[12]) const
    {
      using R = typename SpinorT<P>::R;
      using RX = typename SpinorT<PX>::R;
      const R kcf = R(1.0 / (2.0 * prm->kappa)), m = R(sgn * prm->mu);
      const R alpha = R(st->alpha);
      C<R> v[12];
      pick(t[0], t[1], par).load(ieo, v);
#pragma unroll
      for (int c = 0; c < 12; c++)
        {
          const C<R> im = {-m * v[c].im, m * v[c].re};
          const C<R> h = cscale(acc[c], R(0.5));
          const C<R> k = cscale(v[c], kcf);
          acc[c] = (c < 6) ? cadd(csub(k, h), im) : cadd(csub(h, k), im); // s
        }
      const SpinorT<P> rr = pick(r[0], r[1], par);
      rr.load(ieo, v);
      double n2 = 0.0;
#pragma unroll
      for (int c = 0; c < 12; c++)
        {
          v[c] = csub(v[c], cscale(acc[c], alpha));
          n2 += (double)v[c].re * v[c].re + (double)v[c].im * v[c].im;
        }
      rr.store(ieo, v);
      pick(p[0], p[1], par).load(ieo, v);
      const SpinorT<PX> xx = pick(x[0], x[1], par);
      C<RX> xv[12];
      xx.load(ieo, xv);
      const RX ax = RX(st->alpha);
#pragma unroll
      for (int c = 0; c < 12; c++)
        {
          xv[c].re += ax * RX(v[c].re);
          xv[c].im += ax * RX(v[c].im);
        }
      xx.store(ieo, xv);
      return n2;
    }
  };

  // ----------------------------------------------------- multi-shift CGM
  // cgm_invert, inverters/templates/cgm_invert_template_threaded.hpp:11-295,
  // with one operator application s = Q_W^2 p per iteration split in two
  // launches (t = Q_W p reducing |t|^2 = (p, Q_W^2 p); s = Q_W t fused with
  // r += betaa s reducing |r|^2) and one fused update of p and of every
  // running shift's solution and direction.
  constexpr int CGM_MAX_SHIFTS = 32;

  struct CgmState
  {
    double rr, b2, betaa, betap, alpha, pap;
    int iter, niter_max, nshift, nrun, stop, go;
    double sigma[CGM_MAX_SHIFTS], zps[CGM_MAX_SHIFTS], zas[CGM_MAX_SHIFTS], zfs[CGM_MAX_SHIFTS];
    double betas[CGM_MAX_SHIFTS], alphas[CGM_MAX_SHIFTS], res[CGM_MAX_SHIFTS], target[CGM_MAX_SHIFTS];
    int run[CGM_MAX_SHIFTS], upd[CGM_MAX_SHIFTS];
  };

  // after (p, A p): betaa and the per-shift ratios (:110-158)
  struct FinCgm1
  {
    CgmState* st;
    __device__ void operator()(double pap) const
    {
      st->pap = pap;
      if (!(pap > 0.0) || isnan(pap))
        {
          st->stop = STOP_BREAKDOWN;
          return;
        }
      st->betap = st->betaa;
      st->betaa = -st->rr / pap;
      for (int i = 0; i < st->nshift; i++)
        {
          st->upd[i] = st->run[i];
          if (!st->run[i]) continue;
          const double ratio = st->betap / (st->betaa * st->alpha * (1 - st->zas[i] / st->zps[i]) +
                                            st->betap * (1 - st->sigma[i] * st->betaa));
          if (isnan(ratio))
            {
              st->stop = STOP_BREAKDOWN;
              return;
            }
          st->zfs[i] = st->zas[i] * ratio;
          st->betas[i] = st->betaa * ratio;
        }
      st->go = 1;
    }
  };

  // after |r'|^2: alpha, the per-shift alphas and z shifts, residues and
  // the per-shift stopping test (:164-260)
  struct FinCgm2
  {
    CgmState* st;
    __device__ void operator()(double rfrf) const
    {
      st->alpha = rfrf / st->rr;
      for (int i = 0; i < st->nshift; i++)
        if (st->upd[i])
          {
            st->alphas[i] = st->alpha * st->zfs[i] * st->betas[i] / (st->zas[i] * st->betaa);
            st->zps[i] = st->zas[i];
            st->zas[i] = st->zfs[i];
          }
      st->rr = rfrf;
      st->iter += 1;
      int nrun = 0;
      for (int i = 0; i < st->nshift; i++)
        {
          if (st->upd[i])
            {
              st->res[i] = st->rr * st->zfs[i] * st->zfs[i] / st->b2;
              if (st->res[i] < st->target[i]) st->run[i] = 0;
            }
          nrun += st->run[i];
        }
      st->nrun = nrun;
      if (isnan(rfrf)) st->stop = STOP_BREAKDOWN;
      else if (nrun == 0) st->stop = STOP_CONVERGED;
      else if (st->iter >= st->niter_max) st->stop = STOP_MAXITER;
    }
  };

  // s = Q_W t fused with r += betaa s, reduce |r|^2
  template <int P>
  struct EpiCgm2
  {
    static constexpr bool kReduce = true;
    SpinorT<P> t[2], r[2];
    const OpParams* prm;
    const CgmState* st;
    __device__ __forceinline__ double operator()(int par, int ieo, C<typename SpinorT<P>::R> acc[12]) const
    {
      using R = typename SpinorT<P>::R;
      const R kcf = R(1.0 / (2.0 * prm->kappa)), m = R(prm->mu);
      const R betaa = R(st->betaa);
      C<R> v[12];
      pick(t[0], t[1], par).load(ieo, v);
#pragma unroll
      for (int c = 0; c < 12; c++)
        {
          const C<R> im = {-m * v[c].im, m * v[c].re};
          const C<R> h = cscale(acc[c], R(0.5));
          const C<R> k = cscale(v[c], kcf);
          acc[c] = (c < 6) ? cadd(csub(k, h), im) : cadd(csub(h, k), im); // s
        }
      const SpinorT<P> rr = pick(r[0], r[1], par);
      rr.load(ieo, v);
      double n2 = 0.0;
#pragma unroll
      for (int c = 0; c < 12; c++)
        {
          v[c] = cadd(v[c], cscale(acc[c], betaa));
          n2 += (double)v[c].re * v[c].re + (double)v[c].im * v[c].im;
        }
      rr.store(ieo, v);
      return n2;
    }
  };

  // opens an iteration: the update kernel of the previous one may not run again
  static __global__ void cgm_begin_kernel(CgmState* st) { st->go = 0; }

  // p = r + alpha p ; for every shift updated this iteration:
  // sol_i -= betas_i ps_i ; ps_i = zfs_i r + alphas_i ps_i   (:150-158, :185-228)
  template <int P>
  __global__ void __launch_bounds__(256)
    cgm_update_kernel(int n, SpinorT<P> r, SpinorT<P> p, SpinorT<P> x0, SpinorT<P> ps0, size_t shift_elems,
                      const CgmState* __restrict__ st)
  {
    using R = typename SpinorT<P>::R;
    if (!st->go) return;
    const int i = blockIdx.x * 256 + threadIdx.x;
    if (i >= n) return;
    C<R> rv[12], v[12], w[12];
    r.load(i, rv);
    p.load(i, v);
    const R alpha = R(st->alpha);
#pragma unroll
    for (int c = 0; c < 12; c++) v[c] = cadd(rv[c], cscale(v[c], alpha));
    p.store(i, v);
    const int ns = st->nshift;
    for (int k = 0; k < ns; k++)
      {
        if (!st->upd[k]) continue;
        SpinorT<P> xk = x0, pk = ps0;
        xk.d += k * shift_elems;
        pk.d += k * shift_elems;
        if (xk.n) xk.n += k * (size_t)x0.stride;
        if (pk.n) pk.n += k * (size_t)ps0.stride;
        const R bs = R(st->betas[k]), z = R(st->zfs[k]), as = R(st->alphas[k]);
        pk.load(i, v);
        xk.load(i, w);
#pragma unroll
        for (int c = 0; c < 12; c++) w[c] = csub(w[c], cscale(v[c], bs));
        xk.store(i, w);
#pragma unroll
        for (int c = 0; c < 12; c++) v[c] = cadd(cscale(rv[c], z), cscale(v[c], as));
        pk.store(i, v);
      }
  }

  // ---------------------------------------------------------- hop kernel
  // Launch: one thread per output site; npar = 1 computes the parity
  // par_out only, npar = 2 both parities (grid over 2*Vh).
  // Launch shapes the autotuner chooses from (per precision):
  //   CFG 0: 128 threads, no register cap
  //   CFG 1: 128 threads, registers capped for 4 (FP64) / 8 (FP32, FP16) resident blocks per SM
  //   CFG 2: 256 threads, registers capped for 2 (FP64) / 4 (FP32, FP16) resident blocks per SM
  template <int P, int CFG>
  struct HopCfg
  {
    static constexpr int NT = (CFG == 2) ? 256 : 128;
    static constexpr int MINB = (CFG == 0) ? 1 : (CFG == 1) ? (P == PREC_F64 ? 4 : 8) : (P == PREC_F64 ? 2 : 4);
  };
  constexpr int HOP_CFGS = 3;      // launch shapes of the one-site kernel
  constexpr int HOP_CFGS_ALL = 8;  // FP32 arithmetic: 3 the two-site packed kernel with the cp.async
                                   // pipeline and 4 the two-site packed kernel (both T % 4 == 0), 5 one
                                   // site per thread, spin rows packed, 6 the same with its gathers
                                   // streamed through shared memory by cp.async (tms_hop_sp.cuh), 7 tiles
                                   // of rows staged in shared memory by bulk copies (tms_hop_tma.cuh)

  template <int P, int LF, class Epi, class Fin, int CFG = 0>
  __global__ void __launch_bounds__(HopCfg<P, CFG>::NT, HopCfg<P, CFG>::MINB)
    hop_kernel(Lattice g, int par_out, int npar, SpinorT<P> in_e, SpinorT<P> in_o, LinkT<LF> U, const OpParams* prm,
               Epi epi, Reducer red, Fin fin, const int* __restrict__ stop)
  {
    using R = typename SpinorT<P>::R;
    constexpr int NT = HopCfg<P, CFG>::NT;
    pdl_enter();
    if (stop && *stop) return;
    const int idx = blockIdx.x * NT + threadIdx.x;
    int p = par_out, ieo = idx;
    if (npar == 2)
      {
        p = (idx >= g.Vh) ? 1 : 0;
        ieo = idx - (p ? (int)g.Vh : 0);
      }
    const bool active = (idx < npar * g.Vh);
    double part = 0.0;
    if (active)
      {
        C<R> acc[12];
        const R anis = R(prm->anis);
        hop_site<P, LF>(g, p, ieo, p ? in_e : in_o, U, anis, acc);
        part = epi(p, ieo, acc);
      }
    if (Epi::kReduce) grid_reduce<NT>(part, red, fin);
  }

  // ------------------------------------------- two sites per thread, packed
  // For the FP32-arithmetic hops (FP32 and FP16 spinors) one thread computes
  // the sites (t,x,y,z) and (t+T/2,x,y,z), t < T/2.  When T/2 is even the two
  // have the same parity, e/o indices ieo and ieo + Vh/2, and the same spatial
  // neighbour offsets.  Each real of the first site sits in lane x and the same
  // real of the second in lane y of a float2, so the stencil runs on Blackwell's
  // packed FP32 instructions (two lanes per instruction), halving the
  // floating-point instruction count that bounds the low-precision hops.
  struct P2
  {
    float2 v;
  };
  __device__ __forceinline__ P2 p2(float a, float b) { return {make_float2(a, b)}; }
  __device__ __forceinline__ P2 operator+(P2 a, P2 b) { return {__fadd2_rn(a.v, b.v)}; }
  __device__ __forceinline__ P2 operator-(P2 a) { return {make_float2(-a.v.x, -a.v.y)}; }
  __device__ __forceinline__ P2 operator-(P2 a, P2 b) { return {__fadd2_rn(a.v, make_float2(-b.v.x, -b.v.y))}; }
  __device__ __forceinline__ P2 operator*(P2 a, P2 b) { return {__fmul2_rn(a.v, b.v)}; }
  __device__ __forceinline__ P2 fma2(P2 a, P2 b, P2 c) { return {__ffma2_rn(a.v, b.v, c.v)}; }

  __device__ __forceinline__ C<P2> zip(C<float> a, C<float> b) { return {p2(a.re, b.re), p2(a.im, b.im)}; }

  // an element of row 2 of a special-unitary link, conj(a d - b c), packed
  __device__ __forceinline__ C<P2> row2_elem(C<P2> a, C<P2> b, C<P2> c, C<P2> d)
  {
    // conj(a d - b c)
    P2 re = a.re * d.re;
    re = fma2(-a.im, d.im, re);
    re = fma2(-b.re, c.re, re);
    re = fma2(b.im, c.im, re);
    P2 im = (-a.re) * d.im;
    im = fma2(-a.im, d.re, im);
    im = fma2(b.re, c.im, im);
    im = fma2(b.im, c.re, im);
    return {re, im};
  }

  // link of site a (lane x) and site b (lane y) in stored units; its products
  // are to be multiplied by LinkT::kUnit
  template <int LF>
  __device__ __forceinline__ void load_link2(const LinkT<LF>& U, int par, int mu, int sa, int sb, C<P2> L[9])
  {
    constexpr int NR = LinkT<LF>::kRows;
    C<float> a[3 * NR], b[3 * NR];
    U.load_rows(par, mu, sa, a);
    U.load_rows(par, mu, sb, b);
#pragma unroll
    for (int k = 0; k < 3 * NR; k++) L[k] = zip(a[k], b[k]);
    if (NR == 2)
      {
        L[6] = row2_elem(L[1], L[2], L[4], L[5]);
        L[7] = row2_elem(L[2], L[0], L[5], L[3]);
        L[8] = row2_elem(L[0], L[1], L[3], L[4]);
        // in stored units: the products of two stored values carry one unit too many
        if (LinkT<LF>::kUnit != 1.0f)
          {
            const P2 unit = p2(LinkT<LF>::kUnit, LinkT<LF>::kUnit);
#pragma unroll
            for (int k = 6; k < 9; k++) L[k] = {L[k].re * unit, L[k].im * unit};
          }
      }
  }

  // u = U h (FWD) or U^+ h (backward), packed
  template <bool FWD>
  __device__ __forceinline__ void link_mul2(const C<P2> U[9], const C<P2> h[3], C<P2> u[3])
  {
#pragma unroll
    for (int i = 0; i < 3; i++)
      {
        C<P2> a;
#pragma unroll
        for (int j = 0; j < 3; j++)
          {
            const C<P2> w = FWD ? U[3 * i + j] : U[3 * j + i];
            const P2 wim = FWD ? w.im : -w.im;
            if (j == 0)
              {
                a.re = w.re * h[j].re;
                a.im = w.re * h[j].im;
              }
            else
              {
                a.re = fma2(w.re, h[j].re, a.re);
                a.im = fma2(w.re, h[j].im, a.im);
              }
            a.re = fma2(-wim, h[j].im, a.re);
            a.im = fma2(wim, h[j].re, a.im);
          }
        u[i] = a;
      }
  }

  // acc += f u, acc -= f u, acc += i f u, acc -= i f u (nf = -f)
  __device__ __forceinline__ void acc_add(C<P2>& acc, C<P2> u, P2 f, P2 nf)
  {
    acc.re = fma2(f, u.re, acc.re);
    acc.im = fma2(f, u.im, acc.im);
  }
  __device__ __forceinline__ void acc_sub(C<P2>& acc, C<P2> u, P2 f, P2 nf) { acc_add(acc, u, nf, f); }
  __device__ __forceinline__ void acc_iadd(C<P2>& acc, C<P2> u, P2 f, P2 nf)
  {
    acc.re = fma2(nf, u.im, acc.re);
    acc.im = fma2(f, u.re, acc.im);
  }
  __device__ __forceinline__ void acc_isub(C<P2>& acc, C<P2> u, P2 f, P2 nf) { acc_iadd(acc, u, nf, f); }

  // the reconstruction of `reconstruct`, with the hop factor folded into its fused multiply-adds
  template <int MU, bool FWD>
  __device__ __forceinline__ void reconstruct2(C<P2> acc[12], const C<P2> u0[3], const C<P2> u1[3], P2 f)
  {
    const P2 nf = -f;
#pragma unroll
    for (int c = 0; c < 3; c++)
      {
        acc_add(acc[c], u0[c], f, nf);
        acc_add(acc[3 + c], u1[c], f, nf);
        if (FWD)
          {
            if (MU == 0) { acc_add(acc[6 + c], u0[c], f, nf); acc_add(acc[9 + c], u1[c], f, nf); }
            if (MU == 1) { acc_isub(acc[6 + c], u1[c], f, nf); acc_isub(acc[9 + c], u0[c], f, nf); }
            if (MU == 2) { acc_sub(acc[6 + c], u1[c], f, nf); acc_add(acc[9 + c], u0[c], f, nf); }
            if (MU == 3) { acc_isub(acc[6 + c], u0[c], f, nf); acc_iadd(acc[9 + c], u1[c], f, nf); }
          }
        else
          {
            if (MU == 0) { acc_sub(acc[6 + c], u0[c], f, nf); acc_sub(acc[9 + c], u1[c], f, nf); }
            if (MU == 1) { acc_iadd(acc[6 + c], u1[c], f, nf); acc_iadd(acc[9 + c], u0[c], f, nf); }
            if (MU == 2) { acc_add(acc[6 + c], u1[c], f, nf); acc_sub(acc[9 + c], u0[c], f, nf); }
            if (MU == 3) { acc_iadd(acc[6 + c], u0[c], f, nf); acc_isub(acc[9 + c], u1[c], f, nf); }
          }
      }
  }

  // neighbour of the second site from that of the first: half a volume of
  // e/o indices away, modulo Vh
  __device__ __forceinline__ int partner(int n, int hv) { return (n >= hv) ? n - hv : n + hv; }

  template <int MU, bool FWD, int P, int LF>
  __device__ __forceinline__ void hop_dir2(const Lattice& g, const Site& s, int p, int ieo, int hv,
                                           const SpinorT<P>& in, const LinkT<LF>& U, float anis, C<P2> acc[12])
  {
    const float fmu = (MU > 0) ? anis : 1.0f;
    bool wa;
    const int na = FWD ? nbr_up<MU>(g, s, wa) : nbr_dw<MU>(g, s, wa);
    const int nb = partner(na, hv);
    // the second site (time t + T/2) crosses the boundary forward from t = T-1;
    // backward it never does (t + T/2 >= 1)
    const bool wb = (MU == 0) && FWD && (s.t == (g.T >> 1) - 1);
    C<P2> sp[12], h0[3], h1[3], u0[3], u1[3], L[9];
    {
      C<float> a[12], b[12];
      float sa, sb;
      in.load_raw(na, a, sa);
      in.load_raw(nb, b, sb);
#pragma unroll
      for (int c = 0; c < 12; c++) sp[c] = zip(a[c], b[c]);
      const float fbc = fmu * float(g.bc_t);
      const float k = LinkT<LF>::kUnit;
      const P2 f = p2((wa ? fbc : fmu) * sa * k, (wb ? fbc : fmu) * sb * k);
      project<MU, FWD>(sp, h0, h1);
      if (FWD) load_link2(U, p, MU, ieo, ieo + hv, L);
      else load_link2(U, 1 - p, MU, na, nb, L);
      link_mul2<FWD>(L, h0, u0);
      link_mul2<FWD>(L, h1, u1);
      reconstruct2<MU, FWD>(acc, u0, u1, f);
    }
  }

  constexpr int HOP2_THREADS = 128;

  // registers capped for 3 resident blocks per SM
  template <int P, int LF, class Epi, class Fin>
  __global__ void __launch_bounds__(HOP2_THREADS, 3)
    hop2_kernel(Lattice g, int par_out, int npar, SpinorT<P> in_e, SpinorT<P> in_o, LinkT<LF> U, const OpParams* prm,
                Epi epi, Reducer red, Fin fin, const int* __restrict__ stop)
  {
    pdl_enter();
    if (stop && *stop) return;
    const int hv = (int)(g.Vh >> 1);
    const int idx = blockIdx.x * HOP2_THREADS + threadIdx.x;
    int p = par_out, ieo = idx;
    if (npar == 2)
      {
        p = (idx >= hv) ? 1 : 0;
        ieo = idx - (p ? hv : 0);
      }
    const bool active = (idx < npar * hv);
    double part = 0.0;
    if (active)
      {
        C<P2> acc[12];
#pragma unroll
        for (int c = 0; c < 12; c++) acc[c] = {p2(0.f, 0.f), p2(0.f, 0.f)};
        const float anis = float(prm->anis);
        const Site s = eo_site(g, p, ieo);
        const SpinorT<P> in = p ? in_e : in_o;
        hop_dir2<0, true, P, LF>(g, s, p, ieo, hv, in, U, anis, acc);
        hop_dir2<0, false, P, LF>(g, s, p, ieo, hv, in, U, anis, acc);
        hop_dir2<1, true, P, LF>(g, s, p, ieo, hv, in, U, anis, acc);
        hop_dir2<1, false, P, LF>(g, s, p, ieo, hv, in, U, anis, acc);
        hop_dir2<2, true, P, LF>(g, s, p, ieo, hv, in, U, anis, acc);
        hop_dir2<2, false, P, LF>(g, s, p, ieo, hv, in, U, anis, acc);
        hop_dir2<3, true, P, LF>(g, s, p, ieo, hv, in, U, anis, acc);
        hop_dir2<3, false, P, LF>(g, s, p, ieo, hv, in, U, anis, acc);
        C<float> a[12], b[12];
#pragma unroll
        for (int c = 0; c < 12; c++)
          {
            a[c] = {acc[c].re.v.x, acc[c].im.v.x};
            b[c] = {acc[c].re.v.y, acc[c].im.v.y};
          }
        part = epi(p, ieo, a);
        part += epi(p, ieo + hv, b);
      }
    if (Epi::kReduce) grid_reduce<HOP2_THREADS>(part, red, fin);
  }

  // ------------------------------------------------------- BLAS kernels
  constexpr int BLAS_THREADS = 256;

  // p = r + beta p  (cg_invert_template_threaded.hpp:115-124)
  template <int P>
  static __global__ void __launch_bounds__(BLAS_THREADS)
    xpay_kernel(int n, SpinorT<P> r, SpinorT<P> p, const CgState* st, const int* __restrict__ stop)
  {
    using R = typename SpinorT<P>::R;
    pdl_enter();
    if (stop && *stop) return;
    const int i = blockIdx.x * BLAS_THREADS + threadIdx.x;
    if (i >= n) return;
    const R beta = R(st->beta);
    C<R> a[12], b[12];
    r.load(i, a);
    p.load(i, b);
#pragma unroll
    for (int c = 0; c < 12; c++) b[c] = cadd(a[c], cscale(b[c], beta));
    p.store(i, b);
  }

  // pout = r + beta pin (the paired CG keeps two directions)
  template <int P>
  static __global__ void __launch_bounds__(BLAS_THREADS)
    xpay_to_kernel(int n, SpinorT<P> r, SpinorT<P> pin, SpinorT<P> pout, const CgState* st,
                   const int* __restrict__ stop)
  {
    using R = typename SpinorT<P>::R;
    pdl_enter();
    if (stop && *stop) return;
    const int i = blockIdx.x * BLAS_THREADS + threadIdx.x;
    if (i >= n) return;
    const R beta = R(st->beta);
    C<R> a[12], b[12];
    r.load(i, a);
    pin.load(i, b);
#pragma unroll
    for (int c = 0; c < 12; c++) b[c] = cadd(a[c], cscale(b[c], beta));
    pout.store(i, b);
  }

  // generic: reduce |a|^2 (or Re(a,b)) over n sites
  template <int P, bool DOT>
  static __global__ void __launch_bounds__(BLAS_THREADS)
    norm_kernel(int n, SpinorT<P> a, SpinorT<P> b, Reducer red)
  {
    using R = typename SpinorT<P>::R;
    const int i = blockIdx.x * BLAS_THREADS + threadIdx.x;
    double s = 0.0;
    if (i < n)
      {
        C<R> x[12];
        a.load(i, x);
        if (DOT)
          {
            C<R> y[12];
            b.load(i, y);
#pragma unroll
            for (int c = 0; c < 12; c++) s += (double)x[c].re * y[c].re + (double)x[c].im * y[c].im;
          }
        else
#pragma unroll
          for (int c = 0; c < 12; c++) s += (double)x[c].re * x[c].re + (double)x[c].im * x[c].im;
      }
    grid_reduce<BLAS_THREADS>(s, red, NoFin{});
  }

  // out = a*x + b*y (any precisions)
  template <int PO, int PX, int PY>
  static __global__ void __launch_bounds__(BLAS_THREADS)
    axpby_kernel(int n, double a, SpinorT<PX> x, double b, SpinorT<PY> y, SpinorT<PO> out)
  {
    using RO = typename SpinorT<PO>::R;
    using RX = typename SpinorT<PX>::R;
    using RY = typename SpinorT<PY>::R;
    const int i = blockIdx.x * BLAS_THREADS + threadIdx.x;
    if (i >= n) return;
    C<RX> u[12];
    C<RY> v[12];
    C<RO> w[12];
    x.load(i, u);
    if (b != 0.0) y.load(i, v);
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
    out.store(i, w);
  }

  // r = b - s and reduce |r|^2 (true residual), FP64
  static __global__ void __launch_bounds__(BLAS_THREADS)
    residual_kernel(int n, SpinorT<PREC_F64> b, SpinorT<PREC_F64> s, SpinorT<PREC_F64> r, Reducer red)
  {
    const int i = blockIdx.x * BLAS_THREADS + threadIdx.x;
    double acc = 0.0;
    if (i < n)
      {
        C<double> u[12], v[12];
        b.load(i, u);
        s.load(i, v);
#pragma unroll
        for (int c = 0; c < 12; c++)
          {
            u[c] = csub(u[c], v[c]);
            acc += u[c].re * u[c].re + u[c].im * u[c].im;
          }
        r.store(i, u);
      }
    grid_reduce<BLAS_THREADS>(acc, red, NoFin{});
  }

  // reduce |g5 q - eta|^2 (the lx residual check of cg_invert_tmD_eoprec.cpp:192-212)
  static __global__ void __launch_bounds__(BLAS_THREADS)
    g5_residual_kernel(int n, SpinorT<PREC_F64> q, SpinorT<PREC_F64> eta, Reducer red)
  {
    const int i = blockIdx.x * BLAS_THREADS + threadIdx.x;
    double acc = 0.0;
    if (i < n)
      {
        C<double> u[12], v[12];
        q.load(i, u);
        eta.load(i, v);
#pragma unroll
        for (int c = 0; c < 12; c++)
          {
            const C<double> g = (c < 6) ? u[c] : cscale(u[c], -1.0);
            const C<double> d = csub(g, v[c]);
            acc += d.re * d.re + d.im * d.im;
          }
      }
    grid_reduce<BLAS_THREADS>(acc, red, NoFin{});
  }

  // out = g5 in, FP64 (g5 = diag(1,1,-1,-1), new_types/dirac.cpp:48)
  static __global__ void __launch_bounds__(BLAS_THREADS)
    g5_copy_kernel(int n, SpinorT<PREC_F64> in, SpinorT<PREC_F64> out)
  {
    const int i = blockIdx.x * BLAS_THREADS + threadIdx.x;
    if (i >= n) return;
    C<double> u[12];
    in.load(i, u);
#pragma unroll
    for (int c = 6; c < 12; c++) u[c] = {-u[c].re, -u[c].im};
    out.store(i, u);
  }

  // --------------------------------------------------- layout conversion
  // host-order AoS doubles (site-major, 24 per site) <-> SoA device spinor.
  // site_map (optional) gives the AoS row of SoA site i (used for lx <-> eo).
  template <int P>
  __global__ void aos_to_soa_kernel(int n, const double* __restrict__ aos, const int* __restrict__ site_map,
                                    SpinorT<P> out)
  {
    using R = typename SpinorT<P>::R;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const size_t row = site_map ? (size_t)site_map[i] : (size_t)i;
    const double* a = aos + row * 24; // 8-byte accesses: the caller's buffer need not be 16-byte aligned
    C<R> v[12];
#pragma unroll
    for (int c = 0; c < 12; c++) v[c] = {R(a[2 * c]), R(a[2 * c + 1])};
    out.store(i, v);
  }

  template <int P>
  __global__ void soa_to_aos_kernel(int n, SpinorT<P> in, const int* __restrict__ site_map, double* __restrict__ aos)
  {
    using R = typename SpinorT<P>::R;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const size_t row = site_map ? (size_t)site_map[i] : (size_t)i;
    C<R> v[12];
    in.load(i, v);
    double* a = aos + row * 24;
#pragma unroll
    for (int c = 0; c < 12; c++)
      {
        a[2 * c] = (double)v[c].re;
        a[2 * c + 1] = (double)v[c].im;
      }
  }

  // split_lx_vector_into_eo_parts / paste_eo_parts_into_lx_vector for whole
  // lx spinors: a block takes LXCOPY_THREADS consecutive lx sites, the AoS side
  // moves through shared memory as one contiguous run of doubles (coalesced,
  // 8-byte accesses), the SoA side at e/o index lx/2 of the site's parity
  // (the e/o numbering keeps lx order within a parity and LZ is even).
  constexpr int LXCOPY_THREADS = 128;
  constexpr int LXCOPY_PITCH = 25; // doubles per staged site (24 + 1 against bank conflicts)

  __device__ __forceinline__ int lx_parity(const Lattice& g, unsigned lx)
  {
    const unsigned z = lx % (unsigned)g.LZ;
    unsigned q = lx / (unsigned)g.LZ;
    const unsigned y = q % (unsigned)g.LY;
    q /= (unsigned)g.LY;
    const unsigned x = q % (unsigned)g.LX;
    const unsigned t = q / (unsigned)g.LX;
    return (int)((t + x + y + z) & 1u);
  }

  template <int P>
  __global__ void __launch_bounds__(LXCOPY_THREADS)
    lx_split_kernel(Lattice g, const double* __restrict__ aos, SpinorT<P> ev, SpinorT<P> od)
  {
    using R = typename SpinorT<P>::R;
    __shared__ double sh[LXCOPY_THREADS * LXCOPY_PITCH];
    const int64_t base = (int64_t)blockIdx.x * LXCOPY_THREADS;
    const int nsite = (int)min((int64_t)LXCOPY_THREADS, g.V - base);
    const double* in = aos + base * 24;
    for (int k = threadIdx.x; k < nsite * 24; k += LXCOPY_THREADS) sh[(k / 24) * LXCOPY_PITCH + k % 24] = in[k];
    __syncthreads();
    if ((int)threadIdx.x >= nsite) return;
    const unsigned lx = (unsigned)(base + threadIdx.x);
    const double* v = sh + threadIdx.x * LXCOPY_PITCH;
    C<R> c[12];
#pragma unroll
    for (int k = 0; k < 12; k++) c[k] = {R(v[2 * k]), R(v[2 * k + 1])};
    (lx_parity(g, lx) ? od : ev).store((int)(lx >> 1), c);
  }

  template <int P>
  __global__ void __launch_bounds__(LXCOPY_THREADS)
    lx_paste_kernel(Lattice g, SpinorT<P> ev, SpinorT<P> od, double* __restrict__ aos)
  {
    using R = typename SpinorT<P>::R;
    __shared__ double sh[LXCOPY_THREADS * LXCOPY_PITCH];
    const int64_t base = (int64_t)blockIdx.x * LXCOPY_THREADS;
    const int nsite = (int)min((int64_t)LXCOPY_THREADS, g.V - base);
    if ((int)threadIdx.x < nsite)
      {
        const unsigned lx = (unsigned)(base + threadIdx.x);
        C<R> c[12];
        (lx_parity(g, lx) ? od : ev).load((int)(lx >> 1), c);
        double* v = sh + threadIdx.x * LXCOPY_PITCH;
#pragma unroll
        for (int k = 0; k < 12; k++)
          {
            v[2 * k] = (double)c[k].re;
            v[2 * k + 1] = (double)c[k].im;
          }
      }
    __syncthreads();
    double* out = aos + base * 24;
    for (int k = threadIdx.x; k < nsite * 24; k += LXCOPY_THREADS) out[k] = sh[(k / 24) * LXCOPY_PITCH + k % 24];
  }
}
