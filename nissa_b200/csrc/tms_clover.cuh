// Twisted-clover e/o operator: device data and the epilogues that fuse the
// clover diagonal terms into the hopping kernel.
//
// The clover term of a site is four SU(3)-shaped blocks (the reference's
// clover_term_t, new_types/su3.hpp:57-60): on the spins (0,1) the 6x6
// Hermitian block [[c0, c1^+], [c1, -c0]], on the spins (2,3) the same with
// c2, c3 (unsafe_apply_point_chromo_operator_to_spincolor,
// operations/su3_paths/clover_term.hpp:14-30).  The e/o operator adds the
// twisted diagonal z = 1/2k +- i mu on the two chiralities
// (apply_point_twisted_clover_term_to_halfspincolor, clover_term.hpp:114-141)
// and needs on the even sites the inverse of that 12x12 (two 6x6 blocks)
// matrix (invert_twisted_clover_term, clover_term.hpp:143-262; the lower
// chirality's inverse with -mu is the Hermitian conjugate of the +mu one).
//
// Layout in HBM (structure of arrays, planes of Vh sites):
//   clover term   V2 cl[par][36][Vh]     plane = block*9 + row*3 + col
//   inverse       V2 icl[2][6][6][Vh]    even sites, chirality, row, col
// with V2 = double2 for the FP64 operator and float2 for the inner solvers.
#pragma once

#include <type_traits>

#include "tms_kernels.cuh"

namespace tms
{
  template <int P>
  struct ClovT
  {
    using R = typename SpinorT<P>::R;
    using V2 = typename std::conditional<P == PREC_F64, double2, float2>::type;
    const V2* __restrict__ cl;  // [par][36][Vh]
    const V2* __restrict__ icl; // [72][Vh], even sites
    int Vh;
    __device__ __forceinline__ C<R> cl_elem(int par, int k, int site) const
    {
      const V2 w = __ldg(cl + ((size_t)par * 36 + k) * Vh + site);
      return {R(w.x), R(w.y)};
    }
    __device__ __forceinline__ C<R> icl_elem(int k, int site) const
    {
      const V2 w = __ldg(icl + (size_t)k * Vh + site);
      return {R(w.x), R(w.y)};
    }

    // o = (z + block of chirality b) in on spins 2b, 2b+1 (twisted diagonal z)
    __device__ __forceinline__ void apply_block(int par, int b, int site, C<R> z, const C<R> in[12], C<R> o[12]) const
    {
      const C<R>* i0 = in + 6 * b;
      const C<R>* i1 = in + 6 * b + 3;
      C<R>* o0 = o + 6 * b;
      C<R>* o1 = o + 6 * b + 3;
#pragma unroll
      for (int a = 0; a < 3; a++)
        {
          o0[a] = cmul(z, i0[a]);
          o1[a] = cmul(z, i1[a]);
        }
      // c0: o0 += c0 i0 ; o1 -= c0 i1
#pragma unroll
      for (int a = 0; a < 3; a++)
#pragma unroll
        for (int e = 0; e < 3; e++)
          {
            const C<R> c = cl_elem(par, (2 * b) * 9 + 3 * a + e, site);
            o0[a] = cadd(o0[a], cmul(c, i0[e]));
            o1[a] = csub(o1[a], cmul(c, i1[e]));
          }
      // c1: o0 += c1^+ i1 ; o1 += c1 i0
#pragma unroll
      for (int a = 0; a < 3; a++)
#pragma unroll
        for (int e = 0; e < 3; e++)
          {
            const C<R> c = cl_elem(par, (2 * b + 1) * 9 + 3 * a + e, site);
            o1[a] = cadd(o1[a], cmul(c, i0[e]));
            o0[e] = cadd(o0[e], cjmul(c, i1[a]));
          }
    }

    // tmclovDee_or_oo_eos (dirac_operator_tmclovD_eoprec_portable.cpp:18-40): o = T(mu') in with
    // mu' = -mu when dag; the upper chirality takes +mu', the lower -mu'
    __device__ __forceinline__ void diag(int par, int site, R kcf, R mu, bool dag, const C<R> in[12],
                                         C<R> o[12]) const
    {
      const R m = dag ? -mu : mu;
      apply_block(par, 0, site, C<R>{kcf, m}, in, o);
      apply_block(par, 1, site, C<R>{kcf, -m}, in, o);
    }

    // inv_tmclovDee_or_oo_eos (dirac_operator_tmclovD_eoprec.hpp:24-44) on an even site:
    // the chirality `high` (0, or 1 when dag) takes the stored inverse, the other its conjugate
    __device__ __forceinline__ void inv(int site, bool dag, const C<R> in[12], C<R> o[12]) const
    {
      const int high = dag ? 1 : 0;
#pragma unroll
      for (int b = 0; b < 2; b++)
#pragma unroll
        for (int r = 0; r < 6; r++)
          {
            C<R> s = {R(0), R(0)};
#pragma unroll
            for (int c = 0; c < 6; c++)
              {
                if (b == high) s = cadd(s, cmul(icl_elem(b * 36 + r * 6 + c, site), in[6 * b + c]));
                else s = cadd(s, cjmul(icl_elem(b * 36 + c * 6 + r, site), in[6 * b + c]));
              }
            o[6 * b + r] = s;
          }
    }
  };

  // out = T_ee^-1(dag) hop   (the first half of tmclovDkern_eoprec_eos, on even sites)
  template <int P>
  struct EpiInvClov
  {
    static constexpr bool kReduce = false;
    SpinorT<P> out[2];
    ClovT<P> cl;
    int dag;
    __device__ __forceinline__ double operator()(int p, int ieo, C<typename SpinorT<P>::R> acc[12]) const
    {
      C<typename SpinorT<P>::R> o[12];
      cl.inv(ieo, dag != 0, acc, o);
      pick(out[0], out[1], p).store(ieo, o);
      return 0.0;
    }
  };

  // out = g5 ( T_oo(dag) x - hop/4 ): tmclovDkern_eoprec_eos
  // (dirac_operator_tmclovD_eoprec_portable.cpp:42-68).  Optionally reduces |out|^2.
  template <int P, bool RED>
  struct EpiClovKern
  {
    static constexpr bool kReduce = RED;
    SpinorT<P> out[2];
    SpinorT<P> x[2];
    ClovT<P> cl;
    const OpParams* prm;
    int dag;
    __device__ __forceinline__ double operator()(int p, int ieo, C<typename SpinorT<P>::R> acc[12]) const
    {
      using R = typename SpinorT<P>::R;
      C<R> xv[12], d[12];
      pick(x[0], x[1], p).load(ieo, xv);
      cl.diag(p, ieo, R(1.0 / (2.0 * prm->kappa)), R(prm->mu), dag != 0, xv, d);
      double n2 = 0.0;
#pragma unroll
      for (int c = 0; c < 12; c++)
        {
          const C<R> q = cscale(acc[c], R(0.25));
          acc[c] = (c < 6) ? csub(d[c], q) : csub(q, d[c]);
          if (RED) n2 += (double)acc[c].re * acc[c].re + (double)acc[c].im * acc[c].im;
        }
      pick(out[0], out[1], p).store(ieo, acc);
      return n2;
    }
  };

  // the second K of the CG matrix fused with the CG update:
  //   s = K(dag=false) t1 ;  x += alpha p ;  r -= alpha s ;  reduce |r|^2
  // XM selects the x update as in EpiKernCgUpdate: 1 x += alpha p; 0 none;
  // 2 x += alpha_prev pp + alpha p (paired, every other iteration)
  template <int P, int PX, int XM = 1>
  struct EpiClovKernCgUpdate
  {
    static constexpr bool kReduce = true;
    SpinorT<P> t1, r, p;
    SpinorT<PX> x;
    ClovT<P> cl;
    const OpParams* prm;
    const CgState* st;
    SpinorT<P> pp; // XM == 2: the previous direction
    __device__ __forceinline__ double operator()(int par, int ieo, C<typename SpinorT<P>::R> acc[12]) const
    {
      using R = typename SpinorT<P>::R;
      using RX = typename SpinorT<PX>::R;
      const R alpha = R(st->alpha);
      C<R> v[12], d[12];
      t1.load(ieo, v);
      cl.diag(par, ieo, R(1.0 / (2.0 * prm->kappa)), R(prm->mu), false, v, d);
#pragma unroll
      for (int c = 0; c < 12; c++)
        {
          const C<R> q = cscale(acc[c], R(0.25));
          acc[c] = (c < 6) ? csub(d[c], q) : csub(q, d[c]); // s
        }
      r.load(ieo, v);
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

  // psi_e = T_ee^-1 (eta_e + hop/2): Eq. (11) of the clover solve
  // (cg_invert_tmclovD_eoprec.cpp:104-107)
  template <int P>
  struct EpiClovReco
  {
    static constexpr bool kReduce = false;
    SpinorT<P> out[2];
    SpinorT<P> eta[2];
    ClovT<P> cl;
    __device__ __forceinline__ double operator()(int p, int ieo, C<typename SpinorT<P>::R> acc[12]) const
    {
      using R = typename SpinorT<P>::R;
      C<R> e[12], o[12];
      pick(eta[0], eta[1], p).load(ieo, e);
#pragma unroll
      for (int c = 0; c < 12; c++) e[c] = cadd(e[c], cscale(acc[c], R(0.5)));
      cl.inv(ieo, false, e, o);
      pick(out[0], out[1], p).store(ieo, o);
      return 0.0;
    }
  };

  // Full-lattice Q = g5 D_tmclov (apply_tmclovQ, dirac_operators/tmclovQ/dirac_operator_tmclovQ.cpp:15-170):
  // the twisted-mass Q plus g5 times the clover term.  Both parities in one launch.
  template <int P>
  struct EpiTmClovQ
  {
    static constexpr bool kReduce = false;
    SpinorT<P> out[2];
    SpinorT<P> x[2];
    ClovT<P> cl;
    const OpParams* prm;
    __device__ __forceinline__ double operator()(int p, int ieo, C<typename SpinorT<P>::R> acc[12]) const
    {
      using R = typename SpinorT<P>::R;
      const R kcf = R(1.0 / (2.0 * prm->kappa)), m = R(prm->mu);
      C<R> xv[12], d[12];
      pick(x[0], x[1], p).load(ieo, xv);
      // clover term alone: the block with z = 0
      cl.apply_block(p, 0, ieo, C<R>{R(0), R(0)}, xv, d);
      cl.apply_block(p, 1, ieo, C<R>{R(0), R(0)}, xv, d);
#pragma unroll
      for (int c = 0; c < 12; c++)
        {
          const C<R> im = {-m * xv[c].im, m * xv[c].re};
          const C<R> h = cscale(acc[c], R(0.5));
          const C<R> k = cscale(xv[c], kcf);
          acc[c] = (c < 6) ? cadd(cadd(d[c], csub(k, h)), im) : cadd(csub(csub(h, k), d[c]), im);
        }
      pick(out[0], out[1], p).store(ieo, acc);
      return 0.0;
    }
  };
}
