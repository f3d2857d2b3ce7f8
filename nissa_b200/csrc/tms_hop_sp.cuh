// One site per thread with the two spin rows of every half spinor in the two
// lanes of Blackwell's packed FP32 instructions (launch shape 5 of the
// FP32-arithmetic hops: FP32 and FP16 spinors).
//
// The projection to half spinors, the SU(3) products and the reconstruction
// of tmn2Deo_or_tmn2Doe_eos (dirac_operator_tmD_eoprec_portable.hpp:56-166)
// all act identically on the two rows h0, h1 of a half spinor: both rows
// multiply the same link.  Here lane x of a float2 holds a real of row 0 (spin
// 0, or spin 2 of the lower pair) and lane y the same real of row 1 (spin 1,
// or spin 3), so that
//   * the projection is one packed add (or fused multiply-add with a lane sign
//     pair) per colour and real part: the neighbour's spins are converted
//     straight into (s0, s1) and (s2, s3) pairs, or (s3, s2) for the
//     directions whose projection crosses them (mu = x, y);
//   * U h for both rows is four packed FMAs per link element, each link real
//     broadcast to both lanes (the two-site shape 4 doubles the accumulators
//     for the same saving; this one keeps the register count of one site);
//   * the reconstruction folds the hop factor (anisotropy, time-boundary sign,
//     FP16 per-site scale, 16-bit link unit) into packed FMAs on the
//     accumulators; for mu = x, y the lower spin pair receives the rows
//     crossed, which costs scalar FMAs there.
// The arithmetic is that of the scalar kernel up to the order of FP32
// roundings (the hop factor is applied in the accumulating FMA).
#pragma once

#include "tms_kernels.cuh"

namespace tms
{
  __device__ __forceinline__ P2 bcast(float a) { return {make_float2(a, a)}; }
  // a - b, packed (no packed subtract: a fused multiply-add by -1)
  __device__ __forceinline__ P2 sub2(P2 a, P2 b) { return fma2(p2(-1.f, -1.f), b, a); }

  // row 2 of a special-unitary link from rows 0 and 1, conj(row0 x row1), in
  // the square of the rows' units (the caller scales its products)
  __device__ __forceinline__ void row2_unscaled(C<float> u[9])
  {
    u[6] = cconj(csub(cmul(u[1], u[5]), cmul(u[2], u[4])));
    u[7] = cconj(csub(cmul(u[2], u[3]), cmul(u[0], u[5])));
    u[8] = cconj(csub(cmul(u[0], u[4]), cmul(u[1], u[3])));
  }

  // One direction from the neighbour's spinor sp (in stored units), its link L
  // and the hop factor f that scales their product.
  // With ROW2K, row 2 of L is in k2 times the units of rows 0 and 1 (16-bit
  // links: row 2 rebuilt from raw rows); its products are scaled by k2 on the
  // packed pairs (forward: the output row 2; backward: the input row h_2)
  // rather than on the nine reals of the row.
  template <int MU, bool FWD, bool ROW2K = false>
  __device__ __forceinline__ void sp_dir_compute(const C<float> sp[12], const C<float> L[9], float f, C<P2> A01[3],
                                                 C<P2> A23[3], float k2 = 1.0f)
  {
    // (h0, h1) per colour, real and imaginary parts in packed pairs
    constexpr bool CROSS = (MU == 1 || MU == 2); // projection pairs spin 0 with 3 and 1 with 2
    const P2 pm = p2(1.f, -1.f), mp = p2(-1.f, 1.f);
    C<P2> H[3];
#pragma unroll
    for (int c = 0; c < 3; c++)
      {
        const C<P2> a = zip(sp[c], sp[3 + c]);
        const C<P2> b = CROSS ? zip(sp[9 + c], sp[6 + c]) : zip(sp[6 + c], sp[9 + c]);
        if (MU == 0) H[c] = FWD ? C<P2>{a.re + b.re, a.im + b.im} : C<P2>{sub2(a.re, b.re), sub2(a.im, b.im)};
        if (MU == 1) H[c] = FWD ? C<P2>{sub2(a.re, b.im), a.im + b.re} : C<P2>{a.re + b.im, sub2(a.im, b.re)};
        if (MU == 2)
          H[c] = FWD ? C<P2>{fma2(pm, b.re, a.re), fma2(pm, b.im, a.im)} : C<P2>{fma2(mp, b.re, a.re), fma2(mp, b.im, a.im)};
        if (MU == 3)
          H[c] = FWD ? C<P2>{fma2(mp, b.im, a.re), fma2(pm, b.re, a.im)} : C<P2>{fma2(pm, b.im, a.re), fma2(mp, b.re, a.im)};
      }

    // u = U h (forward) or U^+ h (backward) for both rows at once:
    //   forward  re += Ur hr - Ui hi, im += Ur hi + Ui hr
    //   backward re += Ur hr + Ui hi, im += Ur hi - Ui hr
    // with the one negated part of h formed once per colour
    if (ROW2K && !FWD) H[2] = {H[2].re * bcast(k2), H[2].im * bcast(k2)};
    C<P2> u[3], Hn[3];
#pragma unroll
    for (int j = 0; j < 3; j++)
      Hn[j] = FWD ? C<P2>{H[j].re, H[j].im * p2(-1.f, -1.f)} : C<P2>{H[j].re * p2(-1.f, -1.f), H[j].im};
#pragma unroll
    for (int i = 0; i < 3; i++)
      {
#pragma unroll
        for (int j = 0; j < 3; j++)
          {
            const C<float> e = FWD ? L[3 * i + j] : L[3 * j + i];
            const P2 er = bcast(e.re), ei = bcast(e.im);
            if (j == 0)
              {
                u[i].re = er * H[j].re;
                u[i].im = er * H[j].im;
              }
            else
              {
                u[i].re = fma2(er, H[j].re, u[i].re);
                u[i].im = fma2(er, H[j].im, u[i].im);
              }
            u[i].re = fma2(ei, FWD ? Hn[j].im : H[j].im, u[i].re);
            u[i].im = fma2(ei, FWD ? H[j].re : Hn[j].re, u[i].im);
          }
      }
    if (ROW2K && FWD) u[2] = {u[2].re * bcast(k2), u[2].im * bcast(k2)};

    // accumulate f u into spins (0, 1) and, per the reference's reconstruction, into spins (2, 3)
    const P2 F = bcast(f), NF = bcast(-f), Fpm = p2(f, -f), Fmp = p2(-f, f);
#pragma unroll
    for (int c = 0; c < 3; c++)
      {
        A01[c].re = fma2(F, u[c].re, A01[c].re);
        A01[c].im = fma2(F, u[c].im, A01[c].im);
        C<P2>& A = A23[c];
        const C<P2> v = u[c];
        if (MU == 0)
          {
            A.re = fma2(FWD ? F : NF, v.re, A.re);
            A.im = fma2(FWD ? F : NF, v.im, A.im);
          }
        if (MU == 3)
          {
            // forward: (acc2, acc3) += (-i u0, +i u1); backward: (+i u0, -i u1)
            A.re = fma2(FWD ? Fpm : Fmp, v.im, A.re);
            A.im = fma2(FWD ? Fmp : Fpm, v.re, A.im);
          }
        if (MU == 1)
          {
            // forward: acc2 -= i u1, acc3 -= i u0; backward: acc2 += i u1, acc3 += i u0
            const float sg = FWD ? f : -f;
            A.re.v.x = fmaf(sg, v.im.v.y, A.re.v.x);
            A.im.v.x = fmaf(-sg, v.re.v.y, A.im.v.x);
            A.re.v.y = fmaf(sg, v.im.v.x, A.re.v.y);
            A.im.v.y = fmaf(-sg, v.re.v.x, A.im.v.y);
          }
        if (MU == 2)
          {
            // forward: acc2 -= u1, acc3 += u0; backward: acc2 += u1, acc3 -= u0
            const float sg = FWD ? f : -f;
            A.re.v.x = fmaf(-sg, v.re.v.y, A.re.v.x);
            A.im.v.x = fmaf(-sg, v.im.v.y, A.im.v.x);
            A.re.v.y = fmaf(sg, v.re.v.x, A.re.v.y);
            A.im.v.y = fmaf(sg, v.im.v.x, A.im.v.y);
          }
      }
  }

  template <int MU, bool FWD, int P, int LF>
  __device__ __forceinline__ void hop_dir_sp(const Lattice& g, const Site& s, int p, int ieo, const SpinorT<P>& in,
                                             const LinkT<LF>& U, float fmu, C<P2> A01[3], C<P2> A23[3])
  {
    bool w;
    const int n = FWD ? nbr_up<MU>(g, s, w) : nbr_dw<MU>(g, s, w);
    C<float> sp[12], L[9];
    float ss, ls;
    in.load_raw(n, sp, ss);
    if constexpr (LF == LINK_I16_12)
      {
        // raw 16-bit rows, row 2 rebuilt in raw^2 units
        if (FWD) U.load_rows(p, MU, ieo, L);
        else U.load_rows(1 - p, MU, n, L);
        row2_unscaled(L);
        ls = LinkT<LF>::kUnit;
      }
    else
      {
        if (FWD) U.load_scaled(p, MU, ieo, L, ls);
        else U.load_scaled(1 - p, MU, n, L, ls);
      }
    const float f = (w ? fmu * float(g.bc_t) : fmu) * ss * ls;
    sp_dir_compute<MU, FWD, LF == LINK_I16_12>(sp, L, f, A01, A23, LinkT<LF>::kUnit);
  }

  // the hop of one site, returned unpacked in the accumulator layout of hop_site
  template <int P, int LF>
  __device__ __forceinline__ void hop_site_sp(const Lattice& g, int p, int ieo, const SpinorT<P>& in,
                                              const LinkT<LF>& U, float anis, C<float> acc[12])
  {
    C<P2> A01[3], A23[3];
#pragma unroll
    for (int c = 0; c < 3; c++)
      {
        A01[c] = {p2(0.f, 0.f), p2(0.f, 0.f)};
        A23[c] = {p2(0.f, 0.f), p2(0.f, 0.f)};
      }
    const Site s = eo_site(g, p, ieo);
    hop_dir_sp<0, true, P, LF>(g, s, p, ieo, in, U, 1.0f, A01, A23);
    hop_dir_sp<0, false, P, LF>(g, s, p, ieo, in, U, 1.0f, A01, A23);
    hop_dir_sp<1, true, P, LF>(g, s, p, ieo, in, U, anis, A01, A23);
    hop_dir_sp<1, false, P, LF>(g, s, p, ieo, in, U, anis, A01, A23);
    hop_dir_sp<2, true, P, LF>(g, s, p, ieo, in, U, anis, A01, A23);
    hop_dir_sp<2, false, P, LF>(g, s, p, ieo, in, U, anis, A01, A23);
    hop_dir_sp<3, true, P, LF>(g, s, p, ieo, in, U, anis, A01, A23);
    hop_dir_sp<3, false, P, LF>(g, s, p, ieo, in, U, anis, A01, A23);
#pragma unroll
    for (int c = 0; c < 3; c++)
      {
        acc[c] = {A01[c].re.v.x, A01[c].im.v.x};
        acc[3 + c] = {A01[c].re.v.y, A01[c].im.v.y};
        acc[6 + c] = {A23[c].re.v.x, A23[c].im.v.x};
        acc[9 + c] = {A23[c].re.v.y, A23[c].im.v.y};
      }
  }

  constexpr int HOP_SP_THREADS = 128;

  template <int P, int LF, class Epi, class Fin>
  __global__ void __launch_bounds__(HOP_SP_THREADS)
    hop_sp_kernel(Lattice g, int par_out, int npar, SpinorT<P> in_e, SpinorT<P> in_o, LinkT<LF> U, const OpParams* prm,
                  Epi epi, Reducer red, Fin fin, const int* __restrict__ stop)
  {
    pdl_enter();
    if (stop && *stop) return;
    const int idx = blockIdx.x * HOP_SP_THREADS + threadIdx.x;
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
        C<float> acc[12];
        hop_site_sp<P, LF>(g, p, ieo, p ? in_e : in_o, U, float(prm->anis), acc);
        part = epi(p, ieo, acc);
      }
    if (Epi::kReduce) grid_reduce<HOP_SP_THREADS>(part, red, fin);
  }
}

// ---------------------------------------------------------------------------
// The same one-site packed kernel with the neighbours' data streamed into the
// thread's own shared-memory slots by cp.async, DIST directions ahead of the
// direction it computes (launch shape 6, DIST = 2).  The gather needs many loads in
// flight; in registers they cost occupancy, in shared memory they cost
// nothing while the arithmetic of the earlier directions runs.  A thread reads
// back only what it copied itself, so the only synchronisation is
// cp.async.wait_group on its own copies; a slot is refilled one direction
// after it was read (DIST + 1 slots), when the values read from it have been
// consumed by that direction's arithmetic.
#include "tms_pipe.cuh"

namespace tms
{
  constexpr int SPP_THREADS = 128;

  template <int P, int LF>
  struct SppFmt
  {
    static constexpr int KS = (P == PREC_F16) ? 3 : 6;                                 // spinor, 16-byte words
    static constexpr int HASN = (P == PREC_F16) ? 1 : 0;                               // FP16 per-site factor
    static constexpr int KL16 = (LF == LINK_F32_12) ? 3 : (LF == LINK_I16_12 || LF == LINK_H16_12) ? 1 : 0; // link, 16-byte words
    static constexpr int KL8 = (LF == LINK_I16_12 || LF == LINK_H16_12) ? 1 : (LF == LINK_F32_18) ? 9 : 0;  // link, 8-byte words
    static constexpr int W16 = KS + KL16;
    static constexpr int SLOT_BYTES = W16 * 16 + KL8 * 8 + HASN * 4;
    template <int DIST>
    static constexpr int smem() { return (DIST + 1) * SLOT_BYTES * SPP_THREADS; }
  };

  // the thread's slots: words interleaved across the block's threads
  template <int P, int LF, int SLOTS>
  struct SppSlots
  {
    using F = SppFmt<P, LF>;
    char* base;
    int tid;
    __device__ __forceinline__ uint4* w16(int slot, int k) const
    {
      return reinterpret_cast<uint4*>(base) + (slot * F::W16 + k) * SPP_THREADS + tid;
    }
    __device__ __forceinline__ uint2* w8(int slot, int k) const
    {
      return reinterpret_cast<uint2*>(base + SLOTS * F::W16 * 16 * SPP_THREADS) + (slot * F::KL8 + k) * SPP_THREADS + tid;
    }
    __device__ __forceinline__ float* nrm(int slot) const
    {
      return reinterpret_cast<float*>(base + SLOTS * (F::W16 * 16 + F::KL8 * 8) * SPP_THREADS) + slot * SPP_THREADS + tid;
    }
  };

  template <int D, int P, int LF, int SLOTS>
  __device__ __forceinline__ void spp_issue(const SppSlots<P, LF, SLOTS>& sl, int slot, const Lattice& g, const Site& s,
                                            int p, int ieo, const SpinorT<P>& in, const LinkT<LF>& U, bool& w)
  {
    using F = SppFmt<P, LF>;
    constexpr int MU = D / 2;
    constexpr bool FWD = (D % 2) == 0;
    const int n = FWD ? nbr_up<MU>(g, s, w) : nbr_dw<MU>(g, s, w);
    const int lpar = FWD ? p : 1 - p, ls = FWD ? ieo : n;
    const uint4* sp = reinterpret_cast<const uint4*>(in.d);
#pragma unroll
    for (int k = 0; k < F::KS; k++) cp_async16(sl.w16(slot, k), sp + (size_t)k * in.stride + n);
    if (F::HASN) cp_async4(sl.nrm(slot), in.n + n);
    if constexpr (LF == LINK_I16_12 || LF == LINK_H16_12)
      {
        // the 16-byte word past L1 (a link is read once), the 8-byte word through it
        cp_async16_stream(sl.w16(slot, F::KS), U.w16(lpar, MU) + ls);
        cp_async8(sl.w8(slot, 0), U.w8(lpar, MU) + ls);
      }
    else
      {
        if (F::KL16)
          {
            const uint4* b = reinterpret_cast<const uint4*>(U.d) + ((size_t)(lpar * 4 + MU) * 3) * U.Vh + ls;
#pragma unroll
            for (int k = 0; k < F::KL16; k++) cp_async16_stream(sl.w16(slot, F::KS + k), b + (size_t)k * U.Vh);
          }
        if (F::KL8)
          {
            const uint2* b = reinterpret_cast<const uint2*>(U.d) + ((size_t)(lpar * 4 + MU) * F::KL8) * U.Vh + ls;
#pragma unroll
            for (int k = 0; k < F::KL8; k++) cp_async8(sl.w8(slot, k), b + (size_t)k * U.Vh);
          }
      }
  }

  // the staged spinor (stored units and factor) and link of a slot (16-bit links:
  // raw rows, row 2 in raw^2 units; otherwise the units of LinkT::load_scaled)
  template <int P, int LF, int SLOTS>
  __device__ __forceinline__ void spp_read(const SppSlots<P, LF, SLOTS>& sl, int slot, C<float> v[12], float& ss,
                                           C<float> u[9], float& ls)
  {
    if (P == PREC_F16)
      {
        ss = *sl.nrm(slot);
#pragma unroll
        for (int k = 0; k < 3; k++)
          {
            const uint4 w = *sl.w16(slot, k);
            const unsigned q[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
            for (int j = 0; j < 4; j++)
              {
                const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&q[j]));
                v[4 * k + j] = {f.x, f.y};
              }
          }
      }
    else
      {
        ss = 1.0f;
#pragma unroll
        for (int k = 0; k < 6; k++)
          {
            const float4 f = *reinterpret_cast<const float4*>(sl.w16(slot, k));
            v[2 * k] = {f.x, f.y};
            v[2 * k + 1] = {f.z, f.w};
          }
      }
    if constexpr (LF == LINK_I16_12)
      {
        LinkT<LINK_I16_12>::decode_raw(*sl.w16(slot, SppFmt<P, LF>::KS), *sl.w8(slot, 0), u);
        row2_unscaled(u); // in raw^2 units: sp_dir_compute scales its products by k
        ls = 1.0f / 32767.0f;
      }
    else if (LF == LINK_F32_12)
      {
        constexpr int KS = SppFmt<P, LF>::KS;
#pragma unroll
        for (int r = 0; r < 3; r++)
          {
            const float4 f = *reinterpret_cast<const float4*>(sl.w16(slot, KS + r));
            u[2 * r] = {f.x, f.y};
            u[2 * r + 1] = {f.z, f.w};
          }
        u[6] = cconj(csub(cmul(u[1], u[5]), cmul(u[2], u[4])));
        u[7] = cconj(csub(cmul(u[2], u[3]), cmul(u[0], u[5])));
        u[8] = cconj(csub(cmul(u[0], u[4]), cmul(u[1], u[3])));
        ls = 1.0f;
      }
    else
      {
#pragma unroll
        for (int r = 0; r < 9; r++)
          {
            const float2 f = *reinterpret_cast<const float2*>(sl.w8(slot, r));
            u[r] = {f.x, f.y};
          }
        ls = 1.0f;
      }
  }

  // One direction in FP16 arithmetic (the FP16-arithmetic hop, links LINK_H16_12):
  // the neighbour's stored half2 words w[12] ((re, im) of component spin*3 +
  // colour, in stored units) are projected in half2 arithmetic with the two
  // spin rows in the lanes, row 2 of the link is rebuilt from the FP16 rows 0
  // and 1 (complex multiply-adds on (re, im) half2), the SU(3) product runs in
  // half2 fused multiply-adds with each link element broadcast to both lanes,
  // and the result is widened to FP32 pairs and accumulated times f as in
  // sp_dir_compute.  FP16 products and sums add a rounding of 2^-11 relative to
  // the FP16 storage of the spinors (5.9e-4 from the FP32-arithmetic hop on
  // random fields at 32^3x64).
  template <int MU, bool FWD>
  __device__ __forceinline__ void hp_dir_compute(const unsigned w[12], const __half2 lr[6], float f, C<P2> A01[3],
                                                 C<P2> A23[3])
  {
    constexpr bool CROSS = (MU == 1 || MU == 2);
    const __half2 pm = __floats2half2_rn(1.f, -1.f), mp = __floats2half2_rn(-1.f, 1.f);
    __half2 Hre[3], Him[3];
#pragma unroll
    for (int c = 0; c < 3; c++)
      {
        const __half2 s0 = *reinterpret_cast<const __half2*>(&w[c]), s1 = *reinterpret_cast<const __half2*>(&w[3 + c]);
        const __half2 s2 = *reinterpret_cast<const __half2*>(&w[6 + c]), s3 = *reinterpret_cast<const __half2*>(&w[9 + c]);
        const __half2 are = __lows2half2(s0, s1), aim = __highs2half2(s0, s1);
        const __half2 bre = CROSS ? __lows2half2(s3, s2) : __lows2half2(s2, s3);
        const __half2 bim = CROSS ? __highs2half2(s3, s2) : __highs2half2(s2, s3);
        if (MU == 0)
          {
            Hre[c] = FWD ? __hadd2(are, bre) : __hsub2(are, bre);
            Him[c] = FWD ? __hadd2(aim, bim) : __hsub2(aim, bim);
          }
        if (MU == 1)
          {
            Hre[c] = FWD ? __hsub2(are, bim) : __hadd2(are, bim);
            Him[c] = FWD ? __hadd2(aim, bre) : __hsub2(aim, bre);
          }
        if (MU == 2)
          {
            Hre[c] = __hfma2(FWD ? pm : mp, bre, are);
            Him[c] = __hfma2(FWD ? pm : mp, bim, aim);
          }
        if (MU == 3)
          {
            Hre[c] = __hfma2(FWD ? mp : pm, bim, are);
            Him[c] = __hfma2(FWD ? pm : mp, bre, aim);
          }
      }
    // row 2 = conj(row0 x row1)
    const __half2 cj = __floats2half2_rn(1.f, -1.f), zero = __float2half2_rn(0.f);
    __half2 L[9];
#pragma unroll
    for (int k = 0; k < 6; k++) L[k] = lr[k];
    L[6] = __hmul2(cj, __hcmadd(lr[1], lr[5], __hneg2(__hcmadd(lr[2], lr[4], zero))));
    L[7] = __hmul2(cj, __hcmadd(lr[2], lr[3], __hneg2(__hcmadd(lr[0], lr[5], zero))));
    L[8] = __hmul2(cj, __hcmadd(lr[0], lr[4], __hneg2(__hcmadd(lr[1], lr[3], zero))));
    // forward: re += er hr - ei hi, im += er hi + ei hr; backward (U^+): re += er hr + ei hi, im += er hi - ei hr
    C<P2> u[3];
#pragma unroll
    for (int i = 0; i < 3; i++)
      {
        __half2 ure, uim;
#pragma unroll
        for (int j = 0; j < 3; j++)
          {
            const __half2 e = FWD ? L[3 * i + j] : L[3 * j + i];
            const __half2 er = __low2half2(e), ei = __high2half2(e);
            if (j == 0)
              {
                ure = __hmul2(er, Hre[j]);
                uim = __hmul2(er, Him[j]);
              }
            else
              {
                ure = __hfma2(er, Hre[j], ure);
                uim = __hfma2(er, Him[j], uim);
              }
            ure = __hfma2(FWD ? __hneg2(ei) : ei, Him[j], ure);
            uim = __hfma2(FWD ? ei : __hneg2(ei), Hre[j], uim);
          }
        u[i].re = P2{__half22float2(ure)};
        u[i].im = P2{__half22float2(uim)};
      }
    const P2 F = bcast(f), NF = bcast(-f), Fpm = p2(f, -f), Fmp = p2(-f, f);
#pragma unroll
    for (int c = 0; c < 3; c++)
      {
        A01[c].re = fma2(F, u[c].re, A01[c].re);
        A01[c].im = fma2(F, u[c].im, A01[c].im);
        C<P2>& A = A23[c];
        const C<P2> v = u[c];
        if (MU == 0)
          {
            A.re = fma2(FWD ? F : NF, v.re, A.re);
            A.im = fma2(FWD ? F : NF, v.im, A.im);
          }
        if (MU == 3)
          {
            A.re = fma2(FWD ? Fpm : Fmp, v.im, A.re);
            A.im = fma2(FWD ? Fmp : Fpm, v.re, A.im);
          }
        if (MU == 1)
          {
            const float sg = FWD ? f : -f;
            A.re.v.x = fmaf(sg, v.im.v.y, A.re.v.x);
            A.im.v.x = fmaf(-sg, v.re.v.y, A.im.v.x);
            A.re.v.y = fmaf(sg, v.im.v.x, A.re.v.y);
            A.im.v.y = fmaf(-sg, v.re.v.x, A.im.v.y);
          }
        if (MU == 2)
          {
            const float sg = FWD ? f : -f;
            A.re.v.x = fmaf(-sg, v.re.v.y, A.re.v.x);
            A.im.v.x = fmaf(-sg, v.im.v.y, A.im.v.x);
            A.re.v.y = fmaf(sg, v.re.v.x, A.re.v.y);
            A.im.v.y = fmaf(sg, v.im.v.x, A.im.v.y);
          }
      }
  }

  template <int D, int P, int LF, int SLOTS>
  __device__ __forceinline__ void spp_compute(const SppSlots<P, LF, SLOTS>& sl, const Lattice& g, bool w, float anis,
                                              C<P2> A01[3], C<P2> A23[3])
  {
    constexpr int MU = D / 2;
    const float fmu = MU ? anis : 1.0f;
    if constexpr (LF == LINK_H16_12)
      {
        // FP16 spinor words and FP16 link rows straight from the slot
        const int slot = D % SLOTS;
        unsigned sw[12];
#pragma unroll
        for (int k = 0; k < 3; k++)
          {
            const uint4 x = *sl.w16(slot, k);
            sw[4 * k] = x.x;
            sw[4 * k + 1] = x.y;
            sw[4 * k + 2] = x.z;
            sw[4 * k + 3] = x.w;
          }
        const uint4 a = *sl.w16(slot, SppFmt<P, LF>::KS);
        const uint2 b = *sl.w8(slot, 0);
        const unsigned lw[6] = {a.x, a.y, a.z, a.w, b.x, b.y};
        __half2 lr[6];
#pragma unroll
        for (int k = 0; k < 6; k++) lr[k] = *reinterpret_cast<const __half2*>(&lw[k]);
        const float f = (w ? fmu * float(g.bc_t) : fmu) * *sl.nrm(slot);
        hp_dir_compute<MU, (D % 2) == 0>(sw, lr, f, A01, A23);
      }
    else
      {
        C<float> sp[12], L[9];
        float ss, ls;
        spp_read<P, LF, SLOTS>(sl, D % SLOTS, sp, ss, L, ls);
        const float f = (w ? fmu * float(g.bc_t) : fmu) * ss * ls;
        sp_dir_compute<MU, (D % 2) == 0, LF == LINK_I16_12>(sp, L, f, A01, A23, 1.0f / 32767.0f);
      }
  }

  // an FP16 field at site `site` into a slot's spinor words (an epilogue operand)
  template <int P, int LF, int SLOTS>
  __device__ __forceinline__ void spp_stage(const SppSlots<P, LF, SLOTS>& sl, int slot, const SpinorT<P>& f, int site)
  {
    const uint4* sp = reinterpret_cast<const uint4*>(f.d);
#pragma unroll
    for (int k = 0; k < 3; k++) cp_async16(sl.w16(slot, k), sp + (size_t)k * f.stride + site);
    cp_async4(sl.nrm(slot), f.n + site);
  }

  // The loader an epilogue gets from the pipelined hop: operand k < n is read
  // from slot (8 + k) % SLOTS, where the hop staged it (the same arithmetic as
  // SpinorT<PREC_F16>::load), any other from global memory.
  template <int P, int LF, int SLOTS>
  struct SppStagedLoad
  {
    SppSlots<P, LF, SLOTS> sl;
    int n;
    template <int Q>
    __device__ __forceinline__ void operator()(int k, const SpinorT<Q>& f, int site,
                                               C<typename SpinorT<Q>::R> v[12]) const
    {
      if constexpr (Q == PREC_F16)
        if (k < n)
          {
            const int slot = (8 + k) % SLOTS;
            const float s = *sl.nrm(slot);
#pragma unroll
            for (int w = 0; w < 3; w++)
              {
                const uint4 x = *sl.w16(slot, w);
                const unsigned u[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
                for (int j = 0; j < 4; j++)
                  {
                    const float2 h = __half22float2(*reinterpret_cast<const __half2*>(&u[j]));
                    v[4 * w + j] = {h.x * s, h.y * s};
                  }
              }
            return;
          }
      f.load(site, v);
    }
  };

  // the hop of site (p, ieo) with the thread's gathers pipelined through its
  // slots of `smem` (SppFmt::smem<DIST>() bytes for the block), in the
  // accumulator layout of hop_site.  With nstaged > 0 (at most DIST), the
  // FP16 fields staged[k] at the site itself are copied into the slots freed
  // by the last directions (for the epilogue: SppStagedLoad), and have landed
  // on return.
  template <int P, int LF, int DIST, int NSTAGED = 0>
  __device__ __forceinline__ void spp_hop_site(char* smem, const Lattice& g, int p, int ieo, const SpinorT<P>& in,
                                               const LinkT<LF>& U, float anis, C<float> acc[12],
                                               const SpinorT<P>* staged = nullptr)
  {
    static_assert(NSTAGED <= DIST && (NSTAGED == 0 || P == PREC_F16), "operands staged in the free slots");
    constexpr int SLOTS = DIST + 1;
    const SppSlots<P, LF, SLOTS> sl{smem, (int)(threadIdx.x % SPP_THREADS)};
    const Site s = eo_site(g, p, ieo);
    C<P2> A01[3], A23[3];
#pragma unroll
    for (int c = 0; c < 3; c++)
      {
        A01[c] = {p2(0.f, 0.f), p2(0.f, 0.f)};
        A23[c] = {p2(0.f, 0.f), p2(0.f, 0.f)};
      }
    bool w[8];
    // the copies of the first DIST directions, one commit group each
#define TMS_SPP_ISSUE(D)                                                                                           \
  if ((D) < 8) spp_issue<((D) < 8 ? (D) : 0), P, LF, SLOTS>(sl, (D) % SLOTS, g, s, p, ieo, in, U, w[(D) < 8 ? (D) : 0]); \
  else if ((D) - 8 < NSTAGED) spp_stage(sl, (D) % SLOTS, staged[(D) >= 8 ? (D) - 8 : 0], ieo);                  \
  cp_async_commit();
#define TMS_SPP_STEP(D)                                                                                            \
  TMS_SPP_ISSUE((D) + DIST)                                                                                        \
  cp_async_wait<DIST>();                                                                                           \
  spp_compute<D, P, LF, SLOTS>(sl, g, w[D], anis, A01, A23);
    TMS_SPP_ISSUE(0)
    if (DIST > 1) { TMS_SPP_ISSUE(1) }
    if (DIST > 2) { TMS_SPP_ISSUE(2) }
    TMS_SPP_STEP(0)
    TMS_SPP_STEP(1)
    TMS_SPP_STEP(2)
    TMS_SPP_STEP(3)
    TMS_SPP_STEP(4)
    TMS_SPP_STEP(5)
    TMS_SPP_STEP(6)
    TMS_SPP_STEP(7)
#undef TMS_SPP_STEP
#undef TMS_SPP_ISSUE
    if (NSTAGED > 0) cp_async_wait<0>();
#pragma unroll
    for (int c = 0; c < 3; c++)
      {
        acc[c] = {A01[c].re.v.x, A01[c].im.v.x};
        acc[3 + c] = {A01[c].re.v.y, A01[c].im.v.y};
        acc[6 + c] = {A23[c].re.v.x, A23[c].im.v.x};
        acc[9 + c] = {A23[c].re.v.y, A23[c].im.v.y};
      }
  }

  template <int P, int LF, class Epi, class Fin, int DIST, int MINB = 1>
  __global__ void __launch_bounds__(SPP_THREADS, MINB)
    hop_spp_kernel(Lattice g, int par_out, int npar, SpinorT<P> in_e, SpinorT<P> in_o, LinkT<LF> U,
                   const OpParams* prm, Epi epi, Reducer red, Fin fin, const int* __restrict__ stop)
  {
    extern __shared__ __align__(16) char spp_smem[];
    pdl_enter();
    if (stop && *stop) return;
    const int idx = blockIdx.x * SPP_THREADS + threadIdx.x;
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
        C<float> acc[12];
        // the epilogue's FP16 operands ride in the slots the last directions free
        constexpr int NS = (P == PREC_F16) ? (EpiStaged<Epi>::n < DIST ? EpiStaged<Epi>::n : DIST) : 0;
        if constexpr (NS > 0)
          {
            SpinorT<P> stg[NS];
#pragma unroll
            for (int k = 0; k < NS; k++) stg[k] = epi.staged(p, k);
            spp_hop_site<P, LF, DIST, NS>(spp_smem, g, p, ieo, p ? in_e : in_o, U, float(prm->anis), acc, stg);
            part = epi.run(p, ieo, acc,
                           SppStagedLoad<P, LF, DIST + 1>{{spp_smem, (int)(threadIdx.x % SPP_THREADS)}, NS});
          }
        else
          {
            spp_hop_site<P, LF, DIST>(spp_smem, g, p, ieo, p ? in_e : in_o, U, float(prm->anis), acc);
            part = epi(p, ieo, acc);
          }
      }
    if (Epi::kReduce) grid_reduce<SPP_THREADS>(part, red, fin);
  }
}
