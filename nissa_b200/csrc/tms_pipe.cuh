// Low-precision hopping kernel with an asynchronous-copy pipeline.
//
// The FP32-arithmetic hops (FP16 and FP32 spinors, 16-bit or FP32 links) are
// bound by memory latency once their instruction count is halved by packing
// two sites per thread (hop2_kernel): each warp waits on the gathers of the
// eight neighbours.  Here every thread streams the neighbour spinors and links
// of its two sites (t and t+T/2) into its own slots of shared memory with
// cp.async, three directions (FP32 spinors: two) ahead of the one it computes,
// so that those loads are in flight without holding registers.  A thread
// reads back only what it copied itself: the only synchronisation is
// cp.async.wait_group on its own copies.  A slot is refilled one direction
// after it was last read (one slot more than the directions in flight): its
// shared-memory reads were issued a whole direction of arithmetic before the
// copy that overwrites it, whose write lands only after a global round trip.
#pragma once

#include "tms_kernels.cuh"

namespace tms
{
  constexpr int PIPE_THREADS = 128;

  // staged words per site and direction
  template <int P, int LF>
  struct PipeFmt
  {
    static constexpr int KS16 = (P == PREC_F16) ? 3 : 6;                                 // spinor, 16-byte words
    static constexpr int HASN = (P == PREC_F16) ? 1 : 0;                                 // FP16 per-site factor
    static constexpr int KL16 = (LF == LINK_F32_12) ? 3 : (LF == LINK_I16_12) ? 1 : 0;   // link, 16-byte words
    static constexpr int KL8 = (LF == LINK_I16_12) ? 1 : (LF == LINK_F32_18) ? 9 : 0;    // link, 8-byte words
    static constexpr int W16 = KS16 + KL16;
    // directions in flight + 1 (fewer for FP32 spinors, to keep two blocks per SM)
    static constexpr int SLOTS = (P == PREC_F16) ? 4 : 3;
    static constexpr int SITE_BYTES = W16 * 16 + KL8 * 8 + HASN * 4;
    static constexpr int SMEM = SLOTS * 2 * SITE_BYTES * PIPE_THREADS;
  };

  __device__ __forceinline__ void cp_async16(void* s, const void* g)
  {
    const unsigned a = (unsigned)__cvta_generic_to_shared(s);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(a), "l"(g) : "memory");
  }
  __device__ __forceinline__ void cp_async16_stream(void* s, const void* g)
  {
    const unsigned a = (unsigned)__cvta_generic_to_shared(s);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(a), "l"(g) : "memory");
  }
  __device__ __forceinline__ void cp_async8(void* s, const void* g)
  {
    const unsigned a = (unsigned)__cvta_generic_to_shared(s);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(a), "l"(g) : "memory");
  }
  __device__ __forceinline__ void cp_async4(void* s, const void* g)
  {
    const unsigned a = (unsigned)__cvta_generic_to_shared(s);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(a), "l"(g) : "memory");
  }
  __device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
  template <int N>
  __device__ __forceinline__ void cp_async_wait()
  {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
  }

  // the thread's slots in dynamic shared memory
  template <int P, int LF>
  struct PipeSmem
  {
    using F = PipeFmt<P, LF>;
    uint4* s16; // [SLOTS][2][W16][NT]
    uint2* s8;  // [SLOTS][2][KL8][NT]
    float* sn;  // [SLOTS][2][NT]
    int tid;
    __device__ __forceinline__ uint4* w16(int slot, int j, int k) const
    {
      return s16 + ((slot * 2 + j) * F::W16 + k) * PIPE_THREADS + tid;
    }
    __device__ __forceinline__ uint2* w8(int slot, int j, int k) const
    {
      return s8 + ((slot * 2 + j) * F::KL8 + k) * PIPE_THREADS + tid;
    }
    __device__ __forceinline__ float* nrm(int slot, int j) const { return sn + (slot * 2 + j) * PIPE_THREADS + tid; }
  };

  // issue the copies of direction D (mu = D/2, forward for even D) into `slot`
  template <int D, int P, int LF>
  __device__ __forceinline__ void pipe_issue(const PipeSmem<P, LF>& sm, int slot, const Lattice& g, const Site& s,
                                             int p, int ieo, int hv, const SpinorT<P>& in, const LinkT<LF>& U)
  {
    using F = PipeFmt<P, LF>;
    constexpr int MU = D / 2;
    constexpr bool FWD = (D % 2) == 0;
    bool w;
    const int na = FWD ? nbr_up<MU>(g, s, w) : nbr_dw<MU>(g, s, w);
    const int nb = partner(na, hv);
    const int lpar = FWD ? p : 1 - p;
#pragma unroll
    for (int j = 0; j < 2; j++)
      {
        const int n = j ? nb : na;
        const int ls = FWD ? (j ? ieo + hv : ieo) : n;
        const uint4* sp = reinterpret_cast<const uint4*>(in.d);
#pragma unroll
        for (int k = 0; k < F::KS16; k++) cp_async16(sm.w16(slot, j, k), sp + (size_t)k * in.stride + n);
        if (F::HASN) cp_async4(sm.nrm(slot, j), in.n + n);
        if constexpr (LF == LINK_I16_12)
          {
            cp_async16_stream(sm.w16(slot, j, F::KS16), U.w16(lpar, MU) + ls);
            cp_async8(sm.w8(slot, j, 0), U.w8(lpar, MU) + ls);
          }
        else
          {
            if (F::KL16)
              {
                const uint4* b = reinterpret_cast<const uint4*>(U.d) + ((size_t)(lpar * 4 + MU) * 3) * U.Vh + ls;
#pragma unroll
                for (int k = 0; k < F::KL16; k++)
                  cp_async16_stream(sm.w16(slot, j, F::KS16 + k), b + (size_t)k * U.Vh);
              }
            if (F::KL8)
              {
                const uint2* b = reinterpret_cast<const uint2*>(U.d) + ((size_t)(lpar * 4 + MU) * F::KL8) * U.Vh + ls;
#pragma unroll
                for (int k = 0; k < F::KL8; k++) cp_async8(sm.w8(slot, j, k), b + (size_t)k * U.Vh);
              }
          }
      }
  }

  // spinor of site j of a slot, in stored units, and its factor
  template <int P, int LF>
  __device__ __forceinline__ void pipe_spinor(const PipeSmem<P, LF>& sm, int slot, int j, C<float> v[12], float& scale)
  {
    using F = PipeFmt<P, LF>;
    if (P == PREC_F16)
      {
        scale = *sm.nrm(slot, j);
#pragma unroll
        for (int k = 0; k < 3; k++)
          {
            const uint4 w = *sm.w16(slot, j, k);
            const unsigned u[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
            for (int q = 0; q < 4; q++)
              {
                const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&u[q]));
                v[4 * k + q] = {f.x, f.y};
              }
          }
      }
    else
      {
        scale = 1.0f;
#pragma unroll
        for (int k = 0; k < F::KS16; k++)
          {
            const float4 w = *reinterpret_cast<const float4*>(sm.w16(slot, j, k));
            v[2 * k] = {w.x, w.y};
            v[2 * k + 1] = {w.z, w.w};
          }
      }
  }

  // stored rows of the link of site j of a slot (2 rows for the 12-real formats)
  template <int P, int LF>
  __device__ __forceinline__ void pipe_link_rows(const PipeSmem<P, LF>& sm, int slot, int j, C<float> u[9])
  {
    using F = PipeFmt<P, LF>;
    if (LF == LINK_F32_12)
      {
#pragma unroll
        for (int k = 0; k < 3; k++)
          {
            const float4 w = *reinterpret_cast<const float4*>(sm.w16(slot, j, F::KS16 + k));
            u[2 * k] = {w.x, w.y};
            u[2 * k + 1] = {w.z, w.w};
          }
      }
    else if constexpr (LF == LINK_I16_12)
      LinkT<LINK_I16_12>::decode_raw(*sm.w16(slot, j, F::KS16), *sm.w8(slot, j, 0), u);
    else
      {
#pragma unroll
        for (int k = 0; k < 9; k++)
          {
            const float2 w = *reinterpret_cast<const float2*>(sm.w8(slot, j, k));
            u[k] = {w.x, w.y};
          }
      }
  }

  template <int D, int P, int LF>
  __device__ __forceinline__ void pipe_compute(const PipeSmem<P, LF>& sm, int slot, const Lattice& g, const Site& s,
                                               float anis, C<P2> acc[12])
  {
    constexpr int MU = D / 2;
    constexpr bool FWD = (D % 2) == 0;
    constexpr int NR = LinkT<LF>::kRows;
    const float fmu = (MU > 0) ? anis : 1.0f;
    // time-boundary crossings: the first site (t < T/2) only backward from t = 0,
    // the second (t + T/2) only forward from t = T-1
    const bool wa = (MU == 0) && !FWD && (s.t == 0);
    const bool wb = (MU == 0) && FWD && (s.t == (g.T >> 1) - 1);
    C<P2> sp[12], h0[3], h1[3], u0[3], u1[3], L[9];
    float sa, sb;
    {
      C<float> a[12], b[12];
      pipe_spinor(sm, slot, 0, a, sa);
      pipe_spinor(sm, slot, 1, b, sb);
#pragma unroll
      for (int c = 0; c < 12; c++) sp[c] = zip(a[c], b[c]);
    }
    project<MU, FWD>(sp, h0, h1);
    {
      C<float> a[9], b[9];
      pipe_link_rows(sm, slot, 0, a);
      pipe_link_rows(sm, slot, 1, b);
#pragma unroll
      for (int k = 0; k < 3 * NR; k++) L[k] = zip(a[k], b[k]);
    }
    if (NR == 2)
      {
        L[6] = row2_elem(L[1], L[2], L[4], L[5]);
        L[7] = row2_elem(L[2], L[0], L[5], L[3]);
        L[8] = row2_elem(L[0], L[1], L[3], L[4]);
        if (LinkT<LF>::kUnit != 1.0f)
          {
            const P2 unit = p2(LinkT<LF>::kUnit, LinkT<LF>::kUnit);
#pragma unroll
            for (int k = 6; k < 9; k++) L[k] = {L[k].re * unit, L[k].im * unit};
          }
      }
    const float fbc = fmu * float(g.bc_t);
    const float k = LinkT<LF>::kUnit;
    const P2 f = p2((wa ? fbc : fmu) * sa * k, (wb ? fbc : fmu) * sb * k);
    link_mul2<FWD>(L, h0, u0);
    link_mul2<FWD>(L, h1, u1);
    reconstruct2<MU, FWD>(acc, u0, u1, f);
  }

  // copies of directions 0 .. S-2 into slots 0 .. S-2
  template <int D, int S, int P, int LF>
  __device__ __forceinline__ void pipe_prologue(const PipeSmem<P, LF>& sm, const Lattice& g, const Site& s, int p,
                                                int ieo, int hv, const SpinorT<P>& in, const LinkT<LF>& U)
  {
    if constexpr (D < S - 1)
      {
        pipe_issue<D>(sm, D, g, s, p, ieo, hv, in, U);
        cp_async_commit();
        pipe_prologue<D + 1, S>(sm, g, s, p, ieo, hv, in, U);
      }
  }

  // direction D: wait for its copies (those of later directions may stay in
  // flight), compute it, then issue direction D+S-1 into the slot that
  // direction D-1 used
  template <int D, int S, int P, int LF>
  __device__ __forceinline__ void pipe_steps(const PipeSmem<P, LF>& sm, const Lattice& g, const Site& s, int p, int ieo,
                                             int hv, const SpinorT<P>& in, const LinkT<LF>& U, float anis,
                                             C<P2> acc[12])
  {
    if constexpr (D < 8)
      {
        constexpr int pending = (7 - D < S - 2) ? 7 - D : S - 2;
        cp_async_wait<pending>();
        pipe_compute<D>(sm, D % S, g, s, anis, acc);
        if constexpr (D + S - 1 < 8)
          {
            pipe_issue<D + S - 1>(sm, (D + S - 1) % S, g, s, p, ieo, hv, in, U);
            cp_async_commit();
          }
        pipe_steps<D + 1, S>(sm, g, s, p, ieo, hv, in, U, anis, acc);
      }
  }

  template <int P, int LF, class Epi, class Fin>
  __global__ void __launch_bounds__(PIPE_THREADS, 2)
    hop_pipe_kernel(Lattice g, int par_out, int npar, SpinorT<P> in_e, SpinorT<P> in_o, LinkT<LF> U,
                    const OpParams* prm, Epi epi, Reducer red, Fin fin, const int* __restrict__ stop)
  {
    using F = PipeFmt<P, LF>;
    extern __shared__ __align__(16) unsigned char pipe_smem[];
    pdl_enter();
    if (stop && *stop) return;
    const int hv = (int)(g.Vh >> 1);
    const int idx = blockIdx.x * PIPE_THREADS + threadIdx.x;
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
        PipeSmem<P, LF> sm;
        sm.s16 = reinterpret_cast<uint4*>(pipe_smem);
        sm.s8 = reinterpret_cast<uint2*>(sm.s16 + F::SLOTS * 2 * F::W16 * PIPE_THREADS);
        sm.sn = reinterpret_cast<float*>(sm.s8 + F::SLOTS * 2 * F::KL8 * PIPE_THREADS);
        sm.tid = threadIdx.x;
        const Site s = eo_site(g, p, ieo);
        const SpinorT<P> in = p ? in_e : in_o;
        const float anis = float(prm->anis);
        C<P2> acc[12];
#pragma unroll
        for (int c = 0; c < 12; c++) acc[c] = {p2(0.f, 0.f), p2(0.f, 0.f)};
        pipe_prologue<0, F::SLOTS>(sm, g, s, p, ieo, hv, in, U);
        pipe_steps<0, F::SLOTS>(sm, g, s, p, ieo, hv, in, U, anis, acc);
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
    if (Epi::kReduce) grid_reduce<PIPE_THREADS>(part, red, fin);
  }
}
