// The e/o hopping kernel with its neighbour faces staged in shared memory by
// bulk asynchronous copies (launch shape 7 of the FP32-arithmetic hops).
//
// The one-thread-per-site kernels gather eight neighbour spinors and eight
// links per site straight from global memory; their loads in flight are
// bounded by the registers of the resident warps, and the low-precision hops
// stall on that latency (long-scoreboard stalls dominate once the packed-FP32
// arithmetic has cut the instruction count).  Here a CTA owns a tile of R
// consecutive rows of one (t, x) plane of output sites (a row: the LZ/2 sites
// of one parity at fixed t, x, y, consecutive in the e/o numbering), and one
// warp issues, before any arithmetic, bulk copies global -> shared
// (cp.async.bulk, completion counted on one mbarrier) of everything the tile
// reads:
//   * the input field on the tile's rows of the same plane with one halo row
//     above and below (the z and y neighbours; the whole plane when R = LY),
//   * the input field on the tile's rows of the planes (t, x+-1) and (t+-1, x)
//     (the x and t neighbours: same rows, same positions),
//   * the 12 forward link planes of the tile's own sites, and the backward
//     links of the neighbours: the same rows of the other parity (z), the rows
//     shifted by one (y) and the tile's rows of the planes (t, x-1), (t-1, x).
// Every copy is a contiguous run of whole rows of one component plane, so
// its global and shared addresses and its size are multiples of 16 bytes
// when LZ is a multiple of 8 (the FP16 per-site scales are 4 bytes a site).
// The copies of a tile are in flight together without registers, and
// several CTAs per SM overlap one tile's copies with another's arithmetic.
// The arithmetic is that of tms_hop_sp.cuh (spin rows in packed FP32 lanes),
// reading the gathered data from shared memory.
//
// Waits on the mbarrier are bounded: after kTmaWaitLimit polls the CTA
// counts a timeout in the caller's device word TmaGeom::timeouts, waits once
// more (bounded) for its copies still in flight, and returns without writing
// its outputs.
#pragma once

#include "tms_hop_sp.cuh"

namespace tms
{
  constexpr int HOP_TMA_THREADS = 128;
  constexpr long kTmaWaitLimit = 1L << 22;

  // tile geometry: h sites per row, R rows per tile (R divides LY), ns = R*h <= HOP_TMA_THREADS
  struct TmaGeom
  {
    int h, R, ns, LY, NP;  // NP = LY*h sites per (t, x) plane
    int full;              // R == LY: the whole plane, no halo rows
    int nc;                // centre slots: (R + 2) h, or NP when full
    unsigned* timeouts;    // device counter of timed-out tile waits (stays 0 unless a copy never lands)
  };

  // component planes of a field in the shared-memory staging: count, bytes
  // per site of each, and the base of component c in global memory
  template <int P> struct StageSp;
  template <> struct StageSp<PREC_F16>
  {
    static constexpr int NC = 4;
    static constexpr int kBytes = 52;
    __device__ static int es(int c) { return c < 3 ? 16 : 4; }
    __device__ static const char* src(const SpinorT<PREC_F16>& f, int c)
    {
      return c < 3 ? reinterpret_cast<const char*>(f.d + (size_t)c * f.stride) : reinterpret_cast<const char*>(f.n);
    }
    // the stored halves of slot q (components at base + offsets of an nslots-long buffer) and their scale
    __device__ static void load(const char* base, int nslots, int q, C<float> v[12], float& scale)
    {
      const uint4* w = reinterpret_cast<const uint4*>(base);
      scale = reinterpret_cast<const float*>(base + (size_t)nslots * 48)[q];
#pragma unroll
      for (int k = 0; k < 3; k++)
        {
          const uint4 x = w[k * nslots + q];
          const unsigned u[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
          for (int j = 0; j < 4; j++)
            {
              __half2 hh = *reinterpret_cast<const __half2*>(&u[j]);
              const float2 f = __half22float2(hh);
              v[4 * k + j] = {f.x, f.y};
            }
        }
    }
  };
  template <> struct StageSp<PREC_F32>
  {
    static constexpr int NC = 6;
    static constexpr int kBytes = 96;
    __device__ static int es(int) { return 16; }
    __device__ static const char* src(const SpinorT<PREC_F32>& f, int c)
    {
      return reinterpret_cast<const char*>(f.d + (size_t)c * f.stride);
    }
    __device__ static void load(const char* base, int nslots, int q, C<float> v[12], float& scale)
    {
      const float4* w = reinterpret_cast<const float4*>(base);
      scale = 1.0f;
#pragma unroll
      for (int k = 0; k < 6; k++)
        {
          const float4 x = w[k * nslots + q];
          v[2 * k] = {x.x, x.y};
          v[2 * k + 1] = {x.z, x.w};
        }
    }
  };

  template <int LF> struct StageLk;
  template <> struct StageLk<LINK_I16_12>
  {
    static constexpr int NC = 2;  // planes per (parity, direction): the 16-byte and the 8-byte word
    static constexpr int KB = 24; // bytes per site of all planes
    __device__ static int es(int c) { return c ? 8 : 16; }
    __device__ static int off(int c) { return c ? 16 : 0; } // bytes per site before plane c
    __device__ static const char* src(const LinkT<LINK_I16_12>& U, int par, int mu, int c)
    {
      return c ? reinterpret_cast<const char*>(U.w8(par, mu)) : reinterpret_cast<const char*>(U.w16(par, mu));
    }
    // the link of slot q: raw rows 0 and 1, row 2 rebuilt in raw^2 units
    __device__ static void load(const char* base, int nslots, int q, C<float> u[9], float& scale)
    {
      LinkT<LINK_I16_12>::decode_raw(reinterpret_cast<const uint4*>(base)[q],
                                     reinterpret_cast<const uint2*>(base + (size_t)16 * nslots)[q], u);
      row2_unscaled(u); // raw^2 units: the arithmetic scales row 2's products by k
      scale = 1.0f / 32767.0f;
    }
  };
  template <> struct StageLk<LINK_F32_12>
  {
    static constexpr int NC = 3;
    static constexpr int KB = 48;
    __device__ static int es(int) { return 16; }
    __device__ static int off(int c) { return 16 * c; }
    __device__ static const char* src(const LinkT<LINK_F32_12>& U, int par, int mu, int c)
    {
      return reinterpret_cast<const char*>(U.d + ((size_t)(par * 4 + mu) * 3 + c) * U.Vh);
    }
    __device__ static void load(const char* base, int nslots, int q, C<float> u[9], float& scale)
    {
      const float4* b = reinterpret_cast<const float4*>(base);
      const float4 a0 = b[q], a1 = b[nslots + q], a2 = b[2 * nslots + q];
      u[0] = {a0.x, a0.y};
      u[1] = {a0.z, a0.w};
      u[2] = {a1.x, a1.y};
      u[3] = {a1.z, a1.w};
      u[4] = {a2.x, a2.y};
      u[5] = {a2.z, a2.w};
      u[6] = cconj(csub(cmul(u[1], u[5]), cmul(u[2], u[4])));
      u[7] = cconj(csub(cmul(u[2], u[3]), cmul(u[0], u[5])));
      u[8] = cconj(csub(cmul(u[0], u[4]), cmul(u[1], u[3])));
      scale = 1.0f;
    }
  };

  // shared-memory bytes of one tile
  template <int P, int LF>
  __host__ __device__ constexpr size_t tma_smem_bytes(int nc, int ns)
  {
    return (size_t)(nc + 4 * ns) * (P == PREC_F16 ? 52 : 96) + (size_t)8 * ns * (LF == LINK_I16_12 ? 24 : 48);
  }

  // ------------------------------------------------------------ PTX helpers
  __device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

  __device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count)
  {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  }
  __device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes)
  {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(
                   smem_u32(bar)), "r"(bytes)
                 : "memory");
  }
  __device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned phase)
  {
    unsigned ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(smem_u32(bar)), "r"(phase)
                 : "memory");
    return ok != 0;
  }
  // global -> this CTA's shared memory, completion counted in bytes on `bar`
  // (no multicast: the source is this GPU's own memory and only this CTA reads the copy)
  __device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar)
  {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
  }

  // bounded wait for phase 0 of the tile's barrier: false after a timeout
  __device__ __forceinline__ bool tile_wait(uint64_t* bar)
  {
    for (long it = 0; it < kTmaWaitLimit; it++)
      if (mbar_try_wait(bar, 0)) return true;
    return false;
  }

  // where a tile's copies go: offsets (bytes) of the staged buffers in shared memory
  template <int P, int LF>
  struct TmaLayout
  {
    int nc, ns;
    __device__ size_t centre() const { return 0; }
    // X+, X-, T+, T- (b = 0..3)
    __device__ size_t face(int b) const { return (size_t)nc * StageSp<P>::kBytes + (size_t)b * ns * StageSp<P>::kBytes; }
    // link buffers: forward mu (f = 0..3), backward mu (f = 4..7)
    __device__ size_t links(int f) const
    {
      return (size_t)(nc + 4 * ns) * StageSp<P>::kBytes + (size_t)f * ns * StageLk<LF>::KB;
    }
  };

  // The tile's copies, numbered q = 0 .. ncopies-1 (issued by the lanes of warp 0).
  //   spinor component c (NC of them): centre pieces (3, or 1 when full), X+, X-, T+, T-
  //   links: forward (mu, c) 4*NCL; backward z NCL, y 2*NCL, x NCL, t NCL
  template <int P, int LF>
  __device__ __forceinline__ int tma_ncopies(const TmaGeom& G)
  {
    return StageSp<P>::NC * ((G.full ? 1 : 3) + 4) + StageLk<LF>::NC * 9;
  }

  struct CopyDesc
  {
    size_t dst;      // byte offset in shared memory
    const char* src; // global source
    unsigned bytes;  // 0: nothing to copy
  };

  template <int P, int LF>
  __device__ __forceinline__ CopyDesc tma_desc(int q, const TmaGeom& G, const Lattice& g, int p, int t, int x, int r0,
                                               const SpinorT<P>& in, const LinkT<LF>& U)
  {
    const TmaLayout<P, LF> lay{G.nc, G.ns};
    const int h = G.h, R = G.R, LY = G.LY, NP = G.NP;
    const int plane = t * g.LX + x;
    const int nsp = (G.full ? 1 : 3) + 4;
    if (q < StageSp<P>::NC * nsp)
      {
        const int c = q / nsp, k = q % nsp;
        const int es = StageSp<P>::es(c);
        const char* base = StageSp<P>::src(in, c);
        // the offset of component c inside a staged buffer of n slots
        auto comp_off = [&](int n) {
          size_t o = 0;
          for (int cc = 0; cc < c; cc++) o += (size_t)n * StageSp<P>::es(cc);
          return o;
        };
        int src_site, nsites;
        size_t dst;
        if (k < nsp - 4)
          {
            // centre: [halo row above] [tile rows] [halo row below], or the whole plane
            const size_t cb = lay.centre() + comp_off(G.nc);
            if (G.full)
              {
                src_site = plane * NP;
                nsites = NP;
                dst = cb;
              }
            else if (k == 0)
              {
                src_site = plane * NP + ((r0 - 1 + LY) % LY) * h;
                nsites = h;
                dst = cb;
              }
            else if (k == 1)
              {
                src_site = plane * NP + r0 * h;
                nsites = R * h;
                dst = cb + (size_t)h * es;
              }
            else
              {
                src_site = plane * NP + ((r0 + R) % LY) * h;
                nsites = h;
                dst = cb + (size_t)(R + 1) * h * es;
              }
          }
        else
          {
            const int b = k - (nsp - 4); // 0 X+, 1 X-, 2 T+, 3 T-
            int tt = t, xx = x;
            if (b == 0) xx = (x + 1) % g.LX;
            if (b == 1) xx = (x - 1 + g.LX) % g.LX;
            if (b == 2) tt = (t + 1) % g.T;
            if (b == 3) tt = (t - 1 + g.T) % g.T;
            src_site = (tt * g.LX + xx) * NP + r0 * h;
            nsites = G.ns;
            dst = lay.face(b) + comp_off(G.ns);
          }
        return CopyDesc{dst, base + (size_t)src_site * es, (unsigned)(nsites * es)};
      }
    q -= StageSp<P>::NC * nsp;
    constexpr int NCL = StageLk<LF>::NC;
    const int tile0 = plane * NP + r0 * h; // first site of the tile
    int par, mu, c, src_site, nsites;
    size_t dst;
    if (q < 4 * NCL)
      {
        // forward links of the tile's own sites
        mu = q / NCL;
        c = q % NCL;
        par = p;
        src_site = tile0;
        nsites = G.ns;
        dst = lay.links(mu) + (size_t)G.ns * StageLk<LF>::off(c);
      }
    else
      {
        q -= 4 * NCL;
        par = 1 - p;
        if (q < NCL)
          {
            // z: the same rows of the other parity
            mu = 3;
            c = q;
            src_site = tile0;
            nsites = G.ns;
            dst = lay.links(4 + 3) + (size_t)G.ns * StageLk<LF>::off(c);
          }
        else if (q < 3 * NCL)
          {
            // y: slot row s holds row r0 - 1 + s (two pieces: the wrapped first row, the rest)
            mu = 2;
            q -= NCL;
            c = q >> 1;
            const size_t cb = lay.links(4 + 2) + (size_t)G.ns * StageLk<LF>::off(c);
            if ((q & 1) == 0)
              {
                src_site = plane * NP + ((r0 - 1 + LY) % LY) * h;
                nsites = h;
                dst = cb;
              }
            else
              {
                src_site = tile0;
                nsites = (R - 1) * h;
                dst = cb + (size_t)h * StageLk<LF>::es(c);
              }
          }
        else if (q < 4 * NCL)
          {
            // x: the tile's rows of plane (t, x-1)
            mu = 1;
            c = q - 3 * NCL;
            src_site = (t * g.LX + (x - 1 + g.LX) % g.LX) * NP + r0 * h;
            nsites = G.ns;
            dst = lay.links(4 + 1) + (size_t)G.ns * StageLk<LF>::off(c);
          }
        else
          {
            // t: the tile's rows of plane (t-1, x)
            mu = 0;
            c = q - 4 * NCL;
            src_site = (((t - 1 + g.T) % g.T) * g.LX + x) * NP + r0 * h;
            nsites = G.ns;
            dst = lay.links(4 + 0) + (size_t)G.ns * StageLk<LF>::off(c);
          }
      }
    const int esl = StageLk<LF>::es(c);
    return CopyDesc{dst, StageLk<LF>::src(U, par, mu, c) + (size_t)src_site * esl, (unsigned)(nsites * esl)};
  }

  // bytes the tile's copies deliver (the barrier's transaction count)
  template <int P, int LF>
  __device__ __forceinline__ unsigned tma_tile_bytes(const TmaGeom& G)
  {
    return (unsigned)((size_t)(G.nc + 4 * G.ns) * StageSp<P>::kBytes +
                      (size_t)8 * G.ns * StageLk<LF>::KB);
  }

  // one direction of the stencil from the staged data
  template <int MU, bool FWD, int P, int LF>
  __device__ __forceinline__ void tma_dir(const Lattice& g, const TmaGeom& G, const TmaLayout<P, LF>& lay,
                                          const char* sm, const Site& s, int i, int tid, int r, int r0, int j,
                                          float fmu, C<P2> A01[3], C<P2> A23[3])
  {
    bool w;
    const int n = FWD ? nbr_up<MU>(g, s, w) : nbr_dw<MU>(g, s, w);
    // the neighbour's slot in its staged buffer
    auto cslot = [&](int rr) { return G.full ? (rr + G.LY) % G.LY : rr - r0 + 1; };
    const char* sbase;
    int snslots, sq;
    if (MU == 3)
      {
        sbase = sm + lay.centre();
        snslots = G.nc;
        sq = cslot(r) * G.h + j + (n - i);
      }
    else if (MU == 2)
      {
        sbase = sm + lay.centre();
        snslots = G.nc;
        sq = cslot(FWD ? r + 1 : r - 1) * G.h + j;
      }
    else
      {
        sbase = sm + lay.face(MU == 1 ? (FWD ? 0 : 1) : (FWD ? 2 : 3));
        snslots = G.ns;
        sq = tid;
      }
    C<float> sp[12], L[9];
    float ss, ls;
    StageSp<P>::load(sbase, snslots, sq, sp, ss);
    const int lq = (!FWD && MU == 3) ? tid + (n - i) : tid;
    StageLk<LF>::load(sm + lay.links(FWD ? MU : 4 + MU), G.ns, lq, L, ls);
    const float f = (w ? fmu * float(g.bc_t) : fmu) * ss * ls;
    sp_dir_compute<MU, FWD, LF == LINK_I16_12>(sp, L, f, A01, A23, 1.0f / 32767.0f);
  }

  template <int P, int LF, class Epi, class Fin>
  __global__ void __launch_bounds__(HOP_TMA_THREADS)
    hop_tma_kernel(Lattice g, TmaGeom G, int par_out, int npar, SpinorT<P> in_e, SpinorT<P> in_o, LinkT<LF> U,
                   const OpParams* prm, Epi epi, Reducer red, Fin fin, const int* __restrict__ stop)
  {
    extern __shared__ __align__(128) char sm[];
    __shared__ uint64_t bar;
    pdl_enter();
    if (stop && *stop) return;
    // the tile: parity, plane (t, x), first row
    const int tiles_per_plane = G.LY / G.R;
    const int tiles_per_par = (int)(g.Vh / G.ns);
    int tile = blockIdx.x;
    int p = par_out;
    if (npar == 2)
      {
        p = tile >= tiles_per_par ? 1 : 0;
        tile -= p ? tiles_per_par : 0;
      }
    const int plane = tile / tiles_per_plane;
    const int r0 = (tile - plane * tiles_per_plane) * G.R;
    const int t = plane / g.LX, x = plane - t * g.LX;
    const SpinorT<P> in = p ? in_e : in_o;
    const int tid = threadIdx.x;
    const int nq = tma_ncopies<P, LF>(G);
    if (tid == 0)
      {
        mbar_init(&bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
      }
    __syncthreads();
    if (tid < 32)
      {
        if (tid == 0) mbar_arrive_expect_tx(&bar, tma_tile_bytes<P, LF>(G));
        for (int q = tid; q < nq; q += 32)
          {
            const CopyDesc d = tma_desc<P, LF>(q, G, g, p, t, x, r0, in, U);
            if (d.bytes) bulk_g2s(sm + d.dst, d.src, d.bytes, &bar);
          }
      }
    const bool ok = tile_wait(&bar);
    if (!ok)
      {
        if (tid == 0) atomicAdd(G.timeouts, 1u);
        tile_wait(&bar); // the copies still in flight land before the CTA's shared memory is released
      }
    double part = 0.0;
    if (ok && tid < G.ns)
      {
        const int i = plane * G.NP + r0 * G.h + tid;
        const int rr = tid / G.h, j = tid - rr * G.h;
        const int r = r0 + rr;
        const Site s = eo_site(g, p, i);
        const TmaLayout<P, LF> lay{G.nc, G.ns};
        const float anis = float(prm->anis);
        C<P2> A01[3], A23[3];
#pragma unroll
        for (int c = 0; c < 3; c++)
          {
            A01[c] = {p2(0.f, 0.f), p2(0.f, 0.f)};
            A23[c] = {p2(0.f, 0.f), p2(0.f, 0.f)};
          }
        tma_dir<0, true, P, LF>(g, G, lay, sm, s, i, tid, r, r0, j, 1.0f, A01, A23);
        tma_dir<0, false, P, LF>(g, G, lay, sm, s, i, tid, r, r0, j, 1.0f, A01, A23);
        tma_dir<1, true, P, LF>(g, G, lay, sm, s, i, tid, r, r0, j, anis, A01, A23);
        tma_dir<1, false, P, LF>(g, G, lay, sm, s, i, tid, r, r0, j, anis, A01, A23);
        tma_dir<2, true, P, LF>(g, G, lay, sm, s, i, tid, r, r0, j, anis, A01, A23);
        tma_dir<2, false, P, LF>(g, G, lay, sm, s, i, tid, r, r0, j, anis, A01, A23);
        tma_dir<3, true, P, LF>(g, G, lay, sm, s, i, tid, r, r0, j, anis, A01, A23);
        tma_dir<3, false, P, LF>(g, G, lay, sm, s, i, tid, r, r0, j, anis, A01, A23);
        C<float> acc[12];
#pragma unroll
        for (int c = 0; c < 3; c++)
          {
            acc[c] = {A01[c].re.v.x, A01[c].im.v.x};
            acc[3 + c] = {A01[c].re.v.y, A01[c].im.v.y};
            acc[6 + c] = {A23[c].re.v.x, A23[c].im.v.x};
            acc[9 + c] = {A23[c].re.v.y, A23[c].im.v.y};
          }
        part = epi(p, i, acc);
      }
    if (Epi::kReduce) grid_reduce<HOP_TMA_THREADS>(part, red, fin);
  }

  // a row count R the staged kernel can tile a (t, x) plane with: R divides LY,
  // R LZ/2 sites fit the CTA, and a partial plane leaves room for its two halo
  // rows and holds at least 16 sites (at most V/16 tiles: the reduction's capacity)
  inline bool tma_rows_ok(const Lattice& g, int R)
  {
    return R >= 1 && g.LZ % 8 == 0 && g.LZ / 2 <= 64 && g.LY % R == 0 && R * (g.LZ / 2) <= HOP_TMA_THREADS &&
           (R == g.LY || (R + 2 <= g.LY && R * (g.LZ / 2) >= 16));
  }

  // the tile shape for a lattice, or ns = 0 when the staged kernel does not apply
  // (LZ not a multiple of 8 or above 128, or no row count R dividing LY with R*LZ/2 <= the threads);
  // rows > 0 asks for that many rows per tile (the site tiling), 0 for the most that fit
  inline TmaGeom tma_geom(const Lattice& g, unsigned* timeouts, int rows = 0)
  {
    TmaGeom G{};
    G.timeouts = timeouts;
    G.h = g.LZ / 2;
    G.LY = g.LY;
    G.NP = g.LY * G.h;
    if (g.LZ % 8 != 0 || G.h > 64) return G;
    if (rows > 0 && tma_rows_ok(g, rows)) G.R = rows;
    else
      for (int R = g.LY; R >= 1; R--)
        if (tma_rows_ok(g, R))
          {
            G.R = R;
            break;
          }
    if (G.R == 0) return G;
    G.ns = G.R * G.h;
    G.full = (G.R == g.LY);
    G.nc = G.full ? G.NP : (G.R + 2) * G.h;
    return G;
  }
}
