// Shared device types for the B200 twisted-mass Wilson solver.
//
// Data layout in HBM (structure of arrays, one plane per complex component so
// that a warp reads 32 consecutive sites of one component as a contiguous,
// 128-bit-vectorised segment):
//
//   spinor, FP64   double2 s[12][stride]            component c = spin*3 + colour
//   spinor, FP32   float4  s[6][stride]             float4 k = components (2k, 2k+1)
//   spinor, FP16   uint4   s[3][stride] + float n[stride]
//                  twelve half2 per site scaled by the per-site FP32 factor n
//   links,  FP64   double2 U[par][mu][9][Vh]        element (row,col) = row*3+col
//   links,  FP32   float4  U[par][mu][3][Vh]        12 reals: rows 0 and 1; row 2 is
//                                                   rebuilt as conj(row0 x row1)
//   links,  FP32   float2  U[par][mu][9][Vh]        18 reals, for non-SU(3) links
//   links,  I16    uint4 U16[par][mu][Vh], then uint2 U8[par][mu][Vh]
//                                                   12 reals in 16-bit fixed point (value/32767;
//                                                   SU(3) entries are bounded by 1), row 2 rebuilt:
//                                                   the first 8 of the 12 shorts in one 16-byte
//                                                   word (copied past L1, no reuse), the last 4 in
//                                                   one 8-byte word
//   links,  H16    as I16, the 12 reals as FP16 values (FP16-arithmetic hop only)
//
// Sites of one parity are numbered as the reference numbers them
// (geometry_eo.cpp:66-77): lx = ((t*LX + x)*LY + y)*LZ + z, and the e/o index
// of a site is lx>>1 (exact because LZ is even).  Links are stored periodic;
// the time boundary sign (antiperiodic time) is applied inside the stencil.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace tms
{
  enum Prec { PREC_F64 = 0, PREC_F32 = 1, PREC_F16 = 2 };
  enum LinkFmt { LINK_F64_18 = 0, LINK_F32_12 = 1, LINK_F32_18 = 2, LINK_I16_12 = 3, LINK_F64_12 = 4, LINK_H16_12 = 5 };

  // ------------------------------------------------------------- geometry
  struct Lattice
  {
    int T, LX, LY, LZ;
    int64_t V, Vh;
    int stride;       // plane stride (sites) of an e/o field, >= Vh
    double bc_t;      // time boundary sign applied when a hop crosses t=T-1 -> 0
  };

  // coordinates of the e/o site ieo of parity p
  struct Site
  {
    int t, x, y, z;
    int lx;
  };

  __device__ __forceinline__ Site eo_site(const Lattice& g, int p, int ieo)
  {
    Site s;
    const unsigned r = 2u * (unsigned)ieo;
    const unsigned z0 = r % (unsigned)g.LZ;
    unsigned q = r / (unsigned)g.LZ;
    s.y = (int)(q % (unsigned)g.LY);
    q /= (unsigned)g.LY;
    s.x = (int)(q % (unsigned)g.LX);
    s.t = (int)(q / (unsigned)g.LX);
    s.z = (int)z0 + ((p + s.t + s.x + s.y) & 1);
    s.lx = (int)r + (s.z - (int)z0);
    return s;
  }

  // e/o index of the forward / backward neighbour in direction mu (0=t,1=x,2=y,3=z)
  // and whether the hop crosses the time boundary
  template <int MU>
  __device__ __forceinline__ int nbr_up(const Lattice& g, const Site& s, bool& wrap_t)
  {
    int lx;
    wrap_t = false;
    if (MU == 3) lx = (s.z == g.LZ - 1) ? s.lx - (g.LZ - 1) : s.lx + 1;
    else if (MU == 2) lx = (s.y == g.LY - 1) ? s.lx - (g.LY - 1) * g.LZ : s.lx + g.LZ;
    else if (MU == 1) lx = (s.x == g.LX - 1) ? s.lx - (g.LX - 1) * g.LY * g.LZ : s.lx + g.LY * g.LZ;
    else
      {
        const int st = g.LX * g.LY * g.LZ;
        wrap_t = (s.t == g.T - 1);
        lx = wrap_t ? s.lx - (g.T - 1) * st : s.lx + st;
      }
    return lx >> 1;
  }

  template <int MU>
  __device__ __forceinline__ int nbr_dw(const Lattice& g, const Site& s, bool& wrap_t)
  {
    int lx;
    wrap_t = false;
    if (MU == 3) lx = (s.z == 0) ? s.lx + (g.LZ - 1) : s.lx - 1;
    else if (MU == 2) lx = (s.y == 0) ? s.lx + (g.LY - 1) * g.LZ : s.lx - g.LZ;
    else if (MU == 1) lx = (s.x == 0) ? s.lx + (g.LX - 1) * g.LY * g.LZ : s.lx - g.LY * g.LZ;
    else
      {
        const int st = g.LX * g.LY * g.LZ;
        wrap_t = (s.t == 0);
        lx = wrap_t ? s.lx + (g.T - 1) * st : s.lx - st;
      }
    return lx >> 1;
  }

  // ---------------------------------------- programmatic dependent launch
  // A kernel launched with programmatic stream serialisation may start while
  // its predecessor in the stream drains: it waits here, before reading
  // anything the predecessor wrote, for the predecessor's completion and
  // memory flush (a no-op for an ordinary launch), and lets its own successor
  // start launching once all of its blocks have begun.
  __device__ __forceinline__ void pdl_enter()
  {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  }

  // ------------------------------------------------------- complex algebra
  template <typename R>
  struct C
  {
    R re, im;
  };

  template <typename R> __device__ __forceinline__ C<R> cadd(C<R> a, C<R> b) { return {a.re + b.re, a.im + b.im}; }
  template <typename R> __device__ __forceinline__ C<R> csub(C<R> a, C<R> b) { return {a.re - b.re, a.im - b.im}; }
  // a + i b
  template <typename R> __device__ __forceinline__ C<R> ciadd(C<R> a, C<R> b) { return {a.re - b.im, a.im + b.re}; }
  // a - i b
  template <typename R> __device__ __forceinline__ C<R> cisub(C<R> a, C<R> b) { return {a.re + b.im, a.im - b.re}; }
  template <typename R> __device__ __forceinline__ C<R> cmul(C<R> a, C<R> b)
  {
    return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
  }
  // conj(a) * b
  template <typename R> __device__ __forceinline__ C<R> cjmul(C<R> a, C<R> b)
  {
    return {a.re * b.re + a.im * b.im, a.re * b.im - a.im * b.re};
  }
  template <typename R> __device__ __forceinline__ C<R> cscale(C<R> a, R s) { return {a.re * s, a.im * s}; }
  template <typename R> __device__ __forceinline__ C<R> cconj(C<R> a) { return {a.re, -a.im}; }

  // ------------------------------------------------------ spinor accessors
  template <int P> struct SpinorT;

  template <> struct SpinorT<PREC_F64>
  {
    using R = double;
    double2* __restrict__ d;
    float* __restrict__ n; // unused
    int stride;
    // values and a scale to apply to them (1 here: the values are exact)
    __device__ __forceinline__ void load_raw(int site, C<double> v[12], double& scale) const
    {
      load(site, v);
      scale = 1.0;
    }
    __device__ __forceinline__ void load(int site, C<double> v[12]) const
    {
#pragma unroll
      for (int c = 0; c < 12; c++)
        {
          const double2 w = __ldg(d + (size_t)c * stride + site);
          v[c] = {w.x, w.y};
        }
    }
    __device__ __forceinline__ void store(int site, const C<double> v[12]) const
    {
#pragma unroll
      for (int c = 0; c < 12; c++) d[(size_t)c * stride + site] = make_double2(v[c].re, v[c].im);
    }
  };

  template <> struct SpinorT<PREC_F32>
  {
    using R = float;
    float4* __restrict__ d;
    float* __restrict__ n; // unused
    int stride;
    __device__ __forceinline__ void load_raw(int site, C<float> v[12], float& scale) const
    {
      load(site, v);
      scale = 1.0f;
    }
    __device__ __forceinline__ void load(int site, C<float> v[12]) const
    {
#pragma unroll
      for (int k = 0; k < 6; k++)
        {
          const float4 w = __ldg(d + (size_t)k * stride + site);
          v[2 * k] = {w.x, w.y};
          v[2 * k + 1] = {w.z, w.w};
        }
    }
    __device__ __forceinline__ void store(int site, const C<float> v[12]) const
    {
#pragma unroll
      for (int k = 0; k < 6; k++)
        d[(size_t)k * stride + site] = make_float4(v[2 * k].re, v[2 * k].im, v[2 * k + 1].re, v[2 * k + 1].im);
    }
  };

  template <> struct SpinorT<PREC_F16>
  {
    using R = float;
    uint4* __restrict__ d;
    float* __restrict__ n;
    int stride;
    // the stored halves and the per-site factor that scales them
    __device__ __forceinline__ void load_raw(int site, C<float> v[12], float& scale) const
    {
      scale = __ldg(n + site);
#pragma unroll
      for (int k = 0; k < 3; k++)
        {
          const uint4 w = __ldg(d + (size_t)k * stride + site);
          const unsigned u[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
          for (int j = 0; j < 4; j++)
            {
              __half2 h = *reinterpret_cast<const __half2*>(&u[j]);
              const float2 f = __half22float2(h);
              v[4 * k + j] = {f.x, f.y};
            }
        }
    }
    __device__ __forceinline__ void load(int site, C<float> v[12]) const
    {
      const float s = __ldg(n + site);
#pragma unroll
      for (int k = 0; k < 3; k++)
        {
          const uint4 w = __ldg(d + (size_t)k * stride + site);
          const unsigned u[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
          for (int j = 0; j < 4; j++)
            {
              __half2 h = *reinterpret_cast<const __half2*>(&u[j]);
              const float2 f = __half22float2(h);
              v[4 * k + j] = {f.x * s, f.y * s};
            }
        }
    }
    __device__ __forceinline__ void store(int site, const C<float> v[12]) const
    {
      float m = 0.f;
#pragma unroll
      for (int c = 0; c < 12; c++) m = fmaxf(m, fmaxf(fabsf(v[c].re), fabsf(v[c].im)));
      // a site whose largest component is below 1e-30 is stored as zero (its
      // inverse would overflow and 0*inf give NaN)
      const bool live = (m > 1e-30f);
      const float inv = live ? 1.f / m : 0.f;
      n[site] = live ? m : 0.f;
#pragma unroll
      for (int k = 0; k < 3; k++)
        {
          unsigned u[4];
#pragma unroll
          for (int j = 0; j < 4; j++)
            {
              __half2 h = __floats2half2_rn(v[4 * k + j].re * inv, v[4 * k + j].im * inv);
              u[j] = *reinterpret_cast<unsigned*>(&h);
            }
          d[(size_t)k * stride + site] = make_uint4(u[0], u[1], u[2], u[3]);
        }
    }
  };

  // -------------------------------------------------------- link accessors
  // Low-precision links are loaded with the streaming hint (evict first): each
  // link is read once per hop, so it should not displace the neighbour
  // spinors, which are read up to eight times, from L1 and L2.
  template <int F> struct LinkT;

  // a link load: streaming (evict first) by default; kept cached when the
  // same thread reuses the link (the batched kernel applies it to several
  // right-hand sides one group after the other)
  template <bool STREAM, class T>
  __device__ __forceinline__ T ld_link(const T* p)
  {
    if (STREAM) return __ldcs(p);
    return __ldg(p);
  }

  template <> struct LinkT<LINK_F64_18>
  {
    using R = double;
    const double2* __restrict__ d; // [par][mu][9][Vh]
    int Vh;
    // the link and a factor to apply to its products (1 here)
    template <bool STREAM = true>
    __device__ __forceinline__ void load_scaled(int par, int mu, int site, C<double> u[9], double& scale) const
    {
      load<STREAM>(par, mu, site, u);
      scale = double(1);
    }
    template <bool STREAM = true>
    __device__ __forceinline__ void load(int par, int mu, int site, C<double> u[9]) const
    {
      const double2* b = d + ((size_t)(par * 4 + mu) * 9) * Vh + site;
#pragma unroll
      for (int k = 0; k < 9; k++)
        {
          const double2 w = ld_link<STREAM>(b + (size_t)k * Vh);
          u[k] = {w.x, w.y};
        }
    }
  };

  // The FP64 links read as 12 reals: rows 0 and 1 from the first six planes of
  // the 18-real array, row 2 = conj(row0 x row1), which for links that are
  // SU(3) to FP64 rounding is the stored row to rounding (a third less link
  // traffic for the residual recomputations of the mixed solvers)
  template <> struct LinkT<LINK_F64_12>
  {
    using R = double;
    const double2* __restrict__ d; // [par][mu][9][Vh], planes 6-8 not read
    int Vh;
    template <bool STREAM = true>
    __device__ __forceinline__ void load_scaled(int par, int mu, int site, C<double> u[9], double& scale) const
    {
      load<STREAM>(par, mu, site, u);
      scale = double(1);
    }
    template <bool STREAM = true>
    __device__ __forceinline__ void load(int par, int mu, int site, C<double> u[9]) const
    {
      const double2* b = d + ((size_t)(par * 4 + mu) * 9) * Vh + site;
#pragma unroll
      for (int k = 0; k < 6; k++)
        {
          const double2 w = ld_link<STREAM>(b + (size_t)k * Vh);
          u[k] = {w.x, w.y};
        }
      u[6] = cconj(csub(cmul(u[1], u[5]), cmul(u[2], u[4])));
      u[7] = cconj(csub(cmul(u[2], u[3]), cmul(u[0], u[5])));
      u[8] = cconj(csub(cmul(u[0], u[4]), cmul(u[1], u[3])));
    }
  };

  template <> struct LinkT<LINK_F32_18>
  {
    using R = float;
    const float2* __restrict__ d; // [par][mu][9][Vh]
    int Vh;
    // the link and a factor to apply to its products (1 here)
    template <bool STREAM = true>
    __device__ __forceinline__ void load_scaled(int par, int mu, int site, C<float> u[9], float& scale) const
    {
      load<STREAM>(par, mu, site, u);
      scale = float(1);
    }
    // stored rows (all three) in stored units, for the two-site kernels
    static constexpr int kRows = 3;
    static constexpr float kUnit = 1.0f;
    template <bool STREAM = true>
    __device__ __forceinline__ void load_rows(int par, int mu, int site, C<float> u[9]) const { load<STREAM>(par, mu, site, u); }
    template <bool STREAM = true>
    __device__ __forceinline__ void load(int par, int mu, int site, C<float> u[9]) const
    {
      const float2* b = d + ((size_t)(par * 4 + mu) * 9) * Vh + site;
#pragma unroll
      for (int k = 0; k < 9; k++)
        {
          const float2 w = ld_link<STREAM>(b + (size_t)k * Vh);
          u[k] = {w.x, w.y};
        }
    }
  };

  template <> struct LinkT<LINK_F32_12>
  {
    using R = float;
    const float4* __restrict__ d; // [par][mu][3][Vh]
    int Vh;
    // the link and a factor to apply to its products (1 here)
    template <bool STREAM = true>
    __device__ __forceinline__ void load_scaled(int par, int mu, int site, C<float> u[9], float& scale) const
    {
      load<STREAM>(par, mu, site, u);
      scale = float(1);
    }
    // stored rows 0 and 1 in stored units, for the two-site kernels
    static constexpr int kRows = 2;
    static constexpr float kUnit = 1.0f;
    template <bool STREAM = true>
    __device__ __forceinline__ void load_rows(int par, int mu, int site, C<float> u[6]) const
    {
      const float4* b = d + ((size_t)(par * 4 + mu) * 3) * Vh + site;
      const float4 a0 = ld_link<STREAM>(b), a1 = ld_link<STREAM>(b + Vh), a2 = ld_link<STREAM>(b + 2 * (size_t)Vh);
      u[0] = {a0.x, a0.y};
      u[1] = {a0.z, a0.w};
      u[2] = {a1.x, a1.y};
      u[3] = {a1.z, a1.w};
      u[4] = {a2.x, a2.y};
      u[5] = {a2.z, a2.w};
    }
    template <bool STREAM = true>
    __device__ __forceinline__ void load(int par, int mu, int site, C<float> u[9]) const
    {
      const float4* b = d + ((size_t)(par * 4 + mu) * 3) * Vh + site;
      const float4 a0 = ld_link<STREAM>(b), a1 = ld_link<STREAM>(b + Vh), a2 = ld_link<STREAM>(b + 2 * (size_t)Vh);
      u[0] = {a0.x, a0.y};
      u[1] = {a0.z, a0.w};
      u[2] = {a1.x, a1.y};
      u[3] = {a1.z, a1.w};
      u[4] = {a2.x, a2.y};
      u[5] = {a2.z, a2.w};
      // row 2 = conj(row0 x row1): exact for special-unitary links
      u[6] = cconj(csub(cmul(u[1], u[5]), cmul(u[2], u[4])));
      u[7] = cconj(csub(cmul(u[2], u[3]), cmul(u[0], u[5])));
      u[8] = cconj(csub(cmul(u[0], u[4]), cmul(u[1], u[3])));
    }
  };

  template <> struct LinkT<LINK_I16_12>
  {
    using R = float;
    // two arrays of planes: shorts 0-7 of the two stored rows as one 16-byte
    // word per site for every (parity, direction), then shorts 8-11 as one
    // 8-byte word per site (1 % faster than one block of both planes per
    // (parity, direction))
    const char* __restrict__ d;
    int Vh;
    // stored rows 0 and 1 in raw 16-bit units (value = raw * kUnit), for the two-site kernels
    static constexpr int kRows = 2;
    static constexpr float kUnit = 1.0f / 32767.0f;
    // bytes of all links: 8 (parity, direction) pairs x 24 per site
    __host__ __device__ static size_t bytes(int64_t Vh) { return (size_t)192 * Vh; }
    __device__ __forceinline__ const uint4* w16(int par, int mu) const
    {
      return reinterpret_cast<const uint4*>(d) + (size_t)(par * 4 + mu) * Vh;
    }
    __device__ __forceinline__ const uint2* w8(int par, int mu) const
    {
      return reinterpret_cast<const uint2*>(d + (size_t)128 * Vh) + (size_t)(par * 4 + mu) * Vh;
    }
    // the twelve stored shorts of a link (16-byte word a, 8-byte word b) as rows 0 and 1
    __device__ __forceinline__ static void decode_raw(const uint4& a, const uint2& b, C<float> u[6])
    {
      const short4 a0 = *reinterpret_cast<const short4*>(&a.x), a1 = *reinterpret_cast<const short4*>(&a.z);
      const short4 a2 = *reinterpret_cast<const short4*>(&b);
      u[0] = {float(a0.x), float(a0.y)};
      u[1] = {float(a0.z), float(a0.w)};
      u[2] = {float(a1.x), float(a1.y)};
      u[3] = {float(a1.z), float(a1.w)};
      u[4] = {float(a2.x), float(a2.y)};
      u[5] = {float(a2.z), float(a2.w)};
    }
    template <bool STREAM = true>
    __device__ __forceinline__ void load_rows(int par, int mu, int site, C<float> u[6]) const
    {
      decode_raw(ld_link<STREAM>(w16(par, mu) + site), ld_link<STREAM>(w8(par, mu) + site), u);
    }
    // rows 0 and 1 in raw 16-bit units, row 2 rebuilt from them and brought to
    // the same units: the products of this link are to be multiplied by `scale`
    template <bool STREAM = true>
    __device__ __forceinline__ void load_scaled(int par, int mu, int site, C<float> u[9], float& scale) const
    {
      constexpr float k = 1.0f / 32767.0f;
      load_rows<STREAM>(par, mu, site, u);
      u[6] = cscale(cconj(csub(cmul(u[1], u[5]), cmul(u[2], u[4]))), k);
      u[7] = cscale(cconj(csub(cmul(u[2], u[3]), cmul(u[0], u[5]))), k);
      u[8] = cscale(cconj(csub(cmul(u[0], u[4]), cmul(u[1], u[3]))), k);
      scale = k;
    }
    template <bool STREAM = true>
    __device__ __forceinline__ void load(int par, int mu, int site, C<float> u[9]) const
    {
      constexpr float k = 1.0f / 32767.0f;
      load_rows<STREAM>(par, mu, site, u);
#pragma unroll
      for (int c = 0; c < 6; c++) u[c] = {u[c].re * k, u[c].im * k};
      u[6] = cconj(csub(cmul(u[1], u[5]), cmul(u[2], u[4])));
      u[7] = cconj(csub(cmul(u[2], u[3]), cmul(u[0], u[5])));
      u[8] = cconj(csub(cmul(u[0], u[4]), cmul(u[1], u[3])));
    }
  };

  // The 12 reals of rows 0 and 1 as FP16 values (not fixed point), in the same
  // two arrays of planes as LinkT<LINK_I16_12>: read only by the pipelined FP16
  // hop with FP16 arithmetic (tuning "half_arith"), which rebuilds row 2 in FP16
  template <> struct LinkT<LINK_H16_12>
  {
    using R = float;
    const char* __restrict__ d;
    int Vh;
    __host__ __device__ static size_t bytes(int64_t Vh) { return (size_t)192 * Vh; }
    __device__ __forceinline__ const uint4* w16(int par, int mu) const
    {
      return reinterpret_cast<const uint4*>(d) + (size_t)(par * 4 + mu) * Vh;
    }
    __device__ __forceinline__ const uint2* w8(int par, int mu) const
    {
      return reinterpret_cast<const uint2*>(d + (size_t)128 * Vh) + (size_t)(par * 4 + mu) * Vh;
    }
  };

  // -------------------------------------------------- device-side parameters
  // Operator and solver scalars live in device memory so that captured CUDA
  // graphs can be replayed for any kappa, mu or shift.
  struct OpParams
  {
    double kappa;
    double mu;   // twisted mass of the current operator
    double anis; // 1 when the reference's anisotropy is absent
  };

  struct Reducer
  {
    double* partial;       // per-block partial sums
    unsigned* counter;     // blocks finished (reset by the last block)
    double* result;        // final sum
  };
}
