// ILDG gauge-configuration files and the plaquette of the resident conf.
//
// An ILDG file is a LIME container: records of a 144-byte big-endian header
// (magic 0x456789ab, version, flags, 64-bit payload length, 128-byte type
// string) followed by the payload padded to 8 bytes.  The reference reads the
// 'ildg-binary-data' record (io/reader.hpp:75-99, io/ILDG_File.cpp): sites in
// the order t, z, y, x (x fastest), at each site the links of the directions
// x, y, z, t, each a row-major 3x3 complex matrix in big-endian IEEE floats of
// the precision the 'ildg-format' record states (32 or 64).  The reference
// reorders the directions to its t, x, y, z (quad_su3_ildg_to_nissa_reord) and
// its sites to lx = ((t*LX + x)*LY + y)*LZ + z; so do the functions here.
//
// The plaquette is the reference's global_plaquette_lx_conf
// (operations/su3_paths/plaquette.hpp:25-82): the mean of the temporal and
// spatial averages of Re tr(U_mu(x) U_nu(x+mu) U_mu(x+nu)^+ U_nu(x)^+)/3,
// reduced in FP64 per block and then over blocks in a fixed order.
#include "tms_internal.cuh"

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace tms
{
  namespace
  {
    constexpr uint32_t LIME_MAGIC = 0x456789abu;

    uint64_t be_read(const unsigned char* p, int n)
    {
      uint64_t v = 0;
      for (int i = 0; i < n; i++) v = (v << 8) | p[i];
      return v;
    }
    void be_write(unsigned char* p, uint64_t v, int n)
    {
      for (int i = n - 1; i >= 0; i--, v >>= 8) p[i] = (unsigned char)(v & 0xff);
    }

    struct LimeRecord
    {
      std::string type;
      long long offset; // of the payload
      uint64_t length;
    };

    bool lime_scan(FILE* f, std::vector<LimeRecord>& out)
    {
      long long pos = 0;
      unsigned char h[144];
      while (true)
        {
          if (fseeko(f, pos, SEEK_SET) != 0) return false;
          const size_t got = fread(h, 1, sizeof h, f);
          if (got == 0) return true;
          if (got != sizeof h || be_read(h, 4) != LIME_MAGIC) return false;
          LimeRecord r;
          r.length = be_read(h + 8, 8);
          r.offset = pos + 144;
          r.type.assign(reinterpret_cast<const char*>(h + 16), strnlen(reinterpret_cast<const char*>(h + 16), 128));
          out.push_back(r);
          pos = r.offset + (long long)((r.length + 7) / 8 * 8);
        }
    }

    // integer content of <tag>...</tag>, or -1
    long xml_int(const std::string& xml, const char* tag)
    {
      const std::string open = std::string("<") + tag + ">";
      const size_t a = xml.find(open);
      if (a == std::string::npos) return -1;
      return strtol(xml.c_str() + a + open.size(), nullptr, 10);
    }

    // ILDG site index of nissa's lx site and the direction permutation
    inline long long ildg_site(const Lattice& g, long long lx)
    {
      const int z = (int)(lx % g.LZ);
      long long q = lx / g.LZ;
      const int y = (int)(q % g.LY);
      q /= g.LY;
      const int x = (int)(q % g.LX);
      const int t = (int)(q / g.LX);
      return (((long long)t * g.LZ + z) * g.LY + y) * g.LX + x;
    }
    constexpr int ILDG_DIR_OF_MU[4] = {3, 0, 1, 2}; // nissa t,x,y,z -> ILDG x,y,z,t

    tms_status write_record(FILE* f, const char* type, const void* data, uint64_t len, bool begin, bool end)
    {
      unsigned char h[144] = {};
      be_write(h, LIME_MAGIC, 4);
      be_write(h + 4, 1, 2);                                   // version
      be_write(h + 6, (begin ? 0x8000u : 0u) | (end ? 0x4000u : 0u), 2); // message begin / end bits
      be_write(h + 8, len, 8);
      strncpy(reinterpret_cast<char*>(h + 16), type, 127);
      if (fwrite(h, 1, sizeof h, f) != sizeof h) return TMS_ERR_BAD_ARG;
      if (len && fwrite(data, 1, len, f) != len) return TMS_ERR_BAD_ARG;
      static const unsigned char pad[8] = {};
      const size_t npad = (size_t)((8 - len % 8) % 8);
      if (npad && fwrite(pad, 1, npad, f) != npad) return TMS_ERR_BAD_ARG;
      return TMS_OK;
    }
  }

  // ------------------------------------------------------------ plaquette
  __device__ __forceinline__ void load_link64(const Lattice& g, const double2* __restrict__ U, long long lx, int mu,
                                              double sign_t, C<double> u[9])
  {
    const int par = (int)((lx / (g.LX * g.LY * g.LZ) + (lx / (g.LY * g.LZ)) % g.LX + (lx / g.LZ) % g.LY + lx % g.LZ) & 1);
    const long long ieo = lx >> 1;
    const double2* b = U + ((size_t)(par * 4 + mu) * 9) * g.Vh + ieo;
#pragma unroll
    for (int k = 0; k < 9; k++)
      {
        const double2 w = __ldg(b + (size_t)k * g.Vh);
        u[k] = {w.x * sign_t, w.y * sign_t};
      }
  }

  __device__ __forceinline__ void mat_mul3(const C<double> a[9], const C<double> b[9], C<double> c[9])
  {
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
      for (int j = 0; j < 3; j++)
        {
          C<double> s = cmul(a[3 * i], b[j]);
          s = cadd(s, cmul(a[3 * i + 1], b[3 + j]));
          s = cadd(s, cmul(a[3 * i + 2], b[6 + j]));
          c[3 * i + j] = s;
        }
  }

  constexpr int PLAQ_THREADS = 256;

  // per block: the temporal and spatial sums of Re tr of the block's plaquettes
  static __global__ void __launch_bounds__(PLAQ_THREADS)
    plaquette_kernel(Lattice g, const double2* __restrict__ U, int with_bc, double* __restrict__ partial)
  {
    __shared__ double sh[2][PLAQ_THREADS / 32];
    const long long lx = (long long)blockIdx.x * PLAQ_THREADS + threadIdx.x;
    double sum[2] = {0.0, 0.0};
    if (lx < g.V)
      {
        const int L[4] = {g.T, g.LX, g.LY, g.LZ};
        int c[4];
        long long q = lx;
        c[3] = (int)(q % g.LZ);
        q /= g.LZ;
        c[2] = (int)(q % g.LY);
        q /= g.LY;
        c[1] = (int)(q % g.LX);
        c[0] = (int)(q / g.LX);
        const long long stride[4] = {(long long)g.LX * g.LY * g.LZ, (long long)g.LY * g.LZ, g.LZ, 1};
        for (int mu = 0; mu < 4; mu++)
          for (int nu = mu + 1; nu < 4; nu++)
            {
              const long long B = (c[mu] == L[mu] - 1) ? lx - (long long)(L[mu] - 1) * stride[mu] : lx + stride[mu];
              const long long Cs = (c[nu] == L[nu] - 1) ? lx - (long long)(L[nu] - 1) * stride[nu] : lx + stride[nu];
              // links of time direction on t = T-1 carry the boundary sign when asked
              auto sgn = [&](long long site, int d, int t) {
                return (with_bc && d == 0 && t == g.T - 1) ? g.bc_t : 1.0;
              };
              const int tB = (mu == 0) ? (c[0] + 1) % g.T : c[0];
              const int tC = (nu == 0) ? (c[0] + 1) % g.T : c[0];
              C<double> u1[9], u2[9], u3[9], u4[9], ab[9], ac[9];
              load_link64(g, U, lx, mu, sgn(lx, mu, c[0]), u1);
              load_link64(g, U, B, nu, sgn(B, nu, tB), u2);
              load_link64(g, U, lx, nu, sgn(lx, nu, c[0]), u3);
              load_link64(g, U, Cs, mu, sgn(Cs, mu, tC), u4);
              mat_mul3(u1, u2, ab);
              mat_mul3(u3, u4, ac);
              double t = 0.0;
#pragma unroll
              for (int k = 0; k < 9; k++) t += ab[k].re * ac[k].re + ab[k].im * ac[k].im;
              sum[(mu != 0 && nu != 0) ? 1 : 0] += t;
            }
      }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int k = 0; k < 2; k++)
      {
        const double v = warp_sum(sum[k]);
        if (lane == 0) sh[k][w] = v;
      }
    __syncthreads();
    if (threadIdx.x < 2)
      {
        double s = 0.0;
        for (int i = 0; i < PLAQ_THREADS / 32; i++) s += sh[threadIdx.x][i];
        partial[2 * (size_t)blockIdx.x + threadIdx.x] = s;
      }
  }

  // sum of the block partials in a fixed order
  static __global__ void plaquette_finish_kernel(int nblocks, const double* __restrict__ partial, double* out)
  {
    __shared__ double sh[2][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5; // 64 threads: warp 0 temporal, warp 1 spatial
    double s = 0.0;
    for (int i = lane; i < nblocks; i += 32) s += partial[2 * (size_t)i + w];
    s = warp_sum(s);
    if (lane == 0) sh[w][0] = s;
    __syncthreads();
    if (threadIdx.x == 0)
      {
        out[0] = sh[0][0];
        out[1] = sh[1][0];
      }
  }
}

using namespace tms;
using namespace tms_int;

extern "C" {

tms_status tms_read_ildg(tms_ctx* ctx, const char* path, double* conf_lx)
{
  if (!ctx || !path || !conf_lx) return TMS_ERR_BAD_ARG;
  FILE* f = fopen(path, "rb");
  if (!f) return fail(ctx, TMS_ERR_IO, "cannot open %s", path);
  struct Closer
  {
    FILE* f;
    ~Closer() { fclose(f); }
  } closer{f};
  std::vector<LimeRecord> recs;
  if (!lime_scan(f, recs)) return fail(ctx, TMS_ERR_IO, "%s: not a LIME file", path);
  const LimeRecord *fmt = nullptr, *bin = nullptr;
  for (const auto& r : recs)
    {
      if (r.type == "ildg-format" && !fmt) fmt = &r;
      if (r.type == "ildg-binary-data" && !bin) bin = &r;
    }
  if (!bin) return fail(ctx, TMS_ERR_IO, "%s: no ildg-binary-data record", path);
  const Lattice& g = ctx->g;
  const uint64_t nreal = (uint64_t)g.V * 72;
  int prec = 64;
  if (fmt)
    {
      std::string xml(fmt->length, '\0');
      if (fseeko(f, fmt->offset, SEEK_SET) != 0 || fread(&xml[0], 1, fmt->length, f) != fmt->length)
        return fail(ctx, TMS_ERR_IO, "%s: short ildg-format record", path);
      const long p = xml_int(xml, "precision"), lx = xml_int(xml, "lx"), ly = xml_int(xml, "ly"),
                 lz = xml_int(xml, "lz"), lt = xml_int(xml, "lt");
      if (p == 32 || p == 64) prec = (int)p;
      if ((lx > 0 && lx != g.LX) || (ly > 0 && ly != g.LY) || (lz > 0 && lz != g.LZ) || (lt > 0 && lt != g.T))
        return fail(ctx, TMS_ERR_BAD_ARG, "%s: lattice %ldx%ldx%ldx%ld (t x y z) differs from the context's", path, lt,
                    lx, ly, lz);
    }
  const uint64_t bytes = nreal * (prec / 8);
  if (bin->length != bytes)
    return fail(ctx, TMS_ERR_IO, "%s: binary record of %llu bytes, expected %llu", path,
                (unsigned long long)bin->length, (unsigned long long)bytes);
  std::vector<unsigned char> raw(bytes);
  if (fseeko(f, bin->offset, SEEK_SET) != 0 || fread(raw.data(), 1, bytes, f) != bytes)
    return fail(ctx, TMS_ERR_IO, "%s: short binary record", path);
  const int es = prec / 8;
  for (long long lx = 0; lx < g.V; lx++)
    {
      const long long is = ildg_site(g, lx);
      for (int mu = 0; mu < 4; mu++)
        {
          const unsigned char* src = raw.data() + ((size_t)is * 4 + ILDG_DIR_OF_MU[mu]) * 18 * es;
          double* dst = conf_lx + ((size_t)lx * 4 + mu) * 18;
          for (int k = 0; k < 18; k++)
            {
              const uint64_t v = be_read(src + (size_t)k * es, es);
              if (es == 8)
                {
                  double d;
                  memcpy(&d, &v, 8);
                  dst[k] = d;
                }
              else
                {
                  const uint32_t v32 = (uint32_t)v;
                  float fl;
                  memcpy(&fl, &v32, 4);
                  dst[k] = fl;
                }
            }
        }
    }
  return TMS_OK;
}

tms_status tms_write_ildg(tms_ctx* ctx, const char* path, const double* conf_lx, int precision)
{
  if (!ctx || !path || !conf_lx) return TMS_ERR_BAD_ARG;
  if (precision != 32 && precision != 64) return fail(ctx, TMS_ERR_BAD_ARG, "precision: 32 or 64");
  const Lattice& g = ctx->g;
  const int es = precision / 8;
  std::vector<unsigned char> raw((size_t)g.V * 72 * es);
  for (long long lx = 0; lx < g.V; lx++)
    {
      const long long is = ildg_site(g, lx);
      for (int mu = 0; mu < 4; mu++)
        {
          unsigned char* dst = raw.data() + ((size_t)is * 4 + ILDG_DIR_OF_MU[mu]) * 18 * es;
          const double* src = conf_lx + ((size_t)lx * 4 + mu) * 18;
          for (int k = 0; k < 18; k++)
            {
              uint64_t v;
              if (es == 8)
                memcpy(&v, &src[k], 8);
              else
                {
                  const float fl = (float)src[k];
                  uint32_t v32;
                  memcpy(&v32, &fl, 4);
                  v = v32;
                }
              be_write(dst + (size_t)k * es, v, es);
            }
        }
    }
  char xml[512];
  snprintf(xml, sizeof xml,
           "<?xml version=\"1.0\" encoding=\"UTF-8\"?>\n<ildgFormat xmlns=\"http://www.lqcd.org/ildg\">"
           "<version>1.0</version><field>su3gauge</field><precision>%d</precision>"
           "<lx>%d</lx><ly>%d</ly><lz>%d</lz><lt>%d</lt></ildgFormat>",
           precision, g.LX, g.LY, g.LZ, g.T);
  FILE* f = fopen(path, "wb");
  if (!f) return fail(ctx, TMS_ERR_IO, "cannot create %s", path);
  tms_status s = write_record(f, "ildg-format", xml, strlen(xml), true, false);
  if (s == TMS_OK) s = write_record(f, "ildg-binary-data", raw.data(), raw.size(), false, true);
  if (fclose(f) != 0 && s == TMS_OK) s = TMS_ERR_IO;
  if (s != TMS_OK) return fail(ctx, TMS_ERR_IO, "write error on %s", path);
  return TMS_OK;
}

tms_status tms_conf_plaquette(tms_ctx* ctx, int with_bc, double* plaquette)
{
  if (!ctx || !plaquette) return TMS_ERR_BAD_ARG;
  if (!ctx->conf_loaded) return fail(ctx, TMS_ERR_NO_CONF, "no configuration uploaded");
  const Lattice& g = ctx->g;
  const int nb = (int)((g.V + PLAQ_THREADS - 1) / PLAQ_THREADS);
  double* buf = nullptr;
  CU(cudaMalloc(&buf, sizeof(double) * (2 * (size_t)nb + 2)));
  struct Freer
  {
    double* p;
    ~Freer() { cudaFree(p); }
  } freer{buf};
  ctx->launches += 2;
  plaquette_kernel<<<nb, PLAQ_THREADS, 0, ctx->stream>>>(g, ctx->U64, with_bc ? 1 : 0, buf + 2);
  plaquette_finish_kernel<<<1, 64, 0, ctx->stream>>>(nb, buf + 2, buf);
  double h[2];
  CU(cudaMemcpyAsync(h, buf, sizeof h, cudaMemcpyDeviceToHost, ctx->stream));
  CU(cudaStreamSynchronize(ctx->stream));
  const double nplaq = (double)g.V * 3.0 * 3.0; // 3 planes per site and class, tr/3
  *plaquette = (h[0] / nplaq + h[1] / nplaq) / 2.0;
  return TMS_OK;
}

tms_status tms_conf_load_ildg(tms_ctx* ctx, const char* path, int flags)
{
  if (!ctx || !path) return TMS_ERR_BAD_ARG;
  std::vector<double> conf((size_t)ctx->g.V * 72);
  TRY(tms_read_ildg(ctx, path, conf.data()));
  const int mode = ctx->ptr_mode;
  ctx->ptr_mode = TMS_PTR_HOST;
  const tms_status s = tms_conf_upload(ctx, conf.data(), TMS_LAYOUT_LX, flags);
  ctx->ptr_mode = mode;
  return s;
}

} // extern "C"
