// Twisted clover on the device: the clover term from the resident links, its
// twisted inverse on even sites, and the e/o operators (C ABI).
//
//   clover_term         operations/su3_paths/clover_term.hpp:104-112, clover_term.cpp:57-95,
//                       four_leaves_point measures/gauge/topological_charge.hpp:139-212
//   inverse             invert_twisted_clover_term, clover_term.hpp:143-262
//   tmclovDee / inverse dirac_operator_tmclovD_eoprec_portable.cpp:18-40, dirac_operator_tmclovD_eoprec.hpp:24-44
//   tmclovDkern         dirac_operator_tmclovD_eoprec_portable.cpp:42-84
//   apply_tmclovQ       dirac_operators/tmclovQ/dirac_operator_tmclovQ.cpp:15-170
//
// The clover term is computed from the links as the reference's operators
// see them: the time-boundary sign on the t = T-1 time links.  The reference
// inverts each site's twisted block with a point CG to |r|^2 < 1e-32; the
// inverse is unique, so here each 6x6 block is inverted directly
// (Gauss-Jordan with partial pivoting) in FP64.
#include "tms_internal.cuh"

using namespace tms;
using namespace tms_int;

namespace
{
  // ------------------------------------------------------- SU(3) helpers
  struct M3
  {
    C<double> e[9];
  };

  // c = a b, a b^+, a^+ b, a^+ b^+
  __device__ __forceinline__ M3 mm(const M3& a, const M3& b, bool da, bool db)
  {
    M3 c;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
      for (int j = 0; j < 3; j++)
        {
          C<double> s = {0.0, 0.0};
#pragma unroll
          for (int k = 0; k < 3; k++)
            {
              C<double> x = da ? cconj(a.e[3 * k + i]) : a.e[3 * i + k];
              C<double> y = db ? cconj(b.e[3 * j + k]) : b.e[3 * k + j];
              s = cadd(s, cmul(x, y));
            }
          c.e[3 * i + j] = s;
        }
    return c;
  }

  struct LxGeom
  {
    Lattice g;
    __device__ __forceinline__ void coords(long long lx, int c[4]) const
    {
      c[3] = (int)(lx % g.LZ);
      long long q = lx / g.LZ;
      c[2] = (int)(q % g.LY);
      q /= g.LY;
      c[1] = (int)(q % g.LX);
      c[0] = (int)(q / g.LX);
    }
    __device__ __forceinline__ long long stride(int mu) const
    {
      return mu == 0 ? (long long)g.LX * g.LY * g.LZ : mu == 1 ? (long long)g.LY * g.LZ : mu == 2 ? g.LZ : 1;
    }
    __device__ __forceinline__ int extent(int mu) const { return mu == 0 ? g.T : mu == 1 ? g.LX : mu == 2 ? g.LY : g.LZ; }
    __device__ __forceinline__ long long up(long long lx, int mu) const
    {
      int c[4];
      coords(lx, c);
      return (c[mu] == extent(mu) - 1) ? lx - (long long)(extent(mu) - 1) * stride(mu) : lx + stride(mu);
    }
    __device__ __forceinline__ long long dw(long long lx, int mu) const
    {
      int c[4];
      coords(lx, c);
      return (c[mu] == 0) ? lx + (long long)(extent(mu) - 1) * stride(mu) : lx - stride(mu);
    }
    // the link U_mu(lx) with the time-boundary sign, from the periodic FP64 links
    __device__ __forceinline__ M3 link(const double2* __restrict__ U, long long lx, int mu) const
    {
      int c[4];
      coords(lx, c);
      const int par = (c[0] + c[1] + c[2] + c[3]) & 1;
      const double sg = (mu == 0 && c[0] == g.T - 1) ? g.bc_t : 1.0;
      const double2* b = U + ((size_t)(par * 4 + mu) * 9) * g.Vh + (lx >> 1);
      M3 m;
#pragma unroll
      for (int k = 0; k < 9; k++)
        {
          const double2 w = __ldg(b + (size_t)k * g.Vh);
          m.e[k] = {w.x * sg, w.y * sg};
        }
      return m;
    }
  };

  // one thread per lx site: the clover term in the reference's arithmetic order
  __global__ void __launch_bounds__(128)
    clover_term_kernel(Lattice g, const double2* __restrict__ U, double factor, double2* __restrict__ cl64,
                       float2* __restrict__ cl32)
  {
    const long long X = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (X >= g.V) return;
    const LxGeom G{g};
    C<double> P[6][9];
    int munu = 0;
    for (int mu = 0; mu < 4; mu++)
      {
        const long long A = G.up(X, mu), D = G.dw(X, mu);
        for (int nu = mu + 1; nu < 4; nu++, munu++)
          {
            const long long B = G.up(X, nu), F = G.dw(X, nu), Cc = G.up(D, nu), E = G.dw(D, nu), Gs = G.dw(A, nu);
            // leaf 1: X -> A -> Y -> B -> X
            M3 L = mm(mm(mm(G.link(U, X, mu), G.link(U, A, nu), false, false), G.link(U, B, mu), false, true),
                      G.link(U, X, nu), false, true);
            // leaf 2
            M3 t = mm(mm(mm(G.link(U, X, nu), G.link(U, Cc, mu), false, true), G.link(U, D, nu), false, true),
                      G.link(U, D, mu), false, false);
#pragma unroll
            for (int k = 0; k < 9; k++) L.e[k] = cadd(L.e[k], t.e[k]);
            // leaf 3
            t = mm(mm(mm(G.link(U, D, mu), G.link(U, E, nu), true, true), G.link(U, E, mu), false, false),
                   G.link(U, F, nu), false, false);
#pragma unroll
            for (int k = 0; k < 9; k++) L.e[k] = cadd(L.e[k], t.e[k]);
            // leaf 4
            t = mm(mm(mm(G.link(U, F, nu), G.link(U, F, mu), true, false), G.link(U, Gs, nu), false, false),
                   G.link(U, X, mu), false, true);
#pragma unroll
            for (int k = 0; k < 9; k++) L.e[k] = cadd(L.e[k], t.e[k]);
            // anti-symmetrise and divide by 4
#pragma unroll
            for (int a = 0; a < 3; a++)
#pragma unroll
              for (int b = 0; b < 3; b++)
                P[munu][3 * a + b] = {(L.e[3 * a + b].re - L.e[3 * b + a].re) / 4,
                                      (L.e[3 * a + b].im + L.e[3 * b + a].im) / 4};
          }
      }
    int c[4];
    G.coords(X, c);
    const int par = (c[0] + c[1] + c[2] + c[3]) & 1;
    const long long ieo = X >> 1;
    auto put = [&](int k, C<double> v) {
      const size_t i = ((size_t)par * 36 + k) * g.Vh + ieo;
      cl64[i] = make_double2(v.re * factor, v.im * factor);
      cl32[i] = make_float2((float)(v.re * factor), (float)(v.im * factor));
    };
#pragma unroll
    for (int k = 0; k < 9; k++)
      {
        const C<double> A = csub(P[3][k], P[2][k]), B = cadd(P[4][k], P[1][k]), Cm = csub(P[5][k], P[0][k]);
        const C<double> D = cadd(P[3][k], P[2][k]), E = csub(P[4][k], P[1][k]), F = cadd(P[5][k], P[0][k]);
        put(0 * 9 + k, C<double>{-A.im, A.re});
        put(1 * 9 + k, C<double>{B.re - Cm.im, B.im + Cm.re});
        put(2 * 9 + k, C<double>{-D.im, D.re});
        put(3 * 9 + k, C<double>{E.re - F.im, E.im + F.re});
      }
  }

  // one thread per even site: the inverse of the twisted block of each chirality with +mu
  __global__ void __launch_bounds__(128)
    inv_clover_kernel(int Vh, const double2* __restrict__ cl_even, double kcf, double mu, double2* __restrict__ icl64,
                      float2* __restrict__ icl32)
  {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= Vh) return;
    for (int b = 0; b < 2; b++)
      {
        C<double> M[6][6], I[6][6];
        for (int a = 0; a < 3; a++)
          for (int e = 0; e < 3; e++)
            {
              const double2 c0 = cl_even[(size_t)((2 * b) * 9 + 3 * a + e) * Vh + s];
              const double2 c1 = cl_even[(size_t)((2 * b + 1) * 9 + 3 * a + e) * Vh + s];
              const double2 c1t = cl_even[(size_t)((2 * b + 1) * 9 + 3 * e + a) * Vh + s];
              const double dz = (a == e) ? kcf : 0.0, dm = (a == e) ? mu : 0.0;
              M[a][e] = {dz + c0.x, dm + c0.y};
              M[a][3 + e] = {c1t.x, -c1t.y};
              M[3 + a][e] = {c1.x, c1.y};
              M[3 + a][3 + e] = {dz - c0.x, dm - c0.y};
            }
        for (int i = 0; i < 6; i++)
          for (int j = 0; j < 6; j++) I[i][j] = {i == j ? 1.0 : 0.0, 0.0};
        for (int col = 0; col < 6; col++)
          {
            int piv = col;
            double best = -1.0;
            for (int r = col; r < 6; r++)
              {
                const double m = M[r][col].re * M[r][col].re + M[r][col].im * M[r][col].im;
                if (m > best)
                  {
                    best = m;
                    piv = r;
                  }
              }
            for (int j = 0; j < 6; j++)
              {
                C<double> t = M[col][j];
                M[col][j] = M[piv][j];
                M[piv][j] = t;
                t = I[col][j];
                I[col][j] = I[piv][j];
                I[piv][j] = t;
              }
            const double pn = M[col][col].re * M[col][col].re + M[col][col].im * M[col][col].im;
            const C<double> ip = {M[col][col].re / pn, -M[col][col].im / pn};
            for (int j = 0; j < 6; j++)
              {
                M[col][j] = cmul(M[col][j], ip);
                I[col][j] = cmul(I[col][j], ip);
              }
            for (int r = 0; r < 6; r++)
              {
                if (r == col) continue;
                const C<double> f = M[r][col];
                for (int j = 0; j < 6; j++)
                  {
                    M[r][j] = csub(M[r][j], cmul(f, M[col][j]));
                    I[r][j] = csub(I[r][j], cmul(f, I[col][j]));
                  }
              }
          }
        for (int i = 0; i < 6; i++)
          for (int j = 0; j < 6; j++)
            {
              const size_t k = (size_t)(b * 36 + i * 6 + j) * Vh + s;
              icl64[k] = make_double2(I[i][j].re, I[i][j].im);
              icl32[k] = make_float2((float)I[i][j].re, (float)I[i][j].im);
            }
      }
  }

  // the clover term of both parities as the reference's lx AoS [V][4][3][3][2]
  __global__ void clover_to_lx_kernel(Lattice g, const double2* __restrict__ cl64, const int* __restrict__ lx_of_eo,
                                      double* __restrict__ out)
  {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.V) return;
    const int par = i >= g.Vh;
    const long long ieo = i - (par ? g.Vh : 0);
    const long long lx = lx_of_eo[i];
    for (int k = 0; k < 36; k++)
      {
        const double2 v = cl64[((size_t)par * 36 + k) * g.Vh + ieo];
        out[lx * 72 + 2 * k] = v.x;
        out[lx * 72 + 2 * k + 1] = v.y;
      }
  }

  // out = T_ee^-1(dag) in on even sites (no hop)
  template <int P>
  __global__ void inv_clov_apply_kernel(int n, ClovT<P> cl, int dag, SpinorT<P> in, SpinorT<P> out)
  {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    C<typename SpinorT<P>::R> a[12], o[12];
    in.load(s, a);
    cl.inv(s, dag != 0, a, o);
    out.store(s, o);
  }

  // out = T_pp(dag, mu) in on the sites of one parity (no hop)
  template <int P>
  __global__ void clov_diag_kernel(int n, ClovT<P> cl, int par, const OpParams* prm, int dag, SpinorT<P> in,
                                   SpinorT<P> out)
  {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    using R = typename SpinorT<P>::R;
    C<R> a[12], o[12];
    in.load(s, a);
    cl.diag(par, s, R(1.0 / (2.0 * prm->kappa)), R(prm->mu), dag != 0, a, o);
    out.store(s, o);
  }
}

namespace tms_int
{
  tms_status ensure_clover_inverse(tms_ctx* ctx, double kappa, double mu)
  {
    if (ctx->icl_ok && ctx->icl_kappa == kappa && ctx->icl_mu == mu) return TMS_OK;
    const int Vh = (int)ctx->g.Vh;
    ++ctx->launches;
    inv_clover_kernel<<<div_up(Vh, 128), 128, 0, ctx->stream>>>(Vh, ctx->cl64, 1.0 / (2.0 * kappa), mu, ctx->icl64,
                                                                  ctx->icl32);
    CU(cudaGetLastError());
    ctx->icl_ok = true;
    ctx->icl_kappa = kappa;
    ctx->icl_mu = mu;
    return TMS_OK;
  }

  void inv_clov_apply(tms_ctx* c, const Field& in, const Field& out, int dag)
  {
    const int n = (int)c->g.Vh;
    ++c->launches;
    inv_clov_apply_kernel<PREC_F64><<<div_up(n, 128), 128, 0, c->stream>>>(n, clov64(c), dag, view<PREC_F64>(in),
                                                                           view<PREC_F64>(out));
  }
}

extern "C" {

tms_status tms_clover_term(tms_ctx* ctx, double cSW)
{
  TRY(check_conf(ctx));
  if (!std::isfinite(cSW)) return fail(ctx, TMS_ERR_BAD_ARG, "invalid cSW %g", cSW);
  const size_t Vh = ctx->g.Vh;
  if (!ctx->cl64) CU(cudaMalloc(&ctx->cl64, 72 * Vh * sizeof(double2)));
  if (!ctx->cl32) CU(cudaMalloc(&ctx->cl32, 72 * Vh * sizeof(float2)));
  if (!ctx->icl64) CU(cudaMalloc(&ctx->icl64, 72 * Vh * sizeof(double2)));
  if (!ctx->icl32) CU(cudaMalloc(&ctx->icl32, 72 * Vh * sizeof(float2)));
  // chromo_operator_include_cSW: Cl *= chromo_operator_factor(cSW + 1e-16) / chromo_operator_factor(-4)
  const double factor = (-(cSW + 1e-16) / 4) / (-(-4.0) / 4);
  const long long V = ctx->g.V;
  ++ctx->launches;
  clover_term_kernel<<<(unsigned)div_up(V, 128), 128, 0, ctx->stream>>>(ctx->g, ctx->U64, factor, ctx->cl64,
                                                                         ctx->cl32);
  CU(cudaGetLastError());
  ctx->clov_ok = true;
  ctx->icl_ok = false;
  ctx->clov_csw = cSW;
  return finish(ctx);
}

tms_status tms_clover_get(tms_ctx* ctx, double* cl_lx)
{
  TRY(check_clover(ctx));
  if (!cl_lx) return TMS_ERR_BAD_ARG;
  const size_t bytes = (size_t)ctx->g.V * 72 * sizeof(double);
  double* d = cl_lx;
  if (ctx->ptr_mode == TMS_PTR_HOST)
    {
      TRY(ensure_stage(ctx, bytes));
      d = ctx->stage;
    }
  ++ctx->launches;
  clover_to_lx_kernel<<<(unsigned)div_up(ctx->g.V, 128), 128, 0, ctx->stream>>>(ctx->g, ctx->cl64, ctx->lx_of_eo, d);
  CU(cudaGetLastError());
  if (ctx->ptr_mode == TMS_PTR_HOST) CU(cudaMemcpyAsync(cl_lx, ctx->stage, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  return finish(ctx);
}

tms_status tms_tmclovDee(tms_ctx* ctx, int par, double kappa, double mu, int dag, const double* in, double* out)
{
  TRY(check_clover(ctx));
  if (par != 0 && par != 1) return fail(ctx, TMS_ERR_BAD_ARG, "parity 0 or 1");
  TRY(set_params(ctx, kappa, mu, 0, 1.0));
  Field &a = ctx->f64[6], &b = ctx->f64[7];
  TRY(spinor_in(ctx, in, nullptr, ctx->g.Vh, a));
  TRY(alloc_field(ctx, b, PREC_F64));
  const int n = (int)ctx->g.Vh;
  ++ctx->launches;
  clov_diag_kernel<PREC_F64><<<div_up(n, 128), 128, 0, ctx->stream>>>(n, clov64(ctx), par, ctx->prm, dag,
                                                                      view<PREC_F64>(a), view<PREC_F64>(b));
  CU(cudaGetLastError());
  TRY(spinor_out(ctx, b, nullptr, ctx->g.Vh, out, true));
  return finish(ctx);
}

tms_status tms_inv_tmclovDee(tms_ctx* ctx, double kappa, double mu, int dag, const double* in, double* out)
{
  TRY(check_clover(ctx));
  TRY(set_params(ctx, kappa, mu, 0, 1.0));
  TRY(ensure_clover_inverse(ctx, kappa, mu));
  Field &a = ctx->f64[6], &b = ctx->f64[7];
  TRY(spinor_in(ctx, in, nullptr, ctx->g.Vh, a));
  TRY(alloc_field(ctx, b, PREC_F64));
  inv_clov_apply(ctx, a, b, dag);
  CU(cudaGetLastError());
  TRY(spinor_out(ctx, b, nullptr, ctx->g.Vh, out, true));
  return finish(ctx);
}

tms_status tms_tmclovDkern_eoprec(tms_ctx* ctx, double kappa, int has_anis, double anis, double mu, int dag,
                                  const double* in, double* out)
{
  TRY(check_clover(ctx));
  TRY(set_params(ctx, kappa, mu, has_anis, anis));
  TRY(ensure_clover_inverse(ctx, kappa, mu));
  Field &a = ctx->f64[6], &b = ctx->f64[7], &te = ctx->f64[5];
  TRY(spinor_in(ctx, in, nullptr, ctx->g.Vh, a));
  TRY(alloc_field(ctx, b, PREC_F64));
  TRY(alloc_field(ctx, te, PREC_F64));
  clov_kern_op<PREC_F64>(ctx, links64(ctx), clov64(ctx), a, te, b, dag, ctx->prm);
  CU(cudaGetLastError());
  TRY(spinor_out(ctx, b, nullptr, ctx->g.Vh, out, true));
  return finish(ctx);
}

tms_status tms_tmclovDkern_eoprec_square(tms_ctx* ctx, double kappa, int has_anis, double anis, double mu,
                                         const double* in, double* out)
{
  TRY(check_clover(ctx));
  TRY(set_params(ctx, kappa, mu, has_anis, anis));
  TRY(ensure_clover_inverse(ctx, kappa, mu));
  Field &a = ctx->f64[6], &b = ctx->f64[7], &te = ctx->f64[5], &t1 = ctx->f64[4];
  TRY(spinor_in(ctx, in, nullptr, ctx->g.Vh, a));
  TRY(alloc_field(ctx, b, PREC_F64));
  TRY(alloc_field(ctx, te, PREC_F64));
  TRY(alloc_field(ctx, t1, PREC_F64));
  clov_kern_op<PREC_F64>(ctx, links64(ctx), clov64(ctx), a, te, t1, 1, ctx->prm);
  clov_kern_op<PREC_F64>(ctx, links64(ctx), clov64(ctx), t1, te, b, 0, ctx->prm);
  CU(cudaGetLastError());
  TRY(spinor_out(ctx, b, nullptr, ctx->g.Vh, out, true));
  return finish(ctx);
}

tms_status tms_apply_tmclovQ(tms_ctx* ctx, double kappa, int has_anis, double anis, double mu, const double* in,
                             double* out)
{
  TRY(check_clover(ctx));
  TRY(set_params(ctx, kappa, mu, has_anis, anis));
  Field* f = ctx->f64;
  for (int i = 4; i <= 7; i++) TRY(alloc_field(ctx, f[i], PREC_F64));
  const int64_t Vh = ctx->g.Vh;
  TRY(spinor_in(ctx, in, ctx->lx_of_eo, ctx->g.V, f[6]));
  TRY(spinor_in(ctx, in, ctx->lx_of_eo + Vh, ctx->g.V, f[7]));
  tmclovQ_op(ctx, f[6], f[7], f[4], f[5], ctx->prm);
  CU(cudaGetLastError());
  TRY(spinor_out(ctx, f[4], ctx->lx_of_eo, ctx->g.V, out, false));
  TRY(spinor_out(ctx, f[5], ctx->lx_of_eo + Vh, ctx->g.V, out, true));
  return finish(ctx);
}

} // extern "C"
