// Time-slab decomposition of the e/o hop: a context that owns the time
// slices [t0, t0 + T_loc) of a T x LX x LY x LZ lattice, and the face
// exchange that replaces the in-kernel time wrap.
//
// The reference splits the lattice over ranks and exchanges a halo before
// every hop (communicate the border of the input field, base/field.cpp:11-56)
// and all-reduces every scalar product (base/field.hpp:904).  Here the
// decomposition is along time only, and what crosses a slab boundary is the
// half spinor each side needs, not the full border:
//   * a slab's first slice is needed by the previous slab's forward time hop:
//     this slab packs h = (1 - g_t)-projection of its input there (the
//     projection of tmn2Deo_or_tmn2Doe_eos for mu = t, forward);
//   * a slab's last slice is needed by the next slab's backward time hop,
//     which also needs the link U_t of that slice (owned here): this slab packs
//     U^+ (1 + g_t)-projection of its input there, so no link ever crosses.
// Each face holds the 2 x 3 complex of one half spinor for each of the
// LX LY LZ / 2 sites of one parity on one slice, as six double2 planes
// (face index = e/o index - t * face sites).  The receiving hop reads them
// at its first and last slices and does the same arithmetic in the same
// order as the single-context hop, so the slab hop equals it bit for bit.
// The time-boundary sign is applied by the receiver that crosses the
// lattice's t = T-1 -> 0 boundary: the last slab forward, the first slab
// backward.
#include "tms_internal.cuh"

using namespace tms;
using namespace tms_int;

namespace
{
  struct SlabFaces
  {
    const double2* fwd; // half spinors of the next slab's first slice, projected forward [6][face]
    const double2* bwd; // U^+ times the backward projection of the previous slab's last slice [6][face]
    int face;           // sites of one parity on one slice
    double bc_fwd, bc_bwd;
  };

  // sites of one parity on one time slice
  int face_sites(const Lattice& g) { return g.LX * g.LY * g.LZ / 2; }

  // the two faces of input field `in` (parity par_in): fwd from slice 0, bwd from slice T_loc-1
  __global__ void slab_pack_kernel(Lattice g, int par_in, SpinorT<PREC_F64> in, LinkT<LINK_F64_18> U,
                                   double2* __restrict__ fwd, double2* __restrict__ bwd, int face)
  {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 2 * face) return;
    const bool first = i < face;
    const int fi = first ? i : i - face;
    const int ieo = (first ? 0 : g.T - 1) * face + fi;
    C<double> sp[12], h0[3], h1[3];
    in.load(ieo, sp);
    if (first)
      {
        project<0, true>(sp, h0, h1);
#pragma unroll
        for (int c = 0; c < 3; c++)
          {
            fwd[(size_t)c * face + fi] = make_double2(h0[c].re, h0[c].im);
            fwd[(size_t)(3 + c) * face + fi] = make_double2(h1[c].re, h1[c].im);
          }
      }
    else
      {
        project<0, false>(sp, h0, h1);
        C<double> L[9], u0[3], u1[3];
        U.load(par_in, 0, ieo, L);
        link_mul<false>(L, h0, u0, 1.0);
        link_mul<false>(L, h1, u1, 1.0);
#pragma unroll
        for (int c = 0; c < 3; c++)
          {
            bwd[(size_t)c * face + fi] = make_double2(u0[c].re, u0[c].im);
            bwd[(size_t)(3 + c) * face + fi] = make_double2(u1[c].re, u1[c].im);
          }
      }
  }

  // the time direction of the hop of site (p, ieo): interior slices as in
  // hop_dir<0>, the first and last slices from the faces
  __device__ __forceinline__ void slab_time_dir(const Lattice& g, const Site& s, int p, int ieo,
                                                const SpinorT<PREC_F64>& in, const LinkT<LINK_F64_18>& U,
                                                const SlabFaces& F, C<double> acc[12])
  {
    {
      C<double> h0[3], h1[3], u0[3], u1[3], L[9];
      double f = 1.0;
      if (s.t == g.T - 1)
        {
          const int fi = ieo - (g.T - 1) * F.face;
#pragma unroll
          for (int c = 0; c < 3; c++)
            {
              const double2 a = F.fwd[(size_t)c * F.face + fi], b = F.fwd[(size_t)(3 + c) * F.face + fi];
              h0[c] = {a.x, a.y};
              h1[c] = {b.x, b.y};
            }
          f = F.bc_fwd;
        }
      else
        {
          bool w;
          const int n = nbr_up<0>(g, s, w); // interior: never wraps
          C<double> sp[12];
          in.load(n, sp);
          project<0, true>(sp, h0, h1);
        }
      U.load(p, 0, ieo, L);
      link_mul<true>(L, h0, u0, f);
      link_mul<true>(L, h1, u1, f);
      reconstruct<0, true>(acc, u0, u1);
    }
    {
      C<double> u0[3], u1[3];
      if (s.t == 0)
        {
#pragma unroll
          for (int c = 0; c < 3; c++)
            {
              const double2 a = F.bwd[(size_t)c * F.face + ieo], b = F.bwd[(size_t)(3 + c) * F.face + ieo];
              u0[c] = cscale(C<double>{a.x, a.y}, F.bc_bwd);
              u1[c] = cscale(C<double>{b.x, b.y}, F.bc_bwd);
            }
        }
      else
        {
          bool w;
          const int n = nbr_dw<0>(g, s, w);
          C<double> sp[12], h0[3], h1[3], L[9];
          in.load(n, sp);
          project<0, false>(sp, h0, h1);
          U.load(1 - p, 0, n, L);
          link_mul<false>(L, h0, u0, 1.0);
          link_mul<false>(L, h1, u1, 1.0);
        }
      reconstruct<0, false>(acc, u0, u1);
    }
  }

  template <class Epi>
  __global__ void __launch_bounds__(128)
    slab_hop_kernel(Lattice g, int par_out, SpinorT<PREC_F64> in, LinkT<LINK_F64_18> U, const OpParams* prm,
                    SlabFaces F, Epi epi)
  {
    const int ieo = blockIdx.x * 128 + threadIdx.x;
    if (ieo >= g.Vh) return;
    const int p = par_out;
    C<double> acc[12];
#pragma unroll
    for (int c = 0; c < 12; c++) acc[c] = {0.0, 0.0};
    const Site s = eo_site(g, p, ieo);
    const double anis = prm->anis;
    // the order of hop_site: t, x, y, z
    slab_time_dir(g, s, p, ieo, in, U, F, acc);
    hop_dir<1, PREC_F64, LINK_F64_18>(g, s, p, ieo, in, U, anis, acc);
    hop_dir<2, PREC_F64, LINK_F64_18>(g, s, p, ieo, in, U, anis, acc);
    hop_dir<3, PREC_F64, LINK_F64_18>(g, s, p, ieo, in, U, anis, acc);
    epi(p, ieo, acc);
  }

  tms_status check_slab(tms_ctx* ctx)
  {
    TRY(check_conf(ctx));
    if (!ctx->slab) return fail(ctx, TMS_ERR_BAD_ARG, "not a time-slab context (tms_create_slab)");
    return TMS_OK;
  }

  // device copies of the caller's faces (pointer mode) -> 6 double2 planes each
  tms_status faces_in(tms_ctx* ctx, const double* fwd, const double* bwd, double2** dfwd, double2** dbwd)
  {
    const int face = face_sites(ctx->g);
    const size_t bytes = (size_t)face * 6 * sizeof(double2);
    if (!ctx->slab_ghost)
      CU(cudaMalloc(&ctx->slab_ghost, 2 * bytes));
    double2* g0 = reinterpret_cast<double2*>(ctx->slab_ghost);
    const cudaMemcpyKind k = (ctx->ptr_mode == TMS_PTR_HOST) ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    CU(cudaMemcpyAsync(g0, fwd, bytes, k, ctx->stream));
    CU(cudaMemcpyAsync(g0 + (size_t)6 * face, bwd, bytes, k, ctx->stream));
    *dfwd = g0;
    *dbwd = g0 + (size_t)6 * face;
    return TMS_OK;
  }

  template <class Epi>
  tms_status slab_hop_common(tms_ctx* ctx, int par_out, const double* in, const double* ghost_fwd,
                             const double* ghost_bwd, const Field& inf, const Epi& epi)
  {
    double2 *gf, *gb;
    TRY(faces_in(ctx, ghost_fwd, ghost_bwd, &gf, &gb));
    const SlabFaces F{gf, gb, face_sites(ctx->g), ctx->slab_bc_fwd, ctx->slab_bc_bwd};
    const int n = (int)ctx->g.Vh;
    ++ctx->launches;
    slab_hop_kernel<Epi><<<div_up(n, 128), 128, 0, ctx->stream>>>(ctx->g, par_out, view<PREC_F64>(inf), links64(ctx),
                                                                   ctx->prm, F, epi);
    CU(cudaGetLastError());
    return TMS_OK;
  }
}

extern "C" {

tms_status tms_create_slab(tms_ctx** out, int T, int t0, int T_loc, int LX, int LY, int LZ, double bc_t, int device)
{
  if (!out) return TMS_ERR_BAD_ARG;
  *out = nullptr;
  if (T <= 0 || T_loc < 2 || (T_loc & 1) || (t0 & 1) || t0 < 0 || t0 + T_loc > T || (T & 1))
    return TMS_ERR_BAD_ARG;
  // the slab's own geometry; its time-boundary sign is the lattice's only if
  // the slab ends at t = T-1 (conf uploads with the sign folded in unfold it there)
  const double bc_here = (t0 + T_loc == T) ? bc_t : 1.0;
  TRY(tms_create4(out, T_loc, LX, LY, LZ, bc_here, device));
  tms_ctx* ctx = *out;
  ctx->slab = true;
  ctx->slab_T = T;
  ctx->slab_t0 = t0;
  ctx->slab_bc_fwd = bc_here;
  ctx->slab_bc_bwd = (t0 == 0) ? bc_t : 1.0;
  return TMS_OK;
}

int64_t tms_slab_face_sites(const tms_ctx* ctx) { return ctx ? (int64_t)face_sites(ctx->g) : -1; }

tms_status tms_slab_pack(tms_ctx* ctx, int par_in, const double* in, double* face_fwd, double* face_bwd)
{
  TRY(check_slab(ctx));
  if ((par_in != 0 && par_in != 1) || !in || !face_fwd || !face_bwd)
    return fail(ctx, TMS_ERR_BAD_ARG, "bad slab pack arguments");
  Field& a = ctx->f64[6];
  TRY(spinor_in(ctx, in, nullptr, ctx->g.Vh, a));
  const int face = face_sites(ctx->g);
  const size_t bytes = (size_t)face * 6 * sizeof(double2);
  double2* d = nullptr;
  CU(cudaMalloc(&d, 2 * bytes));
  struct Free
  {
    void* p;
    ~Free() { cudaFree(p); }
  } fr{d};
  ++ctx->launches;
  slab_pack_kernel<<<div_up(2 * face, 128), 128, 0, ctx->stream>>>(ctx->g, par_in, view<PREC_F64>(a), links64(ctx), d,
                                                                    d + (size_t)6 * face, face);
  CU(cudaGetLastError());
  const cudaMemcpyKind k = (ctx->ptr_mode == TMS_PTR_HOST) ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
  CU(cudaMemcpyAsync(face_fwd, d, bytes, k, ctx->stream));
  CU(cudaMemcpyAsync(face_bwd, d + (size_t)6 * face, bytes, k, ctx->stream));
  return finish(ctx);
}

tms_status tms_slab_hop(tms_ctx* ctx, int par_out, const double* in, const double* ghost_fwd, const double* ghost_bwd,
                        double* out, int has_anis, double anis)
{
  TRY(check_slab(ctx));
  if ((par_out != 0 && par_out != 1) || !in || !out || !ghost_fwd || !ghost_bwd)
    return fail(ctx, TMS_ERR_BAD_ARG, "bad slab hop arguments");
  TRY(set_params(ctx, 1.0, 0.0, has_anis, anis));
  Field &a = ctx->f64[6], &b = ctx->f64[7];
  TRY(spinor_in(ctx, in, nullptr, ctx->g.Vh, a));
  TRY(alloc_field(ctx, b, PREC_F64));
  EpiPlain<PREC_F64> e{{view<PREC_F64>(b), view<PREC_F64>(b)}};
  TRY(slab_hop_common(ctx, par_out, in, ghost_fwd, ghost_bwd, a, e));
  TRY(spinor_out(ctx, b, nullptr, ctx->g.Vh, out, true));
  return finish(ctx);
}

tms_status tms_slab_kern_half(tms_ctx* ctx, int which, double kappa, double mu, const double* in,
                              const double* ghost_fwd, const double* ghost_bwd, const double* x, double* out,
                              int has_anis, double anis)
{
  TRY(check_slab(ctx));
  if ((which != 0 && which != 1) || !in || !out || !ghost_fwd || !ghost_bwd || (which == 1 && !x))
    return fail(ctx, TMS_ERR_BAD_ARG, "bad slab operator arguments");
  TRY(set_params(ctx, kappa, mu, has_anis, anis));
  Field &a = ctx->f64[6], &b = ctx->f64[7], &xf = ctx->f64[5];
  TRY(spinor_in(ctx, in, nullptr, ctx->g.Vh, a));
  TRY(alloc_field(ctx, b, PREC_F64));
  if (which == 0)
    {
      // even output: (1/2k + i mu g5)^-1 D_eo in (the first half of K_oo)
      EpiInvDiag<PREC_F64> e{{view<PREC_F64>(b), view<PREC_F64>(b)}, ctx->prm, 1.0};
      TRY(slab_hop_common(ctx, 0, in, ghost_fwd, ghost_bwd, a, e));
    }
  else
    {
      // odd output: g5 ((1/2k + i mu g5) x - D_oe in / 4) (the second half, with the gamma5 combine)
      TRY(spinor_in(ctx, x, nullptr, ctx->g.Vh, xf));
      EpiKern<PREC_F64, false> e{{view<PREC_F64>(b), view<PREC_F64>(b)}, {view<PREC_F64>(xf), view<PREC_F64>(xf)},
                                 ctx->prm, 1.0};
      TRY(slab_hop_common(ctx, 1, in, ghost_fwd, ghost_bwd, a, e));
    }
  TRY(spinor_out(ctx, b, nullptr, ctx->g.Vh, out, true));
  return finish(ctx);
}

} // extern "C"
