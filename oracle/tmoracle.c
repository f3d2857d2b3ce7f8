/* CPU oracle: plain-C restatement of the reference library's twisted-mass
 * Wilson hot path.  TEST INFRASTRUCTURE ONLY (see tmoracle.h): the product
 * never links it.  Every function cites the reference file:line it follows;
 * paths are relative to the reference's src/ directory.
 *
 * Arithmetic follows the reference term by term (same projection tables,
 * same complex products, same per-site accumulation order, same pairwise
 * reduction tree) so that floating-point results agree to a few ulps. */
#include "tmoracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef double cpx[2];

struct orc_geom
{
  int T, L;
  int64_t V, Vh;
  int32_t *parity, *eo_of_lx, *lx_of_eo; /* lx_of_eo[par*Vh+ieo] */
  int32_t *nup_lx, *ndw_lx;              /* [V][4] */
  int32_t *nup_eo, *ndw_eo;              /* [par][Vh][4] */
};

/* site size in doubles */
enum { SC = 24, SU3 = 18, QSU3 = 72 };

/* ---------------------------------------------------------------- geometry */

/* lx index of coordinates, t slowest and z fastest: geometry/geometry_lx.cpp:51-60 */
static int64_t lx_of_coord(const int x[4], const int s[4])
{
  int64_t i = 0;
  for (int mu = 0; mu < 4; mu++) i = i * s[mu] + x[mu];
  return i;
}

orc_geom *orc_geom_create(int T, int L)
{
  if (T <= 0 || L <= 0 || (T & 1) || (L & 1)) return NULL; /* geometry_eo.cpp:46-49: sizes must be even */
  orc_geom *g = (orc_geom *)calloc(1, sizeof(orc_geom));
  g->T = T;
  g->L = L;
  g->V = (int64_t)T * L * L * L;
  g->Vh = g->V / 2;
  const int64_t V = g->V, Vh = g->Vh;
  g->parity = (int32_t *)malloc(sizeof(int32_t) * V);
  g->eo_of_lx = (int32_t *)malloc(sizeof(int32_t) * V);
  g->lx_of_eo = (int32_t *)malloc(sizeof(int32_t) * V);
  g->nup_lx = (int32_t *)malloc(sizeof(int32_t) * V * 4);
  g->ndw_lx = (int32_t *)malloc(sizeof(int32_t) * V * 4);
  g->nup_eo = (int32_t *)malloc(sizeof(int32_t) * V * 4);
  g->ndw_eo = (int32_t *)malloc(sizeof(int32_t) * V * 4);
  const int s[4] = {T, L, L, L};
  /* neighbours with periodic wrap on one rank: geometry_lx.cpp:205-226, 403-424 */
  for (int64_t i = 0; i < V; i++)
    {
      int x[4];
      int64_t r = i;
      for (int mu = 3; mu >= 0; mu--)
        {
          x[mu] = (int)(r % s[mu]);
          r /= s[mu];
        }
      g->parity[i] = (x[0] + x[1] + x[2] + x[3]) % 2; /* glb_coord_parity */
      for (int mu = 0; mu < 4; mu++)
        {
          int y[4] = {x[0], x[1], x[2], x[3]};
          y[mu] = (x[mu] + 1) % s[mu];
          g->nup_lx[i * 4 + mu] = (int32_t)lx_of_coord(y, s);
          y[mu] = (x[mu] - 1 + s[mu]) % s[mu];
          g->ndw_lx[i * 4 + mu] = (int32_t)lx_of_coord(y, s);
        }
    }
  /* e/o labelling in lx order within each parity: geometry_eo.cpp:66-77 */
  int64_t cnt[2] = {0, 0};
  for (int64_t i = 0; i < V; i++)
    {
      const int p = g->parity[i];
      g->eo_of_lx[i] = (int32_t)cnt[p];
      g->lx_of_eo[p * Vh + cnt[p]] = (int32_t)i;
      cnt[p]++;
    }
  /* e/o neighbours: geometry_eo.cpp:79-100 */
  for (int p = 0; p < 2; p++)
    for (int64_t e = 0; e < Vh; e++)
      {
        const int64_t i = g->lx_of_eo[p * Vh + e];
        for (int mu = 0; mu < 4; mu++)
          {
            g->nup_eo[(p * Vh + e) * 4 + mu] = g->eo_of_lx[g->nup_lx[i * 4 + mu]];
            g->ndw_eo[(p * Vh + e) * 4 + mu] = g->eo_of_lx[g->ndw_lx[i * 4 + mu]];
          }
      }
  return g;
}

void orc_geom_destroy(orc_geom *g)
{
  if (!g) return;
  free(g->parity);
  free(g->eo_of_lx);
  free(g->lx_of_eo);
  free(g->nup_lx);
  free(g->ndw_lx);
  free(g->nup_eo);
  free(g->ndw_eo);
  free(g);
}

int64_t orc_geom_vol(const orc_geom *g) { return g->V; }

void orc_geom_tables(const orc_geom *g, int32_t *parity, int32_t *eo_of_lx, int32_t *lx_of_eo,
                     int32_t *neighup_eo, int32_t *neighdw_eo, int32_t *neighup_lx, int32_t *neighdw_lx)
{
  const size_t V = (size_t)g->V;
  if (parity) memcpy(parity, g->parity, V * 4);
  if (eo_of_lx) memcpy(eo_of_lx, g->eo_of_lx, V * 4);
  if (lx_of_eo) memcpy(lx_of_eo, g->lx_of_eo, V * 4);
  if (neighup_eo) memcpy(neighup_eo, g->nup_eo, V * 16);
  if (neighdw_eo) memcpy(neighdw_eo, g->ndw_eo, V * 16);
  if (neighup_lx) memcpy(neighup_lx, g->nup_lx, V * 16);
  if (neighdw_lx) memcpy(neighdw_lx, g->ndw_lx, V * 16);
}

/* geometry/geometry_mix.hpp:46-60 */
void orc_split_lx_to_eo(const orc_geom *g, const double *lx, int ndeg, double *eo)
{
#pragma omp parallel for
  for (int64_t i = 0; i < g->V; i++)
    {
      const int64_t dst = (g->parity[i] * g->Vh + g->eo_of_lx[i]) * ndeg;
      memcpy(eo + dst, lx + i * ndeg, sizeof(double) * ndeg);
    }
}

/* geometry/geometry_mix.hpp:19-39 */
void orc_paste_eo_to_lx(const orc_geom *g, const double *eo, int ndeg, double *lx)
{
#pragma omp parallel for
  for (int64_t j = 0; j < g->V; j++)
    memcpy(lx + (int64_t)g->lx_of_eo[j] * ndeg, eo + j * ndeg, sizeof(double) * ndeg);
}

/* ---------------------------------------------------------- colour algebra */
/* new_types/complex.hpp:448-475 and new_types/su3_op.hpp:240-330,1543-1603 */

static inline void csumm(double *a, const double *b, const double *c) { a[0] = b[0] + c[0]; a[1] = b[1] + c[1]; }
static inline void csubt(double *a, const double *b, const double *c) { a[0] = b[0] - c[0]; a[1] = b[1] - c[1]; }
/* a=b+i*c */
static inline void cisumm(double *a, const double *b, const double *c) { a[0] = b[0] - c[1]; a[1] = b[1] + c[0]; }
/* a=b-i*c */
static inline void cisubt(double *a, const double *b, const double *c) { a[0] = b[0] + c[1]; a[1] = b[1] - c[0]; }

#define COLOR_OP(name, op)                                                                                       \
  static inline void name(double *a, const double *b, const double *c)                                          \
  {                                                                                                              \
    for (int ic = 0; ic < 3; ic++) op(a + 2 * ic, b + 2 * ic, c + 2 * ic);                                       \
  }
COLOR_OP(color_summ, csumm)
COLOR_OP(color_subt, csubt)
COLOR_OP(color_isumm, cisumm)
COLOR_OP(color_isubt, cisubt)

/* a=U*c  (unsafe_su3_prod_color, su3_op.hpp:1543-1554) */
static inline void su3_prod_color(double *a, const double *U, const double *c)
{
  for (int i = 0; i < 3; i++)
    {
      const double *u = U + 6 * i;
      a[2 * i + 0] = u[0] * c[0] - u[1] * c[1];
      a[2 * i + 1] = u[0] * c[1] + u[1] * c[0];
      for (int j = 1; j < 3; j++)
        {
          a[2 * i + 0] += u[2 * j] * c[2 * j] - u[2 * j + 1] * c[2 * j + 1];
          a[2 * i + 1] += u[2 * j] * c[2 * j + 1] + u[2 * j + 1] * c[2 * j];
        }
    }
}

/* a=U^dag*c  (unsafe_su3_dag_prod_color, su3_op.hpp:1592-1603) */
static inline void su3_dag_prod_color(double *a, const double *U, const double *c)
{
  for (int i = 0; i < 3; i++)
    {
      const double *u = U + 2 * i; /* column i, row 0 */
      a[2 * i + 0] = u[0] * c[0] + u[1] * c[1];
      a[2 * i + 1] = u[0] * c[1] - u[1] * c[0];
      for (int j = 1; j < 3; j++)
        {
          const double *w = U + 6 * j + 2 * i;
          a[2 * i + 0] += w[0] * c[2 * j] + w[1] * c[2 * j + 1];
          a[2 * i + 1] += w[0] * c[2 * j + 1] - w[1] * c[2 * j];
        }
    }
}

/* ------------------------------------------------------------------ hopping */

/* Accumulate the -2*hopping term of one site; shared by the e/o stencil
 * (dirac_operator_tmD_eoprec_portable.hpp:56-166) and the full-lattice one
 * (dirac_operator_tmQ_portable.cpp:46-158), which are the same body. */
static void hop_site(double *out, const double *const Uf[4], const double *const Ub[4], const double *const sf[4],
                     const double *const sb[4], int has_anis, double anis)
{
  memset(out, 0, sizeof(double) * SC);
  double *o0 = out, *o1 = out + 6, *o2 = out + 12, *o3 = out + 18;
  for (int mu = 0; mu < 4; mu++)
    {
      double t0[6], t1[6], t2[6], t3[6];
      const double *s = sf[mu];
      /* forward projection */
      switch (mu)
        {
        case 0: color_summ(t0, s + 0, s + 12); color_summ(t1, s + 6, s + 18); break;
        case 1: color_isumm(t0, s + 0, s + 18); color_isumm(t1, s + 6, s + 12); break;
        case 2: color_summ(t0, s + 0, s + 18); color_subt(t1, s + 6, s + 12); break;
        case 3: color_isumm(t0, s + 0, s + 12); color_isubt(t1, s + 6, s + 18); break;
        }
      su3_prod_color(t2, Uf[mu], t0);
      su3_prod_color(t3, Uf[mu], t1);
      if (has_anis && mu > 0)
        for (int k = 0; k < 6; k++) { t2[k] *= anis; t3[k] *= anis; }
      color_summ(o0, o0, t2);
      color_summ(o1, o1, t3);
      switch (mu)
        {
        case 0: color_summ(o2, o2, t2); color_summ(o3, o3, t3); break;
        case 1: color_isubt(o2, o2, t3); color_isubt(o3, o3, t2); break;
        case 2: color_subt(o2, o2, t3); color_summ(o3, o3, t2); break;
        case 3: color_isubt(o2, o2, t2); color_isumm(o3, o3, t3); break;
        }
      /* backward projection */
      s = sb[mu];
      switch (mu)
        {
        case 0: color_subt(t0, s + 0, s + 12); color_subt(t1, s + 6, s + 18); break;
        case 1: color_isubt(t0, s + 0, s + 18); color_isubt(t1, s + 6, s + 12); break;
        case 2: color_subt(t0, s + 0, s + 18); color_summ(t1, s + 6, s + 12); break;
        case 3: color_isubt(t0, s + 0, s + 12); color_isumm(t1, s + 6, s + 18); break;
        }
      su3_dag_prod_color(t2, Ub[mu], t0);
      su3_dag_prod_color(t3, Ub[mu], t1);
      if (has_anis && mu > 0)
        for (int k = 0; k < 6; k++) { t2[k] *= anis; t3[k] *= anis; }
      color_summ(o0, o0, t2);
      color_summ(o1, o1, t3);
      switch (mu)
        {
        case 0: color_subt(o2, o2, t2); color_subt(o3, o3, t3); break;
        case 1: color_isumm(o2, o2, t3); color_isumm(o3, o3, t2); break;
        case 2: color_summ(o2, o2, t3); color_subt(o3, o3, t2); break;
        case 3: color_isumm(o2, o2, t2); color_isubt(o3, o3, t3); break;
        }
    }
}

/* tmn2Deo_or_tmn2Doe_eos: dirac_operators/tmD_eoprec/dirac_operator_tmD_eoprec_portable.hpp:33-169.
 * Forward link conf[xPar][X][mu], backward link conf[!xPar][Xdw][mu]. */
void orc_hop_eo(const orc_geom *g, const double *conf_eo, int par_out, int has_anis, double anis,
                const double *in, double *out)
{
  const int64_t Vh = g->Vh;
  const int p = par_out, np = !par_out;
#pragma omp parallel for
  for (int64_t X = 0; X < Vh; X++)
    {
      const double *Uf[4], *Ub[4], *sf[4], *sb[4];
      for (int mu = 0; mu < 4; mu++)
        {
          const int64_t up = g->nup_eo[(p * Vh + X) * 4 + mu], dw = g->ndw_eo[(p * Vh + X) * 4 + mu];
          Uf[mu] = conf_eo + ((p * Vh + X) * 4 + mu) * SU3;
          Ub[mu] = conf_eo + ((np * Vh + dw) * 4 + mu) * SU3;
          sf[mu] = in + up * SC;
          sb[mu] = in + dw * SC;
        }
      hop_site(out + X * SC, Uf, Ub, sf, sb, has_anis, anis);
    }
}

/* tmDee_or_oo_eos: ..._portable.hpp:171-195.  z=1/(2k)+i*mu on spins 0,1, conj(z) on spins 2,3 */
static void diag_mult(int64_t n, double zr, double zi, const double *in, double *out)
{
#pragma omp parallel for
  for (int64_t X = 0; X < n; X++)
    for (int id = 0; id < 4; id++)
      for (int ic = 0; ic < 3; ic++)
        {
          const double *b = in + X * SC + id * 6 + ic * 2;
          double *a = out + X * SC + id * 6 + ic * 2;
          double re, im;
          if (id < 2)
            { /* unsafe_complex_prod */
              re = b[0] * zr - b[1] * zi;
              im = b[0] * zi + b[1] * zr;
            }
          else
            { /* unsafe_complex_conj2_prod */
              re = +b[0] * zr + b[1] * zi;
              im = -b[0] * zi + b[1] * zr;
            }
          a[0] = re;
          a[1] = im;
        }
}

void orc_tmDee(const orc_geom *g, double kappa, double mu, const double *in, double *out)
{
  diag_mult(g->Vh, 1 / (2 * kappa), mu, in, out);
}

/* inv_tmDee_or_oo_eos: ..._portable.hpp:197-222 */
void orc_inv_tmDee(const orc_geom *g, double kappa, double mu, const double *in, double *out)
{
  const double a = 1 / (2 * kappa), b = mu, nrm = a * a + b * b;
  diag_mult(g->Vh, +a / nrm, -b / nrm, in, out);
}

/* tmDkern_eoprec_eos: dirac_operator_tmD_eoprec_portable.cpp:36-51, with the
 * gamma5 combination of :18-33 (out = g5 (temp - out/4)). */
void orc_kern(const orc_geom *g, const double *conf_eo, double kappa, int has_anis, double anis, double mu,
              const double *in, double *out)
{
  const int64_t n = g->Vh * SC;
  double *te = (double *)malloc(sizeof(double) * n), *to = (double *)malloc(sizeof(double) * n);
  orc_hop_eo(g, conf_eo, 0, has_anis, anis, in, to); /* even <- odd */
  orc_inv_tmDee(g, kappa, mu, to, te);
  orc_hop_eo(g, conf_eo, 1, has_anis, anis, te, out); /* odd <- even */
  orc_tmDee(g, kappa, mu, in, te);
#pragma omp parallel for
  for (int64_t X = 0; X < g->Vh; X++)
    for (int k = 0; k < 12; k++)
      {
        double *o = out + X * SC;
        const double *t = te + X * SC;
        o[k] = +t[k] - o[k] * 0.25;
        o[k + 12] = -t[k + 12] + o[k + 12] * 0.25;
      }
  free(te);
  free(to);
}

/* tmDkern_eoprec_square_eos: dirac_operator_tmD_eoprec_portable.cpp:54-65 */
void orc_kern2(const orc_geom *g, const double *conf_eo, double kappa, int has_anis, double anis, double mu,
               const double *in, double *out)
{
  double *t = (double *)malloc(sizeof(double) * g->Vh * SC);
  orc_kern(g, conf_eo, kappa, has_anis, anis, -mu, in, t);
  orc_kern(g, conf_eo, kappa, has_anis, anis, +mu, t, out);
  free(t);
}

/* ---------------------------------------------------------- linear algebra */

/* per-site sum over the internal degrees, then the pairwise halving tree of
 * reduceNoPreserve: base/field.hpp:315-362 and :862-905 */
static double tree_reduce(double *buf, int64_t n)
{
  while (n > 1)
    {
      const int64_t stride = (n + 1) / 2, nred = n / 2;
#pragma omp parallel for
      for (int64_t i = 0; i < nred; i++) buf[i] += buf[i + stride];
      n = stride;
    }
  return buf[0];
}

static double scalar_prod(int64_t nsites, const double *a, const double *b)
{
  double *buf = (double *)malloc(sizeof(double) * (nsites > 0 ? nsites : 1));
#pragma omp parallel for
  for (int64_t s = 0; s < nsites; s++)
    {
      double r = 0;
      for (int k = 0; k < SC; k++) r += a[s * SC + k] * b[s * SC + k];
      buf[s] = r;
    }
  const double res = tree_reduce(buf, nsites);
  free(buf);
  return res;
}

double orc_norm2(int64_t n, const double *v)
{
  double s = 0;
  for (int64_t i = 0; i < n; i++) s += v[i] * v[i];
  return s;
}

/* ----------------------------------------------------------------- solvers */

typedef void (*op_fn)(const void *ctx, const double *in, double *out);

/* cg_invert: inverters/templates/cg_invert_template_threaded.hpp:17-150.
 * Returns final_iter, or -1 for an invalid source norm (the reference CRASHes,
 * :55), -2 for a NaN (:113).  Non-convergence (final_iter==niter) is reported
 * through the return value like the reference's CRASH condition (:146). */
static int cg_invert(int64_t nsites, op_fn f, const void *ctx, int niter, double residue, const double *guess,
                     const double *src, double *sol, double *true_rel_res2)
{
  const int64_t n = nsites * SC;
  double *s = (double *)malloc(sizeof(double) * n), *p = (double *)malloc(sizeof(double) * n),
         *r = (double *)malloc(sizeof(double) * n);
  if (guess) memcpy(sol, guess, sizeof(double) * n);
  else memset(sol, 0, sizeof(double) * n);
  const double sourceNorm2 = scalar_prod(nsites, src, src);
  f(ctx, sol, s);
#pragma omp parallel for
  for (int64_t i = 0; i < n; i++) { r[i] = src[i] - s[i]; p[i] = r[i]; }
  double delta = scalar_prod(nsites, r, r);
  if (sourceNorm2 == 0 || isnan(sourceNorm2))
    {
      free(s); free(p); free(r);
      return -1;
    }
  int iter = 0, final_iter = 0, nan = 0;
  double lambda;
  do
    {
      final_iter = (++iter);
      f(ctx, p, s);
      const double alpha = scalar_prod(nsites, s, p);
      const double omega = delta / alpha;
#pragma omp parallel for
      for (int64_t i = 0; i < n; i++) sol[i] += p[i] * omega;
#pragma omp parallel for
      for (int64_t i = 0; i < n; i++) r[i] -= s[i] * omega;
      lambda = scalar_prod(nsites, r, r);
      const double gammag = lambda / delta;
      delta = lambda;
      if (isnan(gammag)) { nan = 1; break; }
#pragma omp parallel for
      for (int64_t i = 0; i < n; i++) p[i] = r[i] + p[i] * gammag;
    }
  while (lambda >= (residue * sourceNorm2) && iter < niter);
  /* true residual (:131-135) */
  f(ctx, sol, s);
#pragma omp parallel for
  for (int64_t i = 0; i < n; i++) r[i] = src[i] - s[i];
  lambda = scalar_prod(nsites, r, r);
  if (true_rel_res2) *true_rel_res2 = lambda / sourceNorm2;
  free(s); free(p); free(r);
  return nan ? -2 : final_iter;
}

struct kern2_ctx { const orc_geom *g; const double *conf_eo; double kappa; int has_anis; double anis, mu; };

static void kern2_op(const void *c, const double *in, double *out)
{
  const struct kern2_ctx *k = (const struct kern2_ctx *)c;
  orc_kern2(k->g, k->conf_eo, k->kappa, k->has_anis, k->anis, k->mu, in, out);
}

/* inv_tmDkern_eoprec_square_eos_cg -> _cg_64: cg_invert_tmD_eoprec.cpp:61-78, cg_64_invert_tmD_eoprec.hpp:11-40 */
int orc_cg_eos(const orc_geom *g, const double *conf_eo, double kappa, int has_anis, double anis, double mu,
               int niter, double residue, const double *guess, const double *src, double *sol,
               double *true_rel_res2)
{
  struct kern2_ctx k = {g, conf_eo, kappa, has_anis, anis, mu};
  return cg_invert(g->Vh, kern2_op, &k, niter, residue, guess, src, sol, true_rel_res2);
}

/* apply_tmQ: dirac_operators/tmQ/dirac_operator_tmQ_portable.cpp:29-176 */
void orc_tmQ(const orc_geom *g, const double *conf_lx, double kappa, int has_anis, double anis, double mass,
             const double *in, double *out)
{
  const double kcf = 1 / (2 * kappa);
#pragma omp parallel for
  for (int64_t X = 0; X < g->V; X++)
    {
      const double *Uf[4], *Ub[4], *sf[4], *sb[4];
      for (int mu = 0; mu < 4; mu++)
        {
          const int64_t up = g->nup_lx[X * 4 + mu], dw = g->ndw_lx[X * 4 + mu];
          Uf[mu] = conf_lx + (X * 4 + mu) * SU3;
          Ub[mu] = conf_lx + (dw * 4 + mu) * SU3;
          sf[mu] = in + up * SC;
          sb[mu] = in + dw * SC;
        }
      double *o = out + X * SC;
      const double *i = in + X * SC;
      hop_site(o, Uf, Ub, sf, sb, has_anis, anis);
      /* :160-174 */
      for (int c = 0; c < 3; c++)
        {
          for (int id = 0; id < 2; id++)
            {
              double *a = o + id * 6 + c * 2;
              const double *b = i + id * 6 + c * 2;
              a[0] = -0.5 * a[0] + kcf * b[0] - mass * b[1];
              a[1] = -0.5 * a[1] + kcf * b[1] + mass * b[0];
            }
          for (int id = 2; id < 4; id++)
            {
              double *a = o + id * 6 + c * 2;
              const double *b = i + id * 6 + c * 2;
              a[0] = +0.5 * a[0] - kcf * b[0] - mass * b[1];
              a[1] = +0.5 * a[1] - kcf * b[1] + mass * b[0];
            }
        }
    }
}

/* Q(+mu)Q(-mu): apply_tmQ2 in its original form (dirac_operator_tmQ2.cpp:17-30,
 * commented body) and apply_tmclovQ2 (dirac_operator_tmclovQ2.hpp:13-24) */
void orc_tmQ2(const orc_geom *g, const double *conf_lx, double kappa, int has_anis, double anis, double mu,
              const double *in, double *out)
{
  double *t = (double *)malloc(sizeof(double) * g->V * SC);
  orc_tmQ(g, conf_lx, kappa, has_anis, anis, +mu, in, t);
  orc_tmQ(g, conf_lx, kappa, has_anis, anis, -mu, t, out);
  free(t);
}

/* inv_tmD_cg_eoprec_native + the lx residual check of inv_tmD_cg_eoprec:
 * inverters/twisted_mass/cg_invert_tmD_eoprec.cpp:37-58 (Eq. 8b), :81-99
 * (Eq. 11), :102-150, :192-212.  *lx_rel_res2 = |g5 Q sol - src|^2/|src|^2 */
int orc_cg_full(const orc_geom *g, const double *conf_lx, double kappa, int has_anis, double anis, double mass,
                int niter, double residue, const double *src_lx, double *sol_lx, double *lx_rel_res2)
{
  const int64_t Vh = g->Vh, n = Vh * SC;
  double *conf_eo = (double *)malloc(sizeof(double) * g->V * QSU3);
  double *src_eo = (double *)malloc(sizeof(double) * 2 * n), *sol_eo = (double *)malloc(sizeof(double) * 2 * n);
  double *evnTemp = (double *)malloc(sizeof(double) * n), *varphi = (double *)malloc(sizeof(double) * n);
  double *oddTemp = (double *)malloc(sizeof(double) * n);
  orc_split_lx_to_eo(g, conf_lx, QSU3, conf_eo);
  orc_split_lx_to_eo(g, src_lx, SC, src_eo);
  const double *src_e = src_eo, *src_o = src_eo + n;
  /* Eq. 8a */
  orc_inv_tmDee(g, kappa, mass, src_e, evnTemp);
  /* Eq. 8b (:37-58) */
  orc_hop_eo(g, conf_eo, 1, has_anis, anis, evnTemp, varphi);
#pragma omp parallel for
  for (int64_t X = 0; X < Vh; X++)
    for (int k = 0; k < 12; k++)
      {
        double *v = varphi + X * SC;
        const double *s = src_o + X * SC;
        v[k] = +s[k] + v[k] * 0.5;
        v[k + 12] = -s[k + 12] - v[k + 12] * 0.5;
      }
  /* Eq. 9 */
  double cg_res;
  const int it = orc_cg_eos(g, conf_eo, kappa, has_anis, anis, mass, niter, residue, NULL, varphi, oddTemp, &cg_res);
  /* Eq. 10 */
  double *sol_e = sol_eo, *sol_o = sol_eo + n;
  orc_kern(g, conf_eo, kappa, has_anis, anis, -mass, oddTemp, sol_o);
  /* Eq. 11 (:81-99) */
  orc_hop_eo(g, conf_eo, 0, has_anis, anis, sol_o, evnTemp);
#pragma omp parallel for
  for (int64_t i = 0; i < n; i++) evnTemp[i] = src_e[i] + evnTemp[i] * 0.5;
  orc_inv_tmDee(g, kappa, mass, evnTemp, sol_e);
  orc_paste_eo_to_lx(g, sol_eo, SC, sol_lx);
  /* residual check in lx (:192-212) */
  if (lx_rel_res2)
    {
      double *rv = (double *)malloc(sizeof(double) * g->V * SC);
      orc_tmQ(g, conf_lx, kappa, has_anis, anis, mass, sol_lx, rv);
#pragma omp parallel for
      for (int64_t X = 0; X < g->V; X++)
        for (int k = 0; k < SC; k++)
          {
            const double gv = (k < 12 ? 1 : -1) * rv[X * SC + k]; /* gamma5 = diag(1,1,-1,-1), new_types/dirac.cpp:48 */
            rv[X * SC + k] = gv - src_lx[X * SC + k];
          }
      *lx_rel_res2 = scalar_prod(g->V, rv, rv) / scalar_prod(g->V, src_lx, src_lx);
      free(rv);
    }
  free(conf_eo); free(src_eo); free(sol_eo); free(evnTemp); free(varphi); free(oddTemp);
  return it;
}

/* cgm_invert with f(out,sigma,in)=Q(+sqrt(sigma))Q(-sqrt(sigma)) in, the
 * operator of inv_tmclovQ2_cgm at zero clover term:
 * inverters/templates/cgm_invert_template_threaded.hpp:11-295,
 * inverters/twisted_clover/cgm_invert_tmclovQ2.cpp:10-32,
 * dirac_operators/tmclovQ2/dirac_operator_tmclovQ2.hpp:28-101.
 * sols: [nshift][V][24].  Returns final_iter, -1 invalid source, -2 NaN. */
int orc_cgm(const orc_geom *g, const double *conf_lx, double kappa, int has_anis, double anis, int nshift,
            const double *masses, const double *residues, int niter_max, const double *src, double *sols,
            double *true_rel_res2)
{
  const int64_t V = g->V, n = V * SC;
  double *s = (double *)malloc(sizeof(double) * n), *r = (double *)malloc(sizeof(double) * n),
         *p = (double *)malloc(sizeof(double) * n), *ps = (double *)malloc(sizeof(double) * n * nshift);
  double *shifts = (double *)malloc(sizeof(double) * nshift);
  for (int i = 0; i < nshift; i++) shifts[i] = masses[i] * masses[i];
  for (int i = 0; i < nshift; i++)
    {
      memcpy(ps + i * n, src, sizeof(double) * n);
      memset(sols + i * n, 0, sizeof(double) * n);
    }
  memcpy(p, src, sizeof(double) * n);
  memcpy(r, src, sizeof(double) * n);
  const double source_norm2 = scalar_prod(V, r, r);
  if (source_norm2 == 0 || isnan(source_norm2))
    {
      free(s); free(r); free(p); free(ps); free(shifts);
      return -1;
    }
  double *zps = (double *)malloc(sizeof(double) * nshift), *zas = (double *)malloc(sizeof(double) * nshift),
         *alphas = (double *)malloc(sizeof(double) * nshift), *zfs = (double *)malloc(sizeof(double) * nshift),
         *betas = (double *)malloc(sizeof(double) * nshift), *final_res = (double *)malloc(sizeof(double) * nshift);
  int *run_flag = (int *)malloc(sizeof(int) * nshift);
  int nrun_shift = nshift, iter = 0, final_iter = 0, nan = 0;
  double betaa = 1, alpha = 0, rr = source_norm2, rfrf, betap;
  for (int i = 0; i < nshift; i++)
    {
      zps[i] = zas[i] = 1;
      alphas[i] = 0;
      run_flag[i] = 1;
      final_res[i] = 1;
    }
  do
    {
      final_iter = (++iter);
      orc_tmQ2(g, conf_lx, kappa, has_anis, anis, 0.0, p, s); /* f(s,0.0,p) */
      const double pap = scalar_prod(V, p, s);
      betap = betaa;
      betaa = -rr / pap;
      for (int i = 0; i < nshift; i++)
        if (run_flag[i])
          {
            const double ratio = betap / (betaa * alpha * (1 - zas[i] / zps[i]) + betap * (1 - shifts[i] * betaa));
            if (isnan(ratio)) nan = 1;
            zfs[i] = zas[i] * ratio;
            betas[i] = betaa * ratio;
            double *x = sols + i * n;
            const double *psi = ps + i * n;
            const double beta = betas[i];
#pragma omp parallel for
            for (int64_t k = 0; k < n; k++) x[k] -= beta * psi[k];
          }
      if (nan) break;
#pragma omp parallel for
      for (int64_t k = 0; k < n; k++) r[k] += s[k] * betaa;
      rfrf = scalar_prod(V, r, r);
      alpha = rfrf / rr;
#pragma omp parallel for
      for (int64_t k = 0; k < n; k++) p[k] = r[k] + p[k] * alpha;
      for (int i = 0; i < nshift; i++)
        if (run_flag[i])
          {
            alphas[i] = alpha * zfs[i] * betas[i] / (zas[i] * betaa);
            double *psi = ps + i * n;
            const double a = alphas[i], z = zfs[i];
#pragma omp parallel for
            for (int64_t k = 0; k < n; k++) psi[k] = r[k] * z + psi[k] * a;
            zps[i] = zas[i];
            zas[i] = zfs[i];
          }
      rr = rfrf;
      for (int i = 0; i < nshift; i++)
        if (run_flag[i])
          {
            final_res[i] = rr * zfs[i] * zfs[i] / source_norm2;
            if (final_res[i] < residues[i])
              {
                run_flag[i] = 0;
                nrun_shift--;
              }
          }
    }
  while (nrun_shift > 0 && iter < niter_max);
  /* final true residues (:266-279) */
  if (true_rel_res2)
    for (int i = 0; i < nshift; i++)
      {
        orc_tmQ2(g, conf_lx, kappa, has_anis, anis, sqrt(shifts[i]), sols + i * n, s);
#pragma omp parallel for
        for (int64_t k = 0; k < n; k++) s[k] -= src[k];
        true_rel_res2[i] = scalar_prod(V, s, s) / source_norm2;
      }
  free(s); free(r); free(p); free(ps); free(shifts);
  free(zps); free(zas); free(alphas); free(zfs); free(betas); free(final_res); free(run_flag);
  return nan ? -2 : final_iter;
}

/* ---------------------------------------------------------------- plaquette */

/* global_plaquette_lx_conf: operations/su3_paths/plaquette.hpp:25-82.  Mean of
 * the temporal and spatial averages of Re tr(U U U^+ U^+)/3. */
double orc_plaquette(const orc_geom *g, const double *conf_lx)
{
  const int64_t V = g->V;
  double *buf = (double *)malloc(sizeof(double) * V * 2);
#pragma omp parallel for
  for (int64_t A = 0; A < V; A++)
    {
      double lp[2] = {0, 0};
      for (int mu = 0; mu < 4; mu++)
        {
          const int64_t B = g->nup_lx[A * 4 + mu];
          for (int nu = mu + 1; nu < 4; nu++)
            {
              const int64_t C = g->nup_lx[A * 4 + nu];
              const double *U1 = conf_lx + (A * 4 + mu) * SU3, *U2 = conf_lx + (B * 4 + nu) * SU3;
              const double *U3 = conf_lx + (A * 4 + nu) * SU3, *U4 = conf_lx + (C * 4 + mu) * SU3;
              double ABD[18], ACD[18];
              for (int i = 0; i < 3; i++)
                for (int j = 0; j < 3; j++)
                  {
                    double ar = 0, ai = 0, br = 0, bi = 0;
                    for (int k = 0; k < 3; k++)
                      {
                        const double *x = U1 + 6 * i + 2 * k, *y = U2 + 6 * k + 2 * j;
                        ar += x[0] * y[0] - x[1] * y[1];
                        ai += x[0] * y[1] + x[1] * y[0];
                        const double *z = U3 + 6 * i + 2 * k, *w = U4 + 6 * k + 2 * j;
                        br += z[0] * w[0] - z[1] * w[1];
                        bi += z[0] * w[1] + z[1] * w[0];
                      }
                    ABD[6 * i + 2 * j] = ar;
                    ABD[6 * i + 2 * j + 1] = ai;
                    ACD[6 * i + 2 * j] = br;
                    ACD[6 * i + 2 * j + 1] = bi;
                  }
              /* Re tr(ABD ACD^+) = sum_ij Re(ABD_ij conj(ACD_ij)) */
              double t = 0;
              for (int k = 0; k < 9; k++) t += ABD[2 * k] * ACD[2 * k] + ABD[2 * k + 1] * ACD[2 * k + 1];
              lp[(mu != 0 && nu != 0)] += t;
            }
        }
      buf[A] = lp[0];
      buf[V + A] = lp[1];
    }
  const double p0 = tree_reduce(buf, V) / (V * 9.0);
  const double p1 = tree_reduce(buf + V, V) / (V * 9.0);
  free(buf);
  return (p0 + p1) / 2;
}

/* ================================================================ clover */
/* The twisted-clover e/o path.  Layouts (float64, AoS):
 *   clover term   [sites][4][3][3][2]          clover_term_t = su3[4] (new_types/su3.hpp:57-60)
 *   inverse       [sites][2][2][3][2][3][2]    inv_clover_term_t: per chirality a 6x6
 *                                              matrix [id][ic][jd][jc] (su3.hpp:31,62) */

/* c = a*b, a*b^+, a^+*b, a^+*b^+ (unsafe_su3_prod_su3 and variants, su3_op.hpp) */
static void su3_mm(double *c, const double *a, const double *b, int da, int db)
{
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++)
      {
        double re = 0, im = 0;
        for (int k = 0; k < 3; k++)
          {
            const double *x = da ? a + 6 * k + 2 * i : a + 6 * i + 2 * k;
            const double *y = db ? b + 6 * j + 2 * k : b + 6 * k + 2 * j;
            const double xr = x[0], xi = da ? -x[1] : x[1], yr = y[0], yi = db ? -y[1] : y[1];
            re += xr * yr - xi * yi;
            im += xr * yi + xi * yr;
          }
        c[6 * i + 2 * j] = re;
        c[6 * i + 2 * j + 1] = im;
      }
}

/* four_leaves_point: measures/gauge/topological_charge.hpp:139-212; planes in the
 * order of edge_numb (base/init.cpp:705-714): (0,1) (0,2) (0,3) (1,2) (1,3) (2,3) */
static void four_leaves(const orc_geom *g, const double *conf, int64_t X, double *leaves)
{
#define U(site, d) (conf + ((int64_t)(site) * 4 + (d)) * SU3)
  int munu = 0;
  for (int mu = 0; mu < 4; mu++)
    {
      const int64_t A = g->nup_lx[X * 4 + mu], D = g->ndw_lx[X * 4 + mu];
      for (int nu = mu + 1; nu < 4; nu++, munu++)
        {
          const int64_t B = g->nup_lx[X * 4 + nu], F = g->ndw_lx[X * 4 + nu];
          const int64_t C = g->nup_lx[D * 4 + nu], E = g->ndw_lx[D * 4 + nu];
          const int64_t G = g->ndw_lx[A * 4 + nu];
          double *L = leaves + munu * SU3, t1[SU3], t2[SU3];
          /* leaf 1 */
          su3_mm(t1, U(X, mu), U(A, nu), 0, 0);
          su3_mm(t2, t1, U(B, mu), 0, 1);
          su3_mm(L, t2, U(X, nu), 0, 1);
          /* leaf 2 */
          su3_mm(t1, U(X, nu), U(C, mu), 0, 1);
          su3_mm(t2, t1, U(D, nu), 0, 1);
          su3_mm(t1, t2, U(D, mu), 0, 0);
          for (int k = 0; k < SU3; k++) L[k] += t1[k];
          /* leaf 3 */
          su3_mm(t1, U(D, mu), U(E, nu), 1, 1);
          su3_mm(t2, t1, U(E, mu), 0, 0);
          su3_mm(t1, t2, U(F, nu), 0, 0);
          for (int k = 0; k < SU3; k++) L[k] += t1[k];
          /* leaf 4 */
          su3_mm(t1, U(F, nu), U(F, mu), 1, 0);
          su3_mm(t2, t1, U(G, nu), 0, 0);
          su3_mm(t1, t2, U(X, mu), 0, 1);
          for (int k = 0; k < SU3; k++) L[k] += t1[k];
        }
    }
#undef U
}

/* clover_term (operations/su3_paths/clover_term.hpp:104-112): point_chromo_operator
 * (clover_term.cpp:57-95) times chromo_operator_factor(cSW + 1e-16) /
 * chromo_operator_factor(-4) (clover_term.hpp:44-84) */
void orc_clover_term(const orc_geom *g, const double *conf_lx, double cSW, double *Cl)
{
  const double factor = (-(cSW + 1e-16) / 4) / (-(-4.0) / 4);
#pragma omp parallel for
  for (int64_t X = 0; X < g->V; X++)
    {
      double leaves[6 * SU3], P[6][SU3];
      four_leaves(g, conf_lx, X, leaves);
      for (int i = 0; i < 6; i++)
        for (int a = 0; a < 3; a++)
          for (int b = 0; b < 3; b++)
            {
              P[i][6 * a + 2 * b] = (leaves[i * SU3 + 6 * a + 2 * b] - leaves[i * SU3 + 6 * b + 2 * a]) / 4;
              P[i][6 * a + 2 * b + 1] = (leaves[i * SU3 + 6 * a + 2 * b + 1] + leaves[i * SU3 + 6 * b + 2 * a + 1]) / 4;
            }
      double *c = Cl + X * 4 * SU3;
      for (int k = 0; k < SU3; k += 2)
        {
          const double Ar = P[3][k] - P[2][k], Ai = P[3][k + 1] - P[2][k + 1];
          const double Br = P[4][k] + P[1][k], Bi = P[4][k + 1] + P[1][k + 1];
          const double Cr = P[5][k] - P[0][k], Ci = P[5][k + 1] - P[0][k + 1];
          const double Dr = P[3][k] + P[2][k], Di = P[3][k + 1] + P[2][k + 1];
          const double Er = P[4][k] - P[1][k], Ei = P[4][k + 1] - P[1][k + 1];
          const double Fr = P[5][k] + P[0][k], Fi = P[5][k + 1] + P[0][k + 1];
          /* Cl0 = iA, Cl1 = B + iC, Cl2 = iD, Cl3 = E + iF */
          c[0 * SU3 + k] = -Ai * factor;
          c[0 * SU3 + k + 1] = Ar * factor;
          c[1 * SU3 + k] = (Br - Ci) * factor;
          c[1 * SU3 + k + 1] = (Bi + Cr) * factor;
          c[2 * SU3 + k] = -Di * factor;
          c[2 * SU3 + k + 1] = Dr * factor;
          c[3 * SU3 + k] = (Er - Fi) * factor;
          c[3 * SU3 + k + 1] = (Ei + Fr) * factor;
        }
    }
}

/* the 6x6 twisted clover block of chirality b: z 1 + [[c0, c1^+], [c1, -c0]] with
 * z = 1/2k + i mass (apply_point_twisted_clover_term_to_halfspincolor, clover_term.hpp:114-141) */
static void clover_block_z(const double *Cl, int b, double zr, double zi, double M[6][6][2])
{
  const double *c0 = Cl + (2 * b) * SU3, *c1 = Cl + (2 * b + 1) * SU3;
  for (int a = 0; a < 3; a++)
    for (int e = 0; e < 3; e++)
      {
        const double dz = (a == e) ? zr : 0.0, dm = (a == e) ? zi : 0.0;
        M[a][e][0] = dz + c0[6 * a + 2 * e];
        M[a][e][1] = dm + c0[6 * a + 2 * e + 1];
        M[a][3 + e][0] = c1[6 * e + 2 * a];
        M[a][3 + e][1] = -c1[6 * e + 2 * a + 1];
        M[3 + a][e][0] = c1[6 * a + 2 * e];
        M[3 + a][e][1] = c1[6 * a + 2 * e + 1];
        M[3 + a][3 + e][0] = dz - c0[6 * a + 2 * e];
        M[3 + a][3 + e][1] = dm - c0[6 * a + 2 * e + 1];
      }
}

static void clover_block(const double *Cl, int b, double kappa, double mass, double M[6][6][2])
{
  clover_block_z(Cl, b, 1.0 / (2 * kappa), mass, M);
}

/* invert_twisted_clover_term (clover_term.hpp:143-262): per site and chirality the
 * inverse of the block with +mass.  The reference solves for each column with a
 * point CG on the squared block to |r|^2 < 1e-32; the inverse is unique, so this
 * restatement inverts directly (Gauss-Jordan, partial pivoting) in float64. */
void orc_inv_clover_term(int64_t nsites, const double *Cl, double kappa, double mass, double *invCl)
{
#pragma omp parallel for
  for (int64_t X = 0; X < nsites; X++)
    for (int b = 0; b < 2; b++)
      {
        double M[6][6][2], I[6][6][2];
        clover_block(Cl + X * 4 * SU3, b, kappa, mass, M);
        for (int i = 0; i < 6; i++)
          for (int j = 0; j < 6; j++) I[i][j][0] = (i == j), I[i][j][1] = 0;
        for (int col = 0; col < 6; col++)
          {
            int piv = col;
            double best = -1;
            for (int r = col; r < 6; r++)
              {
                const double m = M[r][col][0] * M[r][col][0] + M[r][col][1] * M[r][col][1];
                if (m > best) best = m, piv = r;
              }
            for (int j = 0; j < 6; j++)
              for (int q = 0; q < 2; q++)
                {
                  double t = M[col][j][q]; M[col][j][q] = M[piv][j][q]; M[piv][j][q] = t;
                  t = I[col][j][q]; I[col][j][q] = I[piv][j][q]; I[piv][j][q] = t;
                }
            const double pr = M[col][col][0], pi = M[col][col][1], pn = pr * pr + pi * pi;
            const double ir = pr / pn, ii = -pi / pn;
            for (int j = 0; j < 6; j++)
              {
                double a = M[col][j][0], c = M[col][j][1];
                M[col][j][0] = a * ir - c * ii; M[col][j][1] = a * ii + c * ir;
                a = I[col][j][0]; c = I[col][j][1];
                I[col][j][0] = a * ir - c * ii; I[col][j][1] = a * ii + c * ir;
              }
            for (int r = 0; r < 6; r++)
              {
                if (r == col) continue;
                const double fr = M[r][col][0], fi = M[r][col][1];
                for (int j = 0; j < 6; j++)
                  {
                    M[r][j][0] -= fr * M[col][j][0] - fi * M[col][j][1];
                    M[r][j][1] -= fr * M[col][j][1] + fi * M[col][j][0];
                    I[r][j][0] -= fr * I[col][j][0] - fi * I[col][j][1];
                    I[r][j][1] -= fr * I[col][j][1] + fi * I[col][j][0];
                  }
              }
          }
        double *o = invCl + X * 144 + b * 72;
        for (int i = 0; i < 6; i++)
          for (int j = 0; j < 6; j++)
            {
              o[(i * 6 + j) * 2] = I[i][j][0];
              o[(i * 6 + j) * 2 + 1] = I[i][j][1];
            }
      }
}

/* tmclovDee_or_oo_eos: dirac_operators/tmclovD_eoprec/dirac_operator_tmclovD_eoprec_portable.cpp:18-40 */
void orc_tmclovDee(int64_t nsites, const double *Cl, double kappa, int dag, double mu, const double *in, double *out)
{
  if (dag) mu = -mu;
#pragma omp parallel for
  for (int64_t X = 0; X < nsites; X++)
    for (int b = 0; b < 2; b++)
      {
        double M[6][6][2];
        clover_block(Cl + X * 4 * SU3, b, kappa, b ? -mu : mu, M);
        const double *i = in + X * SC + b * 12;
        double *o = out + X * SC + b * 12;
        for (int r = 0; r < 6; r++)
          {
            double re = 0, im = 0;
            for (int c = 0; c < 6; c++)
              {
                re += M[r][c][0] * i[2 * c] - M[r][c][1] * i[2 * c + 1];
                im += M[r][c][0] * i[2 * c + 1] + M[r][c][1] * i[2 * c];
              }
            o[2 * r] = re;
            o[2 * r + 1] = im;
          }
      }
}

/* inv_tmclovDee_or_oo_eos: dirac_operator_tmclovD_eoprec.hpp:24-44 */
void orc_inv_tmclovDee(int64_t nsites, const double *invCl, int dag, const double *in, double *out)
{
  const int high = dag ? 1 : 0, low = dag ? 0 : 1;
#pragma omp parallel for
  for (int64_t X = 0; X < nsites; X++)
    for (int b = 0; b < 2; b++)
      {
        const double *m = invCl + X * 144 + b * 72;
        const double *i = in + X * SC + b * 12;
        double *o = out + X * SC + b * 12;
        for (int r = 0; r < 6; r++)
          {
            double re = 0, im = 0;
            for (int c = 0; c < 6; c++)
              {
                if (b == high)
                  {
                    const double *e = m + (r * 6 + c) * 2;
                    re += e[0] * i[2 * c] - e[1] * i[2 * c + 1];
                    im += e[0] * i[2 * c + 1] + e[1] * i[2 * c];
                  }
                else
                  {
                    const double *e = m + (c * 6 + r) * 2; /* conj of the transposed element */
                    re += e[0] * i[2 * c] + e[1] * i[2 * c + 1];
                    im += e[0] * i[2 * c + 1] - e[1] * i[2 * c];
                  }
              }
            o[2 * r] = re;
            o[2 * r + 1] = im;
          }
        (void)low;
      }
}

/* tmclovDkern_eoprec_eos: dirac_operator_tmclovD_eoprec_portable.cpp:42-68 */
void orc_tmclov_kern(const orc_geom *g, const double *conf_eo, double kappa, int has_anis, double anis,
                     const double *Cl_odd, const double *invCl_evn, int dag, double mu, const double *in, double *out)
{
  const int64_t n = g->Vh * SC;
  double *te = (double *)malloc(sizeof(double) * n), *to = (double *)malloc(sizeof(double) * n);
  orc_hop_eo(g, conf_eo, 0, has_anis, anis, in, to);
  orc_inv_tmclovDee(g->Vh, invCl_evn, dag, to, te);
  orc_hop_eo(g, conf_eo, 1, has_anis, anis, te, out);
  orc_tmclovDee(g->Vh, Cl_odd, kappa, dag, mu, in, te);
#pragma omp parallel for
  for (int64_t X = 0; X < g->Vh; X++)
    for (int k = 0; k < 12; k++)
      {
        double *o = out + X * SC;
        const double *t = te + X * SC;
        o[k] = +t[k] - o[k] * 0.25;
        o[k + 12] = -t[k + 12] + o[k + 12] * 0.25;
      }
  free(te);
  free(to);
}

/* tmclovDkern_eoprec_square_eos: dirac_operator_tmclovD_eoprec_portable.cpp:70-84 */
void orc_tmclov_kern2(const orc_geom *g, const double *conf_eo, double kappa, int has_anis, double anis,
                      const double *Cl_odd, const double *invCl_evn, double mu, const double *in, double *out)
{
  double *t = (double *)malloc(sizeof(double) * g->Vh * SC);
  orc_tmclov_kern(g, conf_eo, kappa, has_anis, anis, Cl_odd, invCl_evn, 1, mu, in, t);
  orc_tmclov_kern(g, conf_eo, kappa, has_anis, anis, Cl_odd, invCl_evn, 0, mu, t, out);
  free(t);
}

struct clov2_ctx
{
  const orc_geom *g;
  const double *conf_eo, *Cl_odd, *invCl_evn;
  double kappa;
  int has_anis;
  double anis, mu;
};

static void clov2_op(const void *c, const double *in, double *out)
{
  const struct clov2_ctx *k = (const struct clov2_ctx *)c;
  orc_tmclov_kern2(k->g, k->conf_eo, k->kappa, k->has_anis, k->anis, k->Cl_odd, k->invCl_evn, k->mu, in, out);
}

/* inv_tmclovDkern_eoprec_square_eos_cg -> _cg_64: inverters/twisted_clover/cg_invert_tmclovD_eoprec.cpp:33-52,
 * cg_64_invert_tmclovD_eoprec.hpp:11-44 */
int orc_tmclov_cg_eos(const orc_geom *g, const double *conf_eo, double kappa, int has_anis, double anis,
                      const double *Cl_odd, const double *invCl_evn, double mu, int niter, double residue,
                      const double *guess, const double *src, double *sol, double *true_rel_res2)
{
  struct clov2_ctx k = {g, conf_eo, Cl_odd, invCl_evn, kappa, has_anis, anis, mu};
  return cg_invert(g->Vh, clov2_op, &k, niter, residue, guess, src, sol, true_rel_res2);
}

/* apply_tmclovQ: dirac_operators/tmclovQ/dirac_operator_tmclovQ.cpp:15-170 = apply_tmQ plus
 * gamma5 times the chromo operator (unsafe_apply_point_chromo_operator_to_spincolor,
 * clover_term.hpp:14-30) */
void orc_tmclovQ(const orc_geom *g, const double *conf_lx, double kappa, int has_anis, double anis,
                 const double *Cl_lx, double mu, const double *in, double *out)
{
  orc_tmQ(g, conf_lx, kappa, has_anis, anis, mu, in, out);
#pragma omp parallel for
  for (int64_t X = 0; X < g->V; X++)
    for (int b = 0; b < 2; b++)
      {
        double M[6][6][2];
        clover_block_z(Cl_lx + X * 4 * SU3, b, 0.0, 0.0, M); /* the chromo operator block alone */
        const double *i = in + X * SC + b * 12;
        double *o = out + X * SC + b * 12;
        const double sg = b ? -1.0 : 1.0;
        for (int r = 0; r < 6; r++)
          {
            double re = 0, im = 0;
            for (int c = 0; c < 6; c++)
              {
                const double mr = M[r][c][0], mi = M[r][c][1];
                re += mr * i[2 * c] - mi * i[2 * c + 1];
                im += mr * i[2 * c + 1] + mi * i[2 * c];
              }
            o[2 * r] += sg * re;
            o[2 * r + 1] += sg * im;
          }
      }
}

/* inv_tmclovD_cg_eoprec_native + the residual check of inv_tmclovD_cg_eoprec:
 * inverters/twisted_clover/cg_invert_tmclovD_eoprec.cpp:55-120, :135-220.
 * *lx_rel_res2 = |g5 Q_clov sol - src|^2/|src|^2 */
int orc_tmclov_cg_full(const orc_geom *g, const double *conf_lx, double kappa, int has_anis, double anis, double cSW,
                       double mass, int niter, double residue, const double *src_lx, double *sol_lx,
                       double *lx_rel_res2)
{
  const int64_t V = g->V, Vh = g->Vh, n = Vh * SC;
  double *Cl_lx = (double *)malloc(sizeof(double) * V * 4 * SU3);
  double *Cl_eo = (double *)malloc(sizeof(double) * V * 4 * SU3);
  double *invCl_lx = (double *)malloc(sizeof(double) * V * 144);
  double *invCl_eo = (double *)malloc(sizeof(double) * V * 144);
  orc_clover_term(g, conf_lx, cSW, Cl_lx);
  orc_inv_clover_term(V, Cl_lx, kappa, mass, invCl_lx);
  orc_split_lx_to_eo(g, Cl_lx, 4 * SU3, Cl_eo);
  orc_split_lx_to_eo(g, invCl_lx, 144, invCl_eo);
  const double *Cl_odd = Cl_eo + Vh * 4 * SU3, *invCl_evn = invCl_eo;
  double *conf_eo = (double *)malloc(sizeof(double) * V * QSU3);
  double *src_eo = (double *)malloc(sizeof(double) * 2 * n), *sol_eo = (double *)malloc(sizeof(double) * 2 * n);
  double *evnTemp = (double *)malloc(sizeof(double) * n), *varphi = (double *)malloc(sizeof(double) * n);
  double *oddTemp = (double *)malloc(sizeof(double) * n);
  orc_split_lx_to_eo(g, conf_lx, QSU3, conf_eo);
  orc_split_lx_to_eo(g, src_lx, SC, src_eo);
  const double *src_e = src_eo, *src_o = src_eo + n;
  /* Eq. 8a */
  orc_inv_tmclovDee(Vh, invCl_evn, 0, src_e, evnTemp);
  /* Eq. 8b (inv_tmD_cg_eoprec_prepare_source, twisted_mass/cg_invert_tmD_eoprec.cpp:37-58) */
  orc_hop_eo(g, conf_eo, 1, has_anis, anis, evnTemp, varphi);
#pragma omp parallel for
  for (int64_t X = 0; X < Vh; X++)
    for (int k = 0; k < 12; k++)
      {
        double *v = varphi + X * SC;
        const double *s = src_o + X * SC;
        v[k] = +s[k] + v[k] * 0.5;
        v[k + 12] = -s[k + 12] - v[k + 12] * 0.5;
      }
  /* Eq. 9 */
  double cg_res;
  const int it = orc_tmclov_cg_eos(g, conf_eo, kappa, has_anis, anis, Cl_odd, invCl_evn, mass, niter, residue, NULL,
                                   varphi, oddTemp, &cg_res);
  /* Eq. 10 */
  double *sol_e = sol_eo, *sol_o = sol_eo + n;
  orc_tmclov_kern(g, conf_eo, kappa, has_anis, anis, Cl_odd, invCl_evn, 1, mass, oddTemp, sol_o);
  /* Eq. 11 */
  orc_hop_eo(g, conf_eo, 0, has_anis, anis, sol_o, evnTemp);
#pragma omp parallel for
  for (int64_t i = 0; i < n; i++) evnTemp[i] = src_e[i] + evnTemp[i] * 0.5;
  orc_inv_tmclovDee(Vh, invCl_evn, 0, evnTemp, sol_e);
  orc_paste_eo_to_lx(g, sol_eo, SC, sol_lx);
  if (lx_rel_res2)
    {
      double *rv = (double *)malloc(sizeof(double) * V * SC);
      orc_tmclovQ(g, conf_lx, kappa, has_anis, anis, Cl_lx, mass, sol_lx, rv);
#pragma omp parallel for
      for (int64_t X = 0; X < V; X++)
        for (int k = 0; k < SC; k++)
          {
            const double gv = (k < 12 ? 1 : -1) * rv[X * SC + k];
            rv[X * SC + k] = gv - src_lx[X * SC + k];
          }
      *lx_rel_res2 = scalar_prod(V, rv, rv) / scalar_prod(V, src_lx, src_lx);
      free(rv);
    }
  free(Cl_lx); free(Cl_eo); free(invCl_lx); free(invCl_eo);
  free(conf_eo); free(src_eo); free(sol_eo); free(evnTemp); free(varphi); free(oddTemp);
  return it;
}
