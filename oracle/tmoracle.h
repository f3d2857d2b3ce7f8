/* CPU oracle for the twisted-mass Wilson hot path: a plain-C restatement of
 * the reference library's algorithms, used ONLY as the checker by the tests,
 * by __graft_entry__.smoke() and by bench.py's CPU-baseline leg.  The product
 * (nissa_b200/) never links or calls it.
 *
 * Data are float64 in the reference's CPU (AoS) layout:
 *   lx conf   [V][mu][row][col][re,im]          (base/field.hpp:407-416, new_types/su3.hpp:52-55)
 *   eo conf   [par][Vh][mu][row][col][re,im]    (EoField<quad_su3>, base/field.hpp:1580-1805)
 *   spinors   [sites][spin][col][re,im]         (new_types/su3.hpp:33)
 * Lattice sizes follow initGrid(T,L) (base/init.cpp:563): T x L^3, all even.
 * Pinned against the reference itself: tests/golden holds outputs of the
 * reference's own code (built by oracle/ref_build) on seeded inputs. */
#ifndef TMORACLE_H
#define TMORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_geom orc_geom;

orc_geom *orc_geom_create(int T, int L);
void orc_geom_destroy(orc_geom *g);
int64_t orc_geom_vol(const orc_geom *g);

/* tables as the reference builds them (geometry_lx.cpp:403-424, geometry_eo.cpp:66-100):
 * parity[V], eo_of_lx[V], lx_of_eo[2][Vh], neighup_eo/neighdw_eo[2][Vh][4], neighup_lx/neighdw_lx[V][4] */
void orc_geom_tables(const orc_geom *g, int32_t *parity, int32_t *eo_of_lx, int32_t *lx_of_eo,
                     int32_t *neighup_eo, int32_t *neighdw_eo, int32_t *neighup_lx, int32_t *neighdw_lx);

void orc_split_lx_to_eo(const orc_geom *g, const double *lx, int ndeg, double *eo);
void orc_paste_eo_to_lx(const orc_geom *g, const double *eo, int ndeg, double *lx);

/* has_anis=0 means no anisotropy (std::nullopt in the reference) */
void orc_hop_eo(const orc_geom *g, const double *conf_eo, int par_out, int has_anis, double anis,
                const double *in, double *out);
void orc_tmDee(const orc_geom *g, double kappa, double mu, const double *in, double *out);
void orc_inv_tmDee(const orc_geom *g, double kappa, double mu, const double *in, double *out);
void orc_kern(const orc_geom *g, const double *conf_eo, double kappa, int has_anis, double anis, double mu,
              const double *in, double *out);
void orc_kern2(const orc_geom *g, const double *conf_eo, double kappa, int has_anis, double anis, double mu,
               const double *in, double *out);

/* returns the number of iterations (the reference's final_iter); *true_rel_res2 = |b-Ax|^2/|b|^2 */
int orc_cg_eos(const orc_geom *g, const double *conf_eo, double kappa, int has_anis, double anis, double mu,
               int niter, double residue, const double *guess, const double *src, double *sol,
               double *true_rel_res2);
int orc_cg_full(const orc_geom *g, const double *conf_lx, double kappa, int has_anis, double anis, double mu,
                int niter, double residue, const double *src_lx, double *sol_lx, double *lx_rel_res2);

void orc_tmQ(const orc_geom *g, const double *conf_lx, double kappa, int has_anis, double anis, double mu,
             const double *in, double *out);
void orc_tmQ2(const orc_geom *g, const double *conf_lx, double kappa, int has_anis, double anis, double mu,
              const double *in, double *out);
int orc_cgm(const orc_geom *g, const double *conf_lx, double kappa, int has_anis, double anis, int nshift,
            const double *masses, const double *residues, int niter, const double *src, double *sols,
            double *true_rel_res2);

/* twisted clover (clover term [sites][4][3][3][2], inverse [sites][2][6][6][2]) */
void orc_clover_term(const orc_geom *g, const double *conf_lx, double cSW, double *Cl_lx);
void orc_inv_clover_term(int64_t nsites, const double *Cl, double kappa, double mass, double *invCl);
void orc_tmclovDee(int64_t nsites, const double *Cl, double kappa, int dag, double mu, const double *in, double *out);
void orc_inv_tmclovDee(int64_t nsites, const double *invCl, int dag, const double *in, double *out);
void orc_tmclov_kern(const orc_geom *g, const double *conf_eo, double kappa, int has_anis, double anis,
                     const double *Cl_odd, const double *invCl_evn, int dag, double mu, const double *in, double *out);
void orc_tmclov_kern2(const orc_geom *g, const double *conf_eo, double kappa, int has_anis, double anis,
                      const double *Cl_odd, const double *invCl_evn, double mu, const double *in, double *out);
int orc_tmclov_cg_eos(const orc_geom *g, const double *conf_eo, double kappa, int has_anis, double anis,
                      const double *Cl_odd, const double *invCl_evn, double mu, int niter, double residue,
                      const double *guess, const double *src, double *sol, double *true_rel_res2);
void orc_tmclovQ(const orc_geom *g, const double *conf_lx, double kappa, int has_anis, double anis,
                 const double *Cl_lx, double mu, const double *in, double *out);
int orc_tmclov_cg_full(const orc_geom *g, const double *conf_lx, double kappa, int has_anis, double anis, double cSW,
                       double mass, int niter, double residue, const double *src_lx, double *sol_lx,
                       double *lx_rel_res2);

double orc_plaquette(const orc_geom *g, const double *conf_lx);
double orc_norm2(int64_t n, const double *v);

#ifdef __cplusplus
}
#endif
#endif
