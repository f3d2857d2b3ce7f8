/* tmsolve: B200-native twisted-mass Wilson operator and solvers behind a
 * plain C ABI.
 *
 * Each entry point replaces one entry point of the reference library nissa
 * (paths relative to its src/ directory).  Buffers are the reference's own
 * CPU (AoS) layout in float64:
 *   lx conf    V x [mu][row][col][re,im]            (LxField<quad_su3>)
 *   eo conf    [par][Vh] x [mu][row][col][re,im]    (EoField<quad_su3>)
 *   lx spinor  V x [spin][col][re,im]               (LxField<spincolor>)
 *   eo spinor  Vh x [spin][col][re,im]              (EvnField/OddField<spincolor>)
 * with sites numbered as the reference numbers them (lx: t slowest, z
 * fastest; e/o: lx order within each parity).  By default the pointers are
 * host pointers (copied in and out on every call); after
 * tms_set_pointer_mode(ctx, TMS_PTR_DEVICE) they are device pointers to the
 * same layout.  The library works on its own non-blocking stream: device
 * inputs must be complete when a call is made (the caller synchronises the
 * stream that wrote them), and every call that writes outputs has finished
 * them when it returns.  Every function returns a tms_status; none throws.
 *
 * Residues are SQUARED relative residues, |r|^2/|b|^2, as in the reference
 * (inverters/templates/cg_invert_template_threaded.hpp:129).
 */
#ifndef TMSOLVE_H
#define TMSOLVE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum
{
  TMS_OK = 0,
  TMS_ERR_NOT_CONVERGED = 1, /* reference: CRASH("exit without converging") */
  TMS_ERR_NAN = 2,           /* reference: CRASH("nanned") */
  TMS_ERR_BAD_ARG = 3,
  TMS_ERR_OOM = 4,
  TMS_ERR_TIMEOUT = 5,
  TMS_ERR_CUDA = 6,
  TMS_ERR_NO_CONF = 7,
  TMS_ERR_INVALID_SOURCE = 8, /* reference: CRASH("invalid norm") */
  TMS_ERR_IO = 9              /* a file could not be opened, read, written or parsed */
} tms_status;

typedef enum
{
  TMS_PREC_DOUBLE = 0,      /* plain FP64 CG, the reference's arithmetic */
  TMS_PREC_MIXED_SINGLE = 1,/* FP32 inner CG, 12-real 16-bit (or FP32) links, FP64 reliable updates */
  TMS_PREC_MIXED_HALF = 2   /* FP16 spinors with per-site FP32 scale, FP64 reliable updates */
} tms_precision;

typedef enum { TMS_LAYOUT_LX = 0, TMS_LAYOUT_EO = 1 } tms_layout;
typedef enum { TMS_PTR_HOST = 0, TMS_PTR_DEVICE = 1 } tms_ptr_mode;

/* conf upload flags */
#define TMS_CONF_BC_INCLUDED 1 /* links already carry the time boundary sign, as the reference's operators see them */

typedef struct
{
  int32_t status;           /* tms_status of the solve */
  int32_t iterations;       /* inner CG iterations (the reference's final_iter) */
  int32_t reliable_updates; /* FP64 residual recomputations (mixed precision) */
  int32_t pad;
  double iterated_rel_res2; /* |r_iterated|^2/|b|^2 at exit */
  double true_rel_res2;     /* |b - A x|^2/|b|^2 recomputed in FP64 at exit */
  double lx_rel_res2;       /* full solves: |g5 Q x - src|^2/|src|^2 in lx (cg_invert_tmD_eoprec.cpp:192-212) */
  double seconds;           /* device time of the solve */
} tms_stats;

typedef struct tms_ctx tms_ctx;

/* ---- context: one lattice, one resident gauge configuration, one stream ---- */

/* Lattice T x L^3 on CUDA device `device`; time boundary sign bc_t (-1 antiperiodic, +1 periodic).
 * Replaces initGrid(T,L) (base/init.cpp:563-798) and the e/o geometry it builds
 * (geometry/geometry_eo.cpp:41-100), per instance instead of process-global. */
tms_status tms_create(tms_ctx **ctx, int T, int L, double bc_t, int device);
/* General T x LX x LY x LZ form (all even). */
tms_status tms_create4(tms_ctx **ctx, int T, int LX, int LY, int LZ, double bc_t, int device);
tms_status tms_destroy(tms_ctx *ctx);
const char *tms_last_error(const tms_ctx *ctx);
tms_status tms_set_pointer_mode(tms_ctx *ctx, int mode);
int64_t tms_volume(const tms_ctx *ctx);

/* Device copies of the reference's geometry tables, for bit-exact checks against
 * loclx_parity/loceo_of_loclx/loclx_of_loceo/loceo_neighup/loceo_neighdw
 * (geometry/geometry_eo.cpp:66-100).  Host int32 outputs: parity[V], eo_of_lx[V],
 * lx_of_eo[2*Vh], neighup[2*Vh*4], neighdw[2*Vh*4]; any may be NULL. */
tms_status tms_geometry_tables(tms_ctx *ctx, int32_t *parity, int32_t *eo_of_lx, int32_t *lx_of_eo,
                               int32_t *neighup, int32_t *neighdw);

/* Upload the gauge configuration (kept resident until replaced or destroyed).
 * Replaces the conf argument of every operator and split_lx_vector_into_eo_parts
 * of the conf (geometry/geometry_mix.hpp:46-60, done once here instead of per call). */
tms_status tms_conf_upload(tms_ctx *ctx, const double *conf, int layout, int flags);
/* 1 if the links are special unitary (12-real reconstruction enabled for FP32), 0 if not */
int tms_conf_is_su3(const tms_ctx *ctx);

/* ---- operators (e/o) ---- */

/* tmn2Deo_or_tmn2Doe_eos: dirac_operators/tmD_eoprec/dirac_operator_tmD_eoprec_portable.hpp:33-169.
 * out (parity par_out) = -2 x hopping of in (opposite parity). has_anis=0: no anisotropy. */
tms_status tms_hop_eo(tms_ctx *ctx, int par_out, const double *in, double *out, int has_anis, double anis);
/* tmDee_or_oo_eos / inv_tmDee_or_oo_eos: ..._portable.hpp:171-222 */
tms_status tms_tmDee(tms_ctx *ctx, double kappa, double mu, const double *in, double *out);
tms_status tms_inv_tmDee(tms_ctx *ctx, double kappa, double mu, const double *in, double *out);
/* tmDkern_eoprec_eos: dirac_operator_tmD_eoprec_portable.cpp:36-51 (odd -> odd) */
tms_status tms_kern_eoprec(tms_ctx *ctx, double kappa, int has_anis, double anis, double mu, const double *in,
                           double *out);
/* tmDkern_eoprec_square_eos: dirac_operator_tmD_eoprec_portable.cpp:54-65, K(+mu)K(-mu) */
tms_status tms_kern_eoprec_square(tms_ctx *ctx, double kappa, int has_anis, double anis, double mu,
                                  const double *in, double *out);

/* ---- operators (full lattice, lx spinors) ---- */

/* apply_tmQ: dirac_operators/tmQ/dirac_operator_tmQ_portable.cpp:29-176 */
tms_status tms_apply_tmQ(tms_ctx *ctx, double kappa, int has_anis, double anis, double mu, const double *in,
                         double *out);
/* apply_tmQ2: Q(+mu)Q(-mu), dirac_operators/tmQ2/dirac_operator_tmQ2.cpp:17-30 (a stub in the
 * reference; the body there, and apply_tmclovQ2 at zero clover, tmclovQ2/dirac_operator_tmclovQ2.hpp:13-24) */
tms_status tms_apply_tmQ2(tms_ctx *ctx, double kappa, int has_anis, double anis, double mu, const double *in,
                          double *out);

/* ---- solvers ---- */

/* inv_tmDkern_eoprec_square_eos_cg: inverters/twisted_mass/cg_invert_tmD_eoprec.cpp:61-78
 * Solves K(+mu)K(-mu) sol = src on odd sites.  guess may be NULL (sol starts at 0);
 * stops when |r|^2 < residue |src|^2 or after niter iterations. */
tms_status tms_cg_eoprec_square(tms_ctx *ctx, double *sol, const double *guess, const double *src, double kappa,
                                int has_anis, double anis, double mu, int niter, double residue, int precision,
                                tms_stats *stats);
/* inv_tmD_cg_eoprec: inverters/twisted_mass/cg_invert_tmD_eoprec.cpp:102-213
 * Full solve D_tm sol = src on lx spinors via Eq. (8)-(11) of the e/o preconditioning. */
tms_status tms_cg_eoprec(tms_ctx *ctx, double *sol_lx, const double *src_lx, double kappa, int has_anis,
                         double anis, double mu, int niter, double residue, int precision, tms_stats *stats);
/* The same with the reference's optional guess_Koo (inv_tmD_cg_eoprec's second argument,
 * cg_invert_tmD_eoprec.cpp:102-137): an odd-site e/o spinor (Vh rows) from which the Eq. (9) CG
 * starts; NULL for none.  Read only (the reference writes the new Koo solution into its by-value
 * copy of the guess, so its caller sees no change either). */
tms_status tms_cg_eoprec_guess(tms_ctx *ctx, double *sol_lx, const double *guess_Koo, const double *src_lx,
                               double kappa, int has_anis, double anis, double mu, int niter, double residue,
                               int precision, tms_stats *stats);
/* inv_tmD_cg_eoprec for ncols sources one after the other (the loop over the 12 spin-colour columns
 * of a propagator, projects/ib/prop.cpp:41-112, calls it once per column).  Each column is the same
 * solve as tms_cg_eoprec; with host pointers the copy of column k+1's source in and of column k-1's
 * solution out run on a copy stream while column k is solved (page-locked host buffers overlap,
 * pageable ones are copied all the same).  sols_lx/srcs_lx are arrays of ncols lx spinors; stats
 * (may be NULL) receives ncols entries.  Returns the first error, else TMS_ERR_NOT_CONVERGED if a
 * column did not converge (its solution is still written), else TMS_OK; no copy into or out of the
 * caller's buffers is left running when it returns. */
tms_status tms_cg_eoprec_columns(tms_ctx *ctx, int ncols, double *const *sols_lx, const double *const *srcs_lx,
                                 double kappa, int has_anis, double anis, double mu, int niter, double residue,
                                 int precision, tms_stats *stats);

/* inv_tmQ2_cg: inverters/twisted_mass/cg_invert_tmQ2_common.cpp:5 (a CRASH("reimplement") stub in the
 * reference, cg_invert_tmQ2.cpp:12-14).  Full-lattice CG on Q(+m)Q(-m) = Q_W^2 + m^2 (lx spinors);
 * guess may be NULL. */
tms_status tms_cg_tmQ2(tms_ctx *ctx, double *sol_lx, const double *guess_lx, const double *src_lx, double kappa,
                       int has_anis, double anis, double m, int niter, double residue, int precision,
                       tms_stats *stats);
/* inv_tmQ2_cgm: inverters/twisted_mass/cgm_invert_tmQ2.cpp:46-53 (stub behind it) and its working
 * counterpart inv_tmclovQ2_cgm at zero clover (inverters/twisted_clover/cgm_invert_tmclovQ2.cpp:10-32,
 * cgm_invert in inverters/templates/cgm_invert_template_threaded.hpp:11-295).
 * Solves (Q_W^2 + m_k^2) sol_k = src for nmass (<= 32) masses at once; sols is an array of nmass lx
 * spinors (nissa's spincolor**), residues the per-shift squared relative residues.  TMS_PREC_DOUBLE is
 * the reference's FP64 multi-shift CG; the mixed precisions run it in FP32 down to the squared residue
 * "cgm_floor_single" (tms_set_tuning, default 1e-12) and bring each shift to its target by defect
 * correction through the mixed-precision e/o solver (e = D(-m)^-1 g5 D(+m)^-1 g5 r, since
 * Q_W^2 + m^2 = Q(+m) Q(-m) and Q = g5 D), checking every shift's true residual in FP64.
 * stats (may be NULL) receives nmass entries. */
tms_status tms_cgm_tmQ2(tms_ctx *ctx, double *const *sols, const double *src_lx, double kappa, int has_anis,
                        double anis, const double *masses, int nmass, int niter, const double *residues,
                        int precision, tms_stats *stats);

/* Batched inv_tmD_cg_eoprec (the reference solves one right-hand side per call,
 * inverters/twisted_mass/cg_invert_tmD_eoprec.cpp:152-213): nrhs (<= 64) lx sources with one kappa
 * and a twisted mass mus[k] each; the e/o CG of all of them runs in lock step so that each hop reads
 * the links once for every right-hand side.  Each right-hand side stops at its own residues[k]
 * (squared, relative); the FP64 reliable updates of the mixed precisions are per right-hand side.
 * sols_lx/srcs_lx are arrays of nrhs lx spinors; stats (may be NULL) receives nrhs entries. */
tms_status tms_cg_eoprec_batched(tms_ctx *ctx, int nrhs, double *const *sols_lx, const double *const *srcs_lx,
                                 double kappa, int has_anis, double anis, const double *mus, int niter,
                                 const double *residues, int precision, tms_stats *stats);

/* ---- time-slab decomposition (replaces, for a split along time, the reference's halo exchange
 * before each hop, base/field.cpp:11-56, and its all-reduce after each scalar product,
 * base/field.hpp:904) ----
 * A slab context owns the time slices [t0, t0 + T_loc) of a T x LX x LY x LZ lattice (t0, T_loc
 * even); its conf is uploaded as the slab's own links in lx layout (tms_conf_upload: sites of the
 * slab only, local t = 0 .. T_loc-1).  The time hops that leave the slab read two faces of
 * tms_slab_face_sites(ctx) sites x 6 complex (double[face][6][2] laid out as six planes of face
 * complex: plane k = colour k of h0 (k < 3) or colour k-3 of h1) that the neighbouring slabs pack:
 *   face_fwd: packed by the NEXT slab from its first slice (the forward (1 - g_t) projection),
 *   face_bwd: packed by the PREVIOUS slab from its last slice (U_t^+ times the backward projection),
 * so no link crosses a slab boundary.  The time-boundary sign is applied by the slab that receives
 * across t = T-1 -> 0 (the bc_t given at creation).  Slab operators are exactly the single-context
 * ones on the whole lattice. */
tms_status tms_create_slab(tms_ctx **ctx, int T, int t0, int T_loc, int LX, int LY, int LZ, double bc_t, int device);
/* sites of one parity on one time slice (LX LY LZ / 2): the length of a face */
int64_t tms_slab_face_sites(const tms_ctx *ctx);
/* Pack the two faces of e/o spinor `in` (parity par_in, Vh x 24 AoS): face_fwd for the previous
 * slab, face_bwd for the next one (each face_sites x 12 doubles). */
tms_status tms_slab_pack(tms_ctx *ctx, int par_in, const double *in, double *face_fwd, double *face_bwd);
/* tmn2Deo_or_tmn2Doe_eos on the slab: out (parity par_out) from in (the other parity) and the two
 * faces received for `in` (ghost_fwd from the next slab, ghost_bwd from the previous one). */
tms_status tms_slab_hop(tms_ctx *ctx, int par_out, const double *in, const double *ghost_fwd, const double *ghost_bwd,
                        double *out, int has_anis, double anis);
/* The two halves of tmDkern_eoprec_eos (dirac_operator_tmD_eoprec_portable.cpp:36-51) on the slab:
 * which = 0: out_even = (1/2k + i mu g5)^-1 D_eo in_odd; which = 1: out_odd = g5 ((1/2k + i mu g5) x
 * - D_oe in_even / 4), x the odd operand of the first half.  Faces as for tms_slab_hop, packed from
 * the half's own input. */
tms_status tms_slab_kern_half(tms_ctx *ctx, int which, double kappa, double mu, const double *in,
                              const double *ghost_fwd, const double *ghost_bwd, const double *x, double *out,
                              int has_anis, double anis);

/* ---- batch sessions (continuous batching; no reference counterpart) ----
 * A session keeps up to nslots (<= 64) solves of inv_tmD_cg_eoprec in flight on one context, each
 * with its own kappa, mu and residue: submit puts a right-hand side into a free slot (the source is
 * prepared at once, Eq. 8), step runs one CUDA-graph block of lock-step CG iterations for all
 * running slots and reports the slots that finished, collect writes a finished slot's solution
 * (Eq. 10-11) and frees the slot.  New right-hand sides can be submitted between steps while
 * others are still iterating.  One session per context at a time; one host thread per context. */
typedef struct tms_batch tms_batch;
tms_status tms_batch_open(tms_ctx *ctx, int nslots, int precision, int has_anis, double anis, tms_batch **batch);
tms_status tms_batch_submit(tms_batch *batch, int slot, const double *src_lx, double kappa, double mu, int niter,
                            double residue);
/* finished[nslots] (out): 1 for the slots that finished in this step; *nfinished (may be NULL) their count */
tms_status tms_batch_step(tms_batch *batch, int *finished, int *nfinished);
/* returns the solve's status (TMS_OK, TMS_ERR_NOT_CONVERGED, TMS_ERR_NAN) */
tms_status tms_batch_collect(tms_batch *batch, int slot, double *sol_lx, tms_stats *stats);
tms_status tms_batch_close(tms_batch *batch);

/* ---- twisted clover: the reference's tmclov e/o path ---- */

/* clover_term (operations/su3_paths/clover_term.hpp:104-112; chromo_operator clover_term.cpp:57-95,
 * four_leaves_point measures/gauge/topological_charge.hpp:139-212): compute on the device, in FP64,
 * the clover term of the uploaded conf as the reference's operators see it (time-boundary sign
 * on the t = T-1 time links) times -(cSW + 1e-16)/4, and keep it until the next conf upload.
 * The operators below use it; the twisted inverse on even sites (invert_twisted_clover_term,
 * clover_term.hpp:143-262) is computed for each (kappa, mu) on first use and kept. */
tms_status tms_clover_term(tms_ctx *ctx, double cSW);
/* the kept clover term in the reference's lx layout: V x [4][3][3][re,im] (LxField<clover_term_t>) */
tms_status tms_clover_get(tms_ctx *ctx, double *cl_lx);
/* tmclovDee_or_oo_eos (dirac_operators/tmclovD_eoprec/dirac_operator_tmclovD_eoprec_portable.cpp:18-40)
 * on the Vh sites of parity par */
tms_status tms_tmclovDee(tms_ctx *ctx, int par, double kappa, double mu, int dag, const double *in, double *out);
/* inv_tmclovDee_or_oo_eos (dirac_operator_tmclovD_eoprec.hpp:24-44) on the even sites */
tms_status tms_inv_tmclovDee(tms_ctx *ctx, double kappa, double mu, int dag, const double *in, double *out);
/* tmclovDkern_eoprec_eos (dirac_operator_tmclovD_eoprec_portable.cpp:42-68): odd -> odd */
tms_status tms_tmclovDkern_eoprec(tms_ctx *ctx, double kappa, int has_anis, double anis, double mu, int dag,
                                  const double *in, double *out);
/* tmclovDkern_eoprec_square_eos (dirac_operator_tmclovD_eoprec_portable.cpp:70-84): K(false) K(true) */
tms_status tms_tmclovDkern_eoprec_square(tms_ctx *ctx, double kappa, int has_anis, double anis, double mu,
                                         const double *in, double *out);
/* apply_tmclovQ (dirac_operators/tmclovQ/dirac_operator_tmclovQ.cpp:15-170): lx -> lx */
tms_status tms_apply_tmclovQ(tms_ctx *ctx, double kappa, int has_anis, double anis, double mu, const double *in,
                             double *out);
/* inv_tmclovDkern_eoprec_square_eos_cg (inverters/twisted_clover/cg_invert_tmclovD_eoprec.cpp:33-52,
 * cg_64_invert_tmclovD_eoprec.hpp:11-44): CG on K(false)K(true), odd sites, with the kept clover term */
tms_status tms_cg_tmclov_eoprec_square(tms_ctx *ctx, double *sol, const double *guess, const double *src,
                                       double kappa, int has_anis, double anis, double mu, int niter, double residue,
                                       int precision, tms_stats *stats);
/* inv_tmclovD_cg_eoprec (inverters/twisted_clover/cg_invert_tmclovD_eoprec.cpp:55-220): full solve in
 * lx via e/o preconditioning (Eq. 8-11 with the clover diagonal), computing the clover term for cSW
 * when it differs from the kept one; stats->lx_rel_res2 is the reference's final check
 * |g5 Q_clov sol - src|^2/|src|^2 */
tms_status tms_cg_tmclov_eoprec(tms_ctx *ctx, double *sol_lx, const double *src_lx, double kappa, int has_anis,
                                double anis, double cSW, double mu, int niter, double residue, int precision,
                                tms_stats *stats);

/* ---- caller-side steps around a propagator solve ---- */

/* safe_dirac_prod_spincolor with P- (r = 0) or P+ (r = 1), the twisted-basis rotation of
 * projects/ib/prop.cpp:50-59 and :104-112 (tau3 = {-1,+1}, new_types/dirac.hpp:38-41;
 * P+- = (1 +- i g5)/sqrt2, new_types/dirac.cpp:60-61), on an lx spinor */
tms_status tms_rotate_twisted(tms_ctx *ctx, int r, const double *in_lx, double *out_lx);
/* get_qprop (projects/ib/prop.cpp:41-112) without the photon and free-theory branches: the
 * source rotated by P(r) when rotate_source (the reference's twisted_run), the solve
 * (inv_tmclovD_cg_eoprec when cSW != 0, else inv_tmD_cg_eoprec), the sink rotated by P(r),
 * all on the device */
tms_status tms_get_qprop(tms_ctx *ctx, int r, int rotate_source, double kappa, int has_anis, double anis, double cSW,
                         double mu, int niter, double residue, int precision, const double *src_lx, double *out_lx,
                         tms_stats *stats);
/* reconstruct_tm_doublet (dirac_operators/tmQ/reconstruct_tm_doublet.cpp:13-26; a stub there, whose
 * commented body is followed): outminus = Q(+mu) in, outplus = outminus - 2 i mu in */
tms_status tms_reconstruct_tm_doublet(tms_ctx *ctx, double kappa, int has_anis, double anis, double mu,
                                      const double *in_lx, double *outminus_lx, double *outplus_lx);

/* ---- gauge configuration files and checks ---- */

/* read_ildg_gauge_conf (io/reader.hpp:75-99, io/ILDG_File.cpp): read the 'ildg-binary-data'
 * record of an ILDG (LIME) file, big-endian, 32- or 64-bit as its 'ildg-format' record says
 * (whose lattice sizes must match the context's), reordered to the reference's lx sites and
 * t,x,y,z directions, into conf_lx (a HOST buffer of V x 72 doubles, whatever the pointer
 * mode).  No boundary phase is applied (the file holds periodic links). */
tms_status tms_read_ildg(tms_ctx *ctx, const char *path, double *conf_lx);
/* The inverse: write conf_lx (host, the reference's lx layout) as an ILDG file with an
 * 'ildg-format' record and the big-endian 'ildg-binary-data' record; precision 32 or 64. */
tms_status tms_write_ildg(tms_ctx *ctx, const char *path, const double *conf_lx, int precision);
/* tms_read_ildg followed by tms_conf_upload(ctx, conf, TMS_LAYOUT_LX, flags). */
tms_status tms_conf_load_ildg(tms_ctx *ctx, const char *path, int flags);
/* global_plaquette_lx_conf (operations/su3_paths/plaquette.hpp:25-82) of the uploaded conf,
 * computed on the device in FP64: the mean of the temporal and spatial averages of
 * Re tr(U_mu(x) U_nu(x+mu) U_mu(x+nu)^+ U_nu(x)^+)/3.  with_bc = 0: the periodic links as
 * stored; 1: with the context's time-boundary sign on the t = T-1 time links. */
tms_status tms_conf_plaquette(tms_ctx *ctx, int with_bc, double *plaquette);

/* ---- instrumentation (no reference counterpart) ---- */

/* Number of CUDA kernels this context has launched (CUDA-graph replays count their nodes). */
uint64_t tms_launch_count(const tms_ctx *ctx);
/* Tiles of the staged hopping kernel (launch shape 7) whose bounded wait for their shared-memory
 * copies gave up (their outputs are not written): 0 unless the memory system failed to deliver a
 * copy; -1 on a CUDA error.  Waits for the context's stream. */
int64_t tms_hop_stage_timeouts(tms_ctx *ctx);
/* Tuning knobs (no reference counterpart), used by the autotuner: "hop_cfg_double",
 * "hop_cfg_single", "hop_cfg_half" (hopping-kernel launch shape 0..2: one site per thread, 128 threads;
 * 128 threads with registers capped for 4 (FP64) / 8 resident blocks; 256 threads capped for 2 / 4;
 * single and half only, when T is a multiple of 4 (else shape 0 is used): 3 two sites (t, t+T/2) per
 * thread in packed FP32 arithmetic with the neighbours streamed through shared memory by cp.async,
 * 4 two sites per thread in packed FP32 arithmetic; for any T: 5 one site per thread with the two spin
 * rows of each half spinor in the lanes of packed FP32 arithmetic, 6 the same with each thread's
 * neighbour spinors and links streamed through its own shared-memory slots by cp.async, two
 * directions ahead, 7 tiles of lattice rows whose neighbour faces and links are staged
 * in shared memory by bulk asynchronous copies before the same arithmetic (LZ a multiple of 8 and
 * 16-bit or FP32 12-real links, else shape 0 is used)), "tma_rows" (the site tiling of shape 7: lattice
 * rows of LZ/2 sites per tile, a divisor R of LY with R*LZ/2 <= 128 and either R == LY or R + 2 <= LY
 * and R*LZ/2 >= 16; 0
 * (default): the most that fit),
 * "graph_iters" (CG iterations per CUDA graph replay, 1..64), "reliable_delta_single",
 * "reliable_delta_half" (the mixed solvers recompute the FP64 residual when the iterated one has
 * dropped by this factor, 0 < delta < 1), "links_single" (0: the FP32-spinor inner solver reads FP32
 * 12-real links, 1 (default): 16-bit fixed-point 12-real links, as fast or faster from 8^3x16 to 32^3x64), "links_reliable" (1 (default): the FP64
 * residual recomputations of the mixed solvers read the links as 12 reals, row 2 rebuilt, when the conf
 * is SU(3) to 1e-13; 0: always 18 reals), "mrhs_per_thread" (right-hand sides one thread of the
 * batched hopping kernel computes from each link it loads: 1, 2, 4; FP64 uses at most 2; 0: one, with
 * its gathers streamed through the thread's shared-memory slots by cp.async, FP32 arithmetic only),
 * "batch_graph_iters" (CG iterations per batch-session graph block, 0: chosen by batch size),
 * "cgm_refine_batched" (mixed multi-shift solver: 0 (default) corrects the shifts one after the other
 * through the e/o solver, 1 corrects all shifts as two batched e/o solves per round, one right-hand
 * side per shift), 
 * "half_arith" (FP16-spinor e/o twisted-mass solver with SU(3) links: 0 (default) FP32 arithmetic; 1 the
 * pipelined hop in FP16 arithmetic on FP16 12-real links, about 10 % faster per hop, its operator 6e-4 from
 * the FP32-arithmetic one; the solution is still brought to the target by the FP64 reliable updates, in
 * about 15 % more iterations at 32^3x64 with the default reliable_delta_half, 3 % more and 3-5 % less time per
 * solve with reliable_delta_half 0.01),
 * "stream_priority" (the context's stream is recreated with this CUDA stream priority, an integer in the
 * device's range, lower first; contexts of small volumes sharing a GPU with large ones use it).  Results do not depend on the launch shapes. */
tms_status tms_set_tuning(tms_ctx *ctx, const char *key, double value);
/* The current value of a tuning knob (the keys of tms_set_tuning). */
tms_status tms_get_tuning(tms_ctx *ctx, const char *key, double *value);
/* Time the e/o hopping kernel alone with CUDA events on the context's stream: nrep launches,
 * each preceded (untimed) by a 512 MiB write that flushes the L2 when flush=1.
 * precision: tms_precision; variant 0 plain hop, 1 hop + inverse diagonal (CG first half),
 * 2 hop + diagonal + gamma5 combine + |out|^2 reduction (CG second half).
 * Outputs the mean device time per launch and the algorithmic (compulsory) bytes per launch:
 * Vh x (8 links + input spinor + output spinor [+ own-site spinor for variant 2]). */
tms_status tms_bench_hop(tms_ctx *ctx, int precision, int variant, int nrep, int flush, double *ms_per_launch,
                         double *bytes_per_launch);

/* tms_bench_hop for the batched (multi-RHS) hopping kernel with the inverse-diagonal epilogue:
 * nrhs right-hand sides per launch; algorithmic bytes = Vh x (8 links + 2 nrhs spinors). */
tms_status tms_bench_hop_batched(tms_ctx *ctx, int precision, int nrhs, int nrep, int flush, double *ms_per_launch,
                                 double *bytes_per_launch);

/* ---- allocation-free hopping (no counterpart in the reference) ---- */

/* Lattices of at most this many sites are accepted by tms_hop_eo_noalloc. */
#define TMS_NOALLOC_MAX_SITES 16384

/* The e/o hopping of tms_hop_eo for callers that cannot let a library allocate
 * device memory (an application whose own pool owns all device memory, or a
 * phase where cudaMalloc/cudaFree would synchronise the device).  Needs no
 * context: the caller passes the gauge configuration each call, like the
 * reference's operators, and all buffers are DEVICE pointers in the layouts
 * above (conf: layout TMS_LAYOUT_LX or TMS_LAYOUT_EO, flags as for
 * tms_conf_upload; in/out: Vh e/o spinors).  Runs on the caller's current
 * device and on `stream` (NULL: the legacy default stream), and returns after
 * the stream has finished the work.
 *
 * It calls no cudaMalloc/cudaFree and no allocating library routine: its
 * scratch is one fixed device array of TMS_NOALLOC_MAX_SITES*768+256 bytes
 * (12 MiB) that every GPU loading this library holds until the process exits.
 * The first call on a device is its set-up: with the device current it looks
 * up that array's device address (cudaGetSymbolAddress), which under CUDA's
 * default lazy module loading also loads the library's device code there and
 * materialises the array; make that first call before any stream capture and
 * outside any phase that must not see device memory appear.  The address is
 * kept for the life of the process, so the entry point is not for use across a
 * cudaDeviceReset.  All calls share the array: calls that overlap on the GPU
 * race and must be serialised by the caller.  Lattices larger than
 * TMS_NOALLOC_MAX_SITES are rejected with TMS_ERR_BAD_ARG; `err` (may be NULL)
 * receives a message of at most errlen bytes. */
tms_status tms_hop_eo_noalloc(int T, int L, double bc_t, const double *conf, int layout, int flags, int par_out,
                              const double *in, double *out, int has_anis, double anis, void *stream, char *err,
                              int errlen);

#ifdef __cplusplus
}
#endif
#endif
