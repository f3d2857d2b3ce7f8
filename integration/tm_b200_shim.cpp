// The reference's twisted-mass e/o entry points on libtmsolve (B200).
//
// Linked into the reference library in place of three of its translation
// units (dirac_operators/tmD_eoprec/dirac_operator_tmD_eoprec.cpp,
// dirac_operators/tmQ/dirac_operator_tmQ.cpp,
// inverters/twisted_mass/cg_invert_tmD_eoprec.cpp) and of the stub of the
// multi-mass entry point (inverters/twisted_mass/cgm_invert_tmQ2.cpp), it
// keeps their C++ signatures, so every caller (projects/ib/prop.cpp:96 and
// the rest) is unchanged, and forwards to the C ABI of include/tmsolve.h.
//
// * One context per process, as the reference's geometry is process-global
//   (initGrid, base/init.cpp:563); one rank only: the shim refuses nranks > 1.
// * Links are used exactly as the caller passes them, boundary phases
//   included (the context is periodic in time and nothing is unfolded), as
//   the reference's operators use them.
// * The uploaded configuration is kept until the caller's conf changes: the
//   cache key is the conf's address and size plus a hash of 4096 links
//   sampled evenly through it, so a conf rewritten in place (the same
//   allocation handed back by the reference's memory manager,
//   base/memory_manager.hpp:221) is uploaded again.  A caller that changes
//   only a few links in place calls nissa::b200::conf_changed().
// * Arithmetic: FP64, the reference's precision, unless the caller opts in
//   to a mixed-precision inner solver (same true residual, recomputed in
//   FP64, faster): NISSA_B200_PRECISION=single|half in the environment, or
//   nissa::b200::set_precision().
// * Tuning knobs of the library (tms_set_tuning: launch shapes, the
//   FP16-arithmetic hop, reliable-update factors, ...) from the environment:
//   NISSA_B200_TUNING="key=value,key=value", applied when the context is
//   created; an unknown key or a refused value stops the program (CRASH).
// * Failures keep the reference's semantics: CRASH (base/debug.hpp:25) on a
//   non-converged solve, a NaN or an invalid source, with the library's
//   message.
#include <config.hpp>

#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <optional>
#include <string>
#include <vector>

#include "base/debug.hpp"
#include "base/field.hpp"
#include "inverters/twisted_mass/cgm_invert_tmQ2.hpp"
#include "geometry/geometry_eo.hpp"
#include "geometry/geometry_lx.hpp"
#include "new_types/su3.hpp"
#include "routines/mpi_routines.hpp"

#include <tmsolve.h>

namespace nissa
{
  namespace b200
  {
    namespace
    {
      tms_ctx* ctx = nullptr;
      int precision = -1;
      uint64_t uploaded_key = 0;
      bool have_conf = false;

      void check(tms_status s, const char* what)
      {
        if (s == TMS_OK) return;
        CRASH("%s failed (%d): %s", what, (int)s, ctx ? tms_last_error(ctx) : "no context");
      }

      tms_ctx* context()
      {
        if (ctx) return ctx;
        if (nranks > 1) CRASH("the B200 shim runs on one rank (nranks=%d)", nranks);
        check(tms_create4(&ctx, glbSize[0], glbSize[1], glbSize[2], glbSize[3], +1.0, 0), "tms_create4");
        if (const char* e = std::getenv("NISSA_B200_TUNING"))
          {
            // "key=value,key=value"
            std::string all(e);
            size_t pos = 0;
            while (pos < all.size())
              {
                size_t end = all.find(',', pos);
                if (end == std::string::npos) end = all.size();
                const std::string kv = all.substr(pos, end - pos);
                const size_t eq = kv.find('=');
                if (eq == std::string::npos || eq == 0) CRASH("NISSA_B200_TUNING: '%s' is not key=value", kv.c_str());
                const std::string key = kv.substr(0, eq);
                char* rest = nullptr;
                const double value = std::strtod(kv.c_str() + eq + 1, &rest);
                if (rest == kv.c_str() + eq + 1 || *rest) CRASH("NISSA_B200_TUNING: bad value in '%s'", kv.c_str());
                check(tms_set_tuning(ctx, key.c_str(), value), "tms_set_tuning");
                pos = end + 1;
              }
          }
        return ctx;
      }

      int prec()
      {
        if (precision < 0)
          {
            const char* e = std::getenv("NISSA_B200_PRECISION");
            precision = TMS_PREC_DOUBLE;
            if (e && !std::strcmp(e, "single")) precision = TMS_PREC_MIXED_SINGLE;
            if (e && !std::strcmp(e, "half")) precision = TMS_PREC_MIXED_HALF;
          }
        return precision;
      }

      uint64_t key_of(const void* a, const void* b, size_t ndoubles)
      {
        uint64_t h = 1469598103934665603ull;
        auto mix = [&](uint64_t v) {
          for (int i = 0; i < 8; i++)
            {
              h ^= (v >> (8 * i)) & 0xff;
              h *= 1099511628211ull;
            }
        };
        mix((uint64_t)(uintptr_t)a);
        mix((uint64_t)(uintptr_t)b);
        mix(ndoubles);
        const size_t half = b ? ndoubles / 2 : ndoubles;
        for (const void* part : {a, b})
          {
            if (!part) continue;
            const double* p = static_cast<const double*>(part);
            const size_t step = half > 4096 ? half / 4096 : 1;
            for (size_t i = 0; i < half; i += step)
              {
                uint64_t v;
                std::memcpy(&v, p + i, 8);
                mix(v);
              }
          }
        return h;
      }

      void ensure(const LxField<quad_su3>& conf)
      {
        tms_ctx* c = context();
        const double* p = conf.template getPtr<MemorySpace::CPU>();
        const uint64_t k = key_of(p, nullptr, (size_t)locVol * 72);
        if (have_conf && k == uploaded_key) return;
        check(tms_set_pointer_mode(c, TMS_PTR_HOST), "tms_set_pointer_mode");
        check(tms_conf_upload(c, p, TMS_LAYOUT_LX, 0), "tms_conf_upload");
        uploaded_key = k;
        have_conf = true;
      }

      // a raw lx conf (the multi-mass entry point's quad_su3*)
      void ensure_raw(const quad_su3* conf)
      {
        tms_ctx* c = context();
        const double* p = reinterpret_cast<const double*>(conf);
        const uint64_t k = key_of(p, nullptr, (size_t)locVol * 72);
        if (have_conf && k == uploaded_key) return;
        check(tms_set_pointer_mode(c, TMS_PTR_HOST), "tms_set_pointer_mode");
        check(tms_conf_upload(c, p, TMS_LAYOUT_LX, 0), "tms_conf_upload");
        uploaded_key = k;
        have_conf = true;
      }

      // EoField<quad_su3> keeps its two parities in two allocations: packed once per change
      void ensure(const EoField<quad_su3>& conf)
      {
        tms_ctx* c = context();
        const double* e = conf.evenPart.template getPtr<MemorySpace::CPU>();
        const double* o = conf.oddPart.template getPtr<MemorySpace::CPU>();
        const size_t n = (size_t)locVolh * 72;
        const uint64_t k = key_of(e, o, 2 * n);
        if (have_conf && k == uploaded_key) return;
        std::vector<double> both(2 * n);
        std::memcpy(both.data(), e, n * sizeof(double));
        std::memcpy(both.data() + n, o, n * sizeof(double));
        check(tms_set_pointer_mode(c, TMS_PTR_HOST), "tms_set_pointer_mode");
        check(tms_conf_upload(c, both.data(), TMS_LAYOUT_EO, 0), "tms_conf_upload");
        uploaded_key = k;
        have_conf = true;
      }

      int anis_flag(const std::optional<double>& a) { return a.has_value() ? 1 : 0; }
      double anis_val(const std::optional<double>& a) { return a.value_or(1.0); }
    }

    // the next call uploads the conf again (for callers that change a few links in place)
    void conf_changed() { have_conf = false; }

    // TMS_PREC_DOUBLE (default), TMS_PREC_MIXED_SINGLE or TMS_PREC_MIXED_HALF for the solvers
    void set_precision(int p) { precision = p; }
  }

  // dirac_operator_tmD_eoprec_portable.cpp:18-33: out = g5 (temp - out / 4) on the host
  void tmDkern_eoprec_eos_put_together_and_include_gamma5(OddField<spincolor>& out, const OddField<spincolor>& temp)
  {
    double* o = out.template getPtr<MemorySpace::CPU>();
    const double* t = temp.template getPtr<MemorySpace::CPU>();
    for (int64_t i = 0; i < (int64_t)locVolh; i++)
      for (int k = 0; k < 24; k++)
        {
          double& v = o[i * 24 + k];
          v = (k < 12) ? t[i * 24 + k] - v * 0.25 : -t[i * 24 + k] + v * 0.25;
        }
    out.invalidateHalo();
  }

  // dirac_operator_tmD_eoprec_portable.cpp:36-51
  void tmDkern_eoprec_eos(OddField<spincolor>& out, EvnField<spincolor>&, const EoField<quad_su3>& conf,
                          const double& kappa, const std::optional<double>& anis, const double& mu,
                          const OddField<spincolor>& in)
  {
    b200::ensure(conf);
    b200::check(tms_kern_eoprec(b200::ctx, kappa, b200::anis_flag(anis), b200::anis_val(anis), mu,
                                in.template getPtr<MemorySpace::CPU>(), out.template getPtr<MemorySpace::CPU>()),
                "tmDkern_eoprec_eos");
    out.invalidateHalo();
  }

  // dirac_operator_tmD_eoprec_portable.cpp:54-65
  void tmDkern_eoprec_square_eos(OddField<spincolor>& out, OddField<spincolor>&, EvnField<spincolor>&,
                                 const EoField<quad_su3>& conf, const double& kappa,
                                 const std::optional<double>& anis, const double& mu, const OddField<spincolor>& in)
  {
    b200::ensure(conf);
    b200::check(tms_kern_eoprec_square(b200::ctx, kappa, b200::anis_flag(anis), b200::anis_val(anis), mu,
                                       in.template getPtr<MemorySpace::CPU>(),
                                       out.template getPtr<MemorySpace::CPU>()),
                "tmDkern_eoprec_square_eos");
    out.invalidateHalo();
  }

  // dirac_operator_tmQ_portable.cpp:29-176
  void apply_tmQ(LxField<spincolor>& out, const LxField<quad_su3>& conf, const double& kappa,
                 const std::optional<double>& anis, const double& mass, const LxField<spincolor>& in)
  {
    b200::ensure(conf);
    b200::check(tms_apply_tmQ(b200::ctx, kappa, b200::anis_flag(anis), b200::anis_val(anis), mass,
                              in.template getPtr<MemorySpace::CPU>(), out.template getPtr<MemorySpace::CPU>()),
                "apply_tmQ");
    out.invalidateHalo();
  }

  // cg_invert_tmD_eoprec.cpp:37-58, Eq. (8b): varphi = g5 (source_odd + hop(eq8a) / 2)
  void inv_tmD_cg_eoprec_prepare_source(OddField<spincolor>& varphi, const EoField<quad_su3>& conf_eos,
                                        const std::optional<double>& anis, const EvnField<spincolor>& eq8a,
                                        const OddField<spincolor>& source_odd)
  {
    b200::ensure(conf_eos);
    double* v = varphi.template getPtr<MemorySpace::CPU>();
    b200::check(tms_hop_eo(b200::ctx, 1, eq8a.template getPtr<MemorySpace::CPU>(), v, b200::anis_flag(anis),
                           b200::anis_val(anis)),
                "inv_tmD_cg_eoprec_prepare_source");
    const double* s = source_odd.template getPtr<MemorySpace::CPU>();
    for (int64_t i = 0; i < (int64_t)locVolh; i++)
      for (int k = 0; k < 24; k++)
        v[i * 24 + k] = (k < 12) ? s[i * 24 + k] + v[i * 24 + k] * 0.5 : -s[i * 24 + k] - v[i * 24 + k] * 0.5;
    varphi.invalidateHalo();
  }

  // cg_invert_tmD_eoprec.cpp:81-99, Eq. (11) up to the inverse diagonal
  void inv_tmD_cg_eoprec_almost_reco_sol(EvnField<spincolor>& varphi, const EoField<quad_su3>& conf_eos,
                                         const std::optional<double>& anis, const OddField<spincolor>& sol_odd,
                                         const EvnField<spincolor>& source_evn)
  {
    b200::ensure(conf_eos);
    double* v = varphi.template getPtr<MemorySpace::CPU>();
    b200::check(tms_hop_eo(b200::ctx, 0, sol_odd.template getPtr<MemorySpace::CPU>(), v, b200::anis_flag(anis),
                           b200::anis_val(anis)),
                "inv_tmD_cg_eoprec_almost_reco_sol");
    const double* s = source_evn.template getPtr<MemorySpace::CPU>();
    for (int64_t i = 0; i < (int64_t)locVolh * 24; i++) v[i] = s[i] + v[i] * 0.5;
    varphi.invalidateHalo();
  }

  // cg_invert_tmD_eoprec.cpp:61-78 (the FP64 CG of cg_64_invert_tmD_eoprec.hpp:11-40)
  void inv_tmDkern_eoprec_square_eos_cg(OddField<spincolor>& sol, std::optional<OddField<spincolor>> guess,
                                        const EoField<quad_su3>& conf, const double& kappa,
                                        const std::optional<double>& anis, const double& mass, const int& nitermax,
                                        const double& residue, const OddField<spincolor>& source)
  {
    b200::ensure(conf);
    tms_stats st{};
    b200::check(tms_cg_eoprec_square(b200::ctx, sol.template getPtr<MemorySpace::CPU>(),
                                     guess ? guess->template getPtr<MemorySpace::CPU>() : nullptr,
                                     source.template getPtr<MemorySpace::CPU>(), kappa, b200::anis_flag(anis),
                                     b200::anis_val(anis), mass, nitermax, residue, b200::prec(), &st),
                "inv_tmDkern_eoprec_square_eos_cg");
    sol.invalidateHalo();
    VERBOSITY_LV1_MASTER_PRINTF(" Total cg iterations: %d\n", st.iterations);
  }

  // cg_invert_tmD_eoprec.cpp:102-150
  void inv_tmD_cg_eoprec_native(LxField<spincolor>& solution_lx, std::optional<OddField<spincolor>> guess_Koo,
                                const LxField<quad_su3>& conf_lx, const double& kappa,
                                const std::optional<double>& anis, const double& mass, const int& nitermax,
                                const double& residue, const LxField<spincolor>& source_lx)
  {
    b200::ensure(conf_lx);
    tms_stats st{};
    // the guess is read only: the reference writes the new Koo into its by-value copy of it (:138)
    b200::check(tms_cg_eoprec_guess(b200::ctx, solution_lx.template getPtr<MemorySpace::CPU>(),
                                    guess_Koo ? guess_Koo->template getPtr<MemorySpace::CPU>() : nullptr,
                                    source_lx.template getPtr<MemorySpace::CPU>(), kappa, b200::anis_flag(anis),
                                    b200::anis_val(anis), mass, nitermax, residue, b200::prec(), &st),
                "inv_tmD_cg_eoprec");
    solution_lx.invalidateHalo();
    VERBOSITY_LV1_MASTER_PRINTF(" Total cg iterations: %d\n", st.iterations);
    MASTER_PRINTF("check solution, residue: %lg, target one: %lg\n", st.lx_rel_res2, residue);
  }

  // inverters/twisted_mass/cgm_invert_tmQ2.cpp:46-53: its body is a stub in the reference
  // (CRASH "reimplement"); here it has the meaning of the working twisted-clover form at zero
  // clover (cgm_invert_tmclovQ2.cpp:10-32): (Q_W^2 + m_i^2) sol_i = source, per-mass squared residues
  void inv_tmQ2_cgm(spincolor** sol, quad_su3* conf, double kappa, const std::vector<double>& m, int nmass,
                    int niter_max, const std::vector<double>& req_res, spincolor* source)
  {
    b200::ensure_raw(conf);
    std::vector<tms_stats> st(nmass);
    std::vector<double*> out(nmass);
    for (int i = 0; i < nmass; i++) out[i] = reinterpret_cast<double*>(sol[i]);
    b200::check(tms_cgm_tmQ2(b200::ctx, out.data(), reinterpret_cast<const double*>(source), kappa, 0, 1.0, m.data(),
                             nmass, niter_max, req_res.data(), b200::prec(), st.data()),
                "inv_tmQ2_cgm");
  }

  // cg_invert_tmD_eoprec.cpp:152-213 (the library's solve ends with the same lx residual check)
  void inv_tmD_cg_eoprec(LxField<spincolor>& solution_lx, std::optional<OddField<spincolor>> guess_Koo,
                         const LxField<quad_su3>& conf_lx, const double& kappa, const std::optional<double>& anis,
                         const double& mass, const int& nitermax, const double& residue,
                         const LxField<spincolor>& source_lx)
  {
    inv_tmD_cg_eoprec_native(solution_lx, guess_Koo, conf_lx, kappa, anis, mass, nitermax, residue, source_lx);
  }
}
