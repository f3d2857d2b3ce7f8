// Command-line driver around the reference library's own twisted-mass code.
//
// Test infrastructure only: it links the reference's unmodified sources
// (compiled in place from the reference tree by oracle/ref_build/Makefile) and
// exposes their entry points on raw binary files so that the oracle and the
// committed golden fixtures can be checked against the reference itself, and
// so that the reference's OpenMP CPU path can be timed as the CPU baseline.
//
// Data files are little-endian float64 in the reference's CPU (AoS) layout:
//   lx conf     : V  x [mu=4][row=3][col=3][re,im]        (field.hpp:407-416, su3.hpp:52-55)
//   lx spinor   : V  x [spin=4][col=3][re,im]             (su3.hpp:33)
//   eo spinor   : Vh x [spin=4][col=3][re,im], sites in loclx_of_loceo order (geometry_eo.cpp:66-77)
//
// Usage: nissa_ref <op> T=<T> L=<L> [key=value ...]
//   ops: geom out=...                           the e/o geometry tables of set_eo_geometry (geometry_eo.cpp:41-100):
//                                                int32 loclx_parity[V], loceo_of_loclx[V], loclx_of_loceo[2][Vh],
//                                                loceo_neighup[2][Vh][4], loceo_neighdw[2][Vh][4], one after the other
//        plaq conf=...                          global_plaquette_lx_conf        (su3_paths/plaquette.hpp:77-82)
//        ildg2raw ildg=... out=...               read_ildg_gauge_conf             (io/reader.hpp:75-99)
//        hop conf in out par=P                   tmn2Deo_or_tmn2Doe_eos           (dirac_operator_tmD_eoprec_portable.hpp:33-169)
//        kern conf in out kappa mu               tmDkern_eoprec_eos               (dirac_operator_tmD_eoprec_portable.cpp:36-51)
//        kern2 conf in out kappa mu              tmDkern_eoprec_square_eos        (dirac_operator_tmD_eoprec_portable.cpp:54-65)
//        kern2twice conf in out kappa mu         the same twice, the x links negated in place in between
//        cg conf in out kappa mu niter residue   inv_tmDkern_eoprec_square_eos_cg (cg_invert_tmD_eoprec.cpp:61-78)
//        cgfull conf in out kappa mu niter residue inv_tmD_cg_eoprec              (cg_invert_tmD_eoprec.cpp:152-213)
//        tmQ conf in out kappa mu                apply_tmQ                        (dirac_operator_tmQ_portable.cpp:29-176)
//        cgm conf in out kappa masses=a,b residues=a,b niter
//                                                inv_tmclovQ2_cgm with a zero clover term (cgm_invert_tmclovQ2.cpp:10-32)
//        clover conf out cSW                     clover_term                      (su3_paths/clover_term.hpp:104-112)
//        invclover conf out cSW kappa mu         invert_twisted_clover_term       (su3_paths/clover_term.hpp:143-262)
//        clovkern conf in out cSW kappa mu dag   tmclovDkern_eoprec_eos           (dirac_operator_tmclovD_eoprec_portable.cpp:42-68)
//        clovkern2 conf in out cSW kappa mu      tmclovDkern_eoprec_square_eos    (dirac_operator_tmclovD_eoprec_portable.cpp:70-84)
//        clovcgfull conf in out cSW kappa mu niter residue
//                                                inv_tmclovD_cg_eoprec            (cg_invert_tmclovD_eoprec.cpp:55-120)
//   common keys: anis=<double> (default: none), reps=<n> (timed repetitions, default 1)
//   cgfull also reports every repetition's own time ("seconds_each"); with
//   point_cols=<n> it ignores `in` and solves, in repetition r, the point source
//   at the origin of spin-colour column r mod n (spin = k/3, colour = k%3); the
//   output is the last repetition's solution
//   cg with sample_iters=N: a bounded sample of the solve.  The reference's CG
//   runs exactly N iterations (niter=N, unreachable residue) plus its final
//   true-residual application, then takes its own non-convergence path
//   (CRASH, cg_invert_template_threaded.hpp:146-147); the driver reports the
//   elapsed time from the reference's crash hook (base/debug.hpp:70) and the
//   process exits through the single-rank MPI_Abort.
// The last stdout line is a JSON record with the time per repetition.

#include <config.hpp>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <optional>
#include <sstream>
#include <string>
#include <vector>

#include <omp.h>

#include "base/init.hpp"
#include "base/field.hpp"
#include "dirac_operators/tmD_eoprec/dirac_operator_tmD_eoprec_portable.hpp"
#include "dirac_operators/tmQ/dirac_operator_tmQ.hpp"
#include "geometry/geometry_eo.hpp"
#include "geometry/geometry_mix.hpp"
#include "inverters/twisted_mass/cg_invert_tmD_eoprec.hpp"
#include "io/reader.hpp"
#include "operations/su3_paths/plaquette.hpp"
#include "operations/su3_paths/clover_term.hpp"
#include "dirac_operators/tmclovD_eoprec/dirac_operator_tmclovD_eoprec.hpp"
#include "inverters/twisted_clover/cg_invert_tmclovD_eoprec.hpp"

namespace nissa
{
  void inv_tmDkern_eoprec_square_eos_cg(OddField<spincolor>& sol,
					std::optional<OddField<spincolor>> guess,
					const EoField<quad_su3>& conf,
					const double& kappa,
					const std::optional<double>& anis,
					const double& mass,
					const int& nitermax,
					const double& residue,
					const OddField<spincolor>& source);

  // defined in inverters/twisted_clover/cgm_invert_tmclovQ2.cpp:10-32 (its header
  // still declares an older signature)
  void inv_tmclovQ2_cgm(std::vector<LxField<spincolor>>& sol,
			const LxField<quad_su3>& conf,
			const double& kappa,
			const std::optional<double>& anis,
			const LxField<clover_term_t>& Cl,
			const std::vector<double>& m,
			const int& niter_max,
			const std::vector<double>& req_res,
			const LxField<spincolor>& source);
}

using namespace nissa;

namespace
{
  std::map<std::string, std::string> args;

  std::string arg(const std::string& k, const std::string& def = "")
  {
    auto it = args.find(k);
    if (it == args.end())
      {
	if (def.empty())
	  {
	    fprintf(stderr, "missing argument %s\n", k.c_str());
	    exit(2);
	  }
	return def;
      }
    return it->second;
  }

  double argd(const std::string& k, const std::string& def = "") { return std::stod(arg(k, def)); }

  std::vector<double> argv_list(const std::string& k)
  {
    std::vector<double> v;
    std::stringstream ss(arg(k));
    std::string item;
    while (std::getline(ss, item, ','))
      v.push_back(std::stod(item));
    return v;
  }

  std::vector<double> read_file(const std::string& path, size_t n)
  {
    std::vector<double> v(n);
    FILE* f = fopen(path.c_str(), "rb");
    if (!f || fread(v.data(), sizeof(double), n, f) != n)
      {
	fprintf(stderr, "cannot read %zu doubles from %s\n", n, path.c_str());
	exit(3);
      }
    fclose(f);
    return v;
  }

  void write_file(const std::string& path, const double* d, size_t n)
  {
    FILE* f = fopen(path.c_str(), "wb");
    if (!f || fwrite(d, sizeof(double), n, f) != n)
      {
	fprintf(stderr, "cannot write %s\n", path.c_str());
	exit(3);
      }
    fclose(f);
  }

  void write_ints(const std::string& path, const std::vector<int>& v)
  {
    FILE* f = fopen(path.c_str(), "wb");
    if (!f || fwrite(v.data(), sizeof(int), v.size(), f) != v.size())
      {
	fprintf(stderr, "cannot write %s\n", path.c_str());
	exit(3);
      }
    fclose(f);
  }

  template <typename F>
  void fill(F& field, const std::vector<double>& v, size_t nsites, size_t ndeg)
  {
    double* p = field.template getPtr<MemorySpace::CPU>();
    std::copy(v.begin(), v.begin() + nsites * ndeg, p);
    field.invalidateHalo();
  }

  template <typename F>
  void dump(const F& field, const std::string& path, size_t nsites, size_t ndeg)
  {
    const double* p = field.template getPtr<MemorySpace::CPU>();
    write_file(path, p, nsites * ndeg);
  }

  std::optional<double> anis_arg()
  {
    if (args.count("anis")) return std::stod(args["anis"]);
    return std::nullopt;
  }

  double now()
  {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
  }

  double sample_t0 = 0;
  int sample_iters = 0;
  int sample_T = 0, sample_L = 0;

  void sample_report()
  {
    printf("{\"op\": \"cg\", \"T\": %d, \"L\": %d, \"sample_iters\": %d, \"threads\": %d, \"seconds\": %.9g}\n",
	   sample_T, sample_L, sample_iters, omp_get_max_threads(), now() - sample_t0);
    fflush(stdout);
  }
}

int main(int narg, char** arg_v)
{
  if (narg < 2)
    {
      fprintf(stderr, "usage: %s op key=value ...\n", arg_v[0]);
      return 2;
    }
  const std::string op = arg_v[1];
  for (int i = 2; i < narg; i++)
    {
      std::string s = arg_v[i];
      auto eq = s.find('=');
      if (eq == std::string::npos) continue;
      args[s.substr(0, eq)] = s.substr(eq + 1);
    }

  setenv("NISSA_DO_NOT_TRAP_SIGNALS", "1", 0);
  char* fake_argv[] = {arg_v[0], nullptr};
  initNissa(1, fake_argv);
  verbosity_lv = (int)argd("verbosity", "1");
  // runtime flag of the reference's config file (io/input.cpp:457-546); its
  // default (communicate.hpp:10) makes cgm_invert CRASH("reimplement") from the
  // second iteration on (cgm_invert_template_threaded.hpp:101-102), so the
  // driver runs with synchronous communications, as a config file can ask
  use_async_communications = 0;
  const int T = (int)argd("T"), L = (int)argd("L");
  initGrid(T, L);

  const size_t V = locVol, Vh = locVolh;
  const int reps = (int)argd("reps", "1");
  const auto anis = anis_arg();
  double t_per_rep = 0;
  std::string extra;

  if (op == "geom")
    {
      // the reference's own tables, as set_eo_geometry left them (one rank: no borders)
      std::vector<int> v;
      for (size_t i = 0; i < V; i++) v.push_back(loclx_parity[i]);
      for (size_t i = 0; i < V; i++) v.push_back(loceo_of_loclx[i]);
      for (int par = 0; par < 2; par++)
	for (size_t i = 0; i < Vh; i++) v.push_back(loclx_of_loceo[par][i]);
      for (int par = 0; par < 2; par++)
	for (size_t i = 0; i < Vh; i++)
	  for (int mu = 0; mu < 4; mu++) v.push_back(loceo_neighup[par][i][mu]);
      for (int par = 0; par < 2; par++)
	for (size_t i = 0; i < Vh; i++)
	  for (int mu = 0; mu < 4; mu++) v.push_back(loceo_neighdw[par][i][mu]);
      write_ints(arg("out"), v);
    }
  else if (op == "ildg2raw")
    {
      LxField<quad_su3> conf("conf", WITH_HALO);
      read_ildg_gauge_conf(conf, arg("ildg"));
      dump(conf, arg("out"), V, 72);
    }
  else
    {
      LxField<quad_su3> conf_lx("conf_lx", WITH_HALO);
      fill(conf_lx, read_file(arg("conf"), V * 72), V, 72);

      // the chromo operator reads the conf's edges: a copy allocated with them
      LxField<quad_su3> conf_edges("conf_edges", WITH_HALO_EDGES);
      if (op == "clover" || op == "invclover" || op == "clovkern" || op == "clovkern2" || op == "clovcgfull")
	fill(conf_edges, read_file(arg("conf"), V * 72), V, 72);
      if (op == "clover" || op == "invclover")
	{
	  LxField<clover_term_t> Cl("Cl");
	  const double t0 = now();
	  for (int r = 0; r < reps; r++) clover_term(Cl, argd("cSW"), conf_edges);
	  if (op == "clover")
	    {
	      t_per_rep = (now() - t0) / reps;
	      dump(Cl, arg("out"), V, 72);
	    }
	  else
	    {
	      LxField<inv_clover_term_t> invCl("invCl");
	      const double t1 = now();
	      for (int r = 0; r < reps; r++) invert_twisted_clover_term(invCl, argd("mu"), argd("kappa"), Cl);
	      t_per_rep = (now() - t1) / reps;
	      dump(invCl, arg("out"), V, 144);
	    }
	}
      else if (op == "clovcgfull")
	{
	  LxField<spincolor> in("in", WITH_HALO);
	  fill(in, read_file(arg("in"), V * 24), V, 24);
	  LxField<spincolor> sol("sol", WITH_HALO);
	  const double t0 = now();
	  for (int r = 0; r < reps; r++)
	    inv_tmclovD_cg_eoprec(sol, std::nullopt, conf_edges, argd("kappa"), anis, argd("cSW"), argd("mu"),
				  (int)argd("niter"), argd("residue"), in);
	  t_per_rep = (now() - t0) / reps;
	  dump(sol, arg("out"), V, 24);
	}
      else if (op == "clovkern" || op == "clovkern2")
	{
	  // the clover fields exactly as inv_tmclovD_cg_eoprec_native builds them
	  const double kappa = argd("kappa"), mu = argd("mu");
	  LxField<clover_term_t> Cl_lx("Cl");
	  clover_term(Cl_lx, argd("cSW"), conf_edges);
	  LxField<inv_clover_term_t> invCl_lx("invCl");
	  invert_twisted_clover_term(invCl_lx, mu, kappa, Cl_lx);
	  OddField<clover_term_t> Cl_odd("Cl_odd");
	  get_evn_or_odd_part_of_lx_vector(Cl_odd, Cl_lx, ODD_SITES);
	  EvnField<inv_clover_term_t> invCl_evn("invCl_evn");
	  get_evn_or_odd_part_of_lx_vector(invCl_evn, invCl_lx, EVEN_SITES);
	  EoField<quad_su3> conf("conf", WITH_HALO);
	  split_lx_vector_into_eo_parts(conf, conf_lx);
	  OddField<spincolor> in("in", WITH_HALO), out("out", WITH_HALO);
	  fill(in, read_file(arg("in"), Vh * 24), Vh, 24);
	  const double t0 = now();
	  if (op == "clovkern")
	    {
	      EvnField<spincolor> tmp("tmp", WITH_HALO);
	      for (int r = 0; r < reps; r++)
		tmclovDkern_eoprec_eos(out, tmp, conf, kappa, anis, Cl_odd, invCl_evn, argd("dag") != 0, mu, in);
	    }
	  else
	    {
	      OddField<spincolor> temp1("temp1", WITH_HALO);
	      EvnField<spincolor> temp2("temp2", WITH_HALO);
	      for (int r = 0; r < reps; r++)
		tmclovDkern_eoprec_square_eos(out, temp1, temp2, conf, kappa, anis, Cl_odd, invCl_evn, mu, in);
	    }
	  t_per_rep = (now() - t0) / reps;
	  dump(out, arg("out"), Vh, 24);
	}
      else if (op == "plaq")
	{
	  const double plaq = global_plaquette_lx_conf(conf_lx);
	  char buf[64];
	  snprintf(buf, sizeof buf, "\"plaquette\": %.17g, ", plaq);
	  extra = buf;
	}
      else if (op == "tmQ" || op == "cgfull" || op == "cgm")
	{
	  LxField<spincolor> in("in", WITH_HALO);
	  const int point_cols = (int)argd("point_cols", "0");
	  if (point_cols == 0) fill(in, read_file(arg("in"), V * 24), V, 24);
	  const double kappa = argd("kappa");
	  if (op == "tmQ")
	    {
	      const double mu = argd("mu");
	      LxField<spincolor> out("out");
	      const double t0 = now();
	      for (int r = 0; r < reps; r++) apply_tmQ(out, conf_lx, kappa, anis, mu, in);
	      t_per_rep = (now() - t0) / reps;
	      dump(out, arg("out"), V, 24);
	    }
	  else if (op == "cgfull")
	    {
	      const double mu = argd("mu");
	      LxField<spincolor> sol("sol", WITH_HALO);
	      const double t0 = now();
	      std::string each = "\"seconds_each\": [";
	      for (int r = 0; r < reps; r++)
		{
		  if (point_cols > 0)
		    {
		      // point source at the origin, spin-colour column r mod point_cols (spin = k / 3, colour = k % 3)
		      std::vector<double> v(V * 24, 0.0);
		      const int k = r % point_cols;
		      v[(k / 3) * 6 + (k % 3) * 2] = 1.0;
		      fill(in, v, V, 24);
		    }
		  const double tr = now();
		  inv_tmD_cg_eoprec(sol, std::nullopt, conf_lx, kappa, anis, mu, (int)argd("niter"), argd("residue"), in);
		  char buf[32];
		  snprintf(buf, sizeof buf, "%s%.9g", r ? ", " : "", now() - tr);
		  each += buf;
		}
	      t_per_rep = (now() - t0) / reps;
	      extra = each + "], ";
	      dump(sol, arg("out"), V, 24);
	    }
	  else
	    {
	      const std::vector<double> masses = argv_list("masses"), res = argv_list("residues");
	      std::vector<LxField<spincolor>> sol;
	      for (size_t i = 0; i < masses.size(); i++) sol.emplace_back("sol", WITH_HALO);
	      LxField<clover_term_t> Cl("Cl");
	      Cl.reset();
	      const double t0 = now();
	      for (int r = 0; r < reps; r++)
		inv_tmclovQ2_cgm(sol, conf_lx, kappa, anis, Cl, masses, (int)argd("niter"), res, in);
	      t_per_rep = (now() - t0) / reps;
	      std::vector<double> all;
	      for (auto& s : sol)
		{
		  const double* p = s.getPtr<MemorySpace::CPU>();
		  all.insert(all.end(), p, p + V * 24);
		}
	      write_file(arg("out"), all.data(), all.size());
	    }
	}
      else
	{
	  EoField<quad_su3> conf("conf", WITH_HALO);
	  split_lx_vector_into_eo_parts(conf, conf_lx);
	  const std::vector<double> vin = read_file(arg("in"), Vh * 24);
	  if (op == "hop")
	    {
	      const int par = (int)argd("par");
	      if (par == 0)
		{
		  OddField<spincolor> in("in", WITH_HALO);
		  EvnField<spincolor> out("out", WITH_HALO);
		  fill(in, vin, Vh, 24);
		  const double t0 = now();
		  for (int r = 0; r < reps; r++) tmn2Deo_or_tmn2Doe_eos(out, conf, anis, in);
		  t_per_rep = (now() - t0) / reps;
		  dump(out, arg("out"), Vh, 24);
		}
	      else
		{
		  EvnField<spincolor> in("in", WITH_HALO);
		  OddField<spincolor> out("out", WITH_HALO);
		  fill(in, vin, Vh, 24);
		  const double t0 = now();
		  for (int r = 0; r < reps; r++) tmn2Deo_or_tmn2Doe_eos(out, conf, anis, in);
		  t_per_rep = (now() - t0) / reps;
		  dump(out, arg("out"), Vh, 24);
		}
	    }
	  else
	    {
	      OddField<spincolor> in("in", WITH_HALO);
	      fill(in, vin, Vh, 24);
	      const double kappa = argd("kappa"), mu = argd("mu");
	      OddField<spincolor> out("out", WITH_HALO);
	      if (op == "kern")
		{
		  EvnField<spincolor> temp("temp", WITH_HALO);
		  const double t0 = now();
		  for (int r = 0; r < reps; r++) tmDkern_eoprec_eos(out, temp, conf, kappa, anis, mu, in);
		  t_per_rep = (now() - t0) / reps;
		}
	      else if (op == "kern2")
		{
		  OddField<spincolor> temp1("temp1", WITH_HALO);
		  EvnField<spincolor> temp2("temp2", WITH_HALO);
		  const double t0 = now();
		  for (int r = 0; r < reps; r++) tmDkern_eoprec_square_eos(out, temp1, temp2, conf, kappa, anis, mu, in);
		  t_per_rep = (now() - t0) / reps;
		}
	      else if (op == "kern2twice")
		{
		  // K^2 twice on one EoField conf whose x links are negated in place in
		  // between (the same allocations): a cache of the conf must notice
		  OddField<spincolor> temp1("temp1", WITH_HALO), mid("mid", WITH_HALO);
		  EvnField<spincolor> temp2("temp2", WITH_HALO);
		  tmDkern_eoprec_square_eos(mid, temp1, temp2, conf, kappa, anis, mu, in);
		  double* parts[2] = {conf.evenPart.template getPtr<MemorySpace::CPU>(),
				      conf.oddPart.template getPtr<MemorySpace::CPU>()};
		  for (double* c : parts)
		    for (size_t i = 0; i < Vh; i++)
		      for (int k = 18; k < 36; k++) c[i * 72 + k] = -c[i * 72 + k];
		  conf.evenPart.invalidateHalo();
		  conf.oddPart.invalidateHalo();
		  tmDkern_eoprec_square_eos(out, temp1, temp2, conf, kappa, anis, mu, mid);
		}
	      else if (op == "cg" && args.count("sample_iters"))
		{
		  sample_iters = (int)argd("sample_iters");
		  sample_T = T;
		  sample_L = L;
		  crashHook = sample_report;
		  sample_t0 = now();
		  inv_tmDkern_eoprec_square_eos_cg(out, std::nullopt, conf, kappa, anis, mu, sample_iters, 1e-300, in);
		  fprintf(stderr, "sample run converged before %d iterations\n", sample_iters);
		  return 4;
		}
	      else if (op == "cg")
		{
		  const double t0 = now();
		  for (int r = 0; r < reps; r++)
		    inv_tmDkern_eoprec_square_eos_cg(out, std::nullopt, conf, kappa, anis, mu, (int)argd("niter"),
						     argd("residue"), in);
		  t_per_rep = (now() - t0) / reps;
		}
	      else
		{
		  fprintf(stderr, "unknown op %s\n", op.c_str());
		  return 2;
		}
	      dump(out, arg("out"), Vh, 24);
	    }
	}
    }

  printf("{\"op\": \"%s\", \"T\": %d, \"L\": %d, %s\"threads\": %d, \"reps\": %d, \"seconds_per_rep\": %.9g}\n", op.c_str(), T, L,
	 extra.c_str(), omp_get_max_threads(), reps, t_per_rep);
  fflush(stdout);
  return 0;
}
