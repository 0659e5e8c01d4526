// vls_main.cpp -- command-line driver with the reference's interface
// (vlasolve.cpp:20-55): options as -group.param v1 v2 ... and/or a parameter
// file given as the first non-dash argument (paramsParser.hxx:134-218), the
// initial-condition profiles UDF, PLDF, Plummer and Hernquist with their
// default grids and solver parameters, or -reload of a .vls restart file,
// then vlasovSolver::run (vlasovSolver.hxx:134-190): restart_%.4f.vls files,
// statistics.txt rows, snapshot_%4.4f.ND files, the "Computed N timesteps in
// Ts" line and the final_%.4f.vls file.  The step runs on the GPU
// through the C-ABI; -solver.precision fp64|fp32|fp32all selects the mode
// (an option the reference does not have; default fp64).
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/vlasolve_b200.hpp"

namespace {

// paramsParser: first definition of a key wins; the command line is parsed
// before the file; a key with no value reads as true; "-3" is a value
class Params {
 public:
  bool parse(int argc, char **argv) {
    int i = 1;
    std::string file = "params.ini";
    bool explicit_file = false;
    if (argc > 1 && argv[1][0] != '-') {
      file = argv[1];
      explicit_file = true;
      i = 2;
    }
    while (i < argc) {
      if (argv[i][0] != '-') {
        std::fprintf(stderr, "ERROR parsing command line.\n  AT: %s\n", argv[i]);
        return false;
      }
      std::string key = argv[i++] + 1;
      std::vector<std::string> vals;
      while (i < argc && (argv[i][0] != '-' || std::isdigit((unsigned char)argv[i][1])))
        vals.push_back(argv[i++]);
      insert(key, vals);
    }
    std::ifstream in(file);
    if (!in) {
      if (explicit_file) {
        std::fprintf(stderr, "ERROR in paramsParser:could not read parameter file '%s'.\n",
                     file.c_str());
        return false;
      }
      return true;
    }
    std::string line;
    while (std::getline(in, line)) {
      const size_t h = line.find('#');
      if (h != std::string::npos) line = line.substr(0, h);
      for (char &c : line)
        if (std::strchr(" =:{}[],\t", c)) c = ' ';
      std::istringstream ss(line);
      std::string key, v;
      if (!(ss >> key)) continue;
      std::vector<std::string> vals;
      while (ss >> v) vals.push_back(v);
      insert(key, vals);
    }
    return true;
  }
  template <typename T>
  T get(const std::string &cat, const std::string &what, T def, int which = -1) const {
    auto it = vals_.find(cat + "." + what);
    if (it == vals_.end()) return def;
    const std::vector<std::string> &v = it->second;
    const int w = which < 0 ? 0 : which;
    if (which >= 0 && (int)v.size() <= which) return def;
    if (v.empty()) return from("1", def);
    return from(v[w], def);
  }
  bool defined(const std::string &cat, const std::string &what) const {
    return vals_.count(cat + "." + what) != 0;
  }

 private:
  void insert(std::string key, const std::vector<std::string> &v) {
    if (key.find('.') == std::string::npos) key = "default." + key;
    if (!vals_.count(key)) vals_[key] = v;
  }
  static double from(const std::string &s, double) { return std::atof(s.c_str()); }
  static int from(const std::string &s, int) { return std::atoi(s.c_str()); }
  static long from(const std::string &s, long) { return std::atol(s.c_str()); }
  static bool from(const std::string &s, bool) { return std::atoi(s.c_str()) != 0 || s == "true"; }
  static std::string from(const std::string &s, const std::string &) { return s; }
  std::map<std::string, std::vector<std::string>> vals_;
};

int scale_of(const std::string &s) {
  if (s == "linear") return VLS_SCALE_LINEAR;
  if (s == "logarithmic") return VLS_SCALE_LOG;
  if (s == "quadratic") return VLS_SCALE_QUADRATIC;
  return -1;
}
const char *scale_name(int s) {
  return s == VLS_SCALE_LINEAR ? "linear" : s == VLS_SCALE_LOG ? "logarithmic" : "quadratic";
}

}  // namespace

int main(int argc, char **argv) {
  Params p;
  if (!p.parse(argc, argv)) return 1;
  const std::string type = p.get<std::string>("init", "type", std::string("UDF"));
  vls_init_desc ini = vls::default_init();
  vls_grid_desc g = vls::default_grid();
  vls_solver_desc s = vls::default_solver();
  // per-profile defaults (initGen_*::defaultGridParams / defaultSolverParams)
  if (type == "UDF") {
    ini.type = VLS_INIT_UDF;
  } else if (type == "PLDF") {
    ini.type = VLS_INIT_PLDF;
    ini.alpha = 2;
    ini.R0_given = 0;
    g.Pmax = 200;
  } else if (type == "Plummer" || type == "Hernquist") {
    ini.type = type == "Plummer" ? VLS_INIT_PLUMMER : VLS_INIT_HERNQUIST;
    ini.R0 = 1;
    g.Pmax = type == "Plummer" ? 100 : 250;
    g.Pres = type == "Plummer" ? 180 : 90;
    g.Umin[0] = -1.45;
    g.Umax[0] = 1.45;
    g.Umin[1] = type == "Plummer" ? 0.0 : 1.0e-4;
    g.Umax[1] = type == "Plummer" ? 3.24 : 12.96;
    g.Ures[0] = 80;
    g.Ures[1] = 80;
    g.Uscale[1] = type == "Plummer" ? VLS_SCALE_QUADRATIC : VLS_SCALE_LOG;
    s.Tmax = 62;
    s.dt = type == "Plummer" ? 0.1 : 0.025;
  } else {
    std::fprintf(stderr, "ERROR: unknown initial conditions type %s\n.", type.c_str());
    return 1;
  }
  const int multi = (ini.type == VLS_INIT_UDF || ini.type == VLS_INIT_PLDF) ? 0 : -1;
  ini.M = p.get("init", "M", ini.M, multi);
  ini.alpha = p.get("init", "alpha", ini.alpha, multi);
  ini.smoothingRadius = p.get("init", "smoothingRadius", ini.smoothingRadius, multi);
  ini.eta = p.get("init", "eta", ini.eta, multi);
  ini.n = p.get("init", "n", ini.n, multi);
  ini.Ra = p.get("init", "Ra", ini.Ra);
  if (p.defined("init", "R0")) {
    ini.R0 = p.get("init", "R0", ini.R0, multi);
    ini.R0_given = 1;
  }
  ini.gap[0] = p.get("init", "gap", 0.0, 0);
  ini.gap[1] = p.get("init", "gap", 0.0, 1);
  if (ini.type == VLS_INIT_PLDF) {
    const double R0 = ini.R0_given ? ini.R0 : 1.0 / ini.eta;
    const double sO = (3.0 - ini.n) / (5.0 - 2 * ini.n) * (ini.M * ini.eta) /
                      (R0 * (ini.alpha * 0.5 + 1));
    const double sig = std::sqrt(sO + 2 * (sO * 0.5 * ini.alpha));
    g.Umin[0] = -16 * sig;
    g.Umax[0] = 16 * sig;
  }
  s.G = p.get("solver", "G", s.G);
  s.T0 = p.get("solver", "T0", s.T0);
  s.Tmax = p.get("solver", "Tmax", s.Tmax);
  s.dt = p.get("solver", "dt", s.dt);
  s.noLinking = p.get("solver", "noLinking", false) ? 1 : 0;
  const std::string kt = p.get<std::string>("solver", "kernelType", std::string("delayed"));
  if (kt != "delayed" && kt != "reflective") {
    std::fprintf(stderr, "ERROR: invalid kernel type '%s'\n", kt.c_str());
    return 1;
  }
  s.kernelType = kt == "delayed" ? VLS_KERNEL_DELAYED : VLS_KERNEL_REFLECTIVE;
  s.kernelBufferSize = p.get("solver", "kernelBufferSize", 0);
  const std::string prec = p.get<std::string>("solver", "precision", std::string("fp64"));
  s.precision = prec == "fp32" ? VLS_FP32_BULK : prec == "fp32all" ? VLS_FP32_ALL : VLS_FP64;
  s.device = p.get("default", "device", 0);
  long statsEvery = p.get("solver", "statsEvery", 25L);
  long snapshotEvery = p.get("solver", "snapshotEvery", 500L);
  long restartEvery = p.get("solver", "restartEvery", 5000L);
  g.Pmin = p.get("grid", "Pmin", g.Pmin, 0);
  g.Pmax = p.get("grid", "Pmax", g.Pmax, 0);
  g.Pres = p.get("grid", "Pres", (int)g.Pres, 0);
  g.Pscale = scale_of(p.get<std::string>("grid", "Pscale", std::string(scale_name(g.Pscale)), 0));
  for (int k = 0; k < 2; k++) {
    g.Umin[k] = p.get("grid", "Umin", g.Umin[k], k);
    g.Umax[k] = p.get("grid", "Umax", g.Umax[k], k);
    g.Ures[k] = p.get("grid", "Ures", (int)g.Ures[k], k);
    g.Uscale[k] =
        scale_of(p.get<std::string>("grid", "Uscale", std::string(scale_name(g.Uscale[k])), k));
  }
  if (g.Pscale < 0 || g.Uscale[0] < 0 || g.Uscale[1] < 0) {
    std::fprintf(stderr, "ERROR: invalid scale type\n");
    return 1;
  }
  // -reload name: the state of name.vls (vlasolve.cpp:46-48,
  // vlasovSolver.hxx:104-131); Tmax, dt and the output intervals may be
  // overridden on the command line, everything else comes from the file
  const std::string reload = p.get<std::string>("default", "reload", std::string(""));
  if (!reload.empty()) {
    const std::string fname = reload + ".vls";
    vls_grid_desc rg{};
    vls_solver_desc rs{};
    int64_t every[3];
    double t;
    int64_t n;
    if (vls_restart_info(fname.c_str(), &rg, &rs, every, &t, &n) != VLS_OK) {
      std::fprintf(stderr, "ERROR: %s\n", vls_last_error(nullptr));
      return 1;
    }
    // the J minimum is not in the file; -grid.Umin's second value or 0
    rg.Umin[1] = p.get("grid", "Umin", 0.0, 1);
    rs.precision = s.precision;
    rs.device = s.device;
    rs.Tmax = p.get("solver", "Tmax", rs.Tmax);
    snapshotEvery = p.get("solver", "snapshotEvery", (long)every[0]);
    restartEvery = p.get("solver", "restartEvery", (long)every[1]);
    statsEvery = p.get("solver", "statsEvery", (long)every[2]);
    if (p.defined("solver", "dt") && p.get("solver", "dt", rs.dt) != rs.dt) {
      std::fprintf(stderr, "ERROR: the time step of a reloaded run is the file's (%g)\n", rs.dt);
      return 1;
    }
    try {
      vls::vlasovSolver21_spline solver(rg, rs, nullptr);
      solver.readRestart(fname.c_str());
      std::printf("Reloaded %s at T=%.5f (step %ld)\n", fname.c_str(), t, (long)n);
      std::printf("Starting at T=%.5f, dt=%g, tmax = %g\n", t, rs.dt, rs.Tmax);
      const auto t0 = std::chrono::steady_clock::now();
      solver.run(statsEvery, snapshotEvery, "statistics.txt", restartEvery, true);
      solver.sync();
      const double T =
          std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      double t1;
      int64_t n1;
      vls_get_time(solver.handle(), &t1, &n1);
      std::printf("\nComputed %ld timesteps in %gs. (%3.3gs / step)\n", (long)n1, T,
                  n1 > n ? T / (n1 - n) : 0.0);
    } catch (const vls::error &e) {
      std::fprintf(stderr, "ERROR (%d): %s\n", e.code(), e.what());
      return 2;
    }
    return 0;
  }
  try {
    vls::vlasovSolver21_spline solver(g, s, ini);
    std::printf("Renormalizing mass : M[0]=%g -> %g.\n", solver.massBeforeRenormalisation(),
                ini.M);
    std::printf("Starting at T=%.5f, dt=%g, tmax = %g\n", s.T0, s.dt, s.Tmax);
    const auto t0 = std::chrono::steady_clock::now();
    solver.run(statsEvery, snapshotEvery, "statistics.txt", restartEvery, true);
    solver.sync();
    const double T =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    double t;
    int64_t n;
    vls_get_time(solver.handle(), &t, &n);
    std::printf("\nComputed %ld timesteps in %gs. (%3.3gs / step)\n", (long)n, T,
                n ? T / n : 0.0);
  } catch (const vls::error &e) {
    std::fprintf(stderr, "ERROR (%d): %s\n", e.code(), e.what());
    return 2;
  }
  return 0;
}
