// Host-side set-up of a PIAFS simulation from its input deck (see deck.h).
#include "deck.h"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>

#include "../../include/piafs_gpu.h"

namespace piafs {

namespace {

// In-memory deck of read_deck_memory (this thread, for the duration of the
// call): key files by name, the interior grid, no field files.
thread_local const DeckMemory* tl_mem = nullptr;

std::string base_name(const std::string& path) {
  const size_t k = path.find_last_of('/');
  return k == std::string::npos ? path : path.substr(k + 1);
}

bool read_tokens(const std::string& path, std::vector<std::string>& toks) {
  if (tl_mem) {
    auto it = tl_mem->files.find(base_name(path));
    if (it == tl_mem->files.end()) return false;
    std::istringstream f(it->second);
    std::string t;
    while (f >> t) toks.push_back(t);
    return true;
  }
  std::ifstream f(path);
  if (!f) return false;
  std::string t;
  while (f >> t) toks.push_back(t);
  return true;
}

bool is_number(const std::string& s) {
  char* end = nullptr;
  std::strtod(s.c_str(), &end);
  return end && *end == 0 && !s.empty();
}

// A "begin <key> <value> ... end" file as key -> tokens.  Multi-valued keys
// (size, size_exact, iproc) collect numbers until the next word.
int read_keyfile(const std::string& path, std::map<std::string, std::vector<std::string>>& kv, bool& found,
                 std::string& err) {
  std::vector<std::string> t;
  found = read_tokens(path, t);
  if (!found) return 0;
  if (t.empty() || t[0] != "begin") {
    err = "illegal format in " + path + " (expected 'begin')";
    return PIAFS_ERR_INPUT;
  }
  size_t i = 1;
  while (i < t.size() && t[i] != "end") {
    std::string k = t[i++];
    std::vector<std::string> v;
    if (k == "size" || k == "size_exact" || k == "iproc") {
      while (i < t.size() && t[i] != "end" && is_number(t[i])) v.push_back(t[i++]);
    } else if (k == "input_mode" || k == "output_mode") {
      if (i < t.size()) v.push_back(t[i++]);
      if (!v.empty() && v[0] != "serial" && i < t.size()) v.push_back(t[i++]);
    } else if (i < t.size()) {
      v.push_back(t[i++]);
    }
    kv[k] = v;
  }
  if (i >= t.size()) {
    err = "missing 'end' in " + path;
    return PIAFS_ERR_INPUT;
  }
  return 0;
}

template <typename T>
void get(const std::map<std::string, std::vector<std::string>>& kv, const char* key, T& out) {
  auto it = kv.find(key);
  if (it == kv.end() || it->second.empty()) return;
  std::istringstream is(it->second[0]);
  is >> out;
}

// FindInterval.c:21-50 on the interior coordinates of one dimension
void find_interval(double a, double b, const double* x, int N, int& imin, int& imax) {
  imax = -1;
  imin = N;
  double min_dx = N > 1 ? x[1] - x[0] : 1.0;
  for (int i = 2; i < N; i++) {
    double dx = x[i] - x[i - 1];
    if (dx < min_dx) min_dx = dx;
  }
  double tol = 1e-10 * min_dx;
  for (int i = 0; i < N; i++)
    if (x[i] <= (b + tol)) imax = i + 1;
  for (int i = N - 1; i > -1; i--)
    if (x[i] >= (a - tol)) imin = i;
}

// Butcher tableaux (TimeExplicitRKInitialize.c:25-95); forward Euler = 1 stage
int set_tableau(Deck& d, std::string& err) {
  const int S = MAX_STAGES;
  for (double& a : d.A) a = 0.0;
  for (int i = 0; i < S; i++) d.b[i] = d.c[i] = 0.0;
  const std::string& t = d.time_scheme_type;
  if (d.time_scheme == "euler" || (d.time_scheme == "rk" && t == "1fe")) {
    d.nstages = 1;
    d.b[0] = 1.0;
  } else if (d.time_scheme != "rk") {
    err = "time_scheme " + d.time_scheme + " is not supported";
    return PIAFS_ERR_UNSUPPORTED;
  } else if (t == "22") {
    d.nstages = 2;
    d.A[1 * S + 0] = 1.0; d.c[1] = 1.0; d.b[0] = d.b[1] = 0.5;
  } else if (t == "33") {
    d.nstages = 3;
    d.A[1 * S + 0] = 2.0 / 3.0; d.A[2 * S + 0] = 2.0 / 3.0 - 1.0 / 4.0; d.A[2 * S + 1] = 1.0 / 4.0;
    d.c[1] = 2.0 / 3.0; d.c[2] = 2.0 / 3.0;
    d.b[0] = 1.0 / 4.0; d.b[1] = -1.0 / 4.0; d.b[2] = 1.0;
  } else if (t == "44") {
    d.nstages = 4;
    d.A[1 * S + 0] = 0.5; d.A[2 * S + 1] = 0.5; d.A[3 * S + 2] = 1.0;
    d.c[1] = d.c[2] = 0.5; d.c[3] = 1.0;
    d.b[0] = 1.0 / 6.0; d.b[1] = 1.0 / 3.0; d.b[2] = 1.0 / 3.0; d.b[3] = 1.0 / 6.0;
  } else if (t == "ssprk3" || t == "tvdrk3") {
    d.nstages = 3;
    d.A[1 * S + 0] = 1.0; d.A[2 * S + 0] = 0.25; d.A[2 * S + 1] = 0.25;
    d.c[1] = 1.0; d.c[2] = 0.5;
    d.b[0] = d.b[1] = 1.0 / 6.0; d.b[2] = 2.0 / 3.0;
  } else {
    err = "RK type " + t + " is not supported";
    return PIAFS_ERR_UNSUPPORTED;
  }
  return 0;
}

// ChemistryInitialize.c:69-481: defaults, chemistry.inp, normalisation.
// Also recomputes gamma, Re and Pr for NS2D (NavierStokes2DInitialize.c:196-215).
int setup_chemistry(const std::string& dir, Deck& d, int nflow, std::string& err) {
  double pi = 4.0 * std::atan(1.0), NA = 6.02214076e23, kB = 1.380649e-23, c = 3.0e8;
  double h = 6.62607015e-34, e = 1.60217663e-19, M_O2 = 0.032, M_CO2 = 0.044;
  double Cp_O2 = 918.45, Cv_O2 = 650.0, Cp_CO2 = 842.86, Cv_CO2 = 654.5;
  double mu0_O2 = 1.99e-5, kappa0_O2 = 2.70e-2, mu0_CO2 = 1.45e-5, kappa0_CO2 = 1.58e-2;
  std::map<std::string, double> v = {
      {"lambda_UV", 2.48e-7}, {"theta", 0.17 * pi / 180}, {"f_CO2", 0.0}, {"f_O3", 0.005},
      {"Ptot", 101325.0}, {"Ti", 288.0}, {"t_start", 0.0}, {"t_pulse", 10 * 1e-9}, {"Lz", 0.03},
      {"z_mm", 0.0}, {"k0a", 0.9 * 3.3e-13}, {"k0b", 0.1 * 3.3e-13}, {"k1a", 0.8 * 3.95e-17},
      {"k1b", 0.2 * 3.95e-17}, {"k2a", 1.2e-16}, {"k2b", 1.2e-16}, {"k3a", 1.2e-17}, {"k3b", 1.0e-17},
      {"k4", 1.1e-16}, {"k5", 2.0e-16}, {"k6", 0.2 * 3.0e-17}, {"F0", 2000.0}, {"sO3", 1.1e-21},
      {"IA", 1.0}, {"IB", 1.0}, {"IC", 0.0}};
  int nz_layers = 22;
  std::map<std::string, std::vector<std::string>> kv;
  bool found;
  if (int r = read_keyfile(dir + "/chemistry.inp", kv, found, err)) return r;
  for (auto& it : kv) {
    if (it.first == "nz") get(kv, "nz", nz_layers);
    else if (it.first == "write_all_zlocs") get(kv, "write_all_zlocs", d.write_all_zlocs);
    else if (v.count(it.first)) get(kv, it.first.c_str(), v[it.first]);
  }
  if (v["f_CO2"] > 1.0 || v["f_CO2"] < 0.0 || v["f_O3"] > 1.0 || v["f_O3"] < 0.0) {
    err = "chemistry.inp: species fractions must lie in [0, 1]";
    return PIAFS_ERR_INPUT;
  }
  double f_CO2 = v["f_CO2"], f_O2 = 1.0 - f_CO2, Ti = v["Ti"], Ptot = v["Ptot"];
  double R = NA * kB / (f_O2 * M_O2 + f_CO2 * M_CO2);
  double Cp = f_O2 * Cp_O2 + f_CO2 * Cp_CO2, Cv = f_O2 * Cv_O2 + f_CO2 * Cv_CO2;
  double gamma = Cp / Cv;
  double mu0 = f_O2 * mu0_O2 + f_CO2 * mu0_CO2, kappa0 = f_O2 * kappa0_O2 + f_CO2 * kappa0_CO2;
  double kUV = 2 * pi / v["lambda_UV"];
  double kg = 2 * kUV * std::sin(v["theta"]);
  double n_O2 = f_O2 * Ptot / (kB * Ti);
  double cs = std::sqrt(gamma * R * Ti);
  double L_ref = 1.0 / kg, v_ref = cs, t_ref = L_ref / v_ref;
  double rho_ref = Ptot / (R * Ti), P_ref = rho_ref * v_ref * v_ref;
  double rate_norm_fac = kg * cs / n_O2;
  const char* kk[11] = {"k0a", "k0b", "k1a", "k1b", "k2a", "k2b", "k3a", "k3b", "k4", "k5", "k6"};
  for (int i = 0; i < 11; i++) d.kn[i] = v[kk[i]] / rate_norm_fac;
  const double qf[11] = {0.73, 2.8, 0.29, 0.84, 4.3, 0.81, 0.42, 1.16, 1.23, 1.81, 0.42};
  double Ei = P_ref / ((gamma - 1.0) * n_O2);
  for (int i = 0; i < 11; i++) d.qn[i] = qf[i] * e / Ei;
  d.chem = true;
  d.chem_gamma = gamma;
  d.I0 = v["F0"] / v["t_pulse"];
  d.ch_c = c;
  d.ch_h = h;
  d.ch_nu = c / v["lambda_UV"];
  d.n_O2 = n_O2;
  d.t_start_norm = v["t_start"] / t_ref;
  d.t_pulse_norm = v["t_pulse"] / t_ref;
  d.sO3 = v["sO3"];
  d.dz = v["Lz"] / nz_layers;
  int z_i = (int)(std::ceil(v["z_mm"] * 0.001 * nz_layers / v["Lz"]));
  d.nz = z_i + 1;
  d.L_ref = L_ref; d.kg = kg; d.IA = v["IA"]; d.IB = v["IB"]; d.IC = v["IC"];
  // physics overrides
  d.gamma = gamma;
  if (d.model == "navierstokes2d") {
    d.Tref = Ti;
    if (d.Re > 0) {
      double T0 = d.T0, TS = d.TS, TA = d.TA, TB = d.TB;
      double mu_ref = mu0 * std::exp(1.5 * std::log(Ti / T0)) * ((T0 + TS) / (Ti + TS));
      double kappa_ref = kappa0 * std::exp(1.5 * std::log(Ti / T0)) *
                         ((T0 + TA * std::exp(-TB / T0)) / (Ti + TA * std::exp(-TB / Ti)));
      d.Re = rho_ref * v_ref * L_ref / mu_ref;
      d.Pr = gamma * R / (gamma - 1) * mu_ref / kappa_ref;
    }
  }
  if (d.nvars != nflow + 7 * d.nz) {
    err = "nvars has to be " + std::to_string(nflow + 7 * d.nz) + " in solver.inp with chemistry";
    return PIAFS_ERR_INPUT;
  }
  return 0;
}

// ghosted coordinates (ReadArray.c:71-91) and 1/dx (InitialSolution.c:73-113)
void ghost_grid(const std::vector<double>& xi, int g, std::vector<double>& X, std::vector<double>& D) {
  int N = (int)xi.size();
  X.assign(N + 2 * g, 0.0);
  D.assign(N + 2 * g, 0.0);
  for (int i = 0; i < N; i++) X[g + i] = xi[i];
  for (int i = 0; i < g; i++) X[i] = X[g] + ((double)(g - i)) * (X[g] - X[g + 1]);
  for (int i = N + g; i < N + 2 * g; i++) X[i] = X[N + g - 1] + ((double)(i - (N + g - 1))) * (X[N + g - 1] - X[N + g - 2]);
  for (int i = 0; i < N; i++) D[i + g] = 2.0 / (X[i + 1 + g] - X[i - 1 + g]);
  for (int i = 0; i < g; i++) D[i] = D[g];
  for (int i = N + g; i < N + 2 * g; i++) D[i] = D[N + g - 1];
}

int read_field(const std::string& path, const Deck& d, int nv, bool ascii, std::vector<double>& xs,
               std::vector<double>& field, bool& found, std::string& err) {
  long long npts = 1, nx = 0;
  for (int s : d.size) { npts *= s; nx += s; }
  xs.assign(nx, 0.0);
  field.assign(npts * nv, 0.0);
  if (!ascii) {
    FILE* f = std::fopen(path.c_str(), "rb");
    found = f != nullptr;
    if (!f) return 0;
    size_t a = std::fread(xs.data(), sizeof(double), nx, f);
    size_t b = std::fread(field.data(), sizeof(double), npts * nv, f);
    std::fclose(f);
    if ((long long)a != nx || (long long)b != npts * nv) {
      err = "short read in " + path;
      return PIAFS_ERR_INPUT;
    }
    return 0;
  }
  // ASCII: grid, then each variable over all points (ReadArray.c:197-225)
  std::ifstream f(path);
  found = (bool)f;
  if (!f) return 0;
  for (long long i = 0; i < nx; i++)
    if (!(f >> xs[i])) { err = "short read in " + path; return PIAFS_ERR_INPUT; }
  for (int v = 0; v < nv; v++)
    for (long long p = 0; p < npts; p++)
      if (!(f >> field[p * nv + v])) { err = "short read in " + path; return PIAFS_ERR_INPUT; }
  return 0;
}

}  // namespace

int read_deck(const std::string& dir, Deck& d, std::string& err) {
  std::map<std::string, std::vector<std::string>> kv;
  bool found = false;
  if (int r = read_keyfile(dir + "/solver.inp", kv, found, err)) return r;
  if (!found) { err = "solver.inp not found in " + dir; return PIAFS_ERR_INPUT; }
  get(kv, "ndims", d.ndims);
  get(kv, "nvars", d.nvars);
  get(kv, "ghost", d.ghosts);
  get(kv, "n_iter", d.n_iter);
  get(kv, "restart_iter", d.restart_iter);
  get(kv, "time_scheme", d.time_scheme);
  get(kv, "time_scheme_type", d.time_scheme_type);
  get(kv, "hyp_space_scheme", d.hyp_space_scheme);
  get(kv, "hyp_interp_type", d.hyp_interp_type);
  get(kv, "par_space_scheme", d.par_space_scheme);
  get(kv, "dt", d.dt);
  get(kv, "conservation_check", d.conservation_check);
  get(kv, "screen_op_iter", d.screen_op_iter);
  get(kv, "file_op_iter", d.file_op_iter);
  get(kv, "op_file_format", d.op_file_format);
  get(kv, "ip_file_type", d.ip_file_type);
  get(kv, "input_mode", d.input_mode);
  get(kv, "output_mode", d.output_mode);
  get(kv, "op_overwrite", d.op_overwrite);
  get(kv, "model", d.model);
  if (kv.count("size")) for (auto& s : kv["size"]) d.size.push_back(std::atoi(s.c_str()));
  if (d.ndims < 1 || d.ndims > 2 || (int)d.size.size() != d.ndims) {
    err = "solver.inp: ndims must be 1 or 2 with one size per dimension";
    return PIAFS_ERR_INPUT;
  }
  if (d.screen_op_iter <= 0) d.screen_op_iter = 1;
  if (d.file_op_iter <= 0) d.file_op_iter = d.n_iter;
  if (d.restart_iter != 0 && d.op_file_format != "binary" && d.op_file_format != "bin") {
    err = "restart is supported only with binary output files";
    return PIAFS_ERR_INPUT;
  }
  if (d.input_mode != "serial") { err = "only input_mode serial is supported"; return PIAFS_ERR_UNSUPPORTED; }
  if (d.conservation_check == "yes") {
    err = "conservation_check yes (boundary flux integrals, TimeRK.c:76-81, TimePostStep.c:66-78) is not on the "
          "GPU path";
    return PIAFS_ERR_UNSUPPORTED;
  }
  // schemes on the GPU path
  if (d.hyp_space_scheme != "weno5" && d.hyp_space_scheme != "crweno5" && d.hyp_space_scheme != "upw5") {
    err = "hyp_space_scheme " + d.hyp_space_scheme + " is not on the GPU path (weno5, crweno5, upw5)";
    return PIAFS_ERR_UNSUPPORTED;
  }
  // interpolation on components or on characteristic variables
  if (d.hyp_interp_type != "components" && d.hyp_interp_type != "characteristic" && d.nvars > 1) {
    err = "hyp_interp_type " + d.hyp_interp_type + " is not a PIAFS interpolation type (components, characteristic)";
    return PIAFS_ERR_UNSUPPORTED;
  }
  if (d.ghosts < 3) { err = "WENO5/CRWENO5 need ghost >= 3"; return PIAFS_ERR_INPUT; }
  if (d.model != "euler1d" && d.model != "navierstokes2d") {
    err = "model " + d.model + " is not on the GPU path (euler1d, navierstokes2d)";
    return PIAFS_ERR_UNSUPPORTED;
  }
  if ((d.model == "euler1d") != (d.ndims == 1)) {
    err = "ndims does not match the model";
    return PIAFS_ERR_INPUT;
  }
  if (d.model == "navierstokes2d" && d.par_space_scheme != "2" && d.par_space_scheme != "4") {
    err = "par_space_scheme " + d.par_space_scheme + " is not a PIAFS parabolic scheme (2, 4)";
    return PIAFS_ERR_UNSUPPORTED;
  }
  if (int r = set_tableau(d, err)) return r;
  // weno.inp
  kv.clear();
  if (int r = read_keyfile(dir + "/weno.inp", kv, found, err)) return r;
  get(kv, "mapped", d.mapped);
  get(kv, "borges", d.borges);
  get(kv, "yc", d.yc);
  get(kv, "no_limiting", d.no_limiting);
  get(kv, "epsilon", d.weno_eps);
  // physics.inp
  kv.clear();
  if (int r = read_keyfile(dir + "/physics.inp", kv, found, err)) return r;
  get(kv, "gamma", d.gamma);
  get(kv, "upwinding", d.upwinding);
  get(kv, "include_chemistry", d.include_chem);
  if (d.model == "navierstokes2d") {
    get(kv, "Pr", d.Pr);
    get(kv, "Re", d.Re);
    get(kv, "T_ref", d.Tref);
    get(kv, "T_0", d.T0);
    get(kv, "T_S", d.TS);
    get(kv, "T_A", d.TA);
    get(kv, "T_B", d.TB);
    get(kv, "write_output", d.write_output);
  }
  if (d.upwinding != "roe" && d.upwinding != "rf-char" && d.upwinding != "llf-char" && d.upwinding != "rusanov") {
    err = "upwinding " + d.upwinding + " is not valid (roe, rf-char, llf-char, rusanov)";
    return PIAFS_ERR_INPUT;
  }
  // The wall boundary conditions keep the physics.inp gamma for NS2D: it is
  // copied into the boundary objects before chemistry replaces the flow gamma
  // (NavierStokes2DInitialize.c:172-174 precede :196-200).  Euler1D never sets
  // it, so its walls see the zero of a calloc'd boundary object.
  d.bc_gamma = d.model == "navierstokes2d" ? d.gamma : 0.0;
  const int nflow = d.model == "navierstokes2d" ? 4 : 3;
  // CRWENO5 on characteristic variables with photochemistry: the reference's
  // 11x11 block inverses (_MatrixInvert_, no pivoting) meet zero pivots on the
  // species rows and its solution is not finite
  if (d.hyp_space_scheme == "crweno5" && d.hyp_interp_type == "characteristic" && d.include_chem == "yes") {
    err = "crweno5 with hyp_interp_type characteristic and photochemistry: the reference's block solve is "
          "singular (use components)";
    return PIAFS_ERR_UNSUPPORTED;
  }
  if (d.include_chem == "yes") {
    if (int r = setup_chemistry(dir, d, nflow, err)) return r;
    // PhysicsOutput: Euler1DWriteChem always (Euler1DInitialize.c:144-145),
    // NavierStokes2DWriteChem with write_output yes (NavierStokes2DInitialize.c:189)
    d.write_species = d.model == "euler1d" || d.write_output == "yes";
  } else if (d.nvars != nflow) {
    err = "nvars has to be " + std::to_string(nflow) + " in solver.inp";
    return PIAFS_ERR_INPUT;
  }
  // grid + initial solution
  const int g = d.ghosts;
  const bool ascii = d.ip_file_type == "ascii";
  std::vector<double> xs, field;
  if (tl_mem) {
    long long nx = 0;
    for (int s : d.size) nx += s;
    if ((long long)tl_mem->grid.size() != nx) { err = "in-memory deck: grid size mismatch"; return PIAFS_ERR_INPUT; }
    xs = tl_mem->grid;
  } else {
    if (int r = read_field(dir + "/initial.inp", d, d.nvars, ascii, xs, field, found, err)) return r;
    if (!found) { err = "initial solution file not found"; return PIAFS_ERR_INPUT; }
  }
  d.grid = xs;
  d.x.clear();
  d.dxinv.clear();
  size_t off = 0;
  for (int k = 0; k < d.ndims; k++) {
    std::vector<double> xi(xs.begin() + off, xs.begin() + off + d.size[k]), X, D;
    off += d.size[k];
    ghost_grid(xi, g, X, D);
    d.x.insert(d.x.end(), X.begin(), X.end());
    d.dxinv.insert(d.dxinv.end(), D.begin(), D.end());
  }
  const int N0 = d.size[0], N1 = d.ndims == 2 ? d.size[1] : 1;
  const int W0 = N0 + 2 * g, W1 = d.ndims == 2 ? N1 + 2 * g : 1, g1 = d.ndims == 2 ? g : 0;
  if (tl_mem) {
    // fields are generated by the caller
    d.u0.clear();
    d.imap.clear();
    goto boundaries;
  }
  d.u0.assign((size_t)W0 * W1 * d.nvars, 0.0);
  for (int j = 0; j < N1; j++)
    for (int i = 0; i < N0; i++)
      for (int v = 0; v < d.nvars; v++)
        d.u0[((size_t)(i + g) + (size_t)W0 * (j + g1)) * d.nvars + v] = field[((size_t)i + (size_t)N0 * j) * d.nvars + v];
  // intensity map (ChemistryInitialize.c:441-476)
  d.imap.assign((size_t)W0 * W1, 0.0);
  if (d.chem) {
    std::vector<double> mx, mf;
    if (int r = read_field(dir + "/imap.inp", d, 1, ascii, mx, mf, found, err)) return r;
    for (int j = 0; j < N1; j++)
      for (int i = 0; i < N0; i++) {
        double val;
        if (found) val = mf[(size_t)i + (size_t)N0 * j];
        else {
          double x0 = d.grid[0], xx = d.grid[i];
          val = d.IA + d.IB * std::cos(d.kg * d.L_ref * (xx - x0) * (1.0 - d.IC * (xx - x0)));
        }
        d.imap[(size_t)(i + g) + (size_t)W0 * (j + g1)] = val;
      }
  }
boundaries:
  // boundary.inp (InitializeBoundaries.c:82-150, CalculateLocalExtent :296-378)
  std::vector<std::string> t;
  if (!read_tokens(dir + "/boundary.inp", t) || t.empty()) {
    err = "boundary.inp not found";
    return PIAFS_ERR_INPUT;
  }
  size_t i = 0;
  int nb = std::atoi(t[i++].c_str());
  if (nb < 0 || nb > MAX_ZONES) { err = "too many boundary zones"; return PIAFS_ERR_UNSUPPORTED; }
  d.zones.clear();
  d.zone_vals.clear();
  d.sponges.clear();
  for (int n = 0; n < nb; n++) {
    if (i + 3 + 2 * d.ndims > t.size()) { err = "boundary.inp: truncated"; return PIAFS_ERR_INPUT; }
    Zone z{};
    std::string type = t[i++];
    z.dim = std::atoi(t[i++].c_str());
    z.face = std::atoi(t[i++].c_str());
    double ext[4] = {0, 0, 0, 0};
    for (int k = 0; k < 2 * d.ndims; k++) ext[k] = std::atof(t[i++].c_str());
    if (type == "sponge") {
      // InitializeBoundaries.c:113-118 (reference state), :313-326 (extent
      // from FindInterval in every dimension); the ghost fill is a no-op
      // (BCSpongeUDummy) and the zone acts through the source (BCSpongeSource)
      if (z.dim < 0 || z.dim >= d.ndims || (z.face != 1 && z.face != -1) || i + d.nvars > t.size()) {
        err = "boundary.inp: bad sponge zone";
        return PIAFS_ERR_INPUT;
      }
      SpongeZone sz{};
      sz.dim = z.dim;
      sz.face = z.face;
      for (int v = 0; v < d.nvars; v++) sz.uref.push_back(std::atof(t[i++].c_str()));
      size_t off = 0;
      for (int k = 0; k < 2; k++) {
        if (k >= d.ndims) { sz.is[k] = 0; sz.ie[k] = 1; continue; }
        find_interval(ext[2 * k], ext[2 * k + 1], d.grid.data() + off, d.size[k], sz.is[k], sz.ie[k]);
        if (k == sz.dim) {
          const double xstart = ext[2 * k], xend = ext[2 * k + 1];
          for (int q = sz.is[k]; q < sz.ie[k]; q++) {
            const double x = d.grid[off + q];   // _GetCoordinate_ (basic.h:34-39)
            sz.sigma.push_back(sz.face > 0 ? (x - xstart) / (xend - xstart) : (x - xend) / (xstart - xend));
          }
        }
        off += d.size[k];
      }
      if (sz.ie[0] > sz.is[0] && sz.ie[1] > sz.is[1]) d.sponges.push_back(sz);
      continue;
    }
    // zone data, in the order the reference reads it (InitializeBoundaries.c:106-168)
    std::vector<double> vals;
    auto next = [&]() { return i < t.size() ? std::atof(t[i++].c_str()) : 0.0; };
    const int nscalars = d.nvars - (2 + d.ndims);
    if (type == "periodic") z.type = BC_PERIODIC;
    else if (type == "extrapolate") z.type = BC_EXTRAPOLATE;
    else if (type == "reflect") z.type = BC_REFLECT;
    else if (type == "dirichlet") {
      z.type = BC_DIRICHLET;
      for (int v = 0; v < d.nvars; v++) vals.push_back(next());
    } else if (type == "slip-wall" || type == "noslip-wall") {
      z.type = type == "slip-wall" ? BC_SLIPWALL : BC_NOSLIP;
      for (int k = 0; k < d.ndims; k++) z.vel[k] = next();
    } else if (type == "subsonic-inflow") {
      z.type = BC_SUB_INFLOW;
      z.rho = next();
      for (int k = 0; k < d.ndims; k++) z.vel[k] = next();
      for (int v = 0; v < nscalars; v++) vals.push_back(next());
    } else if (type == "subsonic-outflow") {
      z.type = BC_SUB_OUTFLOW;
      z.pres = next();
    } else if (type == "subsonic-ambivalent") {
      z.type = BC_SUB_AMBIVALENT;
      z.rho = next();
      for (int k = 0; k < d.ndims; k++) z.vel[k] = next();
      z.pres = next();
    } else if (type == "supersonic-inflow") {
      z.type = BC_SUP_INFLOW;
      z.rho = next();
      for (int k = 0; k < d.ndims; k++) z.vel[k] = next();
      z.pres = next();
      for (int v = 0; v < nscalars; v++) vals.push_back(next());
    } else if (type == "supersonic-outflow") {
      z.type = BC_SUP_OUTFLOW;
    } else {
      err = "boundary type " + type + " is not a PIAFS boundary condition (BCInitialize.c:19-35)";
      return PIAFS_ERR_INPUT;
    }
    if (z.dim < 0 || z.dim >= d.ndims || (z.face != 1 && z.face != -1)) {
      err = "boundary.inp: bad dimension or face";
      return PIAFS_ERR_INPUT;
    }
    size_t xoff = 0;
    for (int k = 0; k < 2; k++) {
      if (k >= d.ndims) { z.is[k] = 0; z.ie[k] = 1; continue; }
      if (k == z.dim) {
        if (z.face == 1) { z.is[k] = -g; z.ie[k] = 0; }
        else { z.is[k] = d.size[k]; z.ie[k] = d.size[k] + g; }
      } else {
        find_interval(ext[2 * k], ext[2 * k + 1], d.grid.data() + xoff, d.size[k], z.is[k], z.ie[k]);
      }
      xoff += d.size[k];
    }
    d.zones.push_back(z);
    d.zone_vals.push_back(vals);
  }
  return 0;
}

int read_exact(const std::string& dir, const Deck& d, std::vector<double>& u, bool& found, std::string& err) {
  std::vector<double> xs;
  return read_field(dir + "/exact.inp", d, d.nvars, d.ip_file_type == "ascii", xs, u, found, err);
}

int restrict_rows(const Deck& d, int rank, int nranks, Deck& out, bool& periodic_y, std::string& err) {
  periodic_y = false;
  if (d.ndims != 2) { err = "a row-slab decomposition needs a 2D grid"; return PIAFS_ERR_UNSUPPORTED; }
  const int N0 = d.size[0], N1 = d.size[1], g = d.ghosts;
  if (nranks < 2 || rank < 0 || rank >= nranks) { err = "bad rank / number of slabs"; return PIAFS_ERR_ARGUMENT; }
  if (N1 % nranks || N0 % nranks) {
    err = "the grid's sides (" + std::to_string(N0) + " x " + std::to_string(N1) + ") must be multiples of the " +
          std::to_string(nranks) + " slabs";
    return PIAFS_ERR_UNSUPPORTED;
  }
  const int n1 = N1 / nranks, j0 = rank * n1;
  if (n1 < g) { err = "slabs thinner than the ghost width"; return PIAFS_ERR_UNSUPPORTED; }
  if (!d.sponges.empty()) { err = "sponge zones are not supported on a decomposed grid"; return PIAFS_ERR_UNSUPPORTED; }
  if (d.model == "navierstokes2d" && d.Re > 0 && d.par_space_scheme == "4") {
    err = "par_space_scheme 4 is not supported on a decomposed grid";
    return PIAFS_ERR_UNSUPPORTED;
  }
  if (d.hyp_interp_type == "characteristic" && d.nvars > 1) {
    err = "hyp_interp_type characteristic is not supported on a decomposed grid";
    return PIAFS_ERR_UNSUPPORTED;
  }
  for (const Zone& z : d.zones) {
    if (z.dim == 0 && (z.is[1] != 0 || z.ie[1] != N1)) {
      err = "x-face boundary zones must span every row on a decomposed grid";
      return PIAFS_ERR_UNSUPPORTED;
    }
    if (z.dim == 1 && z.type == BC_PERIODIC) periodic_y = true;
  }
  out = d;
  out.size[1] = n1;
  out.slab_j0 = j0;
  out.slab_N1 = N1;
  const size_t W0 = (size_t)N0 + 2 * g, W1 = (size_t)N1 + 2 * g, w1 = (size_t)n1 + 2 * g;
  // coordinates and 1/dx: x part whole, y part the slab's ghosted rows
  out.x.assign(d.x.begin(), d.x.begin() + W0);
  out.x.insert(out.x.end(), d.x.begin() + W0 + j0, d.x.begin() + W0 + j0 + w1);
  out.dxinv.assign(d.dxinv.begin(), d.dxinv.begin() + W0);
  out.dxinv.insert(out.dxinv.end(), d.dxinv.begin() + W0 + j0, d.dxinv.begin() + W0 + j0 + w1);
  out.grid.assign(d.grid.begin(), d.grid.begin() + N0);
  out.grid.insert(out.grid.end(), d.grid.begin() + N0 + j0, d.grid.begin() + N0 + j0 + n1);
  // ghosted rows j0 .. j0 + n1 + 2g - 1 of the whole grid (ghosted index)
  if (!d.u0.empty()) {
    const size_t row = W0 * d.nvars;
    out.u0.assign(d.u0.begin() + row * j0, d.u0.begin() + row * (j0 + w1));
  }
  if (!d.imap.empty() && d.imap.size() == W0 * W1) out.imap.assign(d.imap.begin() + W0 * j0, d.imap.begin() + W0 * (j0 + w1));
  out.zones.clear();
  out.zone_vals.clear();
  for (size_t k = 0; k < d.zones.size(); k++) {
    Zone z = d.zones[k];
    if (z.dim == 0) {
      z.ie[1] = n1;
    } else {
      if (z.type == BC_PERIODIC) continue;
      if (z.face == 1 && rank != 0) continue;
      if (z.face == -1 && rank != nranks - 1) continue;
      if (z.face == -1) { z.is[1] = n1; z.ie[1] = n1 + g; }
    }
    out.zones.push_back(z);
    out.zone_vals.push_back(d.zone_vals[k]);
  }
  return 0;
}

int check_deck(const Deck& d, std::string& err) {
  if (d.ndims < 1 || d.ndims > 2 || (int)d.size.size() != d.ndims) {
    err = "ndims must be 1 or 2 with one size per dimension";
    return PIAFS_ERR_INPUT;
  }
  if (d.restart_iter != 0 && d.op_file_format != "binary" && d.op_file_format != "bin") {
    err = "restart is supported only with binary output files";
    return PIAFS_ERR_INPUT;
  }
  if (d.conservation_check == "yes") {
    err = "conservation_check yes (boundary flux integrals, TimeRK.c:76-81, TimePostStep.c:66-78) is not on the "
          "GPU path";
    return PIAFS_ERR_UNSUPPORTED;
  }
  if (d.hyp_space_scheme != "weno5" && d.hyp_space_scheme != "crweno5" && d.hyp_space_scheme != "upw5") {
    err = "hyp_space_scheme " + d.hyp_space_scheme + " is not on the GPU path (weno5, crweno5, upw5)";
    return PIAFS_ERR_UNSUPPORTED;
  }
  if (d.hyp_interp_type != "components" && d.hyp_interp_type != "characteristic" && d.nvars > 1) {
    err = "hyp_interp_type " + d.hyp_interp_type + " is not a PIAFS interpolation type (components, characteristic)";
    return PIAFS_ERR_UNSUPPORTED;
  }
  if (d.ghosts < 3) { err = "WENO5/CRWENO5 need ghost >= 3"; return PIAFS_ERR_INPUT; }
  if (d.model != "euler1d" && d.model != "navierstokes2d") {
    err = "model " + d.model + " is not on the GPU path (euler1d, navierstokes2d)";
    return PIAFS_ERR_UNSUPPORTED;
  }
  if ((d.model == "euler1d") != (d.ndims == 1)) { err = "ndims does not match the model"; return PIAFS_ERR_INPUT; }
  if (d.model == "navierstokes2d" && d.par_space_scheme != "2" && d.par_space_scheme != "4") {
    err = "par_space_scheme " + d.par_space_scheme + " is not a PIAFS parabolic scheme (2, 4)";
    return PIAFS_ERR_UNSUPPORTED;
  }
  if (d.nstages < 1 || d.nstages > MAX_STAGES) { err = "more RK stages than the GPU path holds"; return PIAFS_ERR_UNSUPPORTED; }
  if (d.upwinding != "roe" && d.upwinding != "rf-char" && d.upwinding != "llf-char" && d.upwinding != "rusanov") {
    err = "upwinding " + d.upwinding + " is not valid (roe, rf-char, llf-char, rusanov)";
    return PIAFS_ERR_INPUT;
  }
  if (d.hyp_space_scheme == "crweno5" && d.hyp_interp_type == "characteristic" && d.chem) {
    err = "crweno5 with hyp_interp_type characteristic and photochemistry: the reference's block solve is "
          "singular (use components)";
    return PIAFS_ERR_UNSUPPORTED;
  }
  const int nflow = d.model == "navierstokes2d" ? 4 : 3;
  if (d.nvars != (d.chem ? nflow + 7 * d.nz : nflow)) {
    err = "nvars does not match the model and its chemistry layers";
    return PIAFS_ERR_INPUT;
  }
  return 0;
}

int read_deck_memory(const DeckMemory& m, Deck& d, std::string& err) {
  tl_mem = &m;
  const int r = read_deck("<memory>", d, err);
  tl_mem = nullptr;
  return r;
}

int make_params(const Deck& d, DevParams& P, std::string& err) {
  std::memset(&P, 0, sizeof(P));
  P.ndims = d.ndims;
  P.nvars = d.nvars;
  P.ghosts = d.ghosts;
  P.N0 = d.size[0];
  P.N1 = d.ndims == 2 ? d.size[1] : 1;
  P.W0 = P.N0 + 2 * P.ghosts;
  P.W1 = d.ndims == 2 ? P.N1 + 2 * P.ghosts : 1;
  P.g1 = d.ndims == 2 ? P.ghosts : 0;
  P.jg0 = d.slab_j0;
  P.N1g = d.slab_N1 > 0 ? d.slab_N1 : P.N1;
  P.npg = (long long)P.W0 * P.W1;
  P.ps = (P.npg + 31) / 32 * 32;
  if (d.ndims == 1) {
    P.nint[0] = P.N0 + 1;
    P.nint[1] = 0;
  } else {
    P.nint[0] = (long long)(P.N0 + 1) * P.N1;
    P.nint[1] = (long long)P.N0 * (P.N1 + 1);
  }
  long long nmax = P.nint[0] > P.nint[1] ? P.nint[0] : P.nint[1];
  P.pis = (nmax + 31) / 32 * 32;
  P.model = d.model == "navierstokes2d" ? NS2D : EULER1D;
  P.scheme = d.hyp_space_scheme == "crweno5" ? CRWENO5 : d.hyp_space_scheme == "upw5" ? UPW5 : WENO5;
  P.par4 = d.par_space_scheme == "4" ? 1 : 0;
  P.char_interp = (d.hyp_interp_type == "characteristic" && d.nvars > 1) ? 1 : 0;
  P.upwind = d.upwinding == "roe" ? UPW_ROE : d.upwinding == "rf-char" ? UPW_RF
           : d.upwinding == "llf-char" ? UPW_LLF : UPW_RUSANOV;
  P.weno_type = d.yc ? W_YC : d.borges ? W_BORGES : d.mapped ? W_MAPPED : W_JS;
  P.no_limiting = d.no_limiting;
  P.eps = d.weno_eps;
  P.gamma = d.gamma;
  P.bc_gamma = d.bc_gamma;
  P.Re = d.Re; P.Pr = d.Pr; P.Tref = d.Tref; P.T0 = d.T0; P.TS = d.TS; P.TA = d.TA; P.TB = d.TB;
  P.viscous = (P.model == NS2D && d.Re > 0) ? 1 : 0;
  P.chem = d.chem ? 1 : 0;
  P.nflow = P.model == NS2D ? 4 : 3;
  P.nz = d.nz;
  P.zstride = 7;
  for (int i = 0; i < 11; i++) { P.k[i] = d.kn[i]; P.q[i] = d.qn[i]; }
  P.chem_gamma = d.chem_gamma; P.I0 = d.I0; P.ch_c = d.ch_c; P.ch_h = d.ch_h; P.ch_nu = d.ch_nu;
  P.n_O2 = d.n_O2; P.t_start_norm = d.t_start_norm; P.t_pulse_norm = d.t_pulse_norm; P.sO3 = d.sO3; P.dz = d.dz;
  P.dt = d.dt;
  if (P.scheme == CRWENO5) {
    for (int k = 0; k < d.ndims; k++) {
      if (crweno_cluster_size(d.size[k]) < 0 || d.size[k] < 3) {
        err = "crweno5 lines of " + std::to_string(d.size[k]) + " points are outside the GPU path (3..32769)";
        return PIAFS_ERR_UNSUPPORTED;
      }
    }
  }
  return 0;
}

int write_binary(const std::string& path, const Deck& d, const double* u, std::string& err, int nvars) {
  if (nvars < 0) nvars = d.nvars;
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) {
    err = "could not open " + path + " for writing";
    return PIAFS_ERR_IO;
  }
  int hdr[2] = {d.ndims, nvars};
  long long npts = 1;
  for (int s : d.size) npts *= s;
  bool ok = std::fwrite(hdr, sizeof(int), 2, f) == 2;
  ok = ok && std::fwrite(d.size.data(), sizeof(int), d.ndims, f) == (size_t)d.ndims;
  ok = ok && std::fwrite(d.grid.data(), sizeof(double), d.grid.size(), f) == d.grid.size();
  ok = ok && std::fwrite(u, sizeof(double), npts * nvars, f) == (size_t)(npts * nvars);
  std::fclose(f);
  if (!ok) {
    err = "short write to " + path;
    return PIAFS_ERR_IO;
  }
  return 0;
}

}  // namespace piafs
