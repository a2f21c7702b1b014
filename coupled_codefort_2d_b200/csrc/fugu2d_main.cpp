// fugu2d_main.cpp -- the FUGU-2D driver (src/main.f90:7-262) on the B200 path.
//
// Reads the reference's Fortran namelist file (default input.nml, or argv[1])
// with the /sim_params/ keys of main.f90:32-38, sets up the named case
// (rising_bubble, laplace, poiseuille, cavity, cylinder_flow; main.f90:135-183),
// and runs the time loop of main.f90:193-248 through the C ABI: adaptive dt,
// advance_coupled_step on the device-resident state, a log line every 10
// steps, legacy-VTK output every vtk_freq steps (mod_io.f90:29-164 format) and
// checkpoints every chk_freq steps (mod_io.f90:169-187 byte format).
//
// Extra namelist keys (this build): use_gpu (accepted, the path is the GPU),
// precision ('fp64' | 'mixed'), refine (logical or 0 / 1 / 2), refine_inner_tol, refine_max_inner,
// refine_max_outer, pcg_max_iter, pcg_cap_start, pcd_sweeps, pcd_sweeps_max, pcd_smoother
// ('jacobi' | 'rbsor'), pcd_sor_omega, pcd_visc_scale, graphs (logical), vec_rows, krylov_bc_fix,
// limiter ('vanleer' | 'superbee'),
// free_slip_x, device.
//
//   fugu2d [input.nml]                  run
//   fugu2d --print-params [input.nml]   parse only, print the settings as JSON
#include <sys/stat.h>

#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "fugu_gpu.h"

namespace {

struct Settings {
  // main.f90:55-70 defaults
  std::string case_type = "rising_bubble";
  bool periodic_x = false, periodic_y = false, adaptive_dt = true, consistent_amp = true;
  bool use_bicgstab2 = false, restart = false, use_gpu = true;
  int vtk_freq = 20, chk_freq = 50;
  double u_lid = 1.0, cyl_xc = 0.5, cyl_yc = 0.5, cyl_rad = 0.125, drop_rad = 0.25;
  std::string chk_prefix = "output/chk_fugu2d";
  // mod_params.f90:27-68 defaults
  double Lx = 1.0, Ly = 1.0;
  int Nx_global = 64, Ny_global = 64;
  double rho1 = 1000.0, rho2 = 1.0, mu1 = 1.0, mu2 = 0.01, sigma = 0.0, gx = 0.0, gy = -9.81;
  double dt = 1.0e-3, t_final = 1.0, cfl_target = 0.5;
  int max_time_steps = 10000, time_order = 1;
  double tol_bicgstab2 = 1.0e-6;
  int max_iter_bicgstab2 = 500;
  double alpha_penalty = 1.0e12;
  // extensions
  std::string precision = "fp64", limiter = "vanleer", pcd_smoother = "jacobi";
  int refine = 0, refine_max_inner = 20, refine_max_outer = 30, krylov_bc_fix = 0, free_slip_x = 0, device = 0;
  int pcg_max_iter = 150, pcg_cap_start = 0, pcd_sweeps = 3, pcd_sweeps_max = 0, graphs = 0, vec_rows = 0;
  double refine_inner_tol = 1.0e-2, pcd_sor_omega = 1.0, pcd_visc_scale = 0.0;
};

std::string lower(std::string s) {
  for (auto& ch : s) ch = (char)std::tolower((unsigned char)ch);
  return s;
}
std::string trim(const std::string& s) {
  size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
  return a == std::string::npos ? "" : s.substr(a, b - a + 1);
}

// Parse the /sim_params/ group of a Fortran namelist file into key -> raw value.
bool parse_namelist(const std::string& path, std::map<std::string, std::string>& kv, std::string& err) {
  std::ifstream in(path);
  if (!in) {
    err = "cannot open " + path;
    return false;
  }
  std::stringstream ss;
  ss << in.rdbuf();
  std::string text = ss.str();
  // strip comments ('!' outside quotes)
  std::string clean;
  bool q1 = false, q2 = false, comment = false;
  for (char ch : text) {
    if (comment) {
      if (ch == '\n') { comment = false; clean += '\n'; }
      continue;
    }
    if (ch == '\'' && !q2) q1 = !q1;
    if (ch == '"' && !q1) q2 = !q2;
    if (ch == '!' && !q1 && !q2) { comment = true; continue; }
    clean += ch;
  }
  const std::string low = lower(clean);
  size_t start = low.find("&sim_params");
  if (start == std::string::npos) {
    err = "no &sim_params group";
    return false;
  }
  start += 11;
  // body until the terminating '/' outside quotes
  std::string body;
  q1 = q2 = false;
  size_t i = start;
  for (; i < clean.size(); ++i) {
    char ch = clean[i];
    if (ch == '\'' && !q2) q1 = !q1;
    if (ch == '"' && !q1) q2 = !q2;
    if (ch == '/' && !q1 && !q2) break;
    body += ch;
  }
  // split into name = value items at '=' boundaries
  std::vector<std::pair<std::string, std::string>> items;
  std::string cur_name, cur_val, token;
  size_t p = 0;
  while (p < body.size()) {
    size_t eq = std::string::npos;
    q1 = q2 = false;
    for (size_t k = p; k < body.size(); ++k) {
      char ch = body[k];
      if (ch == '\'' && !q2) q1 = !q1;
      if (ch == '"' && !q1) q2 = !q2;
      if (ch == '=' && !q1 && !q2) { eq = k; break; }
    }
    if (eq == std::string::npos) break;
    // the name is the last identifier before '='; the text before it is the previous value
    std::string before = body.substr(p, eq - p);
    size_t e = before.find_last_not_of(" \t\r\n");
    size_t s = e;
    while (s != std::string::npos && s > 0 && (std::isalnum((unsigned char)before[s - 1]) || before[s - 1] == '_')) --s;
    std::string name = lower(trim(before.substr(s, e - s + 1)));
    std::string prev = trim(before.substr(0, s));
    if (!items.empty()) items.back().second = prev;
    items.push_back({name, ""});
    p = eq + 1;
  }
  if (!items.empty()) items.back().second = trim(body.substr(p));
  for (auto& it : items) {
    std::string v = trim(it.second);
    while (!v.empty() && (v.back() == ',' || std::isspace((unsigned char)v.back()))) v.pop_back();
    kv[it.first] = v;
  }
  return true;
}

double fnum(const std::string& v) {
  std::string s = v;
  for (auto& ch : s)
    if (ch == 'd' || ch == 'D') ch = 'e';
  return std::strtod(s.c_str(), nullptr);
}
bool flog(const std::string& v) {
  std::string s = lower(trim(v));
  return s == ".true." || s == "t" || s == ".t." || s == "true";
}
std::string fstr(const std::string& v) {
  std::string s = trim(v);
  if (s.size() >= 2 && (s[0] == '\'' || s[0] == '"')) s = s.substr(1, s.size() - 2);
  return trim(s);
}

bool apply(Settings& st, const std::map<std::string, std::string>& kv, std::string& err) {
  for (auto& [k, v] : kv) {
    if (k == "case_type") st.case_type = fstr(v);
    else if (k == "lx") st.Lx = fnum(v);
    else if (k == "ly") st.Ly = fnum(v);
    else if (k == "nx_global") st.Nx_global = (int)fnum(v);
    else if (k == "ny_global") st.Ny_global = (int)fnum(v);
    else if (k == "rho1") st.rho1 = fnum(v);
    else if (k == "rho2") st.rho2 = fnum(v);
    else if (k == "mu1") st.mu1 = fnum(v);
    else if (k == "mu2") st.mu2 = fnum(v);
    else if (k == "sigma") st.sigma = fnum(v);
    else if (k == "gx") st.gx = fnum(v);
    else if (k == "gy") st.gy = fnum(v);
    else if (k == "dt") st.dt = fnum(v);
    else if (k == "t_final") st.t_final = fnum(v);
    else if (k == "cfl_target") st.cfl_target = fnum(v);
    else if (k == "max_time_steps") st.max_time_steps = (int)fnum(v);
    else if (k == "time_order") st.time_order = (int)fnum(v);
    else if (k == "tol_bicgstab2") st.tol_bicgstab2 = fnum(v);
    else if (k == "max_iter_bicgstab2") st.max_iter_bicgstab2 = (int)fnum(v);
    else if (k == "alpha_penalty") st.alpha_penalty = fnum(v);
    else if (k == "periodic_x") st.periodic_x = flog(v);
    else if (k == "periodic_y") st.periodic_y = flog(v);
    else if (k == "adaptive_dt") st.adaptive_dt = flog(v);
    else if (k == "consistent_amp") st.consistent_amp = flog(v);
    else if (k == "use_bicgstab2") st.use_bicgstab2 = flog(v);
    else if (k == "restart") st.restart = flog(v);
    else if (k == "vtk_freq") st.vtk_freq = (int)fnum(v);
    else if (k == "chk_freq") st.chk_freq = (int)fnum(v);
    else if (k == "u_lid") st.u_lid = fnum(v);
    else if (k == "cyl_xc") st.cyl_xc = fnum(v);
    else if (k == "cyl_yc") st.cyl_yc = fnum(v);
    else if (k == "cyl_rad") st.cyl_rad = fnum(v);
    else if (k == "drop_rad") st.drop_rad = fnum(v);
    else if (k == "chk_prefix") st.chk_prefix = fstr(v);
    else if (k == "use_gpu") st.use_gpu = flog(v);
    else if (k == "precision") st.precision = lower(fstr(v));
    else if (k == "limiter") st.limiter = lower(fstr(v));
    else if (k == "refine") {
      // logical (.true. = defect correction around the step's BiCGStab) or
      // 0 / 1 / 2 (2 = around flexible GMRES)
      const std::string t = trim(v);
      st.refine = (!t.empty() && std::isdigit((unsigned char)t[0])) ? (int)fnum(t) : (flog(v) ? 1 : 0);
    }
    else if (k == "refine_inner_tol") st.refine_inner_tol = fnum(v);
    else if (k == "refine_max_inner") st.refine_max_inner = (int)fnum(v);
    else if (k == "refine_max_outer") st.refine_max_outer = (int)fnum(v);
    else if (k == "pcg_max_iter") st.pcg_max_iter = (int)fnum(v);
    else if (k == "pcg_cap_start") st.pcg_cap_start = (int)fnum(v);
    else if (k == "pcd_sweeps") st.pcd_sweeps = (int)fnum(v);
    else if (k == "pcd_sweeps_max") st.pcd_sweeps_max = (int)fnum(v);
    else if (k == "pcd_smoother") st.pcd_smoother = lower(fstr(v));
    else if (k == "pcd_sor_omega") st.pcd_sor_omega = fnum(v);
    else if (k == "pcd_visc_scale") st.pcd_visc_scale = fnum(v);
    else if (k == "graphs") st.graphs = flog(v) ? 1 : 0;
    else if (k == "vec_rows") st.vec_rows = (int)fnum(v);
    else if (k == "krylov_bc_fix") st.krylov_bc_fix = flog(v) ? 1 : 0;
    else if (k == "free_slip_x") st.free_slip_x = flog(v) ? 1 : 0;
    else if (k == "device") st.device = (int)fnum(v);
    else {
      err = "unknown namelist key: " + k;  // Fortran's read(nml=) also rejects unknown names
      return false;
    }
  }
  if (st.precision != "fp64" && st.precision != "mixed") {
    err = "precision must be 'fp64' or 'mixed'";
    return false;
  }
  if (st.limiter != "vanleer" && st.limiter != "superbee") {
    err = "limiter must be 'vanleer' or 'superbee'";
    return false;
  }
  if (st.pcd_smoother != "jacobi" && st.pcd_smoother != "rbsor") {
    err = "pcd_smoother must be 'jacobi' or 'rbsor'";
    return false;
  }
  return true;
}

void print_json(const Settings& s) {
  printf("{\"case_type\": \"%s\", \"Lx\": %.17g, \"Ly\": %.17g, \"Nx_global\": %d, \"Ny_global\": %d, "
         "\"rho1\": %.17g, \"rho2\": %.17g, \"mu1\": %.17g, \"mu2\": %.17g, \"sigma\": %.17g, \"gx\": %.17g, "
         "\"gy\": %.17g, \"dt\": %.17g, \"t_final\": %.17g, \"cfl_target\": %.17g, \"max_time_steps\": %d, "
         "\"time_order\": %d, \"tol_bicgstab2\": %.17g, \"max_iter_bicgstab2\": %d, \"alpha_penalty\": %.17g, "
         "\"periodic_x\": %s, \"periodic_y\": %s, \"adaptive_dt\": %s, \"consistent_amp\": %s, "
         "\"use_bicgstab2\": %s, \"restart\": %s, \"vtk_freq\": %d, \"chk_freq\": %d, \"u_lid\": %.17g, "
         "\"cyl_xc\": %.17g, \"cyl_yc\": %.17g, \"cyl_rad\": %.17g, \"drop_rad\": %.17g, \"chk_prefix\": \"%s\", "
         "\"precision\": \"%s\", \"limiter\": \"%s\", \"refine\": %d, \"krylov_bc_fix\": %d, "
         "\"pcd_sweeps\": %d, \"pcd_sweeps_max\": %d, \"pcd_smoother\": \"%s\", \"pcd_sor_omega\": %.17g, "
         "\"graphs\": %d, \"pcd_visc_scale\": %.17g, \"vec_rows\": %d}\n",
         s.case_type.c_str(), s.Lx, s.Ly, s.Nx_global, s.Ny_global, s.rho1, s.rho2, s.mu1, s.mu2, s.sigma, s.gx,
         s.gy, s.dt, s.t_final, s.cfl_target, s.max_time_steps, s.time_order, s.tol_bicgstab2,
         s.max_iter_bicgstab2, s.alpha_penalty, s.periodic_x ? "true" : "false", s.periodic_y ? "true" : "false",
         s.adaptive_dt ? "true" : "false", s.consistent_amp ? "true" : "false",
         s.use_bicgstab2 ? "true" : "false", s.restart ? "true" : "false", s.vtk_freq, s.chk_freq, s.u_lid,
         s.cyl_xc, s.cyl_yc, s.cyl_rad, s.drop_rad, s.chk_prefix.c_str(), s.precision.c_str(), s.limiter.c_str(),
         s.refine, s.krylov_bc_fix, s.pcd_sweeps, s.pcd_sweeps_max, s.pcd_smoother.c_str(), s.pcd_sor_omega,
         s.graphs, s.pcd_visc_scale, s.vec_rows);
}

// ---------------------------------------------------------------- fields
struct Host {
  int nx, ny;
  std::vector<double> f[FUGU_NUM_FIELDS];
  static size_t size(int kind, int nx, int ny) {
    switch (kind) {
      case 1: return (size_t)(nx + 5) * (ny + 4);   // u
      case 2: return (size_t)(nx + 4) * (ny + 5);   // v
      case 3: return (size_t)(nx + 5) * (ny + 5);   // vertex
      default: return (size_t)(nx + 4) * (ny + 4);  // cell
    }
  }
  static int kind(int id) {
    switch (id) {
      case FUGU_F_U_VEL: case FUGU_F_U_PREV: case FUGU_F_RHO_U: case FUGU_F_F_SIGMA_U: case FUGU_F_PHI_S_U: return 1;
      case FUGU_F_V_VEL: case FUGU_F_V_PREV: case FUGU_F_RHO_V: case FUGU_F_F_SIGMA_V: case FUGU_F_PHI_S_V: return 2;
      case FUGU_F_ZETA: case FUGU_F_ETA: return 3;
      default: return 0;
    }
  }
  Host(int nx_, int ny_) : nx(nx_), ny(ny_) {
    for (int i = 0; i < FUGU_NUM_FIELDS; ++i) f[i].assign(size(kind(i), nx, ny), 0.0);
  }
  double& cell(int id, int i, int j) { return f[id][(size_t)(i + 1) + (size_t)(j + 1) * (nx + 4)]; }
};

// case initialisers, main.f90:135-183 (i_start = j_start = 1)
void init_colour(const Settings& s, Host& h, double dx, double dy) {
  for (int j = -1; j <= h.ny + 2; ++j) {
    const double yc = ((double)j - 0.5) * dy;
    for (int i = -1; i <= h.nx + 2; ++i) {
      const double xc = ((double)i - 0.5) * dx;
      double c = 1.0;
      if (s.case_type == "rising_bubble") {
        const double r = std::sqrt((xc - 0.5 * s.Lx) * (xc - 0.5 * s.Lx) + (yc - 0.5) * (yc - 0.5));
        c = r <= s.drop_rad ? 0.0 : 1.0;
      } else if (s.case_type == "laplace") {
        const double r = std::sqrt((xc - 0.5 * s.Lx) * (xc - 0.5 * s.Lx) + (yc - 0.5 * s.Ly) * (yc - 0.5 * s.Ly));
        c = r <= s.drop_rad ? 1.0 : 0.0;
      } else if (s.case_type == "poiseuille") {
        c = yc <= 0.5 * s.Ly ? 1.0 : 0.0;
      }
      h.cell(FUGU_F_C_FIELD, i, j) = c;
    }
  }
}

int write_vtk(const char* path, fugu_ctx* ctx, Host& h, double dx, double dy) {
  const int ids[] = {FUGU_F_P_FIELD, FUGU_F_C_FIELD, FUGU_F_RHO_C, FUGU_F_KAPPA_CURV, FUGU_F_U_VEL, FUGU_F_V_VEL};
  for (int id : ids)
    if (fugu_download(ctx, id, h.f[id].data())) return -1;
  FILE* fp = std::fopen(path, "w");
  if (!fp) return -1;
  const int nx = h.nx, ny = h.ny;
  auto U = [&](int i, int j) { return h.f[FUGU_F_U_VEL][(size_t)(i + 2) + (size_t)(j + 1) * (nx + 5)]; };
  auto V = [&](int i, int j) { return h.f[FUGU_F_V_VEL][(size_t)(i + 1) + (size_t)(j + 2) * (nx + 4)]; };
  std::fprintf(fp, "# vtk DataFile Version 3.0\nFUGU-2D Coupled Two-Phase Solver Output\nASCII\n");
  std::fprintf(fp, "DATASET STRUCTURED_POINTS\nDIMENSIONS %8d%8d%8d\n", nx, ny, 1);
  std::fprintf(fp, "ORIGIN %15.7E%15.7E%15.7E\nSPACING %15.7E%15.7E%15.7E\nPOINT_DATA %10d\n", 0.5 * dx, 0.5 * dy,
               0.0, dx, dy, dx, nx * ny);
  const struct { const char* name; int id; } sc[] = {{"VOF_C", FUGU_F_C_FIELD}, {"Pressure", FUGU_F_P_FIELD},
                                                     {"Density", FUGU_F_RHO_C}, {"Curvature", FUGU_F_KAPPA_CURV}};
  for (auto& s : sc) {
    std::fprintf(fp, "SCALARS %s double 1\nLOOKUP_TABLE default\n", s.name);
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) std::fprintf(fp, "%15.7E\n", h.cell(s.id, i, j));
  }
  std::fprintf(fp, "VECTORS Velocity double\n");
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i)
      std::fprintf(fp, "%15.7E%15.7E%15.7E\n", 0.5 * (U(i - 1, j) + U(i, j)), 0.5 * (V(i, j - 1) + V(i, j)), 0.0);
  return std::fclose(fp) == 0 ? 0 : -1;
}

int fail(fugu_ctx* ctx, const char* what, int rc) {
  std::fprintf(stderr, "fugu2d: %s failed (%d): %s\n", what, rc, ctx ? fugu_last_error(ctx) : "");
  if (ctx) fugu_destroy(ctx);
  return 1;
}

}  // namespace

int main(int argc, char** argv) {
  bool print_only = false;
  std::string nml = "input.nml";
  for (int a = 1; a < argc; ++a) {
    if (std::strcmp(argv[a], "--print-params") == 0) print_only = true;
    else nml = argv[a];
  }
  Settings st;
  struct stat sb;
  if (stat(nml.c_str(), &sb) == 0) {
    std::map<std::string, std::string> kv;
    std::string err;
    if (!parse_namelist(nml, kv, err) || !apply(st, kv, err)) {
      std::fprintf(stderr, "fugu2d: %s: %s\n", nml.c_str(), err.c_str());
      return 2;
    }
  }
  if (print_only) {
    print_json(st);
    return 0;
  }
  const int nx = st.Nx_global, ny = st.Ny_global;
  const double dx = st.Lx / (double)nx, dy = st.Ly / (double)ny;
  mkdir("output", 0755);
  fugu_params p;
  fugu_params_default(&p);
  p.nx = nx; p.ny = ny; p.dx = dx; p.dy = dy;
  p.periodic_x = st.periodic_x; p.periodic_y = st.periodic_y;
  p.rho1 = st.rho1; p.rho2 = st.rho2; p.mu1 = st.mu1; p.mu2 = st.mu2; p.sigma = st.sigma;
  p.gx = st.gx; p.gy = st.gy; p.cfl_target = st.cfl_target; p.alpha_penalty = st.alpha_penalty;
  p.time_order = st.time_order; p.tol_bicgstab2 = st.tol_bicgstab2; p.max_iter_bicgstab2 = st.max_iter_bicgstab2;
  p.limiter = st.limiter == "superbee" ? 1 : 0; p.free_slip_x = st.free_slip_x; p.krylov_bc_fix = st.krylov_bc_fix;
  // mixed precision needs the defect correction; flexible GMRES is its default inner solve
  p.refine = st.refine ? st.refine : (st.precision == "mixed" ? 2 : 0);
  p.refine_inner_tol = st.refine_inner_tol;
  p.refine_max_inner = st.refine_max_inner; p.refine_max_outer = st.refine_max_outer;
  p.pcg_max_iter = st.pcg_max_iter; p.pcg_cap_start = st.pcg_cap_start;
  p.pcd_sweeps = st.pcd_sweeps; p.pcd_sweeps_max = st.pcd_sweeps_max;
  p.pcd_smoother = st.pcd_smoother == "rbsor" ? 1 : 0; p.pcd_sor_omega = st.pcd_sor_omega;
  p.graphs = st.graphs;
  p.pcd_visc_scale = st.pcd_visc_scale;
  p.vec_rows = st.vec_rows;
  p.precision = st.precision == "mixed" ? FUGU_MIXED : FUGU_FP64;
  fugu_ctx* ctx = nullptr;
  int rc = fugu_create(&p, st.device, &ctx);
  if (rc) return fail(nullptr, "fugu_create", rc);
  std::printf("================================================================\n");
  std::printf(" FUGU-2D (B200) : coupled Navier-Stokes / VOF step on %s\n", fugu_version());
  std::printf("================================================================\n");
  std::printf(" Case : %s | Grid : %d x %d | BDF%d | AMP : %s | restart : %s\n", st.case_type.c_str(), nx, ny,
              st.time_order, st.consistent_amp ? "T" : "F", st.restart ? "T" : "F");
  Host h(nx, ny);
  for (auto& v : h.f[FUGU_F_C_FIELD]) v = 1.0;
  const bool has_cyl = st.case_type == "cylinder_flow";
  if (has_cyl) {
    rc = fugu_build_cylinder_mask(ctx, st.cyl_xc, st.cyl_yc, st.cyl_rad, h.f[FUGU_F_PHI_S_U].data(),
                                  h.f[FUGU_F_PHI_S_V].data());
    if (rc) return fail(ctx, "fugu_build_cylinder_mask", rc);
  }
  int start_step = 1;
  double t = 0.0;
  bool restarted = false;
  if (st.restart) {
    const std::string path = st.chk_prefix + "_r0000.bin";
    int step_chk = 0;
    double t_chk = 0.0;
    if (stat(path.c_str(), &sb) == 0 && fugu_read_checkpoint(ctx, path.c_str(), &step_chk, &t_chk) == 0) {
      start_step = step_chk + 1;
      t = t_chk;
      restarted = true;
      std::printf(" Restart from step %6d | t = %10.5f\n", step_chk, t_chk);
      fugu_download(ctx, FUGU_F_C_FIELD, h.f[FUGU_F_C_FIELD].data());
    } else {
      std::printf(" [INFO] no valid checkpoint found, starting at t = 0.\n");
    }
  }
  if (!restarted) {
    init_colour(st, h, dx, dy);
    rc = fugu_halo_scalar(ctx, h.f[FUGU_F_C_FIELD].data());
    if (rc) return fail(ctx, "fugu_halo_scalar", rc);
  }
  // properties from C (main.f90:185-186), then the state on the device
  rc = fugu_compute_mixture_densities(ctx, h.f[FUGU_F_C_FIELD].data(), h.f[FUGU_F_RHO_C].data(),
                                      h.f[FUGU_F_RHO_U].data(), h.f[FUGU_F_RHO_V].data());
  rc = rc ? rc : fugu_compute_mixture_viscosities(ctx, h.f[FUGU_F_C_FIELD].data(), h.f[FUGU_F_KAPPA].data(),
                                                  h.f[FUGU_F_ZETA].data(), h.f[FUGU_F_ETA].data());
  if (rc) return fail(ctx, "properties", rc);
  for (int id = 0; id < FUGU_NUM_FIELDS; ++id) {
    if (restarted && (id == FUGU_F_U_VEL || id == FUGU_F_V_VEL || id == FUGU_F_U_PREV || id == FUGU_F_V_PREV ||
                      id == FUGU_F_P_FIELD || id == FUGU_F_C_FIELD))
      continue;  // already loaded from the checkpoint
    if ((rc = fugu_upload(ctx, id, h.f[id].data()))) return fail(ctx, "fugu_upload", rc);
  }
  if (st.vtk_freq > 0 && start_step == 1) write_vtk("output/fugu2d_0000.vtk", ctx, h, dx, dy);
  fugu_step_opts o;
  std::memset(&o, 0, sizeof(o));
  o.use_bicgstab2 = st.use_bicgstab2;
  o.consistent_amp = st.consistent_amp;
  if (st.case_type == "cavity") {
    o.has_lid = 1;
    o.u_top_lid = st.u_lid;
  }
  o.has_penalty = has_cyl;
  fugu_stats stats;
  for (int step = start_step; step <= st.max_time_steps; ++step) {
    if (t >= st.t_final) break;
    double dt_step = st.dt;
    if (st.adaptive_dt) {
      fugu_download(ctx, FUGU_F_U_VEL, h.f[FUGU_F_U_VEL].data());
      fugu_download(ctx, FUGU_F_V_VEL, h.f[FUGU_F_V_VEL].data());
      rc = fugu_compute_adaptive_dt(ctx, h.f[FUGU_F_U_VEL].data(), h.f[FUGU_F_V_VEL].data(), st.dt, &dt_step);
      if (rc) return fail(ctx, "fugu_compute_adaptive_dt", rc);
    }
    if (t + dt_step > st.t_final) dt_step = st.t_final - t;
    rc = fugu_step(ctx, dt_step, step, &o, &stats);
    if (rc) return fail(ctx, "fugu_step", rc);
    t += dt_step;
    if (step == start_step || step % 10 == 0)
      std::printf(" Step %5d | t = %8.4f | dt = %9.2E | iter = %3d | res = %9.2E\n", step, t, dt_step, stats.iter,
                  stats.res);
    if (st.vtk_freq > 0 && step % st.vtk_freq == 0) {
      char name[256];
      std::snprintf(name, sizeof(name), "output/fugu2d_%04d.vtk", step);
      write_vtk(name, ctx, h, dx, dy);
    }
    if (st.chk_freq > 0 && step % st.chk_freq == 0) {
      const std::string path = st.chk_prefix + "_r0000.bin";
      if ((rc = fugu_write_checkpoint(ctx, path.c_str(), step, t))) return fail(ctx, "fugu_write_checkpoint", rc);
    }
  }
  std::printf("================================================================\n");
  std::printf(" Simulation finished at t = %10.5f\n", t);
  std::printf("================================================================\n");
  fugu_destroy(ctx);
  return 0;
}
