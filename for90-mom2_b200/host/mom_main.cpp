// mom_b200 -- the reference's `mom` command interpreter (msgloop,
// interface.f90:1624-1734) over the C ABI, for the commands of the linear
// PMCHWT scattering path:
//
//   name  mesh  wlrg  wlls  symm  sbnd  nmed  smed  ndom  sdom  fdom  nsrc
//   ssrc  quad  solv  crst  rcst  nfpl  exit
//
// plus two settings this build adds (the reference always computes in FP64):
//
//   prec fp64 | mixed [tol [maxit]]   arithmetic of solv (default fp64;
//                                     mixed: FP32 tensor-core LU + FP64
//                                     refinement to ||r|| <= tol ||b||,
//                                     default tol 1e-12, maxit 30)
//   dev  <index>                      CUDA device (default 0, or $MOM_DEVICE)
//
// Commands read one line each from standard input with Fortran list-directed
// syntax: blanks or commas separate items, strings may be quoted, complex
// values are written (re, im) and exponents may use d (200d-9).  Results go
// to the same files as the reference: `crst` writes <name>-s<source>.crs
// (wavelength, sigma_sca, sigma_abs per row) and `rcst w s nt np` writes
// <name>-wl<w>-s<s>.rcs (nt rows of np values), both as EN15.3 fields with a
// blank line after each row (write_data, aux.f90:192-211); `nfpl` writes the
// field-component files of read_nfpl.
//
// Symmetry groups are products of id and the mirror groups mxp, myp, mzp
// with the xplane / yplane / zplane boundaries of sbnd.  Media may carry a
// centrosymmetric surface nonlinearity (`smed m nlsurf value chi_nnn chi_ntt
// chi_ttn`, with the mirror groups too): solv then also solves the second
// harmonic (solver.f90:143-217) and crst, rcst, nfms, nfem, nfdm and nfpl also write
// its results (-sh files).  Commands of the reference outside this path
// (rotation groups, periodic boundaries and Green's functions, volume
// domains, bulk nonlinearities, diffraction, polarizability, the VIE
// solver, source offsets and scans) print an error and stop, as the
// reference does on invalid input, instead of producing results this build
// does not compute.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/mom_gpu.h"

namespace {

// constants.f90:8-16: pi is a default-real literal, so it carries float
// rounding into c0-derived frequencies and degree conversions.
const double kPi = (double)3.141592653589f;
const double kC0 = 2.997924580003e8;
const double kDegToRad = kPi / 180.0;

using cplx = std::complex<double>;

[[noreturn]] void stop(const std::string &msg) {
  std::printf(" %s\n", msg.c_str());
  std::fflush(stdout);
  std::exit(1);
}

// ---- list-directed input ----

// Items of a list-directed record: quoted strings lose their quotes,
// parenthesised complex values stay one item "(re,im)".
std::vector<std::string> items(const std::string &line) {
  std::vector<std::string> out;
  size_t i = 0;
  const size_t n = line.size();
  while (i < n) {
    const char ch = line[i];
    if (ch == ' ' || ch == '\t' || ch == ',' || ch == '\r') {
      i++;
      continue;
    }
    if (ch == '/') break;  // list-directed input ends at a slash
    if (ch == '\'' || ch == '"') {
      const size_t j = line.find(ch, i + 1);
      if (j == std::string::npos) stop("Error: unterminated string in '" + line + "'");
      out.push_back(line.substr(i + 1, j - i - 1));
      i = j + 1;
      continue;
    }
    if (ch == '(') {
      const size_t j = line.find(')', i + 1);
      if (j == std::string::npos) stop("Error: unterminated complex value in '" + line + "'");
      out.push_back(line.substr(i, j - i + 1));
      i = j + 1;
      continue;
    }
    size_t j = i;
    while (j < n && line[j] != ' ' && line[j] != '\t' && line[j] != ',' && line[j] != '\r') j++;
    out.push_back(line.substr(i, j - i));
    i = j;
  }
  return out;
}

bool to_real(std::string s, double *v) {
  for (char &c : s)
    if (c == 'd' || c == 'D') c = 'e';
  char *end = nullptr;
  *v = std::strtod(s.c_str(), &end);
  return end && *end == '\0' && !s.empty();
}

double real_item(const std::vector<std::string> &it, size_t k, const char *cmd) {
  double v;
  if (k >= it.size() || !to_real(it[k], &v)) stop(std::string("Error: bad or missing number in command ") + cmd);
  return v;
}

int int_item(const std::vector<std::string> &it, size_t k, const char *cmd) {
  const double v = real_item(it, k, cmd);
  if (v != std::floor(v)) stop(std::string("Error: expected an integer in command ") + cmd);
  return (int)v;
}

cplx complex_item(const std::vector<std::string> &it, size_t k, const char *cmd) {
  if (k >= it.size()) stop(std::string("Error: missing complex value in command ") + cmd);
  const std::string &s = it[k];
  if (s.size() < 5 || s.front() != '(' || s.back() != ')')
    stop(std::string("Error: complex values are written (re, im) in command ") + cmd);
  const std::vector<std::string> p = items(s.substr(1, s.size() - 2));
  double re, im;
  if (p.size() != 2 || !to_real(p[0], &re) || !to_real(p[1], &im))
    stop(std::string("Error: bad complex value in command ") + cmd);
  return {re, im};
}

// ---- output ----

// Fortran EN15.3: engineering notation (mantissa in [1, 1000), exponent a
// multiple of three, three decimals), right-justified in 15 columns.
std::string en15_3(double v) {
  char buf[64];
  if (v == 0.0 || !std::isfinite(v)) {
    if (v == 0.0) std::snprintf(buf, sizeof buf, "0.000E+00");
    else std::snprintf(buf, sizeof buf, "%s", std::isnan(v) ? "NaN" : (v > 0 ? "Infinity" : "-Infinity"));
  } else {
    const double a = std::fabs(v);
    int e3 = (int)std::floor(std::log10(a) / 3.0) * 3;
    double m = a / std::pow(10.0, e3);
    if (m < 1.0) {  // log10 rounding just below a power of 1000
      m *= 1000.0;
      e3 -= 3;
    }
    char mb[32];
    std::snprintf(mb, sizeof mb, "%.3f", m);
    if (std::atof(mb) >= 1000.0) {
      m /= 1000.0;
      e3 += 3;
      std::snprintf(mb, sizeof mb, "%.3f", m);
    }
    std::snprintf(buf, sizeof buf, "%s%sE%c%02d", v < 0 ? "-" : "", mb, e3 < 0 ? '-' : '+', std::abs(e3));
  }
  std::string s(buf);
  if (s.size() < 15) s = std::string(15 - s.size(), ' ') + s;
  return s;
}

// write_data (aux.f90:192-211): rows of EN15.3 fields, each row followed by
// an empty record.
void write_data(const std::string &path, const std::vector<std::vector<double>> &rows) {
  std::FILE *f = std::fopen(path.c_str(), "w");
  if (!f) stop("Could not open output file" + path + "!");
  for (const auto &r : rows) {
    for (double v : r) std::fputs(en15_3(v).c_str(), f);
    std::fputs("\n\n", f);
  }
  std::fclose(f);
}

// ---- state: the batch type (common.f90:71-108) reduced to this path ----

struct Domain {
  bool set = false;
  int medium = 0;  // 1-based medium index
};

struct State {
  std::string name = "unnamed";
  std::string quad = "tri_gl13";  // batch_defaults (common.f90:111-122)
  mom_problem *prob = nullptr;
  bool finalized = false;
  std::vector<double> wl;
  std::vector<std::vector<cplx>> media;  // [medium][wavelength]
  std::vector<Domain> doms;
  std::vector<mom_src> src;
  std::vector<bool> src_set;
  int precision = MOM_PREC_FP64;
  double tol = 1e-12;
  int maxit = 30;
  int device = 0;
  mom_ctx *ctx = nullptr;
  bool uploaded = false;
  int64_t n2 = 0;                    // 2N unknowns
  double scale = 1.0;                // scale of the mesh command (b%scale)
  std::vector<std::string> symm;     // named groups of the symmetry group (read_symm)
  int nga = 1;                       // its order
  std::vector<std::vector<double>> x;  // per wavelength: [nsrc][nga][2N] complex, interleaved
  // Second harmonic: per medium the refractive indices at half the
  // wavelength (prop%shri) and the surface nonlinearity; per wavelength the
  // SH solutions and, per domain, the source coefficients of nonlinear ones.
  std::vector<std::vector<cplx>> media_sh;  // [medium][wavelength]
  std::vector<mom_nls> nls;                 // [medium]
  std::vector<std::vector<double>> nlx;     // per wavelength, as x
  std::vector<std::vector<std::vector<double>>> shc;  // [wavelength][domain]: empty if linear
};

void clear_solutions(State &s) {
  s.x.clear();
  s.nlx.clear();
  s.shc.clear();
}

bool any_nls(const State &s) {
  for (const auto &m : s.nls)
    if (m.active) return true;
  return false;
}

void check(State &s, int st, const char *what) {
  if (st == MOM_OK) return;
  std::string msg = std::string("Error in ") + what + ": " + mom_gpu_strerror(st);
  if (s.ctx) {
    const char *le = mom_gpu_last_error(s.ctx);
    if (le && *le) msg += std::string(" (") + le + ")";
  }
  stop(msg);
}

double omega_of(double wl) { return 2.0 * kPi * kC0 / wl; }

// get_refind (aux.f90:100-167): linear interpolation in a (wl, n, k) table;
// the result passes through a default-kind (single precision) complex, and
// wavelengths outside the table give unity.
cplx refind_from_file(const std::string &path, double wl) {
  std::ifstream f(path);
  if (!f) stop("Could not open refractive index lookup file!");
  std::string line;
  auto next = [&](double *w, double *nr, double *ni) -> bool {
    while (std::getline(f, line)) {
      const std::vector<std::string> it = items(line);
      if (it.size() < 3) continue;
      if (to_real(it[0], w) && to_real(it[1], nr) && to_real(it[2], ni)) return true;
    }
    return false;
  };
  auto single = [](double re, double im) { return cplx((double)(float)re, (double)(float)im); };
  double w1, n1, k1, w2, n2, k2;
  if (!next(&w1, &n1, &k1)) stop("Could not read refractive index lookup file!");
  if (wl < w1) {
    std::printf(" Wavelength below refractive index sample range!\n Using unity refractive index.\n");
    return 1.0;
  }
  while (next(&w2, &n2, &k2)) {
    if (w1 <= wl && wl <= w2 && w1 != w2) {
      const double t = (wl - w1) / (w2 - w1);
      return single(n1 + t * (n2 - n1), k1 + t * (k2 - k1));
    } else if (wl == w1) {
      return single(n1, k1);
    } else if (wl == w2) {
      return single(n2, k2);
    } else if (w1 > w2) {
      stop("Refractive index data disordered!");
    }
    w1 = w2;
    n1 = n2;
    k1 = k2;
  }
  std::printf(" Wavelength above refractive index sample range!\n Using unity refractive index.\n");
  return 1.0;
}

void ensure_ctx(State &s) {
  if (s.ctx) return;
  check(s, mom_gpu_create(s.device, &s.ctx), "mom_gpu_create");
}

std::vector<double> ri_table(const State &s, size_t n, bool sh = false) {
  std::vector<double> ri(2 * s.doms.size());
  for (size_t d = 0; d < s.doms.size(); d++) {
    const cplx v = (sh ? s.media_sh : s.media)[s.doms[d].medium - 1][n];
    ri[2 * d] = v.real();
    ri[2 * d + 1] = v.imag();
  }
  return ri;
}

// Refractive index of domain d's medium (1-based), fundamental or second harmonic.
cplx dom_ri(const State &s, int d, int w, bool sh) {
  return (sh ? s.media_sh : s.media)[s.doms[d - 1].medium - 1][w - 1];
}

// solve_batch (solver.f90:17-142): every wavelength, all sources.
void solve_batch(State &s) {
  std::printf(" --- Begin wavelength batch ---\n");
  if (s.wl.empty()) stop("Setup wavelengths prior to solving!");
  if (!s.prob) stop("Load mesh prior to solving!");
  if (s.doms.empty() || !s.finalized) stop("Set up domains prior to solving!");
  if (s.media.empty()) stop("Set up media prior to solving!");
  if (s.src.empty()) stop("Set up source prior to solving!");
  for (size_t i = 0; i < s.src.size(); i++)
    if (!s.src_set[i]) stop("Source " + std::to_string(i + 1) + " has not been set up!");
  for (size_t d = 0; d < s.doms.size(); d++)
    if (!s.doms[d].set || s.doms[d].medium < 1 || s.doms[d].medium > (int)s.media.size())
      stop("Domain " + std::to_string(d + 1) + " has no valid medium!");
  ensure_ctx(s);
  if (!s.uploaded) {
    check(s, mom_problem_upload(s.prob, s.ctx, s.quad.c_str()), "upload of the domains");
    if (!s.symm.empty()) {
      std::vector<int32_t> bnd(mom_problem_nedges(s.prob));
      check(s, mom_problem_edge_bnd(s.prob, bnd.data()), "symm");
      std::vector<const char *> names;
      for (const auto &nm : s.symm) names.push_back(nm.c_str());
      check(s, mom_gpu_set_symmetry(s.ctx, (int32_t)names.size(), names.data(), bnd.data()), "symm");
    }
    s.nga = mom_gpu_group_order(s.ctx);
    s.uploaded = true;
  }
  s.n2 = 2 * (int64_t)mom_problem_nedges(s.prob);
  std::printf(" Name: %s\n Triangle quadrature: %s\n Arithmetic: %s\n", s.name.c_str(), s.quad.c_str(),
              s.precision == MOM_PREC_FP64 ? "FP64" : "mixed (FP32 LU + FP64 refinement)");
  const int nsrc = (int)s.src.size();
  s.x.assign(s.wl.size(), std::vector<double>());
  for (size_t n = 0; n < s.wl.size(); n++) {
    std::printf(" Wavelength: %6.1f nm (%zu of %zu)\n", s.wl[n] * 1e9, n + 1, s.wl.size());
    const std::vector<double> ri = ri_table(s, n);
    for (size_t d = 0; d < s.doms.size(); d++)
      std::printf(" Refractive index of domain %zu: (%6.3f,%6.3f)\n", d + 1, ri[2 * d], ri[2 * d + 1]);
    s.x[n].assign((size_t)2 * s.n2 * s.nga * nsrc, 0.0);
    int32_t iters = 0;
    check(s,
          mom_gpu_solve_wavelength(s.ctx, omega_of(s.wl[n]), ri.data(), nsrc, s.src.data(), s.precision, s.tol,
                                   s.maxit, s.x[n].data(), s.n2, &iters),
          "solv");
    if (s.precision == MOM_PREC_MIXED) std::printf(" Refinement steps: %d\n", iters);
    if (any_nls(s)) {
      // the second-harmonic branch of solve_batch (solver.f90:143-217)
      std::printf(" Solving nonlinear scattering from centrosymmetric material\n");
      if (s.nlx.size() != s.wl.size()) {
        s.nlx.assign(s.wl.size(), std::vector<double>());
        s.shc.assign(s.wl.size(), std::vector<std::vector<double>>(s.doms.size()));
      }
      const std::vector<double> shri = ri_table(s, n, true);
      std::vector<mom_nls> dn(s.doms.size());
      for (size_t d = 0; d < s.doms.size(); d++) dn[d] = s.nls[s.doms[d].medium - 1];
      s.nlx[n].assign((size_t)2 * s.n2 * s.nga * nsrc, 0.0);
      check(s,
            mom_gpu_shg_solve(s.ctx, omega_of(s.wl[n]), ri.data(), shri.data(), dn.data(), s.precision, s.tol,
                              s.maxit, s.nlx[n].data(), s.n2, &iters),
            "solv (second harmonic)");
      for (size_t d = 0; d < s.doms.size(); d++) {
        s.shc[n][d].clear();
        if (!dn[d].active) continue;
        s.shc[n][d].assign((size_t)2 * s.n2 * s.nga * nsrc, 0.0);
        check(s, mom_gpu_shg_source_coef(s.ctx, (int32_t)d, s.shc[n][d].data(), s.n2), "solv (second harmonic)");
      }
    }
  }
  std::fflush(stdout);
}

// read_crst (interface.f90:1384-1475).
void crst(State &s, const std::vector<std::string> &it) {
  int medium = 1, domain = 1;
  double factor = 1.0;
  if (it.size() > 1) {
    medium = int_item(it, 1, "crst");
    domain = int_item(it, 2, "crst");
    factor = real_item(it, 3, "crst");
  }
  if (s.x.empty()) stop("Error: solve (solv) before computing cross sections!");
  if (medium < 1 || medium > (int)s.media.size() || domain < 1 || domain > (int)s.doms.size())
    stop("Error: medium or domain index out of range in crst!");
  std::printf(" Computing extinction cross-section\n");
  const int nsrc = (int)s.src.size();
  std::vector<std::vector<std::vector<double>>> data(nsrc, std::vector<std::vector<double>>(s.wl.size()));
  std::vector<double> csca(nsrc), cabs(nsrc);
  for (size_t n = 0; n < s.wl.size(); n++) {
    const cplx v = s.media[medium - 1][n];
    const double ri[2] = {v.real(), v.imag()};
    check(s,
          mom_gpu_cross_sections(s.ctx, domain - 1, omega_of(s.wl[n]), ri, nsrc, s.src.data(), s.x[n].data(), s.n2,
                                 csca.data(), cabs.data()),
          "crst");
    for (int k = 0; k < nsrc; k++) data[k][n] = {s.wl[n], csca[k] * factor, cabs[k] * factor};
    std::printf(" Wavelength %zu of %zu\n", n + 1, s.wl.size());
  }
  for (int k = 0; k < nsrc; k++) write_data(s.name + "-s" + std::to_string(k + 1) + ".crs", data[k]);
  if (!s.nlx.empty()) {
    // second harmonic: no incident field, 2 omega, the medium's SH index
    const std::vector<mom_src> none(nsrc, mom_src{MOM_SRC_NONE, 0, 0, 0, 0, 0});
    for (size_t n = 0; n < s.wl.size(); n++) {
      const cplx v = s.media_sh[medium - 1][n];
      const double ri[2] = {v.real(), v.imag()};
      check(s,
            mom_gpu_cross_sections(s.ctx, domain - 1, 2.0 * omega_of(s.wl[n]), ri, nsrc, none.data(),
                                   s.nlx[n].data(), s.n2, csca.data(), cabs.data()),
            "crst");
      for (int k = 0; k < nsrc; k++) data[k][n] = {s.wl[n], csca[k] * factor, cabs[k] * factor};
      std::printf(" Wavelength %zu of %zu\n", n + 1, s.wl.size());
    }
    for (int k = 0; k < nsrc; k++) write_data(s.name + "-s" + std::to_string(k + 1) + "-sh.crs", data[k]);
  }
  std::fflush(stdout);
}

// read_rcst (interface.f90:1291-1334).
void rcst(State &s, const std::vector<std::string> &it) {
  const int w = int_item(it, 1, "rcst"), k = int_item(it, 2, "rcst");
  const int nt = int_item(it, 3, "rcst"), np = int_item(it, 4, "rcst");
  if (s.x.empty()) stop("Error: solve (solv) before computing radar cross-sections!");
  if (w < 1 || w > (int)s.wl.size() || k < 1 || k > (int)s.src.size() || nt < 1 || np < 1)
    stop("Error: index or grid size out of range in rcst!");
  std::printf(" Computing radar cross-sections\n");
  for (int sh = 0; sh < (s.nlx.empty() ? 1 : 2); sh++) {
    // the second pass: the SH solutions at 2 omega with domain 1's SH index
    const cplx v = dom_ri(s, 1, w, sh);
    const double ri[2] = {v.real(), v.imag()};
    std::vector<double> out((size_t)nt * np);
    check(s,
          mom_gpu_rcs(s.ctx, 0, (sh ? 2.0 : 1.0) * omega_of(s.wl[w - 1]), ri, k - 1,
                      (sh ? s.nlx : s.x)[w - 1].data(), s.n2, nt, np, out.data()),
          "rcst");
    std::vector<std::vector<double>> rows(nt, std::vector<double>(np));
    for (int i = 0; i < nt; i++)
      for (int j = 0; j < np; j++) rows[i][j] = out[(size_t)j * nt + i];  // rcsdata(1:nt, 1:np), column-major
    write_data(s.name + "-wl" + std::to_string(w) + "-s" + std::to_string(k) + (sh ? "-sh.rcs" : ".rcs"), rows);
  }
  std::fflush(stdout);
}

// read_nfpl (interface.f90:805-894) with field_plane (nfpost.f90:316-374):
// fields of domain d on the n1 x n2 grid origin + i/(n1-1) v1 + j/(n2-1) v2,
// plus the incident field in domain 1, expressed in the basis (v1/|v1|,
// v2/|v2|, their cross product); 12 files per source, each n2 rows of n1.
void nfpl_pass(State &s, int w, int d, int sh, const double *v1, const double *v2, int n1, int n2,
               const std::vector<double> &pts, const std::string &tag);

void nfpl(State &s, const std::vector<std::string> &it) {
  const int w = int_item(it, 1, "nfpl"), d = int_item(it, 2, "nfpl");
  double o[3], v1[3], v2[3];
  for (int i = 0; i < 3; i++) {
    o[i] = real_item(it, 3 + i, "nfpl");
    v1[i] = real_item(it, 6 + i, "nfpl");
    v2[i] = real_item(it, 9 + i, "nfpl");
  }
  const int n1 = int_item(it, 12, "nfpl"), n2 = int_item(it, 13, "nfpl");
  if (it.size() < 15) stop("Error: nfpl needs a tag");
  const std::string tag = it[14];
  if (s.x.empty()) stop("Error: solve (solv) before computing near fields!");
  if (w < 1 || w > (int)s.wl.size() || d < 1 || d > (int)s.doms.size() || n1 < 2 || n2 < 2)
    stop("Error: index or grid size out of range in nfpl (grids need at least 2 x 2 points)");
  const int npts = n1 * n2;
  std::vector<double> pts(3 * (size_t)npts);
  for (int a = 0; a < n1; a++)
    for (int b = 0; b < n2; b++)
      for (int i = 0; i < 3; i++)
        pts[3 * ((size_t)a * n2 + b) + i] = o[i] + (double)a / (n1 - 1) * v1[i] + (double)b / (n2 - 1) * v2[i];
  std::printf(" Computing near fields on a plane\n");
  for (int sh = 0; sh < (s.nlx.empty() ? 1 : 2); sh++)
    nfpl_pass(s, w, d, sh, v1, v2, n1, n2, pts, tag);
  std::fflush(stdout);
}

// One pass of nfpl: the fundamental (incident field added in domain 1) or,
// with sh, the second harmonic (2 omega, SH index, no incident field; file
// stems end in -sh, interface.f90:855-888).
void nfpl_pass(State &s, int w, int d, int sh, const double *v1, const double *v2, int n1, int n2,
               const std::vector<double> &pts, const std::string &tag) {
  const int nsrc = (int)s.src.size(), npts = n1 * n2;
  const cplx v = dom_ri(s, d, w, sh);
  const double ri[2] = {v.real(), v.imag()};
  std::vector<double> e(6 * (size_t)npts * nsrc), h(6 * (size_t)npts * nsrc);
  check(s,
        mom_gpu_scat_fields(s.ctx, d - 1, (sh ? 2.0 : 1.0) * omega_of(s.wl[w - 1]), ri, nsrc,
                            (d == 1 && !sh) ? s.src.data() : nullptr, (sh ? s.nlx : s.x)[w - 1].data(), s.n2, npts,
                            pts.data(), e.data(), h.data()),
        "nfpl");
  double b1[3], b2[3], b3[3];
  const double l1 = std::sqrt(v1[0] * v1[0] + v1[1] * v1[1] + v1[2] * v1[2]);
  const double l2 = std::sqrt(v2[0] * v2[0] + v2[1] * v2[1] + v2[2] * v2[2]);
  for (int i = 0; i < 3; i++) {
    b1[i] = v1[i] / l1;
    b2[i] = v2[i] / l2;
  }
  b3[0] = b1[1] * b2[2] - b1[2] * b2[1];
  b3[1] = b1[2] * b2[0] - b1[0] * b2[2];
  b3[2] = b1[0] * b2[1] - b1[1] * b2[0];
  const double *basis[3] = {b1, b2, b3};
  const char *comp[3] = {"x", "y", "z"};
  for (int k = 0; k < nsrc; k++) {
    const std::string stem = s.name + "-wl" + std::to_string(w) + "-s" + std::to_string(k + 1) + "-d" +
                             std::to_string(d) + "-" + tag + (sh ? "-sh-" : "-");
    for (int f = 0; f < 2; f++) {
      const std::vector<double> &src = f == 0 ? e : h;
      std::vector<std::vector<std::vector<double>>> R(3, std::vector<std::vector<double>>(n2, std::vector<double>(n1)));
      std::vector<std::vector<std::vector<double>>> I(3, std::vector<std::vector<double>>(n2, std::vector<double>(n1)));
      for (int a = 0; a < n1; a++)
        for (int b = 0; b < n2; b++) {
          const double *fv = &src[6 * (((size_t)k * npts) + (size_t)a * n2 + b)];  // 3 complex
          for (int c = 0; c < 3; c++) {
            // dotc (linalg.f90:15-21): no conjugation
            const double *bc = basis[c];
            R[c][b][a] = bc[0] * fv[0] + bc[1] * fv[2] + bc[2] * fv[4];
            I[c][b][a] = bc[0] * fv[1] + bc[1] * fv[3] + bc[2] * fv[5];
          }
        }
      const char fl = f == 0 ? 'e' : 'h';
      for (int c = 0; c < 3; c++) write_data(stem + fl + comp[c] + "-re.dat", R[c]);
      for (int c = 0; c < 3; c++) write_data(stem + fl + comp[c] + "-im.dat", I[c]);
    }
  }
}

// ---- field maps in Gmsh post-processing files (mesh.f90:1740-1978) ----

constexpr int kSteps = 25;  // time steps of the harmonic animation (nsteps)

// REAL(v exp(-i 2 pi l / nsteps)) of a complex value (re, im)
inline double phase_re(const double *v, int l) {
  const double a = -2.0 * kPi * (double)l / kSteps;
  return v[0] * std::cos(a) - v[1] * std::sin(a);
}

// A list-directed record "n value" (WRITE(fid,*) n, ' ', value): the
// reference leaves its layout to the compiler; written here as an integer
// and a 17-digit real.
void list_record(std::FILE *f, int n, double v) { std::fprintf(f, "%12d   %.17E\n", n, v); }

void msh_header(std::FILE *f) { std::fputs("$MeshFormat\n2.1 0 8\n$EndMeshFormat\n", f); }

void msh_node(std::FILE *f, int n, const double *p, double scale) {
  std::fprintf(f, "%d ", n);
  for (int i = 0; i < 3; i++) std::fputs(en15_3(p[i] / scale).c_str(), f);
  std::fputs("\n", f);
}

// save_vector_fields_msh (mesh.f90:1740-1888): the mesh and, per face, 25
// animation frames each of Re(E), Re(H) (3 components), Re(En), Re(Hn) and
// |Re(E)|, |Re(H)|.  e, h: [nfaces][3] complex (6 doubles per face).
void save_vector_fields_msh(const std::string &path, const std::vector<double> &nodes,
                            const std::vector<int> &faces, const std::vector<double> &normals,
                            const std::vector<double> &e, const std::vector<double> &h, double scale) {
  std::FILE *f = std::fopen(path.c_str(), "w");
  if (!f) stop("Could not open output file" + path + "!");
  const int nn = (int)(nodes.size() / 3), nf = (int)(faces.size() / 3);
  msh_header(f);
  std::fprintf(f, "$Nodes\n%d\n", nn);
  for (int n = 0; n < nn; n++) msh_node(f, n + 1, &nodes[3 * (size_t)n], scale);
  std::fprintf(f, "$EndNodes\n$Elements\n%d\n", nf);
  for (int n = 0; n < nf; n++)
    std::fprintf(f, "%d 2 3 0 0 0 %d %d %d\n", n + 1, faces[3 * n] + 1, faces[3 * n + 1] + 1, faces[3 * n + 2] + 1);
  std::fputs("$EndElements\n", f);
  for (int which = 0; which < 2; which++) {
    const std::vector<double> &v = which == 0 ? e : h;
    for (int l = 1; l <= kSteps; l++) {
      std::fprintf(f, "$ElementData\n1\n\"Re(%c)\"\n0\n3\n%d\n3\n%d\n", which == 0 ? 'E' : 'H', l - 1, nf);
      for (int n = 0; n < nf; n++) {
        std::fprintf(f, "%d ", n + 1);
        for (int i = 0; i < 3; i++) std::fputs(en15_3(phase_re(&v[6 * (size_t)n + 2 * i], l)).c_str(), f);
        std::fputs("\n", f);
      }
      std::fputs("$EndElementData\n", f);
    }
  }
  for (int which = 0; which < 2; which++) {
    const std::vector<double> &v = which == 0 ? e : h;
    for (int l = 1; l <= kSteps; l++) {
      std::fprintf(f, "$ElementData\n1\n\"Re(%cn)\"\n0\n3\n%d\n1\n%d\n", which == 0 ? 'E' : 'H', l - 1, nf);
      for (int n = 0; n < nf; n++) {
        // dotc (linalg.f90:15-21): the real normal against the complex field, no conjugation
        double fn[2] = {0, 0};
        for (int i = 0; i < 3; i++) {
          fn[0] += normals[3 * (size_t)n + i] * v[6 * (size_t)n + 2 * i];
          fn[1] += normals[3 * (size_t)n + i] * v[6 * (size_t)n + 2 * i + 1];
        }
        list_record(f, n + 1, phase_re(fn, l));
      }
      std::fputs("$EndElementData\n", f);
    }
  }
  for (int which = 0; which < 2; which++) {
    const std::vector<double> &v = which == 0 ? e : h;
    for (int l = 1; l <= kSteps; l++) {
      std::fprintf(f, "$ElementData\n1\n\"|Re(%c)|\"\n0\n3\n%d\n1\n%d\n", which == 0 ? 'E' : 'H', l - 1, nf);
      for (int n = 0; n < nf; n++) {
        double m = 0;
        for (int i = 0; i < 3; i++) {
          const double c = phase_re(&v[6 * (size_t)n + 2 * i], l);
          m += c * c;
        }
        list_record(f, n + 1, std::sqrt(m));
      }
      std::fputs("$EndElementData\n", f);
    }
  }
  std::fclose(f);
}

// The nodes (metres) and 0-based face nodes of domain d's submesh.
void domain_mesh(State &s, int d, std::vector<double> &nodes, std::vector<int> &faces) {
  mom_mesh m;
  check(s, mom_problem_domain(s.prob, d, &m), "domain mesh");
  nodes.assign(m.nodes, m.nodes + 3 * (size_t)m.nnodes);
  faces.assign(m.face_nodes, m.face_nodes + 3 * (size_t)m.nfaces);
}

void unit_normal(const double *p1, const double *p2, const double *p3, double *n) {
  const double a[3] = {p2[0] - p1[0], p2[1] - p1[1], p2[2] - p1[2]}, b[3] = {p3[0] - p1[0], p3[1] - p1[1],
                                                                               p3[2] - p1[2]};
  n[0] = a[1] * b[2] - a[2] * b[1];
  n[1] = a[2] * b[0] - a[0] * b[2];
  n[2] = a[0] * b[1] - a[1] * b[0];
  const double l = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
  for (int i = 0; i < 3; i++) n[i] /= l;
}

void field_indices(State &s, const std::vector<std::string> &it, const char *what, int *w, int *k, int *d) {
  *w = int_item(it, 1, what);
  *k = int_item(it, 2, what);
  *d = int_item(it, 3, what);
  if (s.x.empty()) stop(std::string("Error: solve (solv) before computing near fields!"));
  if (*w < 1 || *w > (int)s.wl.size() || *k < 1 || *k > (int)s.src.size() || *d < 1 || *d > (int)s.doms.size())
    stop(std::string("Error: index out of range in ") + what);
}

std::string field_name(const State &s, int w, int k, int d, bool sh = false) {
  return s.name + "-wl" + std::to_string(w) + "-s" + std::to_string(k) + "-d" + std::to_string(d) +
         (sh ? "-sh.msh" : ".msh");
}

// Number of passes of a field command: the fundamental, then the second
// harmonic when solv solved one.
int passes(const State &s) { return s.nlx.empty() ? 1 : 2; }

void nfms_pass(State &s, int w, int k, int d, int sh);

// read_nfms (interface.f90:772-803) -> field_mesh (nfpost.f90:167-262): the
// fields on domain d's boundary, on the domain mesh and its images under the
// symmetry group.
void nfms(State &s, const std::vector<std::string> &it) {
  int w, k, d;
  field_indices(s, it, "nfms", &w, &k, &d);
  std::printf(" Computing near fields on particle mesh.\n");
  for (int sh = 0; sh < passes(s); sh++) nfms_pass(s, w, k, d, sh);
  std::fflush(stdout);
}

// One pass of nfms; the second harmonic's at 2 omega with the SH index
// (read_nfms, interface.f90:794-801).
void nfms_pass(State &s, int w, int k, int d, int sh) {
  const cplx v = dom_ri(s, d, w, sh);
  const double ri[2] = {v.real(), v.imag()};
  std::vector<double> nodes;
  std::vector<int> faces;
  domain_mesh(s, d - 1, nodes, faces);
  const int nn = (int)(nodes.size() / 3), nf = (int)(faces.size() / 3), nga = s.nga;
  std::vector<double> e(6 * (size_t)nf * nga), h(6 * (size_t)nf * nga);
  check(s,
        mom_gpu_surface_fields(s.ctx, d - 1, (sh ? 2.0 : 1.0) * omega_of(s.wl[w - 1]), ri, k - 1,
                               (sh ? s.nlx : s.x)[w - 1].data(), s.n2, e.data(), h.data()),
        "nfms");
  // the image mesh: nodes J p, faces renumbered per element, normals J n
  std::vector<double> n2((size_t)3 * nn * nga), nor((size_t)3 * nf * nga);
  std::vector<int> f2((size_t)3 * nf * nga);
  for (int g = 0; g < nga; g++) {
    double J[9], detj;
    check(s, mom_gpu_group_action(s.ctx, g, J, &detj), "nfms");
    for (int n = 0; n < nn; n++)
      for (int i = 0; i < 3; i++)
        n2[3 * ((size_t)g * nn + n) + i] = J[3 * i] * nodes[3 * (size_t)n] + J[3 * i + 1] * nodes[3 * (size_t)n + 1] +
                                           J[3 * i + 2] * nodes[3 * (size_t)n + 2];
    for (int n = 0; n < nf; n++) {
      double n0[3];
      unit_normal(&nodes[3 * (size_t)faces[3 * n]], &nodes[3 * (size_t)faces[3 * n + 1]],
                  &nodes[3 * (size_t)faces[3 * n + 2]], n0);
      for (int i = 0; i < 3; i++) {
        f2[3 * ((size_t)g * nf + n) + i] = faces[3 * n + i] + g * nn;
        nor[3 * ((size_t)g * nf + n) + i] = J[3 * i] * n0[0] + J[3 * i + 1] * n0[1] + J[3 * i + 2] * n0[2];
      }
    }
  }
  save_vector_fields_msh(field_name(s, w, k, d, sh), n2, f2, nor, e, h, s.scale);
  double emax = 0;
  for (size_t n = 0; n < (size_t)nf * nga; n++) {
    double m = 0;
    for (int i = 0; i < 6; i++) m += e[6 * n + i] * e[6 * n + i];
    emax = std::max(emax, std::sqrt(m));
  }
  std::printf(" Maximum of |E| is %.15E\n", emax);
}

// read_nfem (interface.f90:1010-1090) -> field_external_mesh
// (nfpost.f90:264-314): scat_fields of domain d at the face centroids of an
// external mesh (scaled as the problem mesh), plus the incident field when
// asked.
void nfem(State &s, const std::vector<std::string> &it) {
  int w, k, d;
  field_indices(s, it, "nfem", &w, &k, &d);
  if (it.size() < 6) stop("Error: nfem needs a mesh file and true/false");
  const bool addsrc = it[5] == "true";
  mom_problem *ext = nullptr;
  check(s, mom_problem_create(&ext), "nfem");
  if (mom_problem_load_gmsh(ext, it[4].c_str(), s.scale) != MOM_OK) {
    mom_problem_destroy(ext);
    stop("Error in nfem: could not read mesh " + it[4]);
  }
  std::printf(" Computing near fields on external mesh.\n");
  std::vector<double> nodes, pts, nor;
  std::vector<int> faces;
  {
    mom_mesh m;
    if (mom_problem_domain(ext, -1, &m) != MOM_OK || m.nfaces <= 0) {
      mom_problem_destroy(ext);
      stop("Error in nfem: external mesh without faces");
    }
    nodes.assign(m.nodes, m.nodes + 3 * (size_t)m.nnodes);
    faces.assign(m.face_nodes, m.face_nodes + 3 * (size_t)m.nfaces);
    mom_problem_destroy(ext);
    const int nf = m.nfaces;
    pts.resize(3 * (size_t)nf);
    nor.resize(3 * (size_t)nf);
    for (int n = 0; n < nf; n++) {
      const double *p1 = &nodes[3 * (size_t)faces[3 * n]], *p2 = &nodes[3 * (size_t)faces[3 * n + 1]],
                   *p3 = &nodes[3 * (size_t)faces[3 * n + 2]];
      for (int i = 0; i < 3; i++) pts[3 * (size_t)n + i] = (p1[i] + p2[i] + p3[i]) / 3.0;
      unit_normal(p1, p2, p3, &nor[3 * (size_t)n]);
    }
  }
  const int nf = (int)(faces.size() / 3), nsrc = (int)s.src.size();
  for (int sh = 0; sh < passes(s); sh++) {
    // second harmonic: 2 omega, the SH index, no incident field, and in a
    // nonlinear domain the source coefficients added to nlx
    // (interface.f90:1050-1085)
    const cplx v = dom_ri(s, d, w, sh);
    const double ri[2] = {v.real(), v.imag()};
    std::vector<double> xs = (sh ? s.nlx : s.x)[w - 1];
    if (sh && !s.shc[w - 1][d - 1].empty())
      for (size_t i = 0; i < xs.size(); i++) xs[i] += s.shc[w - 1][d - 1][i];
    std::vector<double> e(6 * (size_t)nf * nsrc), h(6 * (size_t)nf * nsrc);
    check(s,
          mom_gpu_scat_fields(s.ctx, d - 1, (sh ? 2.0 : 1.0) * omega_of(s.wl[w - 1]), ri, nsrc,
                              (addsrc && !sh) ? s.src.data() : nullptr, xs.data(), s.n2, nf, pts.data(), e.data(),
                              h.data()),
          "nfem");
    std::vector<double> ek(e.begin() + 6 * (size_t)nf * (k - 1), e.begin() + 6 * (size_t)nf * k),
        hk(h.begin() + 6 * (size_t)nf * (k - 1), h.begin() + 6 * (size_t)nf * k);
    save_vector_fields_msh(field_name(s, w, k, d, sh), nodes, faces, nor, ek, hk, s.scale);
  }
  std::fflush(stdout);
}

void nfdm_pass(State &s, int w, int k, int d, int sh, bool addsrc, const std::vector<double> &pts);

// read_nfdm (interface.f90:1092-1139) -> field_domain (nfpost.f90:85-165):
// scat_fields of domain d on a regular grid of npoints(1:3) points over the
// box origin +- dsize/2 (fractions (n-1)/(np-1) in default-kind reals), plus
// the incident field when asked; the points where |E| exceeds 1% of its
// maximum are written with the domain mesh (save_domain_vector_fields_msh,
// mesh.f90:1890-1978).
void nfdm(State &s, const std::vector<std::string> &it) {
  int w, k, d;
  field_indices(s, it, "nfdm", &w, &k, &d);
  if (it.size() < 14) stop("Error: nfdm needs true/false, an origin, a size and three point counts");
  const bool addsrc = it[4] == "true";
  double org[3], dsz[3];
  int np[3];
  for (int i = 0; i < 3; i++) {
    org[i] = real_item(it, 5 + i, "nfdm");
    dsz[i] = real_item(it, 8 + i, "nfdm");
    np[i] = int_item(it, 11 + i, "nfdm");
    if (np[i] < 2) stop("Error: nfdm needs at least 2 points per axis");
  }
  const int npts = np[0] * np[1] * np[2];
  std::vector<double> pts(3 * (size_t)npts);
  for (int a = 0; a < np[0]; a++)
    for (int b = 0; b < np[1]; b++)
      for (int c = 0; c < np[2]; c++) {
        const size_t idx = (size_t)c + (size_t)b * np[2] + (size_t)a * np[2] * np[1];
        const float fr[3] = {(float)a / (float)(np[0] - 1), (float)b / (float)(np[1] - 1),
                             (float)c / (float)(np[2] - 1)};
        for (int i = 0; i < 3; i++) pts[3 * idx + i] = org[i] - dsz[i] / 2 + dsz[i] * (double)fr[i];
      }
  for (int sh = 0; sh < passes(s); sh++)
    nfdm_pass(s, w, k, d, sh, addsrc && !sh, pts);
  std::fflush(stdout);
}

// One pass of nfdm; the second harmonic's at 2 omega with the SH index and
// no incident field (interface.f90:1126-1137).
void nfdm_pass(State &s, int w, int k, int d, int sh, bool addsrc, const std::vector<double> &pts) {
  const int npts = (int)(pts.size() / 3), nsrc = (int)s.src.size();
  const cplx v = dom_ri(s, d, w, sh);
  const double ri[2] = {v.real(), v.imag()};
  std::vector<double> e(6 * (size_t)npts * nsrc), h(6 * (size_t)npts * nsrc);
  check(s,
        mom_gpu_scat_fields(s.ctx, d - 1, (sh ? 2.0 : 1.0) * omega_of(s.wl[w - 1]), ri, nsrc,
                            addsrc ? s.src.data() : nullptr, (sh ? s.nlx : s.x)[w - 1].data(), s.n2, npts, pts.data(),
                            e.data(), h.data()),
        "nfdm");
  const double *ek = &e[6 * (size_t)npts * (k - 1)], *hk = &h[6 * (size_t)npts * (k - 1)];
  auto mag = [&](size_t n) {
    double m = 0;
    for (int i = 0; i < 6; i++) m += ek[6 * n + i] * ek[6 * n + i];
    return std::sqrt(m);
  };
  double emax = 0;
  for (size_t n = 0; n < (size_t)npts; n++) emax = std::max(emax, mag(n));
  std::vector<size_t> keep;
  for (size_t n = 0; n < (size_t)npts; n++)
    if (mag(n) > emax * 0.01) keep.push_back(n);
  std::vector<double> nodes;
  std::vector<int> faces;
  domain_mesh(s, d - 1, nodes, faces);
  const int nn = (int)(nodes.size() / 3), nf = (int)(faces.size() / 3), m = (int)keep.size();
  const std::string path = field_name(s, w, k, d, sh);
  std::FILE *f = std::fopen(path.c_str(), "w");
  if (!f) stop("Could not open output file" + path + "!");
  msh_header(f);
  std::fprintf(f, "$Nodes\n%d\n", nn + m);
  for (int n = 0; n < nn; n++) msh_node(f, n + 1, &nodes[3 * (size_t)n], s.scale);
  for (int n = 0; n < m; n++) msh_node(f, nn + n + 1, &pts[3 * keep[n]], s.scale);
  std::fprintf(f, "$EndNodes\n$Elements\n%d\n", nf + m);
  for (int n = 0; n < nf; n++)
    std::fprintf(f, "%d 2 3 0 0 0 %d %d %d\n", n + 1, faces[3 * n] + 1, faces[3 * n + 1] + 1, faces[3 * n + 2] + 1);
  for (int n = 0; n < m; n++) std::fprintf(f, "%d 15 3 0 0 0 %d\n", nf + n + 1, nn + n + 1);
  std::fputs("$EndElements\n", f);
  for (int which = 0; which < 2; which++) {
    const double *val = which == 0 ? ek : hk;
    for (int l = 1; l <= kSteps; l++) {
      std::fprintf(f, "$NodeData\n1\n\"Re(%c)\"\n0\n3\n%d\n3\n%d\n", which == 0 ? 'E' : 'H', l - 1, m);
      for (int n = 0; n < m; n++) {
        std::fprintf(f, "%d ", nn + n + 1);
        for (int i = 0; i < 3; i++) std::fputs(en15_3(phase_re(&val[6 * keep[n] + 2 * i], l)).c_str(), f);
        std::fputs("\n", f);
      }
      std::fputs("$EndNodeData\n", f);
    }
  }
  std::fclose(f);
}

void command(State &s, const std::string &cmd, const std::vector<std::string> &it) {
  if (cmd == "name") {
    if (it.size() < 2) stop("Error: name needs a value");
    s.name = it[1];
  } else if (cmd == "mesh") {
    // read_mesh (interface.f90:357-366)
    if (it.size() < 3) stop("Error: mesh needs a file and a scale");
    const double scale = real_item(it, 2, "mesh");
    if (s.prob) mom_problem_destroy(s.prob);
    s.prob = nullptr;
    check(s, mom_problem_create(&s.prob), "mesh");
    check(s, mom_problem_load_gmsh(s.prob, it[1].c_str(), scale), ("mesh " + it[1]).c_str());
    s.scale = scale;
    s.finalized = s.uploaded = false;
    s.doms.clear();
  } else if (cmd == "wlrg") {
    // read_wlrange (interface.f90:368-389)
    const int n = int_item(it, 1, "wlrg");
    const double a = real_item(it, 2, "wlrg"), b = real_item(it, 3, "wlrg");
    if (n < 1) stop("Error: wlrg needs at least one wavelength");
    s.wl.assign(n, a);
    for (int i = 0; n > 1 && i < n; i++) s.wl[i] = a + (b - a) * ((double)i / (double)(n - 1));
    clear_solutions(s);
  } else if (cmd == "wlls") {
    // read_wllist (interface.f90:391-406)
    const int n = int_item(it, 1, "wlls");
    if (n < 1) stop("Error: wlls needs at least one wavelength");
    s.wl.resize(n);
    for (int i = 0; i < n; i++) s.wl[i] = real_item(it, 2 + i, "wlls");
    clear_solutions(s);
  } else if (cmd == "symm") {
    // read_symm (interface.f90:160-210): products of id and the mirror
    // groups mxp, myp, mzp (the rotation groups rN are not supported)
    const int n = int_item(it, 1, "symm");
    std::vector<std::string> names;
    int order = 1;
    for (int i = 0; i < n; i++) {
      if (2 + i >= (int)it.size()) stop("Error: symm lists fewer groups than announced");
      const std::string &g = it[2 + i];
      if (g == "mxp" || g == "myp" || g == "mzp") {
        order *= 2;
      } else if (!g.empty() && g[0] == 'r') {
        stop("Error: rotation symmetry group '" + g + "' is not supported by this build (id, mxp, myp, mzp)");
      } else if (g != "id") {
        std::printf(" Error: unrecognized group!\n");
        return;
      }
      names.push_back(g);
    }
    if (order > MOM_MAX_GROUP) stop("Error: symmetry group too large");
    s.symm = order > 1 ? names : std::vector<std::string>();
    s.uploaded = false;
    clear_solutions(s);
    std::printf(" Created a symmetry group with %d elements.\n", order);
  } else if (cmd == "sbnd") {
    // read_sbnd (interface.f90:125-157) -> classify_edges (mesh.f90:155-175)
    if (!s.prob) stop("Error: master mesh has not been loaded!");
    const int id = int_item(it, 1, "sbnd");
    if (it.size() < 3) stop("Error: sbnd needs an id and a boundary type");
    const std::string &bn = it[2];
    int bnd = 0;
    if (bn == "xplane") bnd = MOM_BND_XPLANE;
    else if (bn == "yplane") bnd = MOM_BND_YPLANE;
    else if (bn == "zplane") bnd = MOM_BND_ZPLANE;
    else if (bn == "prdx1" || bn == "prdx2" || bn == "prdy1" || bn == "prdy2" || bn == "rz1" || bn == "rz2")
      stop("Error: boundary type '" + bn + "' is not supported by this build (xplane, yplane, zplane)");
    else
      stop("Unrecognized boundary type!");
    int32_t cnt = 0;
    check(s, mom_problem_classify_edges(s.prob, id, bnd, &cnt), "sbnd");
    s.uploaded = false;
    std::printf(" Classified %d boundary edges\n", cnt);
  } else if (cmd == "nmed") {
    // read_nmed (interface.f90:213-232)
    if (s.wl.empty()) {
      std::printf(" Error: no wavelengths set up!\n");
      return;
    }
    const int n = int_item(it, 1, "nmed");
    s.media.assign(n, std::vector<cplx>(s.wl.size(), cplx(1.0, 0.0)));
    s.media_sh = s.media;
    s.nls.assign(n, mom_nls{0, {0, 0}, {0, 0}, {0, 0}});
    clear_solutions(s);
    std::printf(" Allocated %d media.\n", n);
  } else if (cmd == "smed") {
    // read_smed (interface.f90:234-355): linear media (refractive indices at
    // the wavelength and at half of it) and surface nonlinearities
    if (s.media.empty()) {
      std::printf(" Error: no media allocated!\n");
      return;
    }
    const int m = int_item(it, 1, "smed");
    if (m < 1 || m > (int)s.media.size()) stop("Error: medium index out of range in smed");
    if (it.size() < 4) stop("Error: smed needs a type, a method and a value");
    if (it[2] != "linear" && it[2] != "nlsurf") {
      if (it[2] == "nlbulk-nonlocal" || it[2] == "nlbulk-dipole")
        stop("Error: medium type '" + it[2] + "' is not supported by this build (linear, nlsurf)");
      std::printf(" Unrecognized material type!\n");
      return;
    }
    s.nls[m - 1].active = 0;  // every smed first makes the medium linear
    clear_solutions(s);
    if (it[2] == "nlsurf") {
      if (it[3] != "value") {
        std::printf(" Unrecongnized method for retrieveing medium properties!\n");
        return;
      }
      const cplx a = complex_item(it, 4, "smed"), b = complex_item(it, 5, "smed"), c = complex_item(it, 6, "smed");
      s.nls[m - 1] = mom_nls{1, {a.real(), a.imag()}, {b.real(), b.imag()}, {c.real(), c.imag()}};
    } else if (it[3] == "value") {
      const cplx v = complex_item(it, 4, "smed");
      for (auto &r : s.media[m - 1]) r = v;
      for (auto &r : s.media_sh[m - 1]) r = v;
      std::printf("Set medium %d refractive index to (%6.3f,%6.3f)\n", m, v.real(), v.imag());
    } else if (it[3] == "file") {
      if (it.size() < 5) stop("Error: smed file needs a file name");
      for (size_t n = 0; n < s.wl.size(); n++) {
        s.media[m - 1][n] = refind_from_file(it[4], s.wl[n]);
        s.media_sh[m - 1][n] = refind_from_file(it[4], s.wl[n] * 0.5);
      }
      std::printf("Set medium %d refractive index to %s\n", m, it[4].c_str());
    } else {
      std::printf(" Unrecongnized method for retrieveing medium properties!\n");
    }
  } else if (cmd == "ndom") {
    // read_ndom (interface.f90:32-42)
    if (!s.prob) stop("Error: master mesh has not been loaded!");
    const int n = int_item(it, 1, "ndom");
    if (n < 1) stop("Error: ndom needs at least one domain");
    check(s, mom_problem_set_ndom(s.prob, n), "ndom");
    s.doms.assign(n, Domain());
    s.finalized = s.uploaded = false;
    std::printf(" Allocated %d domains.\n", n);
  } else if (cmd == "sdom") {
    // read_sdom (interface.f90:44-105): dom nsurf ids... nvol [vol ids] medium gf
    if (s.doms.empty()) stop("Error: no domains allocated!");
    if (!s.prob) stop("Error: master mesh has not been loaded!");
    const int d = int_item(it, 1, "sdom"), ns = int_item(it, 2, "sdom");
    if (d < 1 || d > (int)s.doms.size() || ns < 1) stop("Error: domain index or surface count out of range in sdom");
    std::vector<int32_t> ids(ns);
    for (int i = 0; i < ns; i++) {
      ids[i] = int_item(it, 3 + i, "sdom");
      if (ids[i] == 0) stop("Zero is not a valid surface id!");
    }
    const int nvol = int_item(it, 3 + ns, "sdom");
    if (nvol != 0) stop("Error: volume domains (nvol > 0) are not supported by this build");
    const int medium = int_item(it, 4 + ns, "sdom"), gf = int_item(it, 5 + ns, "sdom");
    if (gf != -1) stop("Error: periodic Green's functions (gf != -1) are not supported by this build");
    check(s, mom_problem_set_domain(s.prob, d - 1, ns, ids.data()), "sdom");
    s.doms[d - 1].set = true;
    s.doms[d - 1].medium = medium;
    s.finalized = s.uploaded = false;
  } else if (cmd == "fdom") {
    // read_fdom (interface.f90:107-123)
    if (!s.prob) stop("Error: master mesh has not been loaded!");
    for (size_t d = 0; d < s.doms.size(); d++)
      if (!s.doms[d].set) stop("Error: domain " + std::to_string(d + 1) + " has not been set up (sdom)");
    check(s, mom_problem_finalize(s.prob), "fdom");
    s.finalized = true;
    s.uploaded = false;
  } else if (cmd == "nsrc") {
    // read_nsrc (interface.f90:460-470)
    const int n = int_item(it, 1, "nsrc");
    if (n < 1) stop("Error: nsrc needs at least one source");
    s.src.assign(n, mom_src());
    s.src_set.assign(n, false);
    clear_solutions(s);
    std::printf(" Allocated %d sources.\n", n);
  } else if (cmd == "ssrc") {
    // read_ssrc (interface.f90:486-550): plane waves only
    if (s.src.empty()) stop("No sources allocated!");
    const int k = int_item(it, 1, "ssrc");
    if (k < 1 || k > (int)s.src.size()) stop("Error: source index out of range in ssrc");
    if (it.size() < 3) stop("Error: ssrc needs a source type");
    mom_src &src = s.src[k - 1];
    src = mom_src();
    if (it[2] == "pw") {
      src.type = MOM_SRC_PW;
      src.theta = real_item(it, 3, "ssrc") * kDegToRad;
      src.phi = real_item(it, 4, "ssrc") * kDegToRad;
      src.psi = real_item(it, 5, "ssrc") * kDegToRad;
    } else if (it[2] == "pw_elliptic") {
      src.type = MOM_SRC_PW_ELLIPTIC;
      src.theta = real_item(it, 3, "ssrc") * kDegToRad;
      src.phi = real_item(it, 4, "ssrc") * kDegToRad;
      const cplx ph = complex_item(it, 5, "ssrc");
      src.phase_re = ph.real();
      src.phase_im = ph.imag();
    } else {
      stop("Error: source type '" + it[2] + "' is not supported by this build (pw, pw_elliptic)");
    }
    s.src_set[k - 1] = true;
    clear_solutions(s);
  } else if (cmd == "quad") {
    // read_quad (interface.f90:18-30): the triangle rule; the tetrahedron rule
    // belongs to the volume solver
    if (it.size() < 2) stop("Error: quad needs a triangle rule name");
    double w[13], q[39];
    if (mom_tri_rule(it[1].c_str(), w, q) < 0) stop("Error: unknown triangle quadrature '" + it[1] + "'");
    s.quad = it[1];
    s.uploaded = false;
  } else if (cmd == "prec") {
    if (it.size() < 2) stop("Error: prec needs fp64 or mixed");
    if (it[1] == "fp64") s.precision = MOM_PREC_FP64;
    else if (it[1] == "mixed") s.precision = MOM_PREC_MIXED;
    else stop("Error: prec takes fp64 or mixed");
    if (it.size() > 2) s.tol = real_item(it, 2, "prec");
    if (it.size() > 3) s.maxit = int_item(it, 3, "prec");
  } else if (cmd == "dev") {
    if (s.ctx) stop("Error: dev must come before the first solv");
    s.device = int_item(it, 1, "dev");
  } else if (cmd == "solv") {
    solve_batch(s);
  } else if (cmd == "crst") {
    crst(s, it);
  } else if (cmd == "rcst") {
    rcst(s, it);
  } else if (cmd == "nfpl") {
    nfpl(s, it);
  } else if (cmd == "nfms") {
    nfms(s, it);
  } else if (cmd == "nfem") {
    nfem(s, it);
  } else if (cmd == "nfdm") {
    nfdm(s, it);
  } else if (cmd == "osrc" || cmd == "npgf" || cmd == "ipgw" || cmd == "nfst" || cmd == "rcs2" || cmd == "rcs3" ||
             cmd == "diff" ||
             cmd == "plrz" || cmd == "scan" || cmd == "trns" || cmd == "csca" || cmd == "test" || cmd == "vsol" ||
             cmd == "vext" || cmd == "viem" || cmd == "msrc") {
    stop("Error: command " + cmd + " is outside the linear PMCHWT path that this build implements");
  } else {
    std::printf(" Unrecognized command %s!\n", cmd.c_str());
  }
}

}  // namespace

int main() {
  State s;
  if (const char *ed = std::getenv("MOM_DEVICE")) s.device = std::atoi(ed);
  std::string line;
  while (true) {
    std::printf("> ");
    std::fflush(stdout);
    if (!std::getline(std::cin, line)) break;
    const std::vector<std::string> it = items(line);
    if (it.empty()) continue;
    if (it[0] == "exit") break;
    command(s, it[0], it);
  }
  std::printf("\n");
  if (s.ctx) mom_gpu_destroy(s.ctx);
  if (s.prob) mom_problem_destroy(s.prob);
  return 0;
}
