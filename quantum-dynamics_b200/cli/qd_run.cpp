// qd_run -- command-line driver of the propagator: reads a plain run file,
// builds the struct that the reference's Matlab drivers build (*/main.m:
// grids, Gauss-Legendre quadrature from GaussLegendre/<n>-LegendreGauss.grids,
// Legendre matrix, potential on the Jacobi grid, absorbers, initial packet,
// eta^2 and dividing surface), and calls qd_time_evolution, the drop-in for
// the MEX entry point (common/TimeEvolutionMex.C:18-78).  The set-up runs on
// the GPU through the library's own entry points; P(E) goes to a CSV file.
//
//   qd_run RUNFILE [--check]        --check: parse and print the resolved
//                                   run as JSON, touch no device
//
// Run file: one `key = value` per line, `#` starts a comment; the keys of
// the struct fields keep the reference's names (common/MatlabStructures.h:
// 12-157: r1.n, theta.m, time.total_steps, CRP.n_gradient_points, ...).
// Keys and defaults (F + H2 on the extended-LEPS surface, as main.m sets up):
//   r1.n 64, r1.min 0.5, r1.max 12 (bohr)     R grid, linspace
//   r2.n 64, r2.min 0.4, r2.max 8             r grid
//   theta.n 40, theta.m theta.n-1             quadrature points, highest order
//   grids DIR                                 read <DIR>/<n>-LegendreGauss.grids
//                                             (default: nodes computed here)
//   masses 18.9984 1.00783 1.00783 (amu)      atom 1, then the diatom 2 3
//   r1.r0 8, r1.delta 0.3, e0 0.5 (eV)        Gaussian packet in R, mean energy
//   v0 0, j0 0                                initial diatom state
//   cs.J 0, cs.K 0                            centrifugal-sudden block
//   pes leps|bkmp2|hsw                        surface (hsw: hsw.dir DIR)
//   leps.ab|bc|ac  De(eV) beta(1/A) re(A) sato   extended-LEPS pairs
//   vmax 2.5 (hartree), rmin 0.4 (bohr)       cap and mask of H3PESJacobi.m:13-27
//   time.total_steps 2000, time.time_step 10, time.steps 0
//   dump.length 2, dump.strength 0.3          quadratic absorbers over the last
//                                             `length` bohr of R and of r
//   CRP.calculate_CRP 1, CRP.r_surface 4.5 (or CRP.n_dividing_surface, 1-based),
//   CRP.n_gradient_points 11, CRP.e_min 0.3, CRP.e_max 1.5 (eV), CRP.n_energies 241
//   options.precision fp64|fp32, options.steps_to_copy_psi_from_device_to_host 0,
//   options.test_name
//   output.crp FILE (default crp.csv), output.psi FILE (raw complex128, optional)
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>
#include "qd.h"

namespace {

constexpr double HARTREE_EV = 27.211386245988;
constexpr double AMU_ME = 1822.888486209;
constexpr double BOHR_PER_ANGSTROM = 1.0 / 0.529177210903;

struct RunFile {
  std::map<std::string, std::string> kv;
  std::map<std::string, bool> used;

  bool has(const std::string &k) const { return kv.count(k) != 0; }
  std::string str(const std::string &k, const std::string &def)
  {
    used[k] = true;
    auto it = kv.find(k);
    return it == kv.end() ? def : it->second;
  }
  double num(const std::string &k, double def)
  {
    const std::string v = str(k, "");
    if (v.empty()) return def;
    char *end = nullptr;
    errno = 0;
    const double x = strtod(v.c_str(), &end);
    if (errno || !end || *end) {
      fprintf(stderr, "qd_run: %s = \"%s\" is not a number\n", k.c_str(), v.c_str());
      exit(2);
    }
    return x;
  }
  int integer(const std::string &k, int def)
  {
    const double x = num(k, def);
    if (x != std::floor(x) || std::fabs(x) > 2e9) {
      fprintf(stderr, "qd_run: %s must be an integer\n", k.c_str());
      exit(2);
    }
    return (int)x;
  }
  std::vector<double> nums(const std::string &k, const std::vector<double> &def)
  {
    const std::string v = str(k, "");
    if (v.empty()) return def;
    std::vector<double> out;
    std::istringstream is(v);
    double x;
    while (is >> x) out.push_back(x);
    if (!is.eof() || out.size() != def.size()) {
      fprintf(stderr, "qd_run: %s needs %zu numbers\n", k.c_str(), def.size());
      exit(2);
    }
    return out;
  }
};

RunFile parse(const char *path)
{
  std::ifstream f(path);
  if (!f) {
    fprintf(stderr, "qd_run: cannot read %s\n", path);
    exit(2);
  }
  RunFile rf;
  std::string line;
  int ln = 0;
  while (std::getline(f, line)) {
    ln++;
    const size_t h = line.find('#');
    if (h != std::string::npos) line.resize(h);
    const size_t b = line.find_first_not_of(" \t\r");
    if (b == std::string::npos) continue;
    const size_t eq = line.find('=');
    if (eq == std::string::npos) {
      fprintf(stderr, "qd_run: %s:%d: expected key = value\n", path, ln);
      exit(2);
    }
    auto trim = [](std::string s) {
      const size_t a = s.find_first_not_of(" \t\r"), z = s.find_last_not_of(" \t\r");
      return a == std::string::npos ? std::string() : s.substr(a, z - a + 1);
    };
    const std::string k = trim(line.substr(0, eq)), v = trim(line.substr(eq + 1));
    if (k.empty()) {
      fprintf(stderr, "qd_run: %s:%d: empty key\n", path, ln);
      exit(2);
    }
    if (rf.kv.count(k)) {
      fprintf(stderr, "qd_run: %s:%d: %s given twice\n", path, ln, k.c_str());
      exit(2);
    }
    rf.kv[k] = v;
  }
  return rf;
}

// Gauss-Legendre nodes (ascending) and weights by Newton iteration on P_n
void gauss_legendre(int n, std::vector<double> &x, std::vector<double> &w)
{
  x.assign(n, 0.0);
  w.assign(n, 0.0);
  for (int i = 0; i < n; i++) {
    double z = std::cos(M_PI * (4 * (i + 1) - 1) / (4.0 * n + 2)) * (1 - (n - 1) / (8.0 * n * n * n));
    double dp = 1.0;
    for (int it = 0; it < 100; it++) {
      double p0 = 1.0, p1 = z;
      for (int k = 2; k <= n; k++) {
        const double p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      if (n == 1) { p1 = z; p0 = 1.0; }
      dp = n > 1 ? n * (z * p1 - p0) / (z * z - 1.0) : 1.0;
      const double dz = p1 / dp;
      z -= dz;
      if (std::fabs(dz) < 1e-17) break;
    }
    double p0 = 1.0, p1 = z;
    for (int k = 2; k <= n; k++) {
      const double p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k;
      p0 = p1;
      p1 = p2;
    }
    if (n == 1) { p1 = z; p0 = 1.0; }
    dp = n > 1 ? n * (z * p1 - p0) / (z * z - 1.0) : 1.0;
    x[n - 1 - i] = z;
    w[n - 1 - i] = 2.0 / ((1.0 - z * z) * dp * dp);
  }
  if (n % 2 == 1) x[n / 2] = 0.0;
}

std::vector<double> linspace(double a, double b, int n)
{
  std::vector<double> v(n);
  for (int i = 0; i < n; i++) v[i] = n > 1 ? a + (b - a) * i / (n - 1) : a;
  return v;
}

std::vector<double> quadratic_absorber(const std::vector<double> &x, double len, double strength)
{
  const double x0 = x.back() - len;
  std::vector<double> d(x.size());
  for (size_t i = 0; i < x.size(); i++) {
    const double u = std::max(0.0, (x[i] - x0) / (x.back() - x0));
    d[i] = std::exp(-strength * u * u);
  }
  return d;
}

qd_leps_pair leps_pair(const std::vector<double> &v)
{
  return {v[0] / HARTREE_EV, v[1] / BOHR_PER_ANGSTROM, v[2] * BOHR_PER_ANGSTROM, v[3]};
}

int check(int rc, const char *what)
{
  if (rc != QD_OK) {
    fprintf(stderr, "qd_run: %s failed (%d): %s\n", what, rc, qd_last_error());
    exit(1);
  }
  return rc;
}

int progress(int32_t step, double norm, const double *, void *)
{
  printf("step %d norm %.15f\n", step, norm);
  fflush(stdout);
  return 0;
}

}  // namespace

int main(int argc, char **argv)
{
  if (argc < 2 || argc > 3 || (argc == 3 && strcmp(argv[2], "--check"))) {
    fprintf(stderr, "usage: qd_run RUNFILE [--check]\n");
    return 2;
  }
  const bool check_only = argc == 3;
  RunFile rf = parse(argv[1]);

  // ---- grids and masses --------------------------------------------------------
  const int n1 = rf.integer("r1.n", 64), n2 = rf.integer("r2.n", 64);
  const std::vector<double> R = linspace(rf.num("r1.min", 0.5), rf.num("r1.max", 12.0), n1);
  const std::vector<double> r = linspace(rf.num("r2.min", 0.4), rf.num("r2.max", 8.0), n2);
  const int nth = rf.integer("theta.n", 40), m = rf.integer("theta.m", nth - 1);
  const std::vector<double> amu = rf.nums("masses", {18.9984, 1.00783, 1.00783});
  const double masses[3] = {amu[0] * AMU_ME, amu[1] * AMU_ME, amu[2] * AMU_ME};
  const double mu_R = masses[0] * (masses[1] + masses[2]) / (masses[0] + masses[1] + masses[2]);
  const double mu_r = masses[1] * masses[2] / (masses[1] + masses[2]);
  const double e0 = rf.num("e0", 0.5) / HARTREE_EV;
  qd_radial r1{n1, R.data(), R[1] - R[0], mu_R, rf.num("r1.r0", 8.0), std::sqrt(2 * mu_R * e0),
               rf.num("r1.delta", 0.3)};
  qd_radial r2{n2, r.data(), r[1] - r[0], mu_r, 0.0, 0.0, 0.0};
  const int v0 = rf.integer("v0", 0), j0 = rf.integer("j0", 0);
  const int J = rf.integer("cs.J", 0), K = rf.integer("cs.K", 0);
  const std::string pes = rf.str("pes", "leps"), grids = rf.str("grids", "");
  const double vmax = rf.num("vmax", 2.5), rmin = rf.num("rmin", 0.4);
  qd_leps leps{leps_pair(rf.nums("leps.ab", {6.12, 2.2187, 0.9170, 0.167})),
               leps_pair(rf.nums("leps.bc", {4.7466, 1.9425, 0.7416, 0.106})),
               leps_pair(rf.nums("leps.ac", {6.12, 2.2187, 0.9170, 0.167}))};
  const std::string hsw_dir = rf.str("hsw.dir", "");

  qd_time tm{rf.integer("time.total_steps", 2000), rf.num("time.time_step", 10.0),
             rf.integer("time.steps", 0)};
  const double dlen = rf.num("dump.length", 2.0), dstr = rf.num("dump.strength", 0.3);
  const int do_crp = rf.integer("CRP.calculate_CRP", 1);
  const int npts = rf.integer("CRP.n_gradient_points", 11);
  const int ne = rf.integer("CRP.n_energies", 241);
  const double emin = rf.num("CRP.e_min", 0.3), emax = rf.num("CRP.e_max", 1.5);
  int n_div;
  if (rf.has("CRP.n_dividing_surface")) {
    n_div = rf.integer("CRP.n_dividing_surface", 0);
  } else {   // the Matlab driver's int32((r_surface - r(1)) / dr), rounded half away from zero
    const double u = (rf.num("CRP.r_surface", 4.5) - r[0]) / r2.dr;
    n_div = (int)std::floor(std::fabs(u) + 0.5) * (u < 0 ? -1 : 1);
  }
  const std::string prec_s = rf.str("options.precision", "fp64");
  if (prec_s != "fp64" && prec_s != "fp32") {
    fprintf(stderr, "qd_run: options.precision must be fp64 or fp32\n");
    return 2;
  }
  const int every = rf.integer("options.steps_to_copy_psi_from_device_to_host", 0);
  const std::string test_name = rf.str("options.test_name", argv[1]);
  const std::string out_crp = rf.str("output.crp", "crp.csv"), out_psi = rf.str("output.psi", "");
  for (const auto &kv : rf.kv)
    if (!rf.used.count(kv.first)) {
      fprintf(stderr, "qd_run: unknown key %s\n", kv.first.c_str());
      return 2;
    }
  if (n1 < 2 || n2 < 2 || nth < 1 || m < 0 || ne < 1 || K < 0 || J < K || v0 < 0 || j0 < 0) {
    fprintf(stderr, "qd_run: grid sizes, orders, energies or (J, K, v0, j0) out of range\n");
    return 2;
  }
  if (check_only) {
    printf("{\"r1\": {\"n\": %d, \"min\": %.17g, \"max\": %.17g, \"dr\": %.17g, \"mass\": %.17g, "
           "\"r0\": %.17g, \"k0\": %.17g, \"delta\": %.17g}, "
           "\"r2\": {\"n\": %d, \"min\": %.17g, \"max\": %.17g, \"dr\": %.17g, \"mass\": %.17g}, "
           "\"theta\": {\"n\": %d, \"m\": %d, \"grids\": \"%s\"}, \"pes\": \"%s\", "
           "\"time\": {\"total_steps\": %d, \"time_step\": %.17g, \"steps\": %d}, "
           "\"CRP\": {\"calculate_CRP\": %d, \"n_dividing_surface\": %d, "
           "\"n_gradient_points\": %d, \"n_energies\": %d, \"e_min\": %.17g, \"e_max\": %.17g}, "
           "\"cs\": {\"J\": %d, \"K\": %d}, \"v0\": %d, \"j0\": %d, \"precision\": \"%s\", "
           "\"steps_to_copy_psi_from_device_to_host\": %d}\n",
           n1, R[0], R.back(), r1.dr, r1.mass, r1.r0, r1.k0, r1.delta, n2, r[0], r.back(), r2.dr,
           r2.mass, nth, m, grids.c_str(), pes.c_str(), tm.total_steps, tm.time_step, tm.steps,
           do_crp, n_div, npts, ne, emin, emax, J, K, v0, j0, prec_s.c_str(), every);
    return 0;
  }

  // ---- quadrature and angular basis ----------------------------------------------
  std::vector<double> x(nth), w(nth), leg((size_t)nth * (m + 1));
  if (!grids.empty()) check(qd_read_grids(grids.c_str(), nth, x.data(), w.data()), "qd_read_grids");
  else gauss_legendre(nth, x, w);
  if (K == 0) check(qd_legendre_matrix(nth, m, x.data(), leg.data()), "qd_legendre_matrix");
  else check(qd_cs_legendre(nth, K, m, x.data(), leg.data()), "qd_cs_legendre");
  qd_angle th{nth, m, x.data(), w.data(), leg.data()};

  // ---- potential and the asymptotic diatom potential -------------------------------
  std::vector<double> pot((size_t)n1 * n2 * nth), vdi(n2);
  qd_hsw *hsw = nullptr;
  if (pes == "hsw") check(qd_hsw_create(hsw_dir.c_str(), &hsw), "qd_hsw_create");
  auto surface = [&](const qd_radial *Rg, const qd_angle *tg, double cut, int cap, double *out) {
    if (pes == "leps") return qd_potential_leps(Rg, &r2, tg, masses, &leps, vmax, cut, cap, out);
    if (pes == "bkmp2") return qd_potential_bkmp2(Rg, &r2, tg, masses, vmax, cut, cap, out);
    if (pes == "hsw") return qd_potential_hsw(Rg, &r2, tg, masses, hsw, vmax, cut, cap, out);
    fprintf(stderr, "qd_run: pes must be leps, bkmp2 or hsw\n");
    exit(2);
  };
  check(surface(&r1, &th, rmin, 1, pot.data()), "potential");
  if (J != 0 || K != 0)   // centrifugal-sudden term (J(J+1) - 2K^2) / (2 mu_R R^2)
    for (size_t g = 0; g < pot.size(); g++) {
      const double Ri = R[g % n1];
      pot[g] += (J * (J + 1.0) - 2.0 * K * K) / (2 * mu_R * Ri * Ri);
    }
  {   // the diatom with the atom 100 bohr away: one R, one angle, no mask or cap
    const double Rfar = 100.0, xfar = 0.0, wfar = 2.0, lfar = 1.0;
    qd_radial rf1{1, &Rfar, 1.0, mu_R, 0, 0, 0};
    qd_angle tf{1, 0, &xfar, &wfar, &lfar};
    check(surface(&rf1, &tf, -1.0, 0, vdi.data()), "diatom potential");
  }
  if (hsw) qd_hsw_destroy(hsw);

  // ---- initial packet, energies, eta^2, absorbers ------------------------------------
  std::vector<double> psi(2 * pot.size()), e_coll(ne), energies(ne), eta(ne), crp(ne, 0.0);
  double e_vj = 0.0;
  check(qd_init_state(&r1, &r2, &th, j0, v0, K, vdi.data(), psi.data(), &e_vj, nullptr),
        "qd_init_state");
  for (int e = 0; e < ne; e++) {
    e_coll[e] = (ne > 1 ? emin + (emax - emin) * e / (ne - 1) : emin) / HARTREE_EV;
    energies[e] = e_coll[e] + e_vj;
  }
  check(qd_eta_sq(&r1, ne, e_coll.data(), eta.data()), "qd_eta_sq");
  const std::vector<double> d1 = quadratic_absorber(R, dlen, dstr);
  const std::vector<double> d2 = quadratic_absorber(r, dlen, dstr);

  qd_data d{};
  d.r1 = r1;
  d.r2 = r2;
  d.theta = th;
  d.pot = pot.data();
  d.psi = psi.data();
  d.time = tm;
  d.options.test_name = test_name.c_str();
  d.options.steps_to_copy_psi_from_device_to_host = every;
  d.options.precision = prec_s == "fp32" ? QD_PREC_FP32 : QD_PREC_FP64;
  d.options.progress = every > 0 ? progress : nullptr;
  if (dlen > 0) {
    d.dump1.dump = d1.data();
    d.dump2.dump = d2.data();
  }
  d.CRP.n_dividing_surface = n_div;
  d.CRP.n_gradient_points = npts;
  d.CRP.n_energies = ne;
  d.CRP.calculate_CRP = do_crp;
  d.CRP.energies = energies.data();
  d.CRP.eta_sq = eta.data();
  d.CRP.CRP = crp.data();
  d.cs.J = J;
  d.cs.K = K;
  printf("qd_run: %s, %d x %d x %d grid, n_l = %d, %s, %d steps, E(v=%d, j=%d) = %.12f hartree\n",
         test_name.c_str(), n1, n2, nth, m + 1, prec_s.c_str(), tm.total_steps, v0, j0, e_vj);
  fflush(stdout);
  check(qd_time_evolution(&d), "qd_time_evolution");
  printf("qd_run: %d steps done\n", d.time.steps);

  if (do_crp) {
    FILE *f = fopen(out_crp.c_str(), "w");
    if (!f) {
      fprintf(stderr, "qd_run: cannot write %s\n", out_crp.c_str());
      return 1;
    }
    fprintf(f, "e_coll_ev,energy_hartree,eta_sq,P\n");
    for (int e = 0; e < ne; e++)
      fprintf(f, "%.17g,%.17g,%.17g,%.17g\n", e_coll[e] * HARTREE_EV, energies[e], eta[e], crp[e]);
    fclose(f);
  }
  if (!out_psi.empty()) {
    FILE *f = fopen(out_psi.c_str(), "wb");
    if (!f || fwrite(psi.data(), sizeof(double), psi.size(), f) != psi.size()) {
      fprintf(stderr, "qd_run: cannot write %s\n", out_psi.c_str());
      return 1;
    }
    fclose(f);
  }
  return 0;
}
