// qd_hsw.cu -- the HSW surface of F + H2 (the Stark-Werner SW1 fit with the
// Hartke-Stark-Werner spin-orbit correction) evaluated on the GPU in FP64,
// behind the same Jacobi-grid entry point as the other device surfaces.
//
// What the reference computes (FH2/HSW/hswpot.F, sospline.F), restated:
//   SW1 (hswpot.F:133-209): with X_q = q exp(-b_q (q - q0)) for q = x, y, z
//     (x = r(F-H1), y = r(H1-H2), z = r(F-H2)),
//     V = sum_i a_i X_x^ix_i X_y^iy_i X_z^iz_i
//       + sum over the three pairs of an extended-Rydberg term
//         -D (1 + c1 s + c2 s^2 + c3 s^3) exp(-c1 s) + V0,  s = r - re,
//     with the F-H parameters p(1..6) on x and z and H-H p(7..12) on y.
//   Spin-orbit correction (hswpot.F:46-98): in the F + H2 valley (V above a
//     cutoff, r(H-H) small, R large) a tricubic Hermite interpolation of a
//     tabulated correction in the Jacobi coordinates (R, r, gamma in degrees,
//     gamma folded into 0..90), clamped to the table's box; the function
//     values and the derivatives d/dx, d/dy, d/dz, d2/dxdy, d2/dxdz, d2/dydz,
//     d3/dxdydz at the nodes come from one-dimensional clamped cubic splines
//     (sospline.F:53-285: end slopes of the value splines from the 4-point
//     Lagrange derivative, zero end slopes for the cross derivatives,
//     tridiagonal solves without pivoting).
//   V_HSW = V_SW1 + correction + 0.0006, the last a default-real (single
//     precision) constant in hswpot.F:98, added as its float value.
// The data (three.param, two.param, so.input, so.param) are the reference's
// own files, read from a directory (HSW_DATA_DIR in FH2/HSW/HSWMex.C:48-56)
// or passed in as arrays.  The spline tables are built once on the host in
// FP64; each grid point is one thread.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include "qd_err.h"

namespace {

constexpr int HSW_MAXPOW = 16;    // powers X^0 .. X^15
constexpr int HSW_MAXTERM = 512;
constexpr int HSW_MAXNODE = 64;   // per spline axis

struct HswTerm {
  double a;
  int ix, iy, iz, pad;
};

struct HswDev {
  const HswTerm *term;   // three-body terms
  int nterm, npow;
  double b[3], q0[3];    // exponents and reference distances of X_x, X_y, X_z
  double p[12];          // two-body parameters (two.param, in file order)
  // spin-orbit correction
  int nx, ny, nz;
  const double *gx, *gy, *gz;   // node coordinates
  const double *tab;            // [node][8]: F, Fx, Fy, Fxy, Fz, Fxz, Fyz, Fxyz
  double esocut, rsolim, rrsolm, raddeg, shift;
};

__device__ double sw1(const HswDev &h, double x, double y, double z)
{
  double px[HSW_MAXPOW], py[HSW_MAXPOW], pz[HSW_MAXPOW];
  const double fx = x * exp(-(h.b[0] * (x - h.q0[0])));
  const double fy = y * exp(-(h.b[1] * (y - h.q0[1])));
  const double fz = z * exp(-(h.b[2] * (z - h.q0[2])));
  px[0] = py[0] = pz[0] = 1.0;
  px[1] = fx; py[1] = fy; pz[1] = fz;
#pragma unroll
  for (int m = 2; m < HSW_MAXPOW; m++) {
    px[m] = px[m - 1] * fx;
    py[m] = py[m - 1] * fy;
    pz[m] = pz[m - 1] * fz;
  }
  double fit = 0.0;
  for (int i = 0; i < h.nterm; i++) {
    const HswTerm t = h.term[i];
    fit = fit + px[t.ix] * py[t.iy] * pz[t.iz] * t.a;
  }
  const double *p = h.p;
  auto ryd = [](double r, double d, double c1, double re, double c2, double c3, double v0) {
    const double s = r - re, s2 = s * s, s3 = s2 * s;
    const double u = -d * (1.0 + c1 * s + c2 * s2 + c3 * s3);
    return u * exp(-c1 * s) + v0;
  };
  const double xv = ryd(x, p[0], p[1], p[2], p[3], p[4], p[5]);
  const double yv = ryd(y, p[6], p[7], p[8], p[9], p[10], p[11]);
  const double zv = ryd(z, p[0], p[1], p[2], p[3], p[4], p[5]);
  return fit + xv + yv + zv;
}

// cell of coordinate c on nodes g[0..n): the first node above c (from 1),
// else the last one
__device__ inline int cell(const double *g, int n, double c)
{
  for (int s = 1; s < n; s++)
    if (c < g[s]) return s;
  return n > 1 ? n - 1 : 1;
}

// the cubic Hermite weights of one axis: value at the cell's upper and
// lower node, slope at the upper and lower node
__device__ inline void hermite(double t, double hstep, double u[4])
{
  const double t2 = t * t, t3 = t * t2;
  u[0] = -2.0 * t3 + 3.0 * t2;
  u[1] = -u[0] + 1.0;
  u[2] = hstep * (t3 - t2);
  u[3] = hstep * (t3 - 2.0 * t2 + t);
}

__device__ double so_correction(const HswDev &h, double c0, double c1, double c2)
{
  const int is = cell(h.gx, h.nx, c0), js = cell(h.gy, h.ny, c1);
  const int ks = h.nz > 1 ? cell(h.gz, h.nz, c2) : 1;
  const double hx = h.gx[is] - h.gx[is - 1], hy = h.gy[js] - h.gy[js - 1];
  const double hz = h.nz > 1 ? h.gz[ks] - h.gz[ks - 1] : 1e20;
  double u[3][4];
  hermite((c0 - h.gx[is - 1]) / hx, hx, u[0]);
  hermite((c1 - h.gy[js - 1]) / hy, hy, u[1]);
  hermite((c2 - h.gz[ks - 1]) / hz, hz, u[2]);
  double f = 0.0;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const int nk = (k & 1) ? ks - 1 : ks, dk = k >> 1;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int nj = (j & 1) ? js - 1 : js, dj = j >> 1;
      const double ukj = u[2][k] * u[1][j];
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const int ni = (i & 1) ? is - 1 : is, di = i >> 1;
        const long node = ((long)(h.nz > 1 ? nk : 0) * h.ny + nj) * h.nx + ni;
        f = f + h.tab[node * 8 + (di + 2 * dj + 4 * dk)] * ukj * u[0][i];
      }
    }
  }
  return f;
}

// V(r(F-H1), r(H1-H2), r(F-H2)) in hartree
__device__ double hsw_pot(const HswDev &h, double rhf1, double r, double rhf2)
{
  const double v = sw1(h, rhf1, r, rhf2);
  const double rbig = sqrt(0.5 * (rhf1 * rhf1 + rhf2 * rhf2 - 0.5 * r * r));
  double c = (rbig * rbig + 0.25 * r * r - rhf1 * rhf1) / rbig / r;
  if (fabs(c) >= 1.0) c = copysign(1.0, c);
  const double gam = acos(c);
  double so = 0.0;
  if (v > h.esocut && r < h.rsolim && rbig > h.rrsolm) {
    double c0 = rbig, c1 = r, c2 = gam * h.raddeg;
    if (c0 < h.gx[0]) c0 = h.gx[0];
    if (c0 > h.gx[h.nx - 1]) c0 = h.gx[h.nx - 1];
    if (c1 < h.gy[0]) c1 = h.gy[0];
    if (c1 > h.gy[h.ny - 1]) c1 = h.gy[h.ny - 1];
    if (c2 > 90.0) c2 = 180.0 - c2;
    so = so_correction(h, c0, c1, c2);
  }
  return v + so + h.shift;
}

__global__ void __launch_bounds__(256) k_hsw_points(HswDev h, long n, const double *a,
                                                    const double *b, const double *c, double *v)
{
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n;
       q += (long)gridDim.x * blockDim.x)
    v[q] = hsw_pot(h, a[q], b[q], c[q]);
}

struct HswGrid {
  int n1, n2, nth;
  const double *R, *r, *x;
  double f2, f3, vmax, rmin;
  int cap;
};

__global__ void __launch_bounds__(256) k_hsw_grid(HswDev h, HswGrid g, double *pot)
{
  const long n = (long)g.n1 * g.n2 * g.nth;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n;
       q += (long)gridDim.x * blockDim.x) {
    const int i = (int)(q % g.n1), j = (int)((q / g.n1) % g.n2), k = (int)(q / ((long)g.n1 * g.n2));
    const double R = g.R[i], r = g.r[j], cth = g.x[k];
    const double a = g.f2 * r, b = g.f3 * r;
    const double r23 = r;
    const double r12 = sqrt(a * a + R * R - 2.0 * g.f2 * r * R * cth);
    const double r13 = sqrt(b * b + R * R + 2.0 * g.f3 * r * R * cth);
    double v = g.vmax;
    if (r12 > g.rmin && r13 > g.rmin && r23 > g.rmin) {
      v = hsw_pot(h, r12, r23, r13);
      if (g.cap) v = fmin(v, g.vmax);
    }
    pot[q] = v;
  }
}

// ---- host: the spline tables ------------------------------------------------

// derivative at x[ip] of the cubic through (x[0..3], y[0..3]) (sospline.F:291-314)
double lagrange_slope(const double *x, const double *y, int ip)
{
  double d = 0.0;
  for (int i = 0; i < 4; i++) {
    if (i == ip) continue;
    double t = y[i];
    for (int j = 0; j < 4; j++)
      if (j != ip && j != i) t *= x[ip] - x[j];
    for (int j = 0; j < 4; j++)
      if (j != i) t /= x[i] - x[j];
    d += t;
  }
  for (int i = 0; i < 4; i++)
    if (i != ip) d += y[ip] / (x[ip] - x[i]);
  return d;
}

// slopes s[0..n) of the clamped cubic spline through f[0..n) at the nodes g,
// end slopes s0, sn (sospline.F:107-126, 316-335)
void spline_slopes(const std::vector<double> &g, const double *f, double s0, double sn,
                   double *s)
{
  const int n = (int)g.size(), n2 = n - 2;
  s[0] = s0;
  s[n - 1] = sn;
  if (n2 < 1) return;
  std::vector<double> h(n - 1), lam(n2), mu(n2), rhs(n2), piv(n2);
  for (int i = 0; i + 1 < n; i++) h[i] = g[i + 1] - g[i];
  for (int i = 0; i < n2; i++) {
    lam[i] = h[i + 1] / (h[i] + h[i + 1]);
    mu[i] = 1.0 - lam[i];
    rhs[i] = 3.0 * lam[i] / h[i] * (f[i + 1] - f[i]) + 3.0 * mu[i] / h[i + 1] * (f[i + 2] - f[i + 1]);
  }
  rhs[0] = rhs[0] - lam[0] * s0;
  rhs[n2 - 1] = rhs[n2 - 1] - mu[n2 - 1] * sn;
  piv[0] = 2.0;
  for (int i = 1; i < n2; i++) {
    piv[i] = 2.0 - lam[i] * mu[i - 1] / piv[i - 1];
    rhs[i] = rhs[i] - lam[i] / piv[i - 1] * rhs[i - 1];
  }
  std::vector<double> x(n2);
  x[n2 - 1] = rhs[n2 - 1] / piv[n2 - 1];
  for (int i = n2 - 2; i >= 0; i--) x[i] = (rhs[i] - x[i + 1] * mu[i]) / piv[i];
  for (int i = 0; i < n2; i++) s[i + 1] = x[i];
}

// tables T[node][t], t = dx + 2 dy + 4 dz, from the values F on the nodes
// (node = (k ny + j) nx + i)
std::vector<double> hermite_tables(const std::vector<double> &gx, const std::vector<double> &gy,
                                   const std::vector<double> &gz, const std::vector<double> &F)
{
  const int nx = (int)gx.size(), ny = (int)gy.size(), nz = (int)gz.size();
  const long nn = (long)nx * ny * nz;
  std::vector<std::vector<double>> T(8, std::vector<double>(nn, 0.0));
  T[0] = F;
  auto at = [&](int i, int j, int k) { return ((long)k * ny + j) * nx + i; };
  std::vector<double> line(HSW_MAXNODE), out(HSW_MAXNODE);
  // one spline family: target t from source src along axis ax; value
  // splines take their end slopes from the Lagrange formula, the cross
  // derivatives zero end slopes
  auto family = [&](int t, int src, int ax, bool value) {
    const std::vector<double> &g = ax == 0 ? gx : ax == 1 ? gy : gz;
    const int n = (int)g.size();
    const int na = ax == 0 ? ny : nx, nb = ax == 2 ? ny : nz;
    for (int a = 0; a < na; a++)
      for (int b = 0; b < nb; b++) {
        for (int m = 0; m < n; m++) {
          const int i = ax == 0 ? m : a, j = ax == 1 ? m : (ax == 0 ? a : b);
          const int k = ax == 2 ? m : b;
          line[m] = T[src][at(i, j, k)];
        }
        double s0 = 0.0, sn = 0.0;
        if (value) {
          s0 = lagrange_slope(g.data(), line.data(), 0);
          sn = lagrange_slope(g.data() + n - 4, line.data() + n - 4, 3);
        }
        spline_slopes(g, line.data(), s0, sn, out.data());
        for (int m = 0; m < n; m++) {
          const int i = ax == 0 ? m : a, j = ax == 1 ? m : (ax == 0 ? a : b);
          const int k = ax == 2 ? m : b;
          T[t][at(i, j, k)] = out[m];
        }
      }
  };
  family(1, 0, 0, true);         // Fx   (sospline.F:107-126)
  family(2, 0, 1, true);         // Fy   (:128-148)
  if (nz > 1) family(4, 0, 2, true);    // Fz   (:150-170)
  family(3, 1, 1, false);        // Fxy  (:172-195)
  if (nz > 1) {
    family(5, 1, 2, false);      // Fxz  (:197-221)
    family(6, 2, 2, false);      // Fyz  (:223-245)
    family(7, 3, 2, false);      // Fxyz (:247-270)
  }
  std::vector<double> tab(nn * 8);
  for (long q = 0; q < nn; q++)
    for (int t = 0; t < 8; t++) tab[q * 8 + t] = T[t][q];
  return tab;
}

}  // namespace

struct qd_hsw {
  HswDev dev{};
  void *mem = nullptr;
  ~qd_hsw() { if (mem) cudaFree(mem); }
};

namespace {

int hsw_build(int n3, const int32_t *ix, const int32_t *iy, const int32_t *iz, const double *a,
              const double p[12], int nx, int ny, int nz, const double *x, const double *y,
              const double *z, const double *so, const double so_param[3], qd_hsw **out)
{
  if (!out || !ix || !iy || !iz || !a || !p || !x || !y || !z || !so || !so_param)
    return qd_errf(QD_ERR_INVALID, "NULL argument");
  *out = nullptr;
  // the last six three-body records are b1 b2 b3 x0 y0 z0 (hswpot.F:146-151)
  if (n3 < 7 || n3 - 6 > HSW_MAXTERM)
    return qd_errf(QD_ERR_INVALID, "three-body parameter count %d out of range", n3);
  if (nx < 4 || ny < 4 || nz < 1 || nz == 2 || nz == 3 || nx > HSW_MAXNODE || ny > HSW_MAXNODE ||
      nz > HSW_MAXNODE)
    return qd_errf(QD_ERR_INVALID, "spin-orbit grid %d x %d x %d not supported", nx, ny, nz);
  std::vector<HswTerm> term(n3 - 6);
  for (int i = 0; i < n3 - 6; i++) {
    if (ix[i] < 0 || iy[i] < 0 || iz[i] < 0 || ix[i] >= HSW_MAXPOW || iy[i] >= HSW_MAXPOW ||
        iz[i] >= HSW_MAXPOW)
      return qd_errf(QD_ERR_INVALID, "three-body term %d has a power beyond %d", i + 1,
                     HSW_MAXPOW - 1);
    term[i] = HswTerm{a[i], ix[i], iy[i], iz[i], 0};
  }
  std::vector<double> gx(x, x + nx), gy(y, y + ny), gz(z, z + nz);
  for (int i = 1; i < nx; i++)
    if (!(gx[i] > gx[i - 1])) return qd_errf(QD_ERR_INVALID, "spin-orbit R nodes not ascending");
  for (int i = 1; i < ny; i++)
    if (!(gy[i] > gy[i - 1])) return qd_errf(QD_ERR_INVALID, "spin-orbit r nodes not ascending");
  for (int i = 1; i < nz; i++)
    if (!(gz[i] > gz[i - 1])) return qd_errf(QD_ERR_INVALID, "spin-orbit angle nodes not ascending");
  // so[] is in file order: i (R) outermost, then j (r), k (angle) innermost
  std::vector<double> F((size_t)nx * ny * nz);
  for (int i = 0; i < nx; i++)
    for (int j = 0; j < ny; j++)
      for (int k = 0; k < nz; k++)
        F[((size_t)k * ny + j) * nx + i] = so[((size_t)i * ny + j) * nz + k];
  const std::vector<double> tab = hermite_tables(gx, gy, gz, F);

  qd_hsw *h = new qd_hsw();
  const size_t tb = sizeof(HswTerm) * term.size(), gb = sizeof(double) * (nx + ny + nz),
               sb = sizeof(double) * tab.size();
  cudaError_t e = cudaMalloc(&h->mem, tb + gb + sb);
  if (e != cudaSuccess) {
    delete h;
    cudaGetLastError();
    return qd_errf(QD_ERR_NOMEM, "qd_hsw: cudaMalloc failed: %s", cudaGetErrorString(e));
  }
  char *m = static_cast<char *>(h->mem);
  std::vector<double> g;
  g.insert(g.end(), gx.begin(), gx.end());
  g.insert(g.end(), gy.begin(), gy.end());
  g.insert(g.end(), gz.begin(), gz.end());
  e = cudaMemcpy(m, term.data(), tb, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(m + tb, g.data(), gb, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(m + tb + gb, tab.data(), sb, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    delete h;
    return qd_errf(QD_ERR_CUDA, "qd_hsw: upload failed: %s", cudaGetErrorString(e));
  }
  HswDev &d = h->dev;
  d.term = reinterpret_cast<const HswTerm *>(m);
  d.nterm = n3 - 6;
  d.npow = HSW_MAXPOW;
  for (int q = 0; q < 3; q++) {
    d.b[q] = a[n3 - 6 + q];
    d.q0[q] = a[n3 - 3 + q];
  }
  for (int q = 0; q < 12; q++) d.p[q] = p[q];
  d.nx = nx; d.ny = ny; d.nz = nz;
  d.gx = reinterpret_cast<const double *>(m + tb);
  d.gy = d.gx + nx;
  d.gz = d.gy + ny;
  d.tab = reinterpret_cast<const double *>(m + tb + gb);
  d.esocut = so_param[0] / 627.5095;               // kcal/mol -> hartree (hswpot.F:17,38)
  d.rsolim = so_param[1];
  d.rrsolm = so_param[2];
  d.raddeg = 180.0 / std::acos(-1.0);
  d.shift = (double)0.0006f;                        // hswpot.F:98, a default-real constant
  *out = h;
  return QD_OK;
}

// first numbers of each line of a text file
bool read_numbers(const std::string &path, std::vector<std::vector<double>> &rows, int per_row)
{
  FILE *f = std::fopen(path.c_str(), "r");
  if (!f) return false;
  char buf[512];
  while (std::fgets(buf, sizeof buf, f)) {
    std::vector<double> row;
    const char *s = buf;
    char *end = nullptr;
    while ((int)row.size() < per_row) {
      const double v = std::strtod(s, &end);
      if (end == s) break;
      row.push_back(v);
      s = end;
    }
    if (!row.empty()) rows.push_back(row);
  }
  std::fclose(f);
  return true;
}

}  // namespace

extern "C" {

int qd_hsw_create_from_tables(int32_t n3, const int32_t *ix, const int32_t *iy,
                              const int32_t *iz, const double *a, const double p[12],
                              int32_t nx, int32_t ny, int32_t nz, const double *x,
                              const double *y, const double *z, const double *so,
                              const double so_param[3], qd_hsw **out)
{
  return hsw_build(n3, ix, iy, iz, a, p, nx, ny, nz, x, y, z, so, so_param, out);
}

int qd_hsw_create(const char *dir, qd_hsw **out)
{
  if (!dir || !out) return qd_errf(QD_ERR_INVALID, "NULL argument");
  const std::string d(dir);
  std::vector<std::vector<double>> three, two, soin, sop;
  if (!read_numbers(d + "/three.param", three, 5) || !read_numbers(d + "/two.param", two, 1) ||
      !read_numbers(d + "/so.input", soin, 4) || !read_numbers(d + "/so.param", sop, 1))
    return qd_errf(QD_ERR_IO, "qd_hsw_create: cannot read the HSW data files in %s", dir);
  if (two.size() < 12 || sop.size() < 3 || soin.empty() || soin[0].size() < 3)
    return qd_errf(QD_ERR_IO, "qd_hsw_create: HSW data files in %s are incomplete", dir);
  std::vector<int32_t> ix, iy, iz;
  std::vector<double> a;
  for (const auto &r : three) {
    if (r.size() < 5) return qd_errf(QD_ERR_IO, "three.param: a record has fewer than 5 fields");
    ix.push_back((int32_t)r[1]);
    iy.push_back((int32_t)r[2]);
    iz.push_back((int32_t)r[3]);
    a.push_back(r[4]);
  }
  double p[12], sp[3];
  for (int q = 0; q < 12; q++) p[q] = two[q][0];
  for (int q = 0; q < 3; q++) sp[q] = sop[q][0];
  const int nx = (int)soin[0][0], ny = (int)soin[0][1], nz = (int)soin[0][2];
  if (nx < 1 || ny < 1 || nz < 1 || soin.size() < 1 + (size_t)nx * ny * nz)
    return qd_errf(QD_ERR_IO, "so.input: %zu records for a %d x %d x %d table", soin.size() - 1,
                   nx, ny, nz);
  std::vector<double> x(nx), y(ny), z(nz), so((size_t)nx * ny * nz);
  size_t rec = 1;
  for (int i = 0; i < nx; i++)
    for (int j = 0; j < ny; j++)
      for (int k = 0; k < nz; k++, rec++) {
        const auto &r = soin[rec];
        if (r.size() < 4) return qd_errf(QD_ERR_IO, "so.input: record %zu has fewer than 4 fields", rec + 1);
        x[i] = r[0]; y[j] = r[1]; z[k] = r[2];
        so[((size_t)i * ny + j) * nz + k] = r[3];
      }
  return hsw_build((int)a.size(), ix.data(), iy.data(), iz.data(), a.data(), p, nx, ny, nz,
                   x.data(), y.data(), z.data(), so.data(), sp, out);
}

int qd_hsw_destroy(qd_hsw *h)
{
  delete h;
  return QD_OK;
}

int qd_hsw_eval(const qd_hsw *h, int64_t n, const double *r_fh1, const double *r_hh,
                const double *r_fh2, double *v_out)
{
  if (!h || (n > 0 && (!r_fh1 || !r_hh || !r_fh2 || !v_out)))
    return qd_errf(QD_ERR_INVALID, "NULL argument");
  if (n <= 0) return QD_OK;
  double *d = nullptr;
  QD_CU(cudaMalloc(&d, sizeof(double) * 4 * (size_t)n));
  cudaError_t e = cudaMemcpy(d, r_fh1, sizeof(double) * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + n, r_hh, sizeof(double) * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + 2 * n, r_fh2, sizeof(double) * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    const long blocks = (n + 255) / 256;
    k_hsw_points<<<(unsigned)(blocks < 148 * 16 ? blocks : 148 * 16), 256>>>(h->dev, n, d, d + n,
                                                                            d + 2 * n, d + 3 * n);
    qd_count_launches(1);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(v_out, d + 3 * n, sizeof(double) * n, cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return qd_errf(QD_ERR_CUDA, "qd_hsw_eval: %s", cudaGetErrorString(e));
  return QD_OK;
}

int qd_potential_hsw(const qd_radial *R, const qd_radial *r, const qd_angle *theta,
                     const double masses[3], const qd_hsw *h, double vmax, double rmin,
                     int32_t cap, double *pot_out)
{
  if (!R || !r || !theta || !masses || !h || !pot_out || !R->r || !r->r || !theta->x)
    return qd_errf(QD_ERR_INVALID, "NULL argument");
  if (R->n < 1 || r->n < 1 || theta->n < 1)
    return qd_errf(QD_ERR_INVALID, "empty grid (%d x %d x %d)", R->n, r->n, theta->n);
  if (!(masses[1] + masses[2] > 0) || !(masses[2] >= 0))
    return qd_errf(QD_ERR_INVALID, "masses of the diatom atoms must be positive");
  HswGrid g{};
  g.n1 = R->n; g.n2 = r->n; g.nth = theta->n;
  g.f2 = masses[2] / (masses[1] + masses[2]);
  g.f3 = 1.0 - g.f2;
  g.vmax = vmax; g.rmin = rmin; g.cap = cap ? 1 : 0;
  const long n = (long)g.n1 * g.n2 * g.nth;
  double *d = nullptr;
  QD_CU(cudaMalloc(&d, sizeof(double) * ((size_t)n + g.n1 + g.n2 + g.nth)));
  double *dR = d + n, *dr = dR + g.n1, *dx = dr + g.n2;
  cudaError_t e = cudaMemcpy(dR, R->r, sizeof(double) * g.n1, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dr, r->r, sizeof(double) * g.n2, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dx, theta->x, sizeof(double) * g.nth, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    g.R = dR; g.r = dr; g.x = dx;
    const long blocks = (n + 255) / 256;
    k_hsw_grid<<<(unsigned)(blocks < 148 * 16 ? blocks : 148 * 16), 256>>>(h->dev, g, d);
    qd_count_launches(1);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(pot_out, d, sizeof(double) * n, cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return qd_errf(QD_ERR_CUDA, "qd_potential_hsw: %s", cudaGetErrorString(e));
  return QD_OK;
}

}  // extern "C"
