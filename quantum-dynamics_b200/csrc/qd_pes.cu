// qd_pes.cu -- the potential on the Jacobi grid, the set-up step the
// reference does in Matlab (H3/H3PESJacobi.m:5-27 with a PES MEX such as
// FH2/HSW/HSWMex.C:29-90):
//   r23 = r,  r12 = sqrt((f2 r)^2 + R^2 - 2 f2 r R cos(theta)),
//   r13 = sqrt((f3 r)^2 + R^2 + 2 f3 r R cos(theta)),  f2 = m3/(m2+m3), f3 = 1-f2,
//   V = PES(r12, r23, r13) where every distance > rmin, else vmax
// (optionally capped at vmax).  qd_potential_jacobi calls a host PES through
// the callback convention of the PES MEX functions (column vectors of the
// three distances in, V out, one call for all points); qd_potential_leps
// evaluates an extended-LEPS surface on the GPU in FP64.
#include <cmath>
#include <vector>
#include "qd_err.h"

namespace {

struct JacobiGrid {
  int n1, n2, nth;
  const double *R, *r, *x;
  double f2, f3, vmax, rmin;
  int cap;
};

__host__ __device__ inline void internuclear(const JacobiGrid &g, long q, double &r12,
                                             double &r23, double &r13)
{
  const int i = (int)(q % g.n1), j = (int)((q / g.n1) % g.n2), k = (int)(q / ((long)g.n1 * g.n2));
  const double R = g.R[i], r = g.r[j], c = g.x[k];
  const double a = g.f2 * r, b = g.f3 * r;
  r23 = r;
  r12 = sqrt(a * a + R * R - 2.0 * g.f2 * r * R * c);
  r13 = sqrt(b * b + R * R + 2.0 * g.f3 * r * R * c);
}

struct LepsDev {
  double de[3], beta[3], re[3], pf[3];   // pairs AB (r12), BC (r23), AC (r13)
};

__device__ inline void coulomb_exchange(const LepsDev &p, int s, double r, double &q, double &jx)
{
  const double y = exp(-p.beta[s] * (r - p.re[s]));
  q = 0.5 * (p.de[s] * (y - 2.0) + p.pf[s] * (y + 2.0)) * y;
  jx = 0.5 * (p.de[s] * (y - 2.0) - p.pf[s] * (y + 2.0)) * y;
}

__global__ void __launch_bounds__(256) k_leps(JacobiGrid g, LepsDev p, double *pot)
{
  const long n = (long)g.n1 * g.n2 * g.nth;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n;
       q += (long)gridDim.x * blockDim.x) {
    double r12, r23, r13;
    internuclear(g, q, r12, r23, r13);
    double v = g.vmax;
    if (r12 > g.rmin && r13 > g.rmin && r23 > g.rmin) {
      double q1, j1, q2, j2, q3, j3;
      coulomb_exchange(p, 0, r12, q1, j1);
      coulomb_exchange(p, 1, r23, q2, j2);
      coulomb_exchange(p, 2, r13, q3, j3);
      const double rad = fmax(j1 * (j1 - j2) + j2 * (j2 - j3) + j3 * (j3 - j1), 0.0);
      v = p.de[1] + q1 + q2 + q3 - sqrt(rad);
      if (g.cap) v = fmin(v, g.vmax);
    }
    pot[q] = v;
  }
}

int grid_args(const qd_radial *R, const qd_radial *r, const qd_angle *theta,
              const double masses[3], double vmax, double rmin, int32_t cap, JacobiGrid &g)
{
  if (!R || !r || !theta || !masses || !R->r || !r->r || !theta->x)
    return qd_errf(QD_ERR_INVALID, "NULL argument");
  if (R->n < 1 || r->n < 1 || theta->n < 1)
    return qd_errf(QD_ERR_INVALID, "empty grid (%d x %d x %d)", R->n, r->n, theta->n);
  if (!(masses[1] + masses[2] > 0) || !(masses[2] >= 0))
    return qd_errf(QD_ERR_INVALID, "masses of the diatom atoms must be positive");
  g.n1 = R->n; g.n2 = r->n; g.nth = theta->n;
  g.R = R->r; g.r = r->r; g.x = theta->x;
  g.f2 = masses[2] / (masses[1] + masses[2]);
  g.f3 = 1.0 - g.f2;
  g.vmax = vmax; g.rmin = rmin; g.cap = cap ? 1 : 0;
  return QD_OK;
}

}  // namespace

extern "C" {

int qd_potential_jacobi(const qd_radial *R, const qd_radial *r, const qd_angle *theta,
                        const double masses[3], qd_pes_fn pes, void *ctx, double vmax,
                        double rmin, int32_t cap, double *pot_out)
{
  JacobiGrid g{};
  int rc = grid_args(R, r, theta, masses, vmax, rmin, cap, g);
  if (rc != QD_OK) return rc;
  if (!pes || !pot_out) return qd_errf(QD_ERR_INVALID, "NULL PES callback or output");
  const long n = (long)g.n1 * g.n2 * g.nth;
  std::vector<long> idx;
  std::vector<double> a, b, c;
  idx.reserve(n);
  for (long q = 0; q < n; q++) {
    double r12, r23, r13;
    internuclear(g, q, r12, r23, r13);
    pot_out[q] = vmax;
    if (r12 > rmin && r13 > rmin && r23 > rmin) {
      idx.push_back(q);
      a.push_back(r12);
      b.push_back(r23);
      c.push_back(r13);
    }
  }
  std::vector<double> v(idx.size());
  if (!idx.empty()) {
    const int st = pes((int64_t)idx.size(), a.data(), b.data(), c.data(), v.data(), ctx);
    if (st != 0) return qd_errf(QD_ERR_PES, "PES callback returned %d", st);
  }
  for (size_t m = 0; m < idx.size(); m++) {
    if (!std::isfinite(v[m]))
      return qd_errf(QD_ERR_PES, "PES callback gave a non-finite value at r12 = %g, r23 = %g, "
                     "r13 = %g", a[m], b[m], c[m]);
    pot_out[idx[m]] = g.cap ? std::fmin(v[m], vmax) : v[m];
  }
  return QD_OK;
}

int qd_potential_leps(const qd_radial *R, const qd_radial *r, const qd_angle *theta,
                      const double masses[3], const qd_leps *leps, double vmax, double rmin,
                      int32_t cap, double *pot_out)
{
  JacobiGrid g{};
  int rc = grid_args(R, r, theta, masses, vmax, rmin, cap, g);
  if (rc != QD_OK) return rc;
  if (!leps || !pot_out) return qd_errf(QD_ERR_INVALID, "NULL LEPS parameters or output");
  LepsDev p{};
  const qd_leps_pair *pr[3] = {&leps->ab, &leps->bc, &leps->ac};
  for (int s = 0; s < 3; s++) {
    if (!(pr[s]->sato > -1.0)) return qd_errf(QD_ERR_INVALID, "Sato parameter must be > -1");
    p.de[s] = pr[s]->de;
    p.beta[s] = pr[s]->beta;
    p.re[s] = pr[s]->re;
    p.pf[s] = 0.5 * pr[s]->de * (1.0 - pr[s]->sato) / (1.0 + pr[s]->sato);
  }
  const long n = (long)g.n1 * g.n2 * g.nth;
  double *d = nullptr;
  QD_CU(cudaMalloc(&d, sizeof(double) * ((size_t)n + g.n1 + g.n2 + g.nth)));
  double *dR = d + n, *dr = dR + g.n1, *dx = dr + g.n2;
  cudaError_t e = cudaMemcpy(dR, g.R, sizeof(double) * g.n1, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dr, g.r, sizeof(double) * g.n2, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dx, g.x, sizeof(double) * g.nth, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    JacobiGrid gd = g;
    gd.R = dR; gd.r = dr; gd.x = dx;
    const long blocks = (n + 255) / 256;
    k_leps<<<(unsigned)(blocks < 148 * 16 ? blocks : 148 * 16), 256>>>(gd, p, d);
    qd_count_launches(1);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(pot_out, d, sizeof(double) * n, cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return qd_errf(QD_ERR_CUDA, "qd_potential_leps: %s", cudaGetErrorString(e));
  return QD_OK;
}

}  // extern "C"
