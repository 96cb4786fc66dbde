// qd_bkmp2.cu -- the BKMP2 surface of H3 (Boothroyd, Keogh, Martin,
// Peterson, J. Chem. Phys. 104, 7139 (1996)) evaluated on the GPU in FP64,
// replacing the PES MEX H3/BKMP2Mex.C:16-60 over the Fortran H3/bkmp2.F (the
// "jun21/95" parameter set that file uses).  Values only; the reference
// also forms dV/dr, which the propagator does not need.
//
// The parts, restated from bkmp2.F and summed in its order (:20-115):
//   London term from the singlet H2 curve vH2opt95 (:252-306) and the
//     triplet curve triplet95 (:176-250, Johnson correction below 1.15 bohr),
//     V_lon = sum Q - sqrt(sum of squared J differences / 2 + 1e-12)
//     (h3lond95 :356-392);
//   asymmetric correction Vascal95 (:419-489), A = |(r1-r2)(r2-r3)(r3-r1)|;
//   bending terms vbcb95 (:724-1417) with B1a = 1 - sum cos(theta_i) and
//     B1b = 1 - (5/8 sum cos 3theta_i + 3/8 sum cos theta_i);
//   for compact geometries (a distance below 1.15 bohr) also csym95
//     (:655-722), casym95 (:553-653) and the Cbend part of vbcb95.
// Where the reference stops the program for an impossible triangle or a
// distance below 0.2 bohr (chgeom :1418-1446), the value here is NaN.
// qd_potential_bkmp2 subtracts vH2Min = -0.174495770896975 as
// H3/H3PESBKMP2.m:23-27 does before the grid is used.
#include <cmath>
#include "qd_err.h"

namespace {

// singlet H2 (vH2opt95): alpha(r) = a0/r + sum_{i>=1} a_i r^(i-1)
__constant__ double kH2A[17] = {
    0.03537359271649620, 2.013977588700072, -2.827452449964767, 2.713257715593500,
    -2.792039234205731, 2.166542078766724, -1.272679684173909, 0.5630423099212294,
    -0.1879397372273814, 0.04719891893374140, -0.008851622656489644, 0.001224998776243630,
    -1.227820520228028e-04, 8.638783190083473e-06, -4.036967926499151e-07,
    1.123286608335365e-08, -1.406619156782167e-10};
constexpr double kH2R0 = 3.5284882, kH2DD = 0.160979391, kC6 = 6.499027, kC8 = 124.3991,
                 kC10 = 3285.828;
// triplet (triplet95)
__constant__ double kT[6] = {-0.0298546962, -23.9604445036, -42.5185569474, 2.0382390988,
                          -11.5214861455, 1.5309487826};
__constant__ double kJ[3] = {-0.4106358351531854, -0.0770355790707090, 0.4303193846943223};
// asymmetric correction (Vascal95)
__constant__ double kAS[7] = {0.3788951192e-02, 0.1478100901e-02, -.1848513849e-03,
                           0.9230803609e-05, -.1293180255e-06, 0.5237179303e+00,
                           -.1112326215e-02};
// compact-geometry corrections (csym95, casym95)
constexpr double kRR = 1.15, kRP = 1.25;
__constant__ double kCS[3] = {-.2071708868e+00, -.5672350377e+00, 0.9058780367e-02};
__constant__ double kCA[13] = {0.2210243144e+00, 0.4367417579e+00, 0.6994985432e-02,
                               0.1491096501e+01, 0.1602896673e+01, -.2821747323e+01,
                               0.4948310833e+00, -.3540394679e-01, -.3305809954e+01,
                               0.3644382172e+01, -.9997570970e+00, 0.7989919534e-01,
                               -.1075807322e-02};
// bending (vbcb95): Vbend sets for B1a and B1b, 16 coefficients each in the
// order p11 p12 p13 p21 p22 p23 p24 p31 p32 p41 p42 p43 p44 p51 p52 p53
constexpr double kB1 = 0.52, kB2 = 0.052, kB3 = 0.79;
__constant__ double kVB[2][16] = {
    {-.1838073394e+03, 0.1334593242e+02, -.2358129537e+00, -.4668193478e+01, 0.7197506670e+01,
     0.2162004275e+02, 0.2106294028e+02, 0.4242962586e+01, 0.4453505045e+01, -.1456918088e+00,
     -.1692657366e-01, 0.1279520698e+01, -.4898940075e+00, 0.1742295219e+03, 0.3142175348e+02,
     0.5152903406e+01},
    {-.4765732725e+02, 0.3648933563e+01, -.7141145244e-01, 0.1002349176e-01, 0.9989856329e-02,
     -.4161953634e-02, 0.9075807910e-03, -.2693628729e+00, -.1399065763e-01, -.1417634346e-01,
     -.4870024792e-03, 0.1312231847e+00, -.4409850519e-01, 0.5382970863e+02, 0.4587102824e+01,
     0.1768550515e+01}};
// Cbend sets for B1a and B1b, 30 coefficients each: q11..q15 q21..q24 q31 q32
// q41..q44 q51..q53 q61..q63 q71..q75 q81..q84
__constant__ double kCB[2][30] = {
    {0.1860299931e+04, -.6134458037e+03, 0.7337207161e+02, -.2676717625e+04, 0.1344099415e+04,
     0.1538913137e+03, 0.4348007369e+02, 0.1719720677e+03, 0.2115963042e+03,
     -.7026089414e+02, -.1300938992e+03,
     0.1310273564e+01, -.6175149574e+00, -.2679089358e+02, 0.5577477171e+01,
     -.3543353539e+04, -.3740709591e+03, 0.7979303144e+02,
     -.1104230585e+04, 0.4603572025e+04, -.5593496634e+04,
     -.1069406434e+02, 0.1021807153e+01, 0.6669828341e-01, 0.4168542348e+02, 0.1751608567e+02,
     0.9486883238e+02, -.1519334221e+02, 0.4024697252e+04, -.2225159395e+02},
    {0.4203543357e+03, -.4922474096e+02, 0.3362942544e+00, -.3827423082e+03, 0.1746726001e+03,
     0.1699995737e-01, 0.1513036778e-01, 0.2659119354e-01, -.5760387483e-02,
     0.1020622621e+02, 0.1050536271e-01,
     0.6836172780e+00, -.1627858240e+00, -.6925485045e+01, 0.1632567385e+01,
     0.1083595009e+04, 0.4641431791e+01, -.8233144461e+00,
     -.6157225942e+02, 0.3094361471e+03, -.3299631143e+03,
     0.8866227120e+01, -.1382126854e+01, 0.7620770145e-01, -.5145757859e+02, 0.2046097265e+01,
     0.2540775558e+01, -.4889246569e+00, -.1127439280e+04, -.2269932295e+01}};
constexpr double kVH2Min = -0.174495770896975;

__device__ double singlet(double r)
{
  double rp[16];
  rp[0] = 1.0;
  rp[1] = r;
#pragma unroll
  for (int i = 2; i < 16; i++) rp[i] = rp[i - 1] * r;
  const double r02 = kH2R0 * kH2R0, r04 = r02 * r02, r06 = r04 * r02;
  const double rr2 = rp[2] + r02, rr4 = rp[4] + r04, rr6 = rp[6] + r06;
  const double rr25 = rr2 * rr2 * rr2 * rr2 * rr2;
  double alpha = kH2A[0] / r + kH2A[1];
#pragma unroll
  for (int i = 2; i < 17; i++) alpha = alpha + kH2A[i] * rp[i - 1];
  const double ex = exp(alpha);
  const double vsr = kH2DD * (ex - 1.0) * (ex - 1.0) - kH2DD;
  const double vlr = -kC6 / rr6 - kC8 / (rr4 * rr4) - kC10 / rr25;
  return vsr + vlr;
}

__device__ double triplet(double r)
{
  if (r >= 1.15)
    return kT[0] * (kT[1] + r + kT[2] * (r * r) + kT[4] * pow(r, -kT[5])) * exp(-kT[3] * r);
  const double dr = r - 0.95, e1 = singlet(r);
  if (r <= 0.95) return e1 + kJ[1] * dr + kJ[2];
  return e1 + kJ[0] * dr * dr * dr + kJ[1] * dr + kJ[2];
}

__device__ double area_term(double r1, double r2, double r3)   // acalc95
{
  return fabs((r1 - r2) * (r2 - r3) * (r3 - r1));
}

// Vbend (k = 0: B1a, k = 1: B1b) of vbcb95
__device__ double vbend(int k, double B1, double R, double Rsq, double B2, double B3, double B3b,
                        double e1, double e2, double e7)
{
  const double *p = kVB[k];
  const double B12 = B1 * B1, B13 = B12 * B1, B14 = B13 * B1, B15 = B14 * B1;
  const double asum = p[0] + p[1] * R + p[2] * Rsq;
  const double bsum = p[3] * B12 + p[4] * B13 + p[5] * B14 + p[6] * B15;
  const double csum = p[7] * B1 * e1 + p[8] * B12 * e2;
  const double d1 = p[9] * e1 + p[10] * e2, d2 = p[11] * e1 + p[12] * e2;
  const double fsum = p[13] + p[14] * R + p[15] * Rsq;
  return B1 * asum * e1 + bsum * e2 + B2 * csum + (B1 * B3 * d1 + B1 * B3b * d2) +
         B1 * fsum * e7;
}

// Cbend of vbcb95 (compact geometries), before the sum T factor
__device__ double cbend(int k, double B1, double R, double Rsq, double B2, double B3, double B3b,
                        double P, double Psq, double e1, double e2, double e7c)
{
  const double *q = kCB[k];
  const double B12 = B1 * B1, B13 = B12 * B1, B14 = B13 * B1, B15 = B14 * B1;
  const double asum = q[0] + q[1] * R + q[2] * Rsq + q[3] / R + q[4] / Rsq;
  const double bsum = q[5] * B12 + q[6] * B13 + q[7] * B14 + q[8] * B15;
  const double csum = q[9] * B1 * e1 + q[10] * B12 * e2;
  const double d1 = q[11] * e1 + q[12] * e2, d2 = q[13] * e1 + q[14] * e2;
  const double fsum = (q[15] + q[28]) + q[16] * R + q[17] * Rsq;   // feb27/91: q51 + q83
  const double gsum = q[18] + q[19] / R + q[20] / Rsq;
  const double aasum = q[21] + q[22] * P + q[23] * Psq + q[24] / P + q[25] / Psq;
  const double ffsum = q[26] * P + q[27] * Psq + q[29] / Psq;
  return B1 * asum * e1 / P + bsum * e2 + B2 * csum + (B1 * B3 * d1 + B1 * B3b * d2) +
         B1 * fsum * e7c / P + B1 * gsum * e7c + B1 * aasum * e2 + B1 * ffsum * e7c;
}

// the MEX value at internuclear distances r1, r2, r3 (bohr), hartree
__device__ double bkmp2(double r1, double r2, double r3)
{
  {
    const double lo = fmin(r1, fmin(r2, r3)), hi = fmax(r1, fmax(r2, r3));
    const double mid = r1 + r2 + r3 - lo - hi;
    if (lo + mid + 1e-5 < hi || lo < 0.2) return nan("");
  }
  const double r[3] = {r1, r2, r3};
  // London
  double sq = 0.0, j[3];
#pragma unroll
  for (int i = 0; i < 3; i++) {
    const double e1 = singlet(r[i]), e3 = triplet(r[i]);
    sq = sq + 0.5 * (e1 + e3);
    j[i] = 0.5 * (e1 - e3);
  }
  const double sj = (j[1] - j[0]) * (j[1] - j[0]) + (j[2] - j[1]) * (j[2] - j[1]) +
                    (j[2] - j[0]) * (j[2] - j[0]);
  const double vlon = sq - sqrt(0.5 * sj + 1e-12);
  // asymmetric correction
  const double R = r1 + r2 + r3, Rsq = R * R, Rcu = Rsq * R;
  const double A = area_term(r1, r2, r3), A2 = A * A, A3 = A2 * A, A4 = A3 * A, A5 = A4 * A;
  const double S = kAS[1] * A2 + kAS[2] * A3 + kAS[3] * A4 + kAS[4] * A5;
  const double vas = S * exp(-kAS[0] * Rcu) + kAS[6] * A2 * exp(-kAS[5] * R) / R;
  // compactness
  int icompc = 0;
  double T[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int i = 0; i < 3; i++)
    if (r[i] < kRR) {
      icompc++;
      const double top = kRR - r[i];
      T[i] = top * top * top / (kRP - r[i]);
    }
  double cal = 0.0, cas = 0.0;
  if (icompc >= 1) {
    const double e3 = exp(-kCS[2] * Rcu);
    double sg = 0.0;
#pragma unroll
    for (int i = 0; i < 3; i++)
      if (r[i] < kRR) {
        const double d = kRR - r[i];
        sg = sg + (d * d * d / (kRP - r[i])) * (kCS[0] + kCS[0] * kCS[1] * r[i]);
      }
    cal = sg * e3;
    const double sumt = T[0] + T[1] + T[2];
    const double Pr = r1 * r2 * r3, Pr2 = Pr * Pr;
    const double *u = kCA;
    const double series = 1.0 + u[3] / Pr2 + u[4] / Pr + u[5] + u[6] * Pr + u[7] * Pr2 +
                          A * (u[8] / Pr2 + u[9] / Pr + u[10] + u[11] * Pr + u[12] * Pr2);
    cas = sumt * A2 * (u[0] / pow(Pr, u[1])) * series * exp(-u[2] * Rcu);
  }
  // bending
  const double t1 = r1 * r1 - r2 * r2 - r3 * r3, t2 = r2 * r2 - r3 * r3 - r1 * r1,
               t3 = r3 * r3 - r1 * r1 - r2 * r2;
  const double c1 = t1 / (-2.0 * r2 * r3), c2 = t2 / (-2.0 * r3 * r1), c3 = t3 / (-2.0 * r1 * r2);
  const double s = c1 + c2 + c3;
  const double B1a = 1.0 - s;
  const double sumb = (4.0 * (c1 * c1 * c1) - 3.0 * c1) + (4.0 * (c2 * c2 * c2) - 3.0 * c2) +
                      (4.0 * (c3 * c3 * c3) - 3.0 * c3);
  const double B1b = 1.0 - (0.625 * sumb + 0.375 * s);
  const double B2 = 1.0 / r1 + 1.0 / r2 + 1.0 / r3;
  const double B3 = (r2 - r1) * (r2 - r1) + (r3 - r2) * (r3 - r2) + (r1 - r3) * (r1 - r3);
  const double B3b = sqrt(B3 + 1e-12);
  const double e1 = exp(-kB1 * R), e2 = exp(-kB2 * Rsq), e7 = exp(-kB3 * R);
  const double vbnda = vbend(0, B1a, R, Rsq, B2, B3, B3b, e1, e2, e7);
  const double vbndb = vbend(1, B1b, R, Rsq, B2, B3, B3b, e1, e2, e7);
  double cbnda = 0.0, cbndb = 0.0;
  if (icompc >= 1) {
    const double sumT = T[0] + T[1] + T[2];
    const double P = r1 * r2 * r3, Psq = P * P, e7c = exp(-kB2 * Rcu);
    cbnda = sumT * cbend(0, B1a, R, Rsq, B2, B3, B3b, P, Psq, e1, e2, e7c);
    cbndb = sumT * cbend(1, B1b, R, Rsq, B2, B3, B3b, P, Psq, e1, e2, e7c);
  }
  return vlon + vas + vbnda + vbndb + cal + cas + cbnda + cbndb;
}

__global__ void __launch_bounds__(256) k_bkmp2_points(long n, const double *a, const double *b,
                                                      const double *c, double *v)
{
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n;
       q += (long)gridDim.x * blockDim.x)
    v[q] = bkmp2(a[q], b[q], c[q]);
}

struct Bk2Grid {
  int n1, n2, nth;
  const double *R, *r, *x;
  double f2, f3, vmax, rmin;
  int cap;
};

__global__ void __launch_bounds__(256) k_bkmp2_grid(Bk2Grid g, double *pot)
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
      v = bkmp2(r12, r23, r13) - kVH2Min;
      if (g.cap) v = fmin(v, g.vmax);
    }
    pot[q] = v;
  }
}

}  // namespace

extern "C" {

int qd_bkmp2_eval(int64_t n, const double *r1, const double *r2, const double *r3,
                  double *v_out)
{
  if (n > 0 && (!r1 || !r2 || !r3 || !v_out)) return qd_errf(QD_ERR_INVALID, "NULL argument");
  if (n <= 0) return QD_OK;
  double *d = nullptr;
  QD_CU(cudaMalloc(&d, sizeof(double) * 4 * (size_t)n));
  cudaError_t e = cudaMemcpy(d, r1, sizeof(double) * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + n, r2, sizeof(double) * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + 2 * n, r3, sizeof(double) * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    const long blocks = (n + 255) / 256;
    k_bkmp2_points<<<(unsigned)(blocks < 148 * 16 ? blocks : 148 * 16), 256>>>(n, d, d + n, d + 2 * n,
                                                                              d + 3 * n);
    qd_count_launches(1);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(v_out, d + 3 * n, sizeof(double) * n, cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return qd_errf(QD_ERR_CUDA, "qd_bkmp2_eval: %s", cudaGetErrorString(e));
  return QD_OK;
}

int qd_potential_bkmp2(const qd_radial *R, const qd_radial *r, const qd_angle *theta,
                       const double masses[3], double vmax, double rmin, int32_t cap,
                       double *pot_out)
{
  if (!R || !r || !theta || !masses || !pot_out || !R->r || !r->r || !theta->x)
    return qd_errf(QD_ERR_INVALID, "NULL argument");
  if (R->n < 1 || r->n < 1 || theta->n < 1)
    return qd_errf(QD_ERR_INVALID, "empty grid (%d x %d x %d)", R->n, r->n, theta->n);
  if (!(masses[1] + masses[2] > 0) || !(masses[2] >= 0))
    return qd_errf(QD_ERR_INVALID, "masses of the diatom atoms must be positive");
  if (!(rmin >= 0.2)) return qd_errf(QD_ERR_INVALID, "rmin must be >= 0.2 bohr for BKMP2");
  Bk2Grid g{};
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
    k_bkmp2_grid<<<(unsigned)(blocks < 148 * 16 ? blocks : 148 * 16), 256>>>(g, d);
    qd_count_launches(1);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(pot_out, d, sizeof(double) * n, cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return qd_errf(QD_ERR_CUDA, "qd_potential_bkmp2: %s", cudaGetErrorString(e));
  return QD_OK;
}

}  // extern "C"
