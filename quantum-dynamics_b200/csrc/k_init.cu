// k_init.cu -- the initial state of a propagation on the GPU, in FP64 (the
// Matlab-side set-up of the reference):
//   diatom eigenstate phi_vj(r): sinc-DVR Hamiltonian (H3/H2VibRotWaveFunction.m:20-46)
//     T_ii = pi^2/3 - 1/(2 i^2),  T_ij = (-1)^(i-j) (2/(i-j)^2 - 2/(i+j)^2),
//     H = T/(2 mu dr^2) + V_diatom(r) + j(j+1)/(2 mu r^2),
//   diagonalised by a parallel cyclic Jacobi method in one CTA (rounds of n/2
//   disjoint rotations, round-robin pairing; the matrix and the accumulated
//   eigenvectors in global memory, L2-resident, ordered by the CTA's
//   barriers); the v-th lowest state, largest component made positive,
//   divided by sqrt(dr).
//   packet psi(R, r, theta_k) = g(R) phi_vj(r) Pbar_j^K(x_k), g = (pi delta^2)^(-1/4)
//     exp(-(R-R0)^2/(2 delta^2) - i k0 R) (H3/InitWavePacket.m:13-31; Pbar_j^0 =
//     sqrt(j+1/2) P_j),
//   eta^2(E) = |pi^(1/4) sqrt(2 mu delta / k) exp(-delta^2 (k - k0)^2 / 2)|^2,
//     k = sqrt(2 mu E_coll) (common/EtaSq.m:12-15, complex for E_coll < 0).
#include <cmath>
#include "qd_err.h"

namespace {

constexpr int JAC_THREADS = 256;
constexpr int JAC_MAX_SWEEPS = 40;

// A and V (n x n, row stride n+1 and n) in global memory; rotation data in
// dynamic shared memory
__global__ void __launch_bounds__(JAC_THREADS) k_dvr_jacobi(int n, double mu, double dr,
                                                            const double *r, const double *vd,
                                                            int jrot, int v, double *A, double *V,
                                                            double *phi, double *e_out,
                                                            int *status)
{
  extern __shared__ double sm[];
  const int ld = n + 1;
  double *cs = sm;                             // [n/2] c
  double *sn = cs + n / 2;                     // [n/2] s
  double *red = sn + n / 2;                    // [32]
  int *pp = reinterpret_cast<int *>(red + 32); // [n/2] p, then [n/2] q
  int *qq = pp + n / 2;
  const int tid = threadIdx.x;
  const double pi = 3.141592653589793238462643383279502884;
  const double kin = 1.0 / (2.0 * mu * dr * dr);
  for (int x = tid; x < n * n; x += JAC_THREADS) {
    const int a = x / n, b = x % n;
    const double ia = a + 1, ib = b + 1;
    double h;
    if (a == b) {
      h = (pi * pi / 3.0 - 1.0 / (2.0 * ia * ia)) * kin + vd[a] +
          jrot * (jrot + 1.0) / (2.0 * mu * r[a] * r[a]);
    } else {
      const double d = ia - ib, s = ia + ib;
      h = (((a - b) & 1) ? -1.0 : 1.0) * (2.0 / (d * d) - 2.0 / (s * s)) * kin;
    }
    A[a * ld + b] = h;
    V[(long)a * n + b] = a == b ? 1.0 : 0.0;
  }
  __syncthreads();
  double off0 = 0.0;
  int sweep = 0;
  for (; sweep < JAC_MAX_SWEEPS; sweep++) {
    // off-diagonal and total norms
    double o = 0.0, t = 0.0;
    for (int x = tid; x < n * n; x += JAC_THREADS) {
      const int a = x / n, b = x % n;
      const double e = A[a * ld + b];
      t += e * e;
      if (a != b) o += e * e;
    }
    for (int m = 16; m > 0; m >>= 1) {
      o += __shfl_xor_sync(0xffffffffu, o, m);
      t += __shfl_xor_sync(0xffffffffu, t, m);
    }
    if ((tid & 31) == 0) { red[tid >> 5] = o; red[16 + (tid >> 5)] = t; }
    __syncthreads();
    double ot = 0.0, tt = 0.0;
    for (int w = 0; w < JAC_THREADS / 32; w++) { ot += red[w]; tt += red[16 + w]; }
    __syncthreads();
    if (sweep == 0) off0 = ot;
    if (ot <= 1e-30 * tt || ot == 0.0) break;
    for (int round = 0; round < n - 1; round++) {
      // round-robin pairs: position 0 fixed, the others rotate
      for (int i = tid; i < n / 2; i += JAC_THREADS) {
        auto pos = [&](int j) { return j == 0 ? 0 : 1 + (j - 1 + round) % (n - 1); };
        int p = pos(i), q = pos(n - 1 - i);
        if (p > q) { const int x = p; p = q; q = x; }
        const double apq = A[p * ld + q];
        double c = 1.0, s = 0.0;
        if (apq != 0.0) {
          const double th = (A[q * ld + q] - A[p * ld + p]) / (2.0 * apq);
          const double tn = (th >= 0.0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1.0));
          c = 1.0 / sqrt(tn * tn + 1.0);
          s = tn * c;
        }
        pp[i] = p; qq[i] = q; cs[i] = c; sn[i] = s;
      }
      __syncthreads();
      // rows p, q of A
      for (int x = tid; x < (n / 2) * n; x += JAC_THREADS) {
        const int i = x / n, k = x % n;
        const int p = pp[i], q = qq[i];
        const double c = cs[i], s = sn[i], ap = A[p * ld + k], aq = A[q * ld + k];
        A[p * ld + k] = c * ap - s * aq;
        A[q * ld + k] = s * ap + c * aq;
      }
      __syncthreads();
      // columns p, q of A and of V
      for (int x = tid; x < (n / 2) * n; x += JAC_THREADS) {
        const int i = x / n, k = x % n;
        const int p = pp[i], q = qq[i];
        const double c = cs[i], s = sn[i];
        const double ap = A[k * ld + p], aq = A[k * ld + q];
        A[k * ld + p] = c * ap - s * aq;
        A[k * ld + q] = s * ap + c * aq;
        const double vp = V[(long)k * n + p], vq = V[(long)k * n + q];
        V[(long)k * n + p] = c * vp - s * vq;
        V[(long)k * n + q] = s * vp + c * vq;
      }
      __syncthreads();
    }
  }
  __syncthreads();
  // the v-th lowest eigenvalue (ties by index) and its vector
  __shared__ int pick;
  if (tid == 0) pick = -1;
  __syncthreads();
  for (int i = tid; i < n; i += JAC_THREADS) {
    const double li = A[i * ld + i];
    int rank = 0;
    for (int j = 0; j < n; j++) {
      const double lj = A[j * ld + j];
      if (lj < li || (lj == li && j < i)) rank++;
    }
    if (rank == v) pick = i;
  }
  __syncthreads();
  if (pick < 0) {
    if (tid == 0) *status = 2;
    return;
  }
  // sign: the largest-magnitude component positive
  if (tid == 0) {
    int imax = 0;
    double amax = 0.0;
    for (int k = 0; k < n; k++) {
      const double a = fabs(V[(long)k * n + pick]);
      if (a > amax) { amax = a; imax = k; }
    }
    red[0] = V[(long)imax * n + pick] < 0.0 ? -1.0 : 1.0;
    *e_out = A[pick * ld + pick];
    *status = sweep >= JAC_MAX_SWEEPS ? 1 : 0;
    (void)off0;
  }
  __syncthreads();
  const double sg = red[0] / sqrt(dr);
  for (int k = tid; k < n; k += JAC_THREADS) phi[k] = V[(long)k * n + pick] * sg;
}

// Pbar_j^K(x) normalised to one on [-1, 1], no Condon-Shortley phase
__device__ double pbar(int j, int K, double x)
{
  double p0 = sqrt(0.5);
  const double s = sqrt(fmax(0.0, 1.0 - x * x));
  for (int m = 1; m <= K; m++) p0 *= sqrt((2.0 * m + 1.0) / (2.0 * m)) * s;
  if (j == K) return p0;
  double p1 = sqrt(2.0 * K + 3.0) * x * p0;
  for (int l = K + 2; l <= j; l++) {
    const double a = sqrt((4.0 * l * l - 1.0) / ((double)l * l - (double)K * K));
    const double b = sqrt(((l - 1.0) * (l - 1.0) - (double)K * K) / (4.0 * (l - 1.0) * (l - 1.0) - 1.0));
    const double p2 = a * (x * p1 - b * p0);
    p0 = p1;
    p1 = p2;
  }
  return p1;
}

__global__ void k_packet(int n1, int n2, int nth, const double *R, double r0, double k0,
                         double delta, const double *x, int j0, int K, const double *phi,
                         double2 *psi)
{
  const long n = (long)n1 * n2 * nth;
  const double pi = 3.141592653589793238462643383279502884;
  const double amp = pow(1.0 / (pi * delta * delta), 0.25);
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n;
       q += (long)gridDim.x * blockDim.x) {
    const int i = (int)(q % n1), j = (int)((q / n1) % n2), k = (int)(q / ((long)n1 * n2));
    const double d = R[i] - r0;
    const double mag = amp * exp(-d * d / (2.0 * delta * delta));
    double sn, cs;
    sincos(-k0 * R[i], &sn, &cs);
    const double ang = K <= j0 ? pbar(j0, K, x[k]) : 0.0;
    const double f = mag * phi[j] * ang;
    psi[q] = make_double2(f * cs, f * sn);
  }
}

__global__ void k_eta_sq(int ne, const double *e, double mu, double delta, double k0, double *out)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ne) return;
  const double pi = 3.141592653589793238462643383279502884;
  // k = sqrt(2 mu E) as a complex number: real for E >= 0, i sqrt(-2 mu E) below
  const double a = 2.0 * mu * e[i];
  const double kr = a >= 0.0 ? sqrt(a) : 0.0, ki = a >= 0.0 ? 0.0 : sqrt(-a);
  // |sqrt(2 mu delta / k)|^2 = 2 mu delta / |k|
  const double kabs = sqrt(kr * kr + ki * ki);
  // |exp(-delta^2 (k - k0)^2 / 2)|^2 = exp(-delta^2 Re((k - k0)^2))
  const double dr = kr - k0, re2 = dr * dr - ki * ki;
  out[i] = sqrt(pi) * (2.0 * mu * delta / kabs) * exp(-delta * delta * re2);
}

}  // namespace

extern "C" {

int qd_init_state(const qd_radial *R, const qd_radial *r, const qd_angle *theta, int32_t j0,
                  int32_t v0, int32_t K, const double *v_diatom, double *psi_out,
                  double *e_vj_out, double *phi_out)
{
  if (!R || !r || !theta || !R->r || !r->r || !theta->x || !v_diatom || !psi_out)
    return qd_errf(QD_ERR_INVALID, "qd_init_state: NULL argument");
  const int n1 = R->n, n2 = r->n, nth = theta->n;
  if (n1 < 1 || n2 < 2 || nth < 1 || n2 % 2 || n2 > 4096 || j0 < 0 || v0 < 0 || v0 >= n2 ||
      K < 0 || !(r->dr > 0) || !(r->mass > 0) || !(R->delta > 0))
    return qd_errf(QD_ERR_INVALID, "qd_init_state: bad sizes or parameters (r2.n even)");
  const size_t smem = sizeof(double) * ((size_t)n2 + 32) + sizeof(int) * n2;
  const long npt = (long)n1 * n2 * nth;
  double *d = nullptr;
  const size_t nd = 2 * npt + (size_t)n2 * (n2 + 1) + (size_t)n2 * n2 + 3 * n2 + n1 + nth + 2;
  QD_CU(cudaMalloc(&d, sizeof(double) * nd));
  double2 *dpsi = reinterpret_cast<double2 *>(d);          // first: 16-byte aligned
  double *dA = d + 2 * npt, *dV = dA + (size_t)n2 * (n2 + 1), *dr_ = dV + (size_t)n2 * n2,
         *dvd = dr_ + n2, *dphi = dvd + n2;
  double *dR = dphi + n2, *dx = dR + n1, *de = dx + nth;
  int *dstat = reinterpret_cast<int *>(de + 1);
  cudaError_t e = cudaFuncSetAttribute(k_dvr_jacobi, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e == cudaSuccess) e = cudaMemcpy(dr_, r->r, sizeof(double) * n2, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dvd, v_diatom, sizeof(double) * n2, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dR, R->r, sizeof(double) * n1, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dx, theta->x, sizeof(double) * nth, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(dstat, 0xff, sizeof(int));
  if (e == cudaSuccess) {
    k_dvr_jacobi<<<1, JAC_THREADS, smem>>>(n2, r->mass, r->dr, dr_, dvd, j0, v0, dA, dV, dphi,
                                           de, dstat);
    k_packet<<<(unsigned)((npt + 255) / 256 < 148 * 16 ? (npt + 255) / 256 : 148 * 16), 256>>>(
        n1, n2, nth, dR, R->r0, R->k0, R->delta, dx, j0, K, dphi, dpsi);
    qd_count_launches(2);
    e = cudaGetLastError();
  }
  int st = 0;
  double evj = 0.0;
  if (e == cudaSuccess) e = cudaMemcpy(&st, dstat, sizeof(int), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(&evj, de, sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(psi_out, dpsi, sizeof(double2) * npt, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && phi_out) e = cudaMemcpy(phi_out, dphi, sizeof(double) * n2, cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return qd_errf(QD_ERR_CUDA, "qd_init_state: %s", cudaGetErrorString(e));
  if (st != 0)
    return qd_errf(QD_ERR_NONFINITE, "qd_init_state: diatom eigensolver %s",
                   st == 1 ? "did not converge" : "found no such state");
  if (e_vj_out) *e_vj_out = evj;
  return QD_OK;
}

int qd_eta_sq(const qd_radial *R, int32_t ne, const double *e_coll, double *eta_sq_out)
{
  if (!R || !e_coll || !eta_sq_out || ne < 1 || !(R->mass > 0) || !(R->delta > 0))
    return qd_errf(QD_ERR_INVALID, "qd_eta_sq: bad argument");
  double *d = nullptr;
  QD_CU(cudaMalloc(&d, sizeof(double) * 2 * ne));
  cudaError_t e = cudaMemcpy(d, e_coll, sizeof(double) * ne, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    k_eta_sq<<<(ne + 255) / 256, 256>>>(ne, d, R->mass, R->delta, R->k0, d + ne);
    qd_count_launches(1);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(eta_sq_out, d + ne, sizeof(double) * ne, cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return qd_errf(QD_ERR_CUDA, "qd_eta_sq: %s", cudaGetErrorString(e));
  return QD_OK;
}

}  // extern "C"
