// qd_kernels.h -- launch interface of the propagator kernels (host side).
//
// Device layout of one propagation (n12 = n1*n2 grid columns, p = j*n1 + i):
//   lpsi   [n_l][n2][n1]      complex<R>  l-space wavepacket (state between steps)
//   psi_z  [n_th][n2][n1]     complex128  theta-space staging (user layout)
//   surf   [2h+1][n_th][n1]   complex<R>  dividing-surface rows of one step
//   ring   [C][n_th][n1]      complex128  psi_s / dpsi_s history for the E-accumulation
//   fai    [n_E][n_th][n1]    complex128  phi_E, dphi_E
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "qd_device.cuh"

// Column pass modes
enum ColumnMode {
  COL_HEAD = 0,   // psi_z (theta) -> [pre-step] -> V -> F -> lpsi
  COL_MID = 1,    // lpsi -> B -> dump -> [flux, norm] -> V -> F -> lpsi
  COL_TAIL = 2,   // lpsi -> B -> dump -> [flux, norm] (-> psi_z if out_z)
};

struct ColumnParams {
  int n1, n2, nth, nl;
  long n12;
  void *lpsi;              // complex<R>
  double2 *psi_z;          // theta-space staging (HEAD in / TAIL out)
  const double *P;         // [nth][nl]  P_l(x_k)
  const double *WP;        // [nth][nl]  (l+1/2) w_k P_l(x_k)
  const float *P32;        // FP32 kernels: P = P32 + P32lo (float + float residual)
  const float *WP32;
  const float *P32lo;
  const float *WP32lo;
  const double2 *expV;     // FP64: exp(-i V dt) [nth][n12]
  const float *vturn;      // FP32: -V dt / 2 pi reduced to [-1/2, 1/2) turns
  const double *pot;       // HEAD: potential (FP64) for the first V phase
  double dt;
  int prestep;             // HEAD: divide by the principal sqrt(exp(-iVdt)) first
  const double *d1, *d2;   // absorbers (null = none)
  int do_flux;             // capture surface rows
  void *surf;              // complex<R> [nrows][nth][n1]
  int surf_j0, surf_nrows;
  const double *w;         // quadrature weights
  double *norm_out;        // accumulate sum_k w_k |psi|^2 (null = skip)
  int out_z;               // TAIL: also write psi_z
};

struct LineParams {
  int n1, n2, nl;
  long n12;
  void *lpsi;              // complex<R>, in place
  const double2 *rot;      // FP64: exp(-i l(l+1)(I1+I2) dt/2) [nl][n12]
  const double2 *kin;      // FP64: exp(-i(T1+T2)dt)/(n1 n2)    [n12]
  const float *rt1, *rt2;  // FP32: rotational phase turns [nl][n1], [nl][n2]
  const float *kt1, *kt2;  // FP32: kinetic phase turns [n1], [n2]
  float kscale, kscale_lo; // FP32: 1/(n1 n2) = kscale + kscale_lo
  const void *tw1, *tw2;   // complex<R> root tables of n1, n2
  FftPlan pl1, pl2;
  int rows_per_cta;        // rows kernels
  int cols_per_cta;        // column kernel
};

struct FluxParams {
  int n1, nth, npts, h;
  const void *surf;        // complex<R> [2h+1][nth][n1]
  double den_dx;           // den * dr2 (Gradient3.F divides by it)
  double2 *ring_psi, *ring_g;
  int slot;                // ring slot of this step
};

struct AccumParams {
  int nq;                  // nth * n1
  int ne;
  int nt;                  // steps in this chunk
  long t0;                 // accumulations done before this chunk
  double dt;
  const double *energies;
  const double2 *ring_psi, *ring_g;
  double2 *fai, *dfai;
};

struct CrpParams {
  int n1, nth, ne;
  const double *w, *eta_sq;
  double dr1_mu2;
  const double2 *fai, *dfai;
  double *crp;
};

// launchers (return cudaGetLastError() after the launch)
template <typename R> cudaError_t launch_column(const ColumnParams &p, int mode, cudaStream_t s);
template <typename R> cudaError_t launch_lines(const LineParams &p, cudaStream_t s);
template <typename R> cudaError_t launch_flux_prep(const FluxParams &p, cudaStream_t s);
cudaError_t launch_flux_accum(const AccumParams &p, cudaStream_t s);
cudaError_t launch_crp(const CrpParams &p, cudaStream_t s);

// set-up kernels
cudaError_t launch_setup_tables_fp64(int n1, int n2, int nth, int nl, double dt,
                                     const double *pot, const double *I1, const double *I2,
                                     const double *T1, const double *T2, double2 *expV,
                                     double2 *rot, double2 *kin, cudaStream_t s);
cudaError_t launch_setup_tables_fp32(int n1, int n2, int nth, int nl, double dt,
                                     const double *pot, const double *I1, const double *I2,
                                     const double *T1, const double *T2, float *vturn,
                                     float *rt1, float *rt2, float *kt1, float *kt2,
                                     cudaStream_t s);
cudaError_t launch_legendre_matrices(int nth, int nl, const double *x, const double *w,
                                     const double *legendre, double *P, double *WP,
                                     float *P32, float *WP32, float *P32lo, float *WP32lo,
                                     cudaStream_t s);
cudaError_t launch_legendre_p2(int n, int m, const double *x, double *legendre, cudaStream_t s);
cudaError_t launch_roots(int n, double2 *tw64, float2 *tw32, cudaStream_t s);

// number of kernel launches that launch_lines<R> issues per call
int lines_launches_per_step(int n1, int n2, int prec);
