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

// Batches: nruns propagations on the same grid advance together.  Per run r:
//   lpsi + r * nl * n12, psi_z + r * nth * n12, surf + r * nrows * nth * n1,
//   expV / expV32 / pot + r * vrun (vrun = 0: one table shared by all runs),
//   norm_out[r].
struct ColumnParams {
  int n1, n2, nth, nl;
  long n12;
  int nruns;
  long vrun;               // per-run stride of the potential tables (0 = shared)
  void *lpsi;              // complex<R>
  double2 *psi_z;          // theta-space staging (HEAD in / TAIL out)
  const double *P;         // [nth][nl]  P_l(x_k)
  const double *WP;        // [nth][nl]  (l+1/2) w_k P_l(x_k)
  const float *P32;        // FP32 kernels: P = P32 + P32lo (float + float residual)
  const float *WP32;
  const float *P32lo;
  const float *WP32lo;
  const double2 *expV;     // FP64: exp(-i V dt) [nth][n12]
  const float2 *expV32;    // FP32: exp(-i V dt) from FP64, rounded to complex64
  const double *pot;       // HEAD: potential (FP64) for the first V phase
  double dt;
  int prestep;             // HEAD: divide by the principal sqrt(exp(-iVdt)) first
  const double *d1, *d2;   // absorbers (null = none)
  int do_flux;             // capture surface rows
  void *surf;              // complex<R> [nrows][nth][n1]
  int surf_j0, surf_nrows;
  const double *w;         // quadrature weights
  double *norm_out;        // [nruns]: accumulate sum_k w_k |psi|^2 (null = skip)
  int out_z;               // TAIL: also write psi_z
  // per-run angular basis: the P/WP matrices of run r start at
  // run_set[r] * set_stride (null: one set); run r stores l < run_nl[r]
  const int *run_set;
  long set_stride;
  const int *run_nl;
  const int *run_order;    // tensor-core pass: tile order over runs (null: 0, 1, ...)
  // energy step (null: none): per run r, esum[3 r + 2] += sum_k w_k sum_ij V |psi|^2 of the
  // theta-space wavepacket after B, before the absorber (potential_energy, timeEvol.C:256-283)
  double *esum;
};

struct FluxParams {
  int n1, nth, npts, h, nruns;
  const void *surf;        // complex<R> [run][2h+1][nth][n1]
  double den_dx;           // den * dr2 (Gradient3.F divides by it)
  double2 *ring_psi, *ring_g;   // [slot][run][nth][n1]
  int slot;                // ring slot of this step
};

// psi_s and d psi_s / dr at point Q = run*nq + k*n1 + i of the dividing
// surface from the 2h+1 captured rows: the central differences of
// Gradient3.F:31-167 with the integer coefficients summed in the same order,
// in FP64.
template <typename C>
__device__ __forceinline__ void flux_point(const FluxParams &p, int Q)
{
  const int nq = p.nth * p.n1;
  const int run = Q / nq, q = Q - run * nq;
  const int h = p.h;
  const C *s = reinterpret_cast<const C *>(p.surf) + (long)run * (2 * h + 1) * nq;
  const double2 v = to_z(s[(long)h * nq + q]);
  double gx = 0.0, gy = 0.0;
#pragma unroll
  for (int t = 0; t < 5; t++) {
    if (t >= h) break;
    const int m = h - t;   // offsets in descending order
    double c;
    switch (h) {
      case 1: c = 1.0; break;
      case 2: c = t == 0 ? -1.0 : 8.0; break;
      case 3: c = t == 0 ? 1.0 : t == 1 ? -9.0 : 45.0; break;
      case 4: c = t == 0 ? -3.0 : t == 1 ? 32.0 : t == 2 ? -168.0 : 672.0; break;
      default: c = t == 0 ? 2.0 : t == 1 ? -25.0 : t == 2 ? 150.0 : t == 3 ? -600.0 : 2100.0; break;
    }
    const double2 a = to_z(s[(long)(h + m) * nq + q]);
    const double2 b = to_z(s[(long)(h - m) * nq + q]);
    const double dx = a.x - b.x, dy = a.y - b.y;
    if (t == 0) { gx = c * dx; gy = c * dy; }   // first term exact (c * d, as Fortran's 0 + c*d)
    else { gx += c * dx; gy += c * dy; }
  }
  const long o = ((long)p.slot * p.nruns + run) * nq + q;
  p.ring_psi[o] = v;
  p.ring_g[o] = make_double2(gx / p.den_dx, gy / p.den_dx);
}

struct LineParams {
  int n1, n2, nl;
  long n12;
  int nruns;               // slices s = run * nl + l, all of the same n1 x n2
  void *lpsi;              // complex<R>, in place
  const double2 *rot;      // FP64: exp(-i l(l+1)(I1+I2) dt/2) [nl][n12]
  const double2 *kin;      // FP64: exp(-i(T1+T2)dt)/(n1 n2)    [n12]
  // FP32: separable phases from FP64, rounded once to complex64:
  //   rot = rc1[l][i] rc2[l][j],  rc1 = exp(-i l(l+1) I1 dt/2), rc2 likewise with I2
  //   kin = kc1[i] kc2[j] (kscale + kscale_lo),  kc1 = exp(-i T1 dt), kc2 likewise
  const float2 *rc1, *rc2;
  const float2 *kc1, *kc2;
  float kscale, kscale_lo; // FP32: 1/(n1 n2) = kscale + kscale_lo
  const void *tw1, *tw2;   // complex<R> root tables of n1, n2
  FftPlan pl1, pl2;
  int rows_per_cta;        // rows kernels
  int cols_per_cta;        // column kernel
  int cluster;             // l-space pass: 0 = split kernels, 1/2/4 = cluster kernel with
                           // that many CTAs per slice, SLICE_RF = register-FFT kernel
  FluxParams flux;         // fused slice kernel: flux preparation of the step ...
  int flux_ctas;           // ... by this many extra CTAs (0 = none)
  int fft_only;            // split kernels: plain forward 2-D DFT, no phases
  // centrifugal-sudden blocks: slice l of run r has j = run_k[r] + l (null: j = l);
  // the rotational tables have jrows rows
  const int *run_k;
  int jrows;
  // energy step (null: none): per run r, esum[3 r] += the kinetic energy sum (the
  // (T1 + T2) |FFT2 psi_l|^2 / (n1 n2) of kinetic_energy_for_legendre_psi,
  // timeEvol.C:390-436) and esum[3 r + 1] += sum j(j+1) (I1 + I2) |psi_l|^2 after the
  // second Rot(dt/2) (rotational_energy, timeEvol.C:323-360), both with the l-space
  // weight 1 / (l + 1/2) (orth = 0; orth = 1: the state is psi_l / sqrt(l + 1/2), weight 1)
  double *esum;
  const double *T1, *T2, *I1, *I2;
  int orth;
};

// Programmatic dependent launch: a hot kernel lets the next one start its
// prologue (trigger at entry) and waits for the previous grid (and its
// memory) before its first read of data that grid produces.  Both are no-ops
// for a kernel launched without the attribute.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
// host: whether launches carry the attribute (QD_PDL=0 turns it off)
bool pdl_enabled();

// rotational-table row of slice sl = run * nl + l, clamped to the table (the
// padded l-slices of runs with fewer angular functions hold zeros)
__device__ __forceinline__ int rot_row(const LineParams &p, int sl)
{
  const int l = sl % p.nl;
  if (!p.run_k) return l;
  const int j = p.run_k[sl / p.nl] + l;
  return j < p.jrows ? j : p.jrows - 1;
}

// energies of one run's theta-space psi (FP64): sums[0] kinetic (before the
// dr1 dr2 / (n1 n2) factor), sums[1] rotational, sums[2] potential
struct EnergyParams {
  int n1, n2, nth, nl;
  long n12;
  const double2 *psi_z;    // [nth][n2][n1]
  const double *pot;       // [nth][n2][n1]
  const double *w, *P, *WP;
  const double *T1, *T2, *I1, *I2;
  const double2 *tw1, *tw2;
  FftPlan pl1, pl2;
  double2 *scratch;        // nth * n12
  double *sums;            // 3
  int K;                   // centrifugal-sudden block: j = K + l in E_rot
};
cudaError_t launch_energies(const EnergyParams &e, cudaStream_t s);
int energies_launches();

// per run r: energies/eta_sq/crp + r * ne, fai/dfai + r * ne * nq,
// ring slot t of run r at (t * nruns + r) * nq
struct AccumParams {
  int nq;                  // nth * n1
  int ne;
  int nruns;
  int nt;                  // steps in this chunk
  long t0;                 // accumulations done before this chunk
  double dt;
  const double *energies;
  const double2 *ring_psi, *ring_g;
  double2 *fai, *dfai;
  double2 *phase;          // workspace [nruns][ne][FLUX_CHUNK] for the chunk's e^{iEt} factors
  int variant;             // GEMM tile variant, 0 .. flux_variants() - 1 (the autotuner's choice)
  // chirp-z form (energies on a uniform grid per run; null czt_b: the GEMM form)
  const double2 *czt_tw;   // [CZT_N] e^{-2 pi i m / CZT_N}
  const double2 *czt_g;    // [nruns][FLUX_CHUNK] e^{i E_0 t dt} c(t)
  const double2 *czt_b;    // [nruns][CZT_N] FFT of b_k = conj(c(k)), divided by CZT_N
  const double *czt_de;    // [nruns] energy spacing dE; c(k) = e^{i dE dt k^2 / 2}
  // P(E) of the updated accumulators fused into the GEMM form (null: off):
  // crp_part[run][e][q tile] = the tile's sum of w_k Im(conj(phi) dphi)
  double *crp_part;
  const double *w;         // theta weights (with crp_part)
  int n1;                  // surface points per theta row (with crp_part)
};
constexpr int CZT_N = 512;       // cyclic convolution length of the chirp-z form
constexpr int CZT_MIN_STEPS = 125;   // chunks of fewer steps take the GEMM form
// tables of the chirp-z form for runs with energies e0[r] + j de[r], j < ne
cudaError_t launch_czt_tables(int nruns, int ne, double dt, const double *e0, const double *de,
                              double2 *tw, double2 *g, double2 *b, cudaStream_t s);
int flux_accum_launches();
int flux_variants();
bool flux_accum_is_czt(const AccumParams &p);   // the chunk takes the chirp-z form
int flux_q_tiles(int nq);                       // surface-point tiles of the GEMM form

struct CrpParams {
  int n1, nth, ne, nruns;
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
// P(E) from the per-tile sums that a fused GEMM-form accumulation wrote
cudaError_t launch_crp_parts(const CrpParams &p, const double *part, int nqt, cudaStream_t s);

// set-up kernels
cudaError_t launch_setup_tables_fp64(int n1, int n2, int nth, int nl, double dt,
                                     const double *pot, const double *I1, const double *I2,
                                     const double *T1, const double *T2, double2 *expV,
                                     double2 *rot, double2 *kin, cudaStream_t s);
cudaError_t launch_setup_tables_fp32(int n1, int n2, int nth, int nl, double dt,
                                     const double *pot, const double *I1, const double *I2,
                                     const double *T1, const double *T2, float2 *expV32,
                                     float2 *rc1, float2 *rc2, float2 *kc1, float2 *kc2,
                                     cudaStream_t s);
// fused slice kernel (FP32): CTAs per slice it can run with for these sizes
// (0 if none), its launch, and the smem bytes it needs
// steps of flux history accumulated into phi_E by one GEMM launch (the ring
// of surface rows and the e^{iEt} table hold that many steps)
constexpr int FLUX_CHUNK = 250;
constexpr int SLICE_RF = 8;    // LineParams::cluster value of the register-FFT slice kernel
constexpr int SLICE_RF2 = 9;   // the same on a 2-CTA cluster per slice
constexpr int SLICE_RF4 = 10;  // the same on a 4-CTA cluster per slice
constexpr int SLICE_RF4W = 11; // the 4-CTA form with 16 x 16 row transforms
inline bool slice_is_rf(int cluster)
{
  return cluster == SLICE_RF || cluster == SLICE_RF2 || cluster == SLICE_RF4 ||
         cluster == SLICE_RF4W;
}
inline int slice_ctas(int cluster)           // CTAs per slice
{
  return cluster == SLICE_RF ? 1 : cluster == SLICE_RF2 ? 2
       : cluster == SLICE_RF4 || cluster == SLICE_RF4W ? 4 : cluster;
}
int slice_cluster_ok(int n1, int n2, int cluster);
int slice_rf_threads(int n1, int n2, int cl); // threads per CTA, 0 if the shape is not built
int slice_threads(int n1, int n2, int cluster);
cudaError_t launch_slice_rf(const LineParams &p, int cl, cudaStream_t s);
bool slice_rf_wide_ok(int n1, int n2);
cudaError_t launch_slice_rf_wide(const LineParams &p, cudaStream_t s);
cudaError_t launch_slice(const LineParams &p, cudaStream_t s);
cudaError_t launch_legendre_matrices(int nth, int nl, const double *x, const double *w,
                                     const double *legendre, double *P, double *WP,
                                     float *P32, float *WP32, float *P32lo, float *WP32lo,
                                     cudaStream_t s);
// complex64 <-> complex128 copies of the theta-space state (n complex values)
cudaError_t launch_widen_c(const float2 *src, double2 *dst, size_t n, cudaStream_t s);
cudaError_t launch_narrow_c(const double2 *src, float2 *dst, size_t n, cudaStream_t s);
cudaError_t launch_legendre_basis(int n, int K, int m, const double *x, double *legendre,
                                  cudaStream_t s);
cudaError_t launch_roots(int n, double2 *tw64, float2 *tw32, cudaStream_t s);
// read a buffer through L2 (the clean-up half of the timed L2 flush)
cudaError_t launch_l2_read(const void *buf, size_t bytes, cudaStream_t s);

// number of kernel launches that launch_lines<R> issues per call
int lines_launches_per_step(int n1, int n2, int prec);
