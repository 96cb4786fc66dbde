// k_flux.cu -- flux through the dividing surface r = r_s and P(E).
//
//   k_flux_prep    psi_s(i,k) and d psi_s/dr by the central differences of
//                  Gradient3.F:31-167 (3..11 points, same coefficient order),
//                  from the surface rows captured by the column pass; stored
//                  in FP64 in a history ring (one slot per step).
//   k_flux_accum   phi_E += sum_t dt e^{iE t} psi_s(t), dphi_E likewise
//                  (PsiTimeToPsiEnergyOnSurface, CRPAux.F:4-31, with the
//                  e^{iEt} recurrence of timeEvol.C:807-817 evaluated
//                  directly): a complex FP64 GEMM over a chunk of steps.
//   k_crp          P(E) = Im(sum_k w_k sum_i conj(phi) dphi) / eta^2 dr1/mu2
//                  (CalculateCRP, CRPAux.F:34-66), warp-shuffle reduction.
#include "qd_kernels.h"

namespace {

template <typename R>
__global__ void k_flux_prep(FluxParams p)
{
  typedef typename Cplx<R>::T C;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < p.nruns * p.nth * p.n1) flux_point<C>(p, q);
}

constexpr int EB = 8;          // energies per CTA
constexpr int TMAX = 128;      // max steps per chunk

__global__ void __launch_bounds__(256) k_flux_accum(AccumParams p)
{
  __shared__ double2 ph[EB][TMAX];
  const int e0 = blockIdx.y * EB;
  const int run = blockIdx.z;
  const double *energies = p.energies + (long)run * p.ne;
  for (int x = threadIdx.x; x < EB * p.nt; x += blockDim.x) {
    const int e = x / p.nt, t = x % p.nt;
    double2 c = make_double2(0.0, 0.0);
    if (e0 + e < p.ne) {
      const double edt = energies[e0 + e] * p.dt;
      double sn, cs;
      sincos(edt * (double)(p.t0 + t + 1), &sn, &cs);
      c = make_double2(p.dt * cs, p.dt * sn);
    }
    ph[e][t] = c;
  }
  __syncthreads();
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= p.nq) return;
  double2 a[EB], b[EB];
#pragma unroll
  for (int e = 0; e < EB; e++) { a[e] = make_double2(0, 0); b[e] = make_double2(0, 0); }
  for (int t = 0; t < p.nt; t++) {
    const long o = ((long)t * p.nruns + run) * p.nq + q;
    const double2 zp = p.ring_psi[o];
    const double2 zg = p.ring_g[o];
#pragma unroll
    for (int e = 0; e < EB; e++) {
      const double2 c = ph[e][t];
      a[e].x += c.x * zp.x - c.y * zp.y; a[e].y += c.x * zp.y + c.y * zp.x;
      b[e].x += c.x * zg.x - c.y * zg.y; b[e].y += c.x * zg.y + c.y * zg.x;
    }
  }
#pragma unroll
  for (int e = 0; e < EB; e++) {
    if (e0 + e >= p.ne) break;
    const long o = ((long)run * p.ne + e0 + e) * p.nq + q;
    double2 f = p.fai[o], df = p.dfai[o];
    f.x += a[e].x; f.y += a[e].y; df.x += b[e].x; df.y += b[e].y;
    p.fai[o] = f; p.dfai[o] = df;
  }
}

__global__ void __launch_bounds__(256) k_crp(CrpParams p)
{
  __shared__ double red[32];
  const int b = blockIdx.x;                    // run * ne + e
  const long nq = (long)p.nth * p.n1;
  const double2 *f = p.fai + (long)b * nq, *df = p.dfai + (long)b * nq;
  double s = 0.0;
  for (long q = threadIdx.x; q < nq; q += blockDim.x) {
    const int k = (int)(q / p.n1);
    const double2 a = f[q], b = df[q];
    s += p.w[k] * (a.x * b.y - a.y * b.x);   // Im(conj(phi) dphi)
  }
  s = block_sum(s, red);
  if (threadIdx.x == 0) p.crp[b] = s / p.eta_sq[b] * p.dr1_mu2;
}

}  // namespace

template <typename R>
cudaError_t launch_flux_prep(const FluxParams &p, cudaStream_t s)
{
  const int nq = p.nruns * p.nth * p.n1;
  k_flux_prep<R><<<(nq + 255) / 256, 256, 0, s>>>(p);
  return cudaGetLastError();
}
template cudaError_t launch_flux_prep<float>(const FluxParams &, cudaStream_t);
template cudaError_t launch_flux_prep<double>(const FluxParams &, cudaStream_t);

cudaError_t launch_flux_accum(const AccumParams &p, cudaStream_t s)
{
  if (p.nt <= 0) return cudaSuccess;
  if (p.nt > TMAX) return cudaErrorInvalidValue;
  dim3 grid((p.nq + 255) / 256, (p.ne + EB - 1) / EB, p.nruns);
  k_flux_accum<<<grid, 256, 0, s>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_crp(const CrpParams &p, cudaStream_t s)
{
  k_crp<<<p.nruns * p.ne, 256, 0, s>>>(p);
  return cudaGetLastError();
}
