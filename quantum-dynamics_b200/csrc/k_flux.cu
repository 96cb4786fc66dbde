// k_flux.cu -- flux through the dividing surface r = r_s and P(E).
//
//   k_flux_prep    psi_s(i,k) and d psi_s/dr by the central differences of
//                  Gradient3.F:31-167 (3..11 points, same coefficient order),
//                  from the surface rows captured by the column pass; stored
//                  in FP64 in a history ring (one slot per step).
//   k_flux_phase   the factors dt e^{iE t} of a chunk of steps (the e^{iEt}
//                  recurrence of timeEvol.C:807-817 evaluated directly, FP64)
//   k_flux_gemm    phi_E += sum_t dt e^{iE t} psi_s(t), dphi_E likewise
//                  (PsiTimeToPsiEnergyOnSurface, CRPAux.F:4-31): a
//                  register-tiled complex FP64 GEMM over the chunk.
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

constexpr int TMAX = FLUX_CHUNK;   // max steps per chunk

// phase[run][e][t] = dt e^{i E_e (t0 + t + 1) dt} of this chunk, FP64
__global__ void __launch_bounds__(256) k_flux_phase(AccumParams p)
{
  const int n = p.nruns * p.ne * p.nt;
  for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < n; x += gridDim.x * blockDim.x) {
    const int t = x % p.nt, re = x / p.nt;                 // re = run * ne + e
    double sn, cs;
    sincos(p.energies[re] * p.dt * (double)(p.t0 + t + 1), &sn, &cs);
    p.phase[(size_t)re * TMAX + t] = make_double2(p.dt * cs, p.dt * sn);
  }
}

// phi[e][q] += sum_t phase[e][t] psi_s[t][q] (and dphi with the gradient), a
// complex FP64 GEMM per run.  CTA tile: GE energies x GQ surface points x
// {psi_s, d psi_s}; each thread owns 4 energies x 4 columns (2 points x 2
// fields) in registers, GE / 4 x 16 threads.  KT steps of phases and history
// are staged in shared memory by asynchronous copies into two buffers, so the
// next KT steps load while the current ones are multiplied; the history is
// read from HBM once per energy tile.  The variant (GE, KT) is picked per
// shape by the autotuner.
constexpr int GQ = 32;

__device__ __forceinline__ void cp16(void *dst, const void *src, bool valid)
{
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  const int n = valid ? 16 : 0;                 // 0: fill the 16 bytes with zeros
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;" :: "r"(d), "l"(src), "r"(n)
               : "memory");
}

template <int GE, int KT>
__global__ void __launch_bounds__(GE * 4) k_flux_gemm(AccumParams p)
{
  constexpr int NT = GE * 4;                    // threads: GE / 4 energy groups x 16
  __shared__ double2 As[2][GE][KT + 1];         // phases (padded rows)
  __shared__ double2 Bs[2][KT][2 * GQ];         // cols 0..GQ-1 psi_s, GQ..2GQ-1 gradient
  const int tid = threadIdx.x;
  const int te = tid >> 4, tc = tid & 15;       // GE/4 energy groups x 16 column groups
  const int e0 = blockIdx.x * GE, q0 = blockIdx.y * GQ, run = blockIdx.z;
  const double2 *ph = p.phase + ((size_t)run * p.ne) * TMAX;
  auto stage = [&](int buf, int t0) {
    for (int x = tid; x < GE * KT; x += NT) {
      const int e = x / KT, t = x % KT;
      const bool ok = e0 + e < p.ne && t0 + t < p.nt;
      cp16(&As[buf][e][t], ok ? ph + (size_t)(e0 + e) * TMAX + t0 + t : ph, ok);
    }
    for (int x = tid; x < KT * 2 * GQ; x += NT) {
      const int t = x / (2 * GQ), c = x % (2 * GQ), q = q0 + (c % GQ);
      const bool ok = t0 + t < p.nt && q < p.nq;
      const size_t o = ok ? ((size_t)(t0 + t) * p.nruns + run) * p.nq + q : 0;
      cp16(&Bs[buf][t][c], (c < GQ ? p.ring_psi : p.ring_g) + o, ok);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  double2 acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) acc[i][j] = make_double2(0.0, 0.0);
  const int nchunk = (p.nt + KT - 1) / KT;
  stage(0, 0);
  for (int ch = 0; ch < nchunk; ch++) {
    const int buf = ch & 1;
    if (ch + 1 < nchunk) {
      stage(buf ^ 1, (ch + 1) * KT);
      asm volatile("cp.async.wait_group 1;" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    }
    __syncthreads();
#pragma unroll 2
    for (int k = 0; k < KT; k++) {             // rows past nt were zero-filled
      double2 a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; i++) a[i] = As[buf][te + (GE / 4) * i][k];
#pragma unroll
      for (int j = 0; j < 4; j++) b[j] = Bs[buf][k][tc + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) {
          acc[i][j].x = fma(a[i].x, b[j].x, fma(-a[i].y, b[j].y, acc[i][j].x));
          acc[i][j].y = fma(a[i].x, b[j].y, fma(a[i].y, b[j].x, acc[i][j].y));
        }
    }
    __syncthreads();                            // buffer free for the stage after next
  }
  // phi += acc, two energy rows at a time: their eight loads are all issued
  // before any of their stores (a store between two loads would make each
  // load wait for the one before, since phi and dphi may alias as far as the
  // compiler knows)
  auto at = [&](int i, int j) -> double2 * {
    const int e = e0 + te + (GE / 4) * i, c = tc + 16 * j, q = q0 + (c % GQ);
    if (e >= p.ne || q >= p.nq) return nullptr;
    return (c < GQ ? p.fai : p.dfai) + ((size_t)run * p.ne + e) * p.nq + q;
  };
#pragma unroll
  for (int h = 0; h < 4; h += 2) {
#pragma unroll
    for (int i = h; i < h + 2; i++)
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const double2 *src = at(i, j);
        if (src) {
          const double2 f = *src;
          acc[i][j].x += f.x;
          acc[i][j].y += f.y;
        }
      }
#pragma unroll
    for (int i = h; i < h + 2; i++)
#pragma unroll
      for (int j = 0; j < 4; j++) {
        double2 *dst = at(i, j);
        if (dst) *dst = acc[i][j];
      }
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

template <int GE, int KT> void launch_gemm(const AccumParams &p, cudaStream_t s)
{
  dim3 grid((p.ne + GE - 1) / GE, (p.nq + GQ - 1) / GQ, p.nruns);
  k_flux_gemm<GE, KT><<<grid, GE * 4, 0, s>>>(p);
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

int flux_variants() { return 4; }

cudaError_t launch_flux_accum(const AccumParams &p, cudaStream_t s)
{
  if (p.nt <= 0) return cudaSuccess;
  if (p.nt > TMAX) return cudaErrorInvalidValue;
  const int n = p.nruns * p.ne * p.nt;
  k_flux_phase<<<(n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096, 256, 0, s>>>(p);
  switch (p.variant) {   // (energies per CTA, steps per staged chunk)
    case 1: launch_gemm<64, 5>(p, s); break;
    case 2: launch_gemm<32, 10>(p, s); break;
    case 3: launch_gemm<32, 15>(p, s); break;
    default: launch_gemm<64, 10>(p, s); break;
  }
  return cudaGetLastError();
}

cudaError_t launch_crp(const CrpParams &p, cudaStream_t s)
{
  k_crp<<<p.nruns * p.ne, 256, 0, s>>>(p);
  return cudaGetLastError();
}

int flux_accum_launches() { return 2; }
