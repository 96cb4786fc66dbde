// k_energy.cu -- energies of the current wavepacket, FP64 (the per-step
// diagnostics of the reference, timeEvol.C:256-360):
//   E_pot = sum_k w_k sum_ij |psi|^2 V                       potential_energy      :256-283
//   E_rot = sum_l l(l+1)/(l+1/2) sum_ij |F psi|^2 (I1 + I2)   rotational_energy     :323-360
//   E_kin = sum_k w_k sum_ij |DFT psi|^2 (T1 + T2) / (n1 n2)  kinetic_energy_for_psi :285-321
// each multiplied by dr1 dr2 on the host.
#include <algorithm>
#include "qd_kernels.h"

namespace {

// a tile of TQ grid columns at a time: their theta-space values are read
// once into shared memory ([n_theta][TQ]), then every order l is contracted
// from there
__global__ void __launch_bounds__(256) k_e_pot_rot(EnergyParams e, int TQ)
{
  extern __shared__ double2 zt[];
  __shared__ double red[32];
  double srot = 0.0, spot = 0.0;
  const long ntile = (e.n12 + TQ - 1) / TQ;
  for (long tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
    const long q0 = tile * TQ;
    __syncthreads();                               // the previous tile's reads are done
    for (int x = threadIdx.x; x < e.nth * TQ; x += blockDim.x) {
      const int k = x / TQ, t = x % TQ;
      const long q = q0 + t;
      double2 z = make_double2(0.0, 0.0);
      if (q < e.n12) {
        z = e.psi_z[(long)k * e.n12 + q];
        spot += e.w[k] * (z.x * z.x + z.y * z.y) * e.pot[(long)k * e.n12 + q];
      }
      zt[x] = z;
    }
    __syncthreads();
    for (int x = threadIdx.x; x < e.nl * TQ; x += blockDim.x) {
      const int l = x / TQ, t = x % TQ;
      const long q = q0 + t;
      if (q >= e.n12 || (e.K == 0 && l == 0)) continue;   // j(j+1) = 0 only for j = 0
      double2 c = make_double2(0.0, 0.0);
      for (int k = 0; k < e.nth; k++) {
        const double2 z = zt[k * TQ + t];
        const double wp = e.WP[k * e.nl + l];
        c.x += z.x * wp;
        c.y += z.y * wp;
      }
      const int j = (int)(q / e.n1), i = (int)(q % e.n1);
      const double jr = (double)(e.K + l);           // j = K + l (centrifugal sudden)
      srot += (c.x * c.x + c.y * c.y) * (e.I1[i] + e.I2[j]) * jr * (jr + 1) / (l + 0.5);
    }
  }
  srot = block_sum(srot, red);
  if (threadIdx.x == 0) atomicAdd(e.sums + 1, srot);
  spot = block_sum(spot, red);
  if (threadIdx.x == 0) atomicAdd(e.sums + 2, spot);
}

__global__ void __launch_bounds__(256) k_e_kin(EnergyParams e)
{
  __shared__ double red[32];
  double s = 0.0;
  const long n = e.n12 * e.nth;
  for (long g = blockIdx.x * (long)blockDim.x + threadIdx.x; g < n;
       g += (long)gridDim.x * blockDim.x) {
    const int k = (int)(g / e.n12);
    const long q = g % e.n12;
    const int j = (int)(q / e.n1), i = (int)(q % e.n1);
    const double2 z = e.scratch[g];
    s += e.w[k] * (z.x * z.x + z.y * z.y) * (e.T1[i] + e.T2[j]);
  }
  s = block_sum(s, red);
  if (threadIdx.x == 0) atomicAdd(e.sums, s);
}

}  // namespace

int energies_launches() { return 5; }

cudaError_t launch_energies(const EnergyParams &e, cudaStream_t s)
{
  const int TQ = (int)std::max(1L, std::min(32L, (long)(96 * 1024 / (16 * e.nth))));
  const size_t sm = sizeof(double2) * e.nth * TQ;
  static bool attr_set = false;
  if (!attr_set) {
    cudaFuncSetAttribute(k_e_pot_rot, cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024);
    attr_set = true;
  }
  k_e_pot_rot<<<2 * 148, 256, sm, s>>>(e, TQ);
  cudaError_t err = cudaMemcpyAsync(e.scratch, e.psi_z, sizeof(double2) * e.n12 * e.nth,
                                    cudaMemcpyDeviceToDevice, s);
  if (err != cudaSuccess) return err;
  LineParams p{};
  p.n1 = e.n1; p.n2 = e.n2; p.nl = e.nth; p.n12 = e.n12; p.nruns = 1;
  p.lpsi = e.scratch; p.tw1 = e.tw1; p.tw2 = e.tw2; p.pl1 = e.pl1; p.pl2 = e.pl2;
  p.fft_only = 1;
  err = launch_lines<double>(p, s);
  if (err != cudaSuccess) return err;
  k_e_kin<<<148 * 4, 256, 0, s>>>(e);
  return cudaGetLastError();
}
