// k_column.cu -- the column pass of one split-operator step, SIMT form.
//
// For a tile of TP grid columns (R_i, r_j) it performs, in shared memory,
//   psi_theta = B psi_l                    BackwardLegendreTransform (LegTransform.F:34-59)
//   psi_theta *= d1(i) d2(j)               dump_psi (timeEvol.C:713-735)
//   surface rows -> surf, norm             Gradient3.F input, module_for_psi (timeEvol.C:220-243)
//   psi_theta *= exp(-i V dt)              evolution_with_potential_dt (timeEvol.C:540-559)
//   psi_l = F psi_theta                    ForwardLegendreTransform (LegTransform.F:6-31)
// i.e. the end of step n and the start of step n+1, so that the l-space
// wavepacket is read and written once per step by this pass.
#include "qd_kernels.h"

namespace {

constexpr int KB = 4;      // outputs per thread along the contracted-to index

template <typename R> struct MatSel;
template <> struct MatSel<double> {
  static __device__ __forceinline__ const double *P(const ColumnParams &p) { return p.P; }
  static __device__ __forceinline__ const double *WP(const ColumnParams &p) { return p.WP; }
  static __device__ __forceinline__ const double *Plo(const ColumnParams &) { return nullptr; }
  static __device__ __forceinline__ const double *WPlo(const ColumnParams &) { return nullptr; }
};
template <> struct MatSel<float> {
  static __device__ __forceinline__ const float *P(const ColumnParams &p) { return p.P32; }
  static __device__ __forceinline__ const float *WP(const ColumnParams &p) { return p.WP32; }
  static __device__ __forceinline__ const float *Plo(const ColumnParams &p) { return p.P32lo; }
  static __device__ __forceinline__ const float *WPlo(const ColumnParams &p) { return p.WP32lo; }
};

__device__ __forceinline__ double2 vphase(const ColumnParams &p, long g, double2)
{ return p.expV[g]; }
__device__ __forceinline__ float2 vphase(const ColumnParams &p, long g, float2)
{ return p.expV32[g]; }

// out[o][t] = sum_c M[o*ldm + c] * in[c][t], o < nout, c < nin, KB outputs / thread;
// M = Mhi + Mlo when Mlo is given (float matrices carried to ~2^-48)
template <typename R, typename C>
__device__ __forceinline__ void contract(const R *__restrict__ M, const R *__restrict__ Mlo,
                                         int ldm, bool trans, const C *in, int nin, C *out,
                                         int nout, int TP)
{
  const int ngroups = (nout + KB - 1) / KB;
  for (int e = threadIdx.x; e < ngroups * TP; e += blockDim.x) {
    const int t = e % TP, o0 = (e / TP) * KB;
    C acc[KB];
#pragma unroll
    for (int b = 0; b < KB; b++) acc[b] = mk((R)0, (R)0);
    for (int c = 0; c < nin; c++) {
      const C v = in[c * TP + t];
#pragma unroll
      for (int b = 0; b < KB; b++) {
        const int o = min(o0 + b, nout - 1);
        const long mi = trans ? (long)c * ldm + o : (long)o * ldm + c;
        const R m = __ldg(M + mi);
        if (Mlo) {
          const R ml = __ldg(Mlo + mi);
          acc[b].x += ml * v.x;
          acc[b].y += ml * v.y;
        }
        acc[b].x += m * v.x;
        acc[b].y += m * v.y;
      }
    }
#pragma unroll
    for (int b = 0; b < KB; b++)
      if (o0 + b < nout) out[(o0 + b) * TP + t] = acc[b];
  }
}

template <typename R>
__global__ void __launch_bounds__(256) k_column(ColumnParams p, int mode, int TP)
{
  typedef typename Cplx<R>::T C;
  extern __shared__ __align__(16) unsigned char smem[];
  C *A = reinterpret_cast<C *>(smem);          // [nl][TP]   l-space tile
  C *B = A + p.nl * TP;                         // [nth][TP]  theta-space tile
  double *red = reinterpret_cast<double *>(B + p.nth * TP);
  const long tiles_per_run = (p.n12 + TP - 1) / TP;
  const int run = (int)(blockIdx.x / tiles_per_run);
  const long p0 = (long)(blockIdx.x % tiles_per_run) * TP;
  C *lpsi = reinterpret_cast<C *>(p.lpsi) + (long)run * p.nl * p.n12;
  const long zoff = (long)run * p.nth * p.n12;      // psi_z of this run
  const long voff = (long)run * p.vrun;             // potential tables of this run
  const long soff = p.run_set ? p.run_set[run] * p.set_stride : 0;   // angular basis of the run
  const R *P = MatSel<R>::P(p) + soff;
  const R *WP = MatSel<R>::WP(p) + soff;
  const R *Plo = MatSel<R>::Plo(p) ? MatSel<R>::Plo(p) + soff : nullptr;
  const R *WPlo = MatSel<R>::WPlo(p) ? MatSel<R>::WPlo(p) + soff : nullptr;

  if (mode == COL_HEAD) {
    for (int e = threadIdx.x; e < p.nth * TP; e += blockDim.x) {
      const int k = e / TP, t = e % TP;
      const long q = p0 + t;
      C v = mk((R)0, (R)0);
      if (q < p.n12) {
        const long g = (long)k * p.n12 + q;
        double2 z = p.psi_z[zoff + g];
        double s, c;
        sincos(p.dt * p.pot[voff + g], &s, &c);   // exp(-i V dt) = (c, -s)
        double2 f = make_double2(c, -s);
        if (p.prestep) {
          // psi / sqrt(v) * v = psi * sqrt(v), principal branch
          // (pre_evolution_with_potential_dt_2, timeEvol.C:519-538)
          double sh, ch;
          sincos(0.5 * atan2(-s, c), &sh, &ch);
          f = make_double2(ch, sh);
        }
        z = cmul(z, f);
        v = from_z<C>(z);
      }
      B[k * TP + t] = v;
    }
  } else {
    for (int e = threadIdx.x; e < p.nl * TP; e += blockDim.x) {
      const int l = e / TP, t = e % TP;
      const long q = p0 + t;
      A[l * TP + t] = q < p.n12 ? lpsi[(long)l * p.n12 + q] : mk((R)0, (R)0);
    }
    __syncthreads();
    // psi_theta(k) = sum_l P[k][l] psi_l(l)
    contract<R, C>(P, Plo, p.nl, false, A, p.nl, B, p.nth, TP);
  }
  __syncthreads();

  if (mode != COL_HEAD) {
    double nsum = 0.0, esum = 0.0;
    C *surf = reinterpret_cast<C *>(p.surf) + (long)run * p.surf_nrows * p.nth * p.n1;
    for (int e = threadIdx.x; e < p.nth * TP; e += blockDim.x) {
      const int k = e / TP, t = e % TP;
      const long q = p0 + t;
      if (q >= p.n12) continue;
      const int j = (int)(q / p.n1), i = (int)(q % p.n1);
      C v = B[k * TP + t];
      const long g = (long)k * p.n12 + q;
      if (p.esum) {                               // potential energy, before the absorber
        const double2 z = to_z(v);
        esum += p.w[k] * (z.x * z.x + z.y * z.y) * p.pot[voff + g];
      }
      if (p.d1) v = cscale(v, (R)(p.d1[i] * p.d2[j]));
      if (p.do_flux && j >= p.surf_j0 && j < p.surf_j0 + p.surf_nrows)
        surf[((long)(j - p.surf_j0) * p.nth + k) * p.n1 + i] = v;
      if (p.norm_out) {
        const double2 z = to_z(v);
        nsum += p.w[k] * (z.x * z.x + z.y * z.y);
      }
      if (p.out_z) p.psi_z[zoff + g] = to_z(v);
      if (mode == COL_MID) v = cmul(v, vphase(p, voff + g, v));
      B[k * TP + t] = v;
    }
    if (p.norm_out) {
      const double s = block_sum(nsum, red);
      if (threadIdx.x == 0) atomicAdd(p.norm_out + run, s);
    }
    if (p.esum) {
      const double s = block_sum(esum, red);
      if (threadIdx.x == 0) atomicAdd(p.esum + 3 * run + 2, s);
    }
    if (mode == COL_TAIL) return;
    __syncthreads();
  }

  // psi_l(l) = sum_k WP[k][l] psi_theta(k)
  contract<R, C>(WP, WPlo, p.nl, true, B, p.nth, A, p.nl, TP);
  __syncthreads();
  for (int e = threadIdx.x; e < p.nl * TP; e += blockDim.x) {
    const int l = e / TP, t = e % TP;
    const long q = p0 + t;
    if (q < p.n12) lpsi[(long)l * p.n12 + q] = A[l * TP + t];
  }
}

}  // namespace

template <typename R>
cudaError_t launch_column(const ColumnParams &p, int mode, cudaStream_t s)
{
  typedef typename Cplx<R>::T C;
  int TP = 32;
  while (TP > 8 && (size_t)(p.nl + p.nth) * TP * sizeof(C) > 96 * 1024) TP /= 2;
  const size_t sm = (size_t)(p.nl + p.nth) * TP * sizeof(C) + 32 * sizeof(double);
  static bool attr_set = false;
  if (!attr_set) {
    cudaFuncSetAttribute(k_column<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    attr_set = true;
  }
  const unsigned grid = (unsigned)((p.n12 + TP - 1) / TP * p.nruns);
  k_column<R><<<grid, 256, sm, s>>>(p, mode, TP);
  return cudaGetLastError();
}

template cudaError_t launch_column<float>(const ColumnParams &, int, cudaStream_t);
template cudaError_t launch_column<double>(const ColumnParams &, int, cudaStream_t);
