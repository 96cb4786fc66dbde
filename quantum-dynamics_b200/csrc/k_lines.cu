// k_lines.cu -- the l-space part of one split-operator step:
//     psi_l <- Rot(dt/2) IFFT2 [exp(-i(T1+T2)dt)/(n1 n2)] FFT2 Rot(dt/2) psi_l
// (evolution_dt, timeEvol.C:625-635; tables timeEvol.C:465-517) as three
// shared-memory Stockham passes over each l-slice:
//   rows kernel    Rot(dt/2), FFT along R (contiguous lines of n1)
//   columns kernel FFT along r, kinetic phase, inverse FFT along r
//   rows kernel    inverse FFT along R, Rot(dt/2)
// The 2-D DFT is the unnormalised FFTW_FORWARD / FFTW_BACKWARD pair of
// fftwinterface.C:70-76; the 1/(n1 n2) sits in the kinetic phase as in
// setup_exp_ikin_dt (timeEvol.C:514).
#include "qd_kernels.h"

namespace {

template <typename R> struct Phase;
template <> struct Phase<double> {
  static __device__ __forceinline__ double2 rot(const LineParams &p, int l, int j, int i)
  { return p.rot[((long)l * p.n2 + j) * p.n1 + i]; }
  static __device__ __forceinline__ double2 kin(const LineParams &p, int j, int i)
  { return p.kin[(long)j * p.n1 + i]; }
};
template <> struct Phase<float> {
  static __device__ __forceinline__ float2 rot(const LineParams &p, int l, int j, int i)
  { return cmul(__ldg(p.rc1 + l * p.n1 + i), __ldg(p.rc2 + l * p.n2 + j)); }
  static __device__ __forceinline__ float2 kin(const LineParams &p, int j, int i)
  { return cscale2(cmul(__ldg(p.kc1 + i), __ldg(p.kc2 + j)), p.kscale, p.kscale_lo); }
};

// dir = -1: Rot then forward FFT along R;  dir = +1: inverse FFT then Rot.
template <typename R>
__global__ void __launch_bounds__(256) k_rows(LineParams p, int dir)
{
  typedef typename Cplx<R>::T C;
  extern __shared__ __align__(16) unsigned char smem[];
  const int rb = p.rows_per_cta;
  C *bufA = reinterpret_cast<C *>(smem);
  C *bufB = bufA + rb * p.n1;
  const int sl = blockIdx.y, l = rot_row(p, sl);  // slice = run * nl + l
  const int j0 = blockIdx.x * rb;
  const int nrows = min(rb, p.n2 - j0);
  C *slice = reinterpret_cast<C *>(p.lpsi) + (long)sl * p.n12 + (long)j0 * p.n1;
  const int nel = nrows * p.n1;
  for (int e = threadIdx.x; e < nel; e += blockDim.x) {
    C v = slice[e];
    if (dir < 0 && !p.fft_only) v = cmul(v, Phase<R>::rot(p, l, j0 + e / p.n1, e % p.n1));
    bufA[e] = v;
  }
  __syncthreads();
  C *res = smem_fft_lines<C>(bufA, bufB, p.pl1, nrows, p.n1, 1, false,
                             reinterpret_cast<const C *>(p.tw1), dir);
  double er = 0.0;                               // energy step: sum (I1 + I2) |psi_l|^2
  for (int e = threadIdx.x; e < nel; e += blockDim.x) {
    C v = res[e];
    if (dir > 0) {
      const int j = j0 + e / p.n1, i = e % p.n1;
      v = cmul(v, Phase<R>::rot(p, l, j, i));
      if (p.esum) {
        const double2 z = to_z(v);
        er += (z.x * z.x + z.y * z.y) * (p.I1[i] + p.I2[j]);
      }
    }
    slice[e] = v;
  }
  if (dir > 0 && p.esum) {
    __shared__ double red[32];
    const int run = sl / p.nl, ll = sl - run * p.nl;
    const double wl = p.orth ? 1.0 : 1.0 / (ll + 0.5);
    const double s = block_sum(er, red);
    if (threadIdx.x == 0) atomicAdd(p.esum + 3 * run + 1, s * (double)l * (l + 1.0) * wl);
  }
}

template <typename R>
__global__ void __launch_bounds__(256) k_cols(LineParams p)
{
  typedef typename Cplx<R>::T C;
  extern __shared__ __align__(16) unsigned char smem[];
  const int cb = p.cols_per_cta;
  C *bufA = reinterpret_cast<C *>(smem);
  C *bufB = bufA + cb * p.n2;
  const int sl = blockIdx.y;                     // slice = run * nl + l
  const int i0 = blockIdx.x * cb;
  const int ncols = min(cb, p.n1 - i0);
  C *slice = reinterpret_cast<C *>(p.lpsi) + (long)sl * p.n12;
  const int nel = ncols * p.n2;
  for (int e = threadIdx.x; e < nel; e += blockDim.x) {
    const int j = e / ncols, c = e % ncols;
    bufA[j * cb + c] = slice[(long)j * p.n1 + i0 + c];
  }
  __syncthreads();
  const C *tw2 = reinterpret_cast<const C *>(p.tw2);
  C *res = smem_fft_lines<C>(bufA, bufB, p.pl2, ncols, 1, cb, true, tw2, -1);
  C *other = (res == bufA) ? bufB : bufA;
  if (p.fft_only) {
    for (int e = threadIdx.x; e < nel; e += blockDim.x) {
      const int j = e / ncols, c = e % ncols;
      slice[(long)j * p.n1 + i0 + c] = res[j * cb + c];
    }
    return;
  }
  double ek = 0.0;                               // energy step: sum (T1 + T2) |FFT2 psi_l|^2
  for (int e = threadIdx.x; e < nel; e += blockDim.x) {
    const int j = e / ncols, c = e % ncols;
    if (p.esum) {
      const double2 z = to_z(res[j * cb + c]);
      ek += (z.x * z.x + z.y * z.y) * (p.T1[i0 + c] + p.T2[j]);
    }
    res[j * cb + c] = cmul(res[j * cb + c], Phase<R>::kin(p, j, i0 + c));
  }
  if (p.esum) {
    __shared__ double red[32];
    const int run = sl / p.nl, ll = sl - run * p.nl;
    const double wl = p.orth ? 1.0 : 1.0 / (ll + 0.5);
    const double s = block_sum(ek, red);
    if (threadIdx.x == 0) atomicAdd(p.esum + 3 * run, s * wl / (double)p.n12);
  }
  __syncthreads();
  res = smem_fft_lines<C>(res, other, p.pl2, ncols, 1, cb, true, tw2, +1);
  for (int e = threadIdx.x; e < nel; e += blockDim.x) {
    const int j = e / ncols, c = e % ncols;
    slice[(long)j * p.n1 + i0 + c] = res[j * cb + c];
  }
}

}  // namespace

template <typename R>
cudaError_t launch_lines(const LineParams &p0, cudaStream_t s)
{
  typedef typename Cplx<R>::T C;
  LineParams p = p0;
  static bool attr_set = false;
  if (!attr_set) {
    cudaFuncSetAttribute(k_rows<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(k_cols<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    attr_set = true;
  }
  const size_t budget = 96 * 1024;
  int rb = (int)(budget / (2 * sizeof(C) * p.n1));
  rb = max(1, min(rb, p.n2));
  int cb = (int)(budget / (2 * sizeof(C) * p.n2));
  cb = max(1, min(cb, min(32, p.n1)));
  p.rows_per_cta = rb;
  p.cols_per_cta = cb;
  const size_t sm_rows = 2 * sizeof(C) * (size_t)rb * p.n1;
  const size_t sm_cols = 2 * sizeof(C) * (size_t)cb * p.n2;
  dim3 grows((p.n2 + rb - 1) / rb, p.nruns * p.nl), gcols((p.n1 + cb - 1) / cb, p.nruns * p.nl);
  k_rows<R><<<grows, 256, sm_rows, s>>>(p, -1);
  k_cols<R><<<gcols, 256, sm_cols, s>>>(p);
  if (!p.fft_only) k_rows<R><<<grows, 256, sm_rows, s>>>(p, +1);
  return cudaGetLastError();
}

int lines_launches_per_step(int, int, int) { return 3; }

template cudaError_t launch_lines<float>(const LineParams &, cudaStream_t);
template cudaError_t launch_lines<double>(const LineParams &, cudaStream_t);
