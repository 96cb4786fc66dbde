// qd_libcmp.cu -- the propagator's two passes in the form the reference's
// GPU code gives them (common-cuda/evolutionCUDA2.cu), on NVIDIA's libraries,
// timed for comparison with this library's own kernels.  Not part of the
// propagator: a separate shared library (libqd_libcmp.so) that only the
// benchmark loads.
//
//   l-space pass  (evolutionCUDA2.cu:318-338 plan, :600-608 exec; the phases
//                  as separate elementwise kernels, like :503-535):
//                  Rot/2, cufftExec forward, kinetic phase / (n1 n2),
//                  cufftExec inverse, Rot/2 -- one batched 2-D plan over all
//                  l-slices of all runs (cufftPlanMany, Z2Z or C2C)
//   column pass   (evolutionCUDA2.cu:566-593): psi_theta = psi_l L (l -> theta),
//                  psi_theta *= exp(-i V dt) * absorber, psi_l = psi_theta W
//                  (theta -> l) -- strided-batched GEMMs over the runs with the
//                  real Legendre matrices (the complex wavepacket read as a
//                  real matrix with 2 n1 n2 rows: the same products as the
//                  reference's Zgemm with a real matrix, half its flops)
//
// Both are timed with CUDA events on one stream over `reps` steps after two
// warm-up steps, on synthetic data of the given shapes, and reported as ms
// per step.  The data are finite and bounded (unit-modulus phases), so the
// timing does not depend on the values.
#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <cufft.h>
#include <cstdio>
#include <cstring>
#include <string>

namespace {

thread_local std::string g_err;

int fail(const char *what, int code)
{
  char b[256];
  snprintf(b, sizeof b, "%s failed (%d)", what, code);
  g_err = b;
  return -1;
}

#define CUDA_OK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { rc = fail(#x, (int)e_); goto done; } } while (0)
#define FFT_OK(x) do { cufftResult e_ = (x); if (e_ != CUFFT_SUCCESS) { rc = fail(#x, (int)e_); goto done; } } while (0)
#define BLAS_OK(x) do { cublasStatus_t e_ = (x); if (e_ != CUBLAS_STATUS_SUCCESS) { rc = fail(#x, (int)e_); goto done; } } while (0)

template <typename C> struct Ops;
template <> struct Ops<float2> {
  static __device__ float2 mul(float2 a, float2 b)
  { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
  static __device__ float2 scale(float2 a, double s)
  { return make_float2(a.x * (float)s, a.y * (float)s); }
  static __device__ float2 phase(double t)
  { float s, c; sincosf((float)t, &s, &c); return make_float2(c, -s); }
};
template <> struct Ops<double2> {
  static __device__ double2 mul(double2 a, double2 b)
  { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
  static __device__ double2 scale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
  static __device__ double2 phase(double t) { double s, c; sincos(t, &s, &c); return make_double2(c, -s); }
};

// synthetic input: psi of modulus <= 1, unit-modulus phase rows
template <typename C> __global__ void k_fill(C *p, size_t n, double f)
{
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    p[i] = Ops<C>::scale(Ops<C>::phase(f * (double)(i % 9973)), 0.5);
}
template <typename R> __global__ void k_fill_real(R *p, size_t n, double f)
{
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    p[i] = (R)(0.1 * sin(f * (double)(i % 7919)));
}

// psi[slice][j][i] *= a[l][i] b[l][j] (scale): the separable rotational or
// kinetic phase of one elementwise kernel (slice = run * nl + l; the kinetic
// phase has one row, nrow = 1)
template <typename C>
__global__ void k_phase2(C *psi, const C *a, const C *b, int n1, int n2, int nl, int nrow,
                         long nslices, double scale)
{
  const long n12 = (long)n1 * n2, tot = n12 * nslices;
  for (long x = blockIdx.x * (long)blockDim.x + threadIdx.x; x < tot;
       x += (long)gridDim.x * blockDim.x) {
    const long s = x / n12;
    const int q = (int)(x - s * n12), j = q / n1, i = q - j * n1;
    const int row = nrow == 1 ? 0 : (int)(s % nl);
    C v = Ops<C>::mul(psi[x], Ops<C>::mul(a[(long)row * n1 + i], b[(long)row * n2 + j]));
    psi[x] = scale != 1.0 ? Ops<C>::scale(v, scale) : v;
  }
}

// psi_theta[run][k][q] *= expV[run][k][q] * d1[i] d2[j]
template <typename C, typename R>
__global__ void k_vphase(C *psi, const C *ev, const R *d, long n12, long total)
{
  for (long x = blockIdx.x * (long)blockDim.x + threadIdx.x; x < total;
       x += (long)gridDim.x * blockDim.x)
    psi[x] = Ops<C>::scale(Ops<C>::mul(psi[x], ev[x]), (double)d[x % n12]);
}

int grid_for(long n)
{
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  long g = (n + 255) / 256;
  return (int)(g < 8L * sms ? g : 8L * sms);
}

template <typename C>
int lspace_cufft(int n1, int n2, int nl, int runs, int reps, double *ms)
{
  int rc = 0;
  const long nsl = (long)nl * runs, n12 = (long)n1 * n2, npt = n12 * nsl;
  C *psi = nullptr, *r1 = nullptr, *r2 = nullptr, *k1 = nullptr, *k2 = nullptr;
  cufftHandle plan = 0;
  bool have_plan = false;
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  const bool f32 = sizeof(C) == 8;
  int dims[2] = {n2, n1};
  float t = 0.f;
  CUDA_OK(cudaStreamCreate(&st));
  CUDA_OK(cudaMalloc(&psi, sizeof(C) * npt));
  CUDA_OK(cudaMalloc(&r1, sizeof(C) * nl * n1));
  CUDA_OK(cudaMalloc(&r2, sizeof(C) * nl * n2));
  CUDA_OK(cudaMalloc(&k1, sizeof(C) * n1));
  CUDA_OK(cudaMalloc(&k2, sizeof(C) * n2));
  k_fill<<<grid_for(npt), 256, 0, st>>>(psi, npt, 0.37);
  k_fill<<<grid_for(nl * n1), 256, 0, st>>>(r1, (size_t)nl * n1, 0.11);
  k_fill<<<grid_for(nl * n2), 256, 0, st>>>(r2, (size_t)nl * n2, 0.13);
  k_fill<<<1, 256, 0, st>>>(k1, n1, 0.17);
  k_fill<<<1, 256, 0, st>>>(k2, n2, 0.19);
  FFT_OK(cufftPlanMany(&plan, 2, dims, nullptr, 1, (int)n12, nullptr, 1, (int)n12,
                       f32 ? CUFFT_C2C : CUFFT_Z2Z, (int)nsl));
  have_plan = true;
  FFT_OK(cufftSetStream(plan, st));
  CUDA_OK(cudaEventCreate(&e0));
  CUDA_OK(cudaEventCreate(&e1));
  for (int it = -2; it < reps; it++) {
    if (it == 0) CUDA_OK(cudaEventRecord(e0, st));
    k_phase2<<<grid_for(npt), 256, 0, st>>>(psi, r1, r2, n1, n2, nl, nl, nsl, 1.0);
    if (f32) FFT_OK(cufftExecC2C(plan, (cufftComplex *)psi, (cufftComplex *)psi, CUFFT_FORWARD));
    else FFT_OK(cufftExecZ2Z(plan, (cufftDoubleComplex *)psi, (cufftDoubleComplex *)psi, CUFFT_FORWARD));
    k_phase2<<<grid_for(npt), 256, 0, st>>>(psi, k1, k2, n1, n2, nl, 1, nsl, 1.0 / (double)n12);
    if (f32) FFT_OK(cufftExecC2C(plan, (cufftComplex *)psi, (cufftComplex *)psi, CUFFT_INVERSE));
    else FFT_OK(cufftExecZ2Z(plan, (cufftDoubleComplex *)psi, (cufftDoubleComplex *)psi, CUFFT_INVERSE));
    k_phase2<<<grid_for(npt), 256, 0, st>>>(psi, r1, r2, n1, n2, nl, nl, nsl, 1.0);
    CUDA_OK(cudaGetLastError());
  }
  CUDA_OK(cudaEventRecord(e1, st));
  CUDA_OK(cudaEventSynchronize(e1));
  CUDA_OK(cudaEventElapsedTime(&t, e0, e1));
  *ms = reps > 0 ? t / reps : 0.0;
done:
  if (have_plan) cufftDestroy(plan);
  if (st) cudaStreamSynchronize(st);
  cudaFree(psi); cudaFree(r1); cudaFree(r2); cudaFree(k1); cudaFree(k2);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (st) cudaStreamDestroy(st);
  return rc;
}

// compute: 0 = FP64 (cublasDgemm), 1 = FP32 SIMT (CUBLAS_COMPUTE_32F),
// 2 = FP32 inputs rounded to TF32 (CUBLAS_COMPUTE_32F_FAST_TF32),
// 3 = FP32 emulated by BF16 splits on the tensor cores
// (CUBLAS_COMPUTE_32F_EMULATED_16BFX9)
template <typename C, typename R>
int column_cublas(int n1, int n2, int nth, int nl, int runs, int compute, int reps, double *ms)
{
  int rc = 0;
  const long n12 = (long)n1 * n2;
  const long nlp = n12 * nl * runs, nthp = n12 * nth * runs;
  C *lpsi = nullptr, *tpsi = nullptr, *ev = nullptr;
  R *L = nullptr, *W = nullptr, *d = nullptr;
  cublasHandle_t hb = nullptr;
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  const R one = 1, zero = 0;
  const int M = (int)(2 * n12);
  cudaDataType_t dt = sizeof(R) == 4 ? CUDA_R_32F : CUDA_R_64F;
  cublasComputeType_t ct = compute == 0 ? CUBLAS_COMPUTE_64F
                         : compute == 1 ? CUBLAS_COMPUTE_32F
                         : compute == 2 ? CUBLAS_COMPUTE_32F_FAST_TF32
                                        : CUBLAS_COMPUTE_32F_EMULATED_16BFX9;
  float t = 0.f;
  CUDA_OK(cudaStreamCreate(&st));
  CUDA_OK(cudaMalloc(&lpsi, sizeof(C) * nlp));
  CUDA_OK(cudaMalloc(&tpsi, sizeof(C) * nthp));
  CUDA_OK(cudaMalloc(&ev, sizeof(C) * nthp));
  CUDA_OK(cudaMalloc(&L, sizeof(R) * nl * nth));
  CUDA_OK(cudaMalloc(&W, sizeof(R) * nl * nth));
  CUDA_OK(cudaMalloc(&d, sizeof(R) * n12));
  k_fill<<<grid_for(nlp), 256, 0, st>>>(lpsi, nlp, 0.37);
  k_fill<<<grid_for(nthp), 256, 0, st>>>(ev, nthp, 0.29);
  k_fill_real<<<grid_for(nl * nth), 256, 0, st>>>(L, (size_t)nl * nth, 0.31);
  k_fill_real<<<grid_for(nl * nth), 256, 0, st>>>(W, (size_t)nl * nth, 0.23);
  k_fill_real<<<grid_for(n12), 256, 0, st>>>(d, n12, 0.07);
  BLAS_OK(cublasCreate(&hb));
  BLAS_OK(cublasSetStream(hb, st));
  CUDA_OK(cudaEventCreate(&e0));
  CUDA_OK(cudaEventCreate(&e1));
  for (int it = -2; it < reps; it++) {
    if (it == 0) CUDA_OK(cudaEventRecord(e0, st));
    // l -> theta: psi_theta[run] (M x nth) = psi_l[run] (M x nl) * L (nl x nth)
    BLAS_OK(cublasGemmStridedBatchedEx(hb, CUBLAS_OP_N, CUBLAS_OP_N, M, nth, nl, &one,
                                       lpsi, dt, M, 2 * n12 * nl, L, dt, nl, 0, &zero,
                                       tpsi, dt, M, 2 * n12 * nth, runs, ct, CUBLAS_GEMM_DEFAULT));
    k_vphase<C, R><<<grid_for(nthp), 256, 0, st>>>(tpsi, ev, d, n12, nthp);
    // theta -> l: psi_l[run] (M x nl) = psi_theta[run] (M x nth) * W (nth x nl)
    BLAS_OK(cublasGemmStridedBatchedEx(hb, CUBLAS_OP_N, CUBLAS_OP_N, M, nl, nth, &one,
                                       tpsi, dt, M, 2 * n12 * nth, W, dt, nth, 0, &zero,
                                       lpsi, dt, M, 2 * n12 * nl, runs, ct, CUBLAS_GEMM_DEFAULT));
    CUDA_OK(cudaGetLastError());
  }
  CUDA_OK(cudaEventRecord(e1, st));
  CUDA_OK(cudaEventSynchronize(e1));
  CUDA_OK(cudaEventElapsedTime(&t, e0, e1));
  *ms = reps > 0 ? t / reps : 0.0;
done:
  if (st) cudaStreamSynchronize(st);
  if (hb) cublasDestroy(hb);
  cudaFree(lpsi); cudaFree(tpsi); cudaFree(ev); cudaFree(L); cudaFree(W); cudaFree(d);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (st) cudaStreamDestroy(st);
  return rc;
}

}  // namespace

extern "C" {

const char *qdc_last_error(void) { return g_err.c_str(); }

int qdc_set_device(int device)
{
  return cudaSetDevice(device) == cudaSuccess ? 0 : fail("cudaSetDevice", device);
}

// ms per step of the library form of the l-space pass: precision 0 = Z2Z
// (complex128), 1 = C2C (complex64)
int qdc_lspace_cufft(int n1, int n2, int nl, int runs, int precision, int reps, double *ms)
{
  if (n1 < 2 || n2 < 2 || nl < 1 || runs < 1 || reps < 1 || !ms) return fail("arguments", 0);
  return precision == 0 ? lspace_cufft<double2>(n1, n2, nl, runs, reps, ms)
                        : lspace_cufft<float2>(n1, n2, nl, runs, reps, ms);
}

// ms per step of the library form of the column pass (compute as above)
int qdc_column_cublas(int n1, int n2, int nth, int nl, int runs, int compute, int reps,
                      double *ms)
{
  if (n1 < 2 || n2 < 2 || nth < 1 || nl < 1 || runs < 1 || reps < 1 || !ms ||
      compute < 0 || compute > 3)
    return fail("arguments", 0);
  if (compute == 0) return column_cublas<double2, double>(n1, n2, nth, nl, runs, 0, reps, ms);
  return column_cublas<float2, float>(n1, n2, nth, nl, runs, compute, reps, ms);
}

}  // extern "C"
