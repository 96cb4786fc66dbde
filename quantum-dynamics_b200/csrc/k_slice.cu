// k_slice.cu -- the l-space part of one complex64 split-operator step in ONE
// kernel: for every l-slice (n1 x n2, R fastest)
//     psi_l <- Rot(dt/2) IFFT2 [exp(-i(T1+T2)dt)/(n1 n2)] FFT2 Rot(dt/2) psi_l
// (evolution_dt, timeEvol.C:625-635; FFTW 2-D DFT pair of
// fftwinterface.C:70-76; tables timeEvol.C:465-517).
//
// A slice is owned by a cluster of CL CTAs (CL = 1, 2, 4; chosen at set-up by
// timing).  CTA `rank` holds rows [rank n2/CL, (rank+1) n2/CL) for the FFTs
// along R and columns [rank n1/CL, ...) for the FFTs along r; between the two
// phases the slice is transposed across the cluster through distributed
// shared memory (plain ld/st to the peers' shared memory, cluster barriers
// around each exchange).  psi_l is read and written once per step.
//
// FFTs are shared-memory Stockham passes (radix 8/4/2/3/5 in registers).
// Row buffers are padded by one element per 8 so that the radix-8 output
// pattern of the row passes is free of bank conflicts; the column passes
// walk consecutive columns across a warp.
#include <cooperative_groups.h>
#include "qd_kernels.h"

namespace cg = cooperative_groups;

namespace {

constexpr int NT = 512;

struct LayRowPad {      // rows of n contiguous elements, one pad per 8
  int rs;
  __device__ __forceinline__ int operator()(int line, int e) const { return line * rs + e + (e >> 3); }
};
struct LayColOnRows {   // columns of a LayRowPad buffer: line = column, e = row
  int rs;
  __device__ __forceinline__ int operator()(int line, int e) const { return e * rs + line + (line >> 3); }
};
struct LayCols {        // [e][line] with leading dimension ld
  int ld;
  __device__ __forceinline__ int operator()(int line, int e) const { return e * ld + line; }
};

template <int RAD, class Lay>
__device__ __forceinline__ void stage(const float2 *__restrict__ src, float2 *__restrict__ dst,
                                      int n, int Ns, int nlines, bool lines_fast, Lay lay,
                                      const float2 *__restrict__ tw, int sgn)
{
  const int nb = n / RAD;
  const int total = nb * nlines;
  const int tstep = n / (Ns * RAD);
  for (int b = threadIdx.x; b < total; b += blockDim.x) {
    int line, j;
    if (lines_fast) { line = b % nlines; j = b / nlines; }
    else            { line = b / nb;     j = b % nb; }
    float2 v[RAD];
#pragma unroll
    for (int r = 0; r < RAD; r++) v[r] = src[lay(line, j + r * nb)];
    const int k = j % Ns;
    if (Ns > 1) {
#pragma unroll
      for (int r = 1; r < RAD; r++) {
        float2 w = tw[r * k * tstep];
        if (sgn > 0) w.y = -w.y;
        v[r] = cmul(v[r], w);
      }
    }
    SmallDFT<RAD, float2>::run(v, sgn, tw, n);
    const int o = (j / Ns) * Ns * RAD + k;
#pragma unroll
    for (int r = 0; r < RAD; r++) dst[lay(line, o + r * Ns)] = v[r];
  }
}

// all lines of a buffer, ping-pong a <-> b; returns the buffer with the result
template <class Lay>
__device__ float2 *fft(float2 *a, float2 *b, const FftPlan &pl, int nlines, bool lines_fast,
                       Lay lay, const float2 *tw, int sgn)
{
  float2 *src = a, *dst = b;
  int Ns = 1;
  for (int s = 0; s < pl.nst; s++) {
    const int R = pl.rad[s];
    switch (R) {
      case 2: stage<2>(src, dst, pl.n, Ns, nlines, lines_fast, lay, tw, sgn); break;
      case 3: stage<3>(src, dst, pl.n, Ns, nlines, lines_fast, lay, tw, sgn); break;
      case 4: stage<4>(src, dst, pl.n, Ns, nlines, lines_fast, lay, tw, sgn); break;
      case 5: stage<5>(src, dst, pl.n, Ns, nlines, lines_fast, lay, tw, sgn); break;
      default: stage<8>(src, dst, pl.n, Ns, nlines, lines_fast, lay, tw, sgn); break;
    }
    __syncthreads();
    float2 *t = src; src = dst; dst = t;
    Ns *= R;
  }
  return src;
}

__device__ __forceinline__ float2 rot(const LineParams &p, int l, int j, int i)
{ return cmul(__ldg(p.rc1 + l * p.n1 + i), __ldg(p.rc2 + l * p.n2 + j)); }
__device__ __forceinline__ float2 kin(const LineParams &p, int j, int i)
{ return cscale2(cmul(__ldg(p.kc1 + i), __ldg(p.kc2 + j)), p.kscale, p.kscale_lo); }

__host__ __device__ inline int slice_buf_elems(int n1, int n2, int CL)
{
  const int rs = n1 + n1 / 8;
  return (n2 / CL) * rs;            // >= n2 * (n1 / CL)
}
__host__ __device__ inline size_t slice_smem_bytes(int n1, int n2, int CL)
{
  return sizeof(float2) * ((size_t)n1 + n2 + 2 * (size_t)slice_buf_elems(n1, n2, CL));
}

template <int CL>
__global__ void __launch_bounds__(NT, 1) k_slice(LineParams p)
{
  extern __shared__ float4 smem4[];
  float2 *sm = reinterpret_cast<float2 *>(smem4);
  const int n1 = p.n1, n2 = p.n2;
  const int rank = CL > 1 ? (int)cg::this_cluster().block_rank() : 0;
  if ((int)blockIdx.x >= p.nruns * p.nl * CL) {   // whole extra clusters: flux preparation
    const int q = ((int)blockIdx.x - p.nruns * p.nl * CL) * NT + (int)threadIdx.x;
    if (q < p.flux.nruns * p.flux.nth * p.flux.n1) flux_point<float2>(p.flux, q);
    return;
  }
  const int sl = blockIdx.x / CL, l = rot_row(p, sl);   // slice = run * nl + l
  const int nrow = n2 / CL, ncol = n1 / CL;
  const int rs = n1 + n1 / 8;
  const int bufsz = slice_buf_elems(n1, n2, CL);
  float2 *tw1 = sm, *tw2 = sm + n1;
  float2 *X = tw2 + n2, *Y = X + bufsz;
  const float2 *gtw1 = reinterpret_cast<const float2 *>(p.tw1);
  const float2 *gtw2 = reinterpret_cast<const float2 *>(p.tw2);
  for (int e = threadIdx.x; e < n1; e += NT) tw1[e] = gtw1[e];
  for (int e = threadIdx.x; e < n2; e += NT) tw2[e] = gtw2[e];

  float2 *slice = reinterpret_cast<float2 *>(p.lpsi) + (long)sl * p.n12;
  const int j0 = rank * nrow;
  const LayRowPad rowlay{rs};
  // 1. own rows, Rot(dt/2)
  for (int e = threadIdx.x; e < nrow * n1; e += NT) {
    const int r = e / n1, i = e - r * n1;
    X[rowlay(r, i)] = cmul(slice[(long)(j0 + r) * n1 + i], rot(p, l, j0 + r, i));
  }
  __syncthreads();
  // 2. FFT along R
  float2 *R1 = fft(X, Y, p.pl1, nrow, false, rowlay, tw1, -1);
  float2 *Rr;
  if (CL == 1) {
    // 3. FFT along r on the same buffer, kinetic phase, inverse FFT along r
    const LayColOnRows collay{rs};
    float2 *C = fft(R1, R1 == X ? Y : X, p.pl2, n1, true, collay, tw2, -1);
    for (int e = threadIdx.x; e < n2 * n1; e += NT) {
      const int j = e / n1, i = e - j * n1;
      C[collay(i, j)] = cmul(C[collay(i, j)], kin(p, j, i));
    }
    __syncthreads();
    Rr = fft(C, C == X ? Y : X, p.pl2, n1, true, collay, tw2, +1);
  } else {
    cg::cluster_group cluster = cg::this_cluster();
    cluster.sync();
    // 3a. gather my columns [rank ncol, ...) of every row from the owners' R1
    float2 *G = R1 == X ? Y : X;
    const LayCols clay{ncol};
    for (int e = threadIdx.x; e < n2 * ncol; e += NT) {
      const int j = e / ncol, c = e - j * ncol;
      const int owner = j / nrow, rr = j - owner * nrow, i = rank * ncol + c;
      const float2 *peer = cluster.map_shared_rank(R1, owner);
      G[clay(c, j)] = peer[rowlay(rr, i)];
    }
    cluster.sync();
    // 3b. FFT along r, kinetic phase, inverse FFT along r
    float2 *C = fft(G, G == X ? Y : X, p.pl2, ncol, true, clay, tw2, -1);
    for (int e = threadIdx.x; e < n2 * ncol; e += NT) {
      const int j = e / ncol, c = e - j * ncol;
      C[clay(c, j)] = cmul(C[clay(c, j)], kin(p, j, rank * ncol + c));
    }
    __syncthreads();
    float2 *C2 = fft(C, C == X ? Y : X, p.pl2, ncol, true, clay, tw2, +1);
    cluster.sync();
    // 3c. gather my rows back from the owners' columns
    Rr = C2 == X ? Y : X;
    for (int e = threadIdx.x; e < nrow * n1; e += NT) {
      const int r = e / n1, i = e - r * n1;
      const int owner = i / ncol, c = i - owner * ncol;
      const float2 *peer = cluster.map_shared_rank(C2, owner);
      Rr[rowlay(r, i)] = peer[clay(c, j0 + r)];
    }
    cluster.sync();
  }
  // 4. inverse FFT along R, Rot(dt/2), store
  float2 *F = fft(Rr, Rr == X ? Y : X, p.pl1, nrow, false, rowlay, tw1, +1);
  for (int e = threadIdx.x; e < nrow * n1; e += NT) {
    const int r = e / n1, i = e - r * n1;
    slice[(long)(j0 + r) * n1 + i] = cmul(F[rowlay(r, i)], rot(p, l, j0 + r, i));
  }
}

// ---------------------------------------------------------------------------
// Compile-time specialisation for the common grid sizes: the same algorithm
// with every size, radix, stride and line count a constant, so that the index
// arithmetic of the Stockham stages reduces to shifts and multiplies.
// ---------------------------------------------------------------------------

// radix of stage s of the plan for n (greedy 8, then 4, 2, 3, 5) -- the same
// factorisation radix_plan() builds on the host
__host__ __device__ constexpr int ct_rad(int n, int s)
{
  int m = n, r = 1;
  for (int k = 0; k <= s; k++) {
    r = (m % 8 == 0) ? 8 : (m % 4 == 0) ? 4 : (m % 2 == 0) ? 2 : (m % 3 == 0) ? 3 : 5;
    m /= r;
  }
  return r;
}
__host__ __device__ constexpr int ct_nst(int n)
{
  int m = n, s = 0;
  while (m > 1) { m /= ct_rad(n, s); s++; }
  return s;
}

template <int RS> struct CRowPad {
  __device__ __forceinline__ int operator()(int line, int e) const { return line * RS + e + (e >> 3); }
};
template <int RS> struct CColOnRows {
  __device__ __forceinline__ int operator()(int line, int e) const { return e * RS + line + (line >> 3); }
};
template <int LD> struct CCols {
  __device__ __forceinline__ int operator()(int line, int e) const { return e * LD + line; }
};

// element loop with a compile-time trip count, unrolled by 4 so that a
// thread's loads are in flight together (deeper unrolling spills)
#define QD_FOR_ELEMS(e, C)                                                \
  _Pragma("unroll 4") for (int it_ = 0; it_ < ((C) + NT - 1) / NT; it_++) \
    if (const int e = it_ * NT + (int)threadIdx.x; e < (C))

template <int N, int RAD, int NS, int NLINES, bool LF, class Lay>
__device__ __forceinline__ void stage_ct(const float2 *__restrict__ src, float2 *__restrict__ dst,
                                         Lay lay, const float2 *__restrict__ tw, int sgn)
{
  constexpr int NB = N / RAD;
  constexpr int TOTAL = NB * NLINES;
  constexpr int TSTEP = N / (NS * RAD);
  QD_FOR_ELEMS(b, TOTAL) {
    const int line = LF ? b % NLINES : b / NB;
    const int j = LF ? b / NLINES : b % NB;
    float2 v[RAD];
#pragma unroll
    for (int r = 0; r < RAD; r++) v[r] = src[lay(line, j + r * NB)];
    const int k = j % NS;
    if (NS > 1) {
#pragma unroll
      for (int r = 1; r < RAD; r++) {
        float2 w = tw[r * k * TSTEP];
        if (sgn > 0) w.y = -w.y;
        v[r] = cmul(v[r], w);
      }
    }
    SmallDFT<RAD, float2>::run(v, sgn, tw, N);
    const int o = (j / NS) * NS * RAD + k;
#pragma unroll
    for (int r = 0; r < RAD; r++) dst[lay(line, o + r * NS)] = v[r];
  }
}

template <int N, int S, int NS, int NLINES, bool LF, class Lay>
__device__ __forceinline__ float2 *fft_ct(float2 *src, float2 *dst, Lay lay, const float2 *tw,
                                          int sgn)
{
  if constexpr (S == ct_nst(N)) {
    return src;
  } else {
    constexpr int R = ct_rad(N, S);
    stage_ct<N, R, NS, NLINES, LF>(src, dst, lay, tw, sgn);
    __syncthreads();
    return fft_ct<N, S + 1, NS * R, NLINES, LF>(dst, src, lay, tw, sgn);
  }
}

// 64 registers per thread so that two CTAs share an SM where shared memory
// allows (the Stockham stages need few live values)
template <int N1, int N2, int CL>
__global__ void __launch_bounds__(NT, 2) k_slice_ct(LineParams p)
{
  constexpr int NROW = N2 / CL, NCOL = N1 / CL;
  constexpr int RS = N1 + N1 / 8;
  constexpr int BUF = NROW * RS;
  extern __shared__ float4 smem4[];
  float2 *sm = reinterpret_cast<float2 *>(smem4);
  const int rank = CL > 1 ? (int)cg::this_cluster().block_rank() : 0;
  if ((int)blockIdx.x >= p.nruns * p.nl * CL) {   // whole extra clusters: flux preparation
    const int q = ((int)blockIdx.x - p.nruns * p.nl * CL) * NT + (int)threadIdx.x;
    if (q < p.flux.nruns * p.flux.nth * p.flux.n1) flux_point<float2>(p.flux, q);
    return;
  }
  const int sl = blockIdx.x / CL, l = rot_row(p, sl);   // slice = run * nl + l
  float2 *tw1 = sm, *tw2 = sm + N1;
  float2 *X = tw2 + N2, *Y = X + BUF;
  const float2 *gtw1 = reinterpret_cast<const float2 *>(p.tw1);
  const float2 *gtw2 = reinterpret_cast<const float2 *>(p.tw2);
  for (int e = threadIdx.x; e < N1; e += NT) tw1[e] = gtw1[e];
  for (int e = threadIdx.x; e < N2; e += NT) tw2[e] = gtw2[e];
  float2 *slice = reinterpret_cast<float2 *>(p.lpsi) + (long)sl * (N1 * N2);
  const float2 *rc1 = p.rc1 + l * N1, *rc2 = p.rc2 + l * N2;
  const int j0 = rank * NROW;
  const CRowPad<RS> rowlay;
  QD_FOR_ELEMS(e, NROW * N1) {
    const int r = e / N1, i = e % N1;
    X[rowlay(r, i)] = cmul(slice[(j0 + r) * N1 + i], cmul(__ldg(rc1 + i), __ldg(rc2 + j0 + r)));
  }
  __syncthreads();
  float2 *R1 = fft_ct<N1, 0, 1, NROW, false>(X, Y, rowlay, tw1, -1);
  float2 *Rr;
  if constexpr (CL == 1) {
    const CColOnRows<RS> collay;
    float2 *C = fft_ct<N2, 0, 1, N1, true>(R1, R1 == X ? Y : X, collay, tw2, -1);
    QD_FOR_ELEMS(e, N2 * N1) {
      const int j = e / N1, i = e % N1;
      C[collay(i, j)] = cmul(C[collay(i, j)], cscale2(cmul(__ldg(p.kc1 + i), __ldg(p.kc2 + j)),
                                                        p.kscale, p.kscale_lo));
    }
    __syncthreads();
    Rr = fft_ct<N2, 0, 1, N1, true>(C, C == X ? Y : X, collay, tw2, +1);
  } else {
    cg::cluster_group cluster = cg::this_cluster();
    cluster.sync();
    float2 *G = R1 == X ? Y : X;
    const CCols<NCOL> clay;
    QD_FOR_ELEMS(e, N2 * NCOL) {
      const int j = e / NCOL, c = e % NCOL;
      const int owner = j / NROW, rr = j % NROW;
      const float2 *peer = cluster.map_shared_rank(R1, owner);
      G[clay(c, j)] = peer[rowlay(rr, rank * NCOL + c)];
    }
    cluster.sync();
    float2 *C = fft_ct<N2, 0, 1, NCOL, true>(G, G == X ? Y : X, clay, tw2, -1);
    QD_FOR_ELEMS(e, N2 * NCOL) {
      const int j = e / NCOL, c = e % NCOL;
      C[clay(c, j)] = cmul(C[clay(c, j)],
                           cscale2(cmul(__ldg(p.kc1 + rank * NCOL + c), __ldg(p.kc2 + j)),
                                   p.kscale, p.kscale_lo));
    }
    __syncthreads();
    float2 *C2 = fft_ct<N2, 0, 1, NCOL, true>(C, C == X ? Y : X, clay, tw2, +1);
    cluster.sync();
    Rr = C2 == X ? Y : X;
    QD_FOR_ELEMS(e, NROW * N1) {
      const int r = e / N1, i = e % N1;
      const int owner = i / NCOL, c = i % NCOL;
      const float2 *peer = cluster.map_shared_rank(C2, owner);
      Rr[rowlay(r, i)] = peer[clay(c, j0 + r)];
    }
    cluster.sync();
  }
  float2 *F = fft_ct<N1, 0, 1, NROW, false>(Rr, Rr == X ? Y : X, rowlay, tw1, +1);
  QD_FOR_ELEMS(e, NROW * N1) {
    const int r = e / N1, i = e % N1;
    slice[(j0 + r) * N1 + i] = cmul(F[rowlay(r, i)], cmul(__ldg(rc1 + i), __ldg(rc2 + j0 + r)));
  }
}

// compile-time kernel for (n1, n2, CL) if one is built, else the runtime one
template <int CL> void *slice_kernel_for(int n1, int n2)
{
#define QD_SLICE_CASE(A, B) \
  if (n1 == A && n2 == B) return reinterpret_cast<void *>(&k_slice_ct<A, B, CL>);
  QD_SLICE_CASE(64, 64)
  QD_SLICE_CASE(128, 128)
  QD_SLICE_CASE(128, 96)
  QD_SLICE_CASE(256, 192)
  QD_SLICE_CASE(256, 256)
#undef QD_SLICE_CASE
  return reinterpret_cast<void *>(&k_slice<CL>);
}

template <int CL> cudaError_t launch_cl(const LineParams &p, cudaStream_t s)
{
  const size_t sm = slice_smem_bytes(p.n1, p.n2, CL);
  const void *kern = slice_kernel_for<CL>(p.n1, p.n2);
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)sm);
  if (e != cudaSuccess) return e;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(p.nruns * p.nl * CL + p.flux_ctas));
  cfg.blockDim = dim3(NT);
  cfg.dynamicSmemBytes = sm;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = CL;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  LineParams pc = p;
  void *args[] = {&pc};
  return cudaLaunchKernelExC(&cfg, kern, args);
}

}  // namespace

int slice_cluster_ok(int n1, int n2, int cl)
{
  if (cl == SLICE_RF4W) return slice_rf_wide_ok(n1, n2) ? 1 : 0;
  if (slice_is_rf(cl)) return slice_rf_threads(n1, n2, slice_ctas(cl)) > 0;
  if (cl != 1 && cl != 2 && cl != 4) return 0;
  if (n1 % cl || n2 % cl) return 0;
  return slice_smem_bytes(n1, n2, cl) <= 227 * 1024 ? 1 : 0;
}

int slice_threads(int n1, int n2, int cl)
{
  return slice_is_rf(cl) ? slice_rf_threads(n1, n2, slice_ctas(cl)) : NT;
}

cudaError_t launch_slice(const LineParams &p, cudaStream_t s)
{
  switch (p.cluster) {
    case SLICE_RF: return launch_slice_rf(p, 1, s);
    case SLICE_RF2: return launch_slice_rf(p, 2, s);
    case SLICE_RF4: return launch_slice_rf(p, 4, s);
    case SLICE_RF4W: return launch_slice_rf_wide(p, s);
    case 1: return launch_cl<1>(p, s);
    case 2: return launch_cl<2>(p, s);
    case 4: return launch_cl<4>(p, s);
    default: return cudaErrorInvalidValue;
  }
}
