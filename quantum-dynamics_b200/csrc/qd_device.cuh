// qd_device.cuh -- device helpers shared by the propagator kernels:
// complex arithmetic on float2/double2 and shared-memory Stockham FFT stages.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

template <typename R> struct Cplx;
template <> struct Cplx<float> { typedef float2 T; };
template <> struct Cplx<double> { typedef double2 T; };

__device__ __forceinline__ float2 mk(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ double2 mk(double a, double b) { return make_double2(a, b); }

template <typename C> __device__ __forceinline__ C cadd(C a, C b) { return mk(a.x + b.x, a.y + b.y); }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { return mk(a.x - b.x, a.y - b.y); }
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
// complex64 sums and real scalings as one paired FP32 instruction (sm_100:
// add/sub/mul/fma on .f32x2, both halves rounded to nearest like the scalar
// forms), the real and imaginary parts in one 64-bit register pair
__device__ __forceinline__ float2 cadd(float2 a, float2 b)
{
  float2 r;
  asm("{\n\t.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
      "add.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
      : "=f"(r.x), "=f"(r.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}
__device__ __forceinline__ float2 csub(float2 a, float2 b)
{
  float2 r;
  asm("{\n\t.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
      "sub.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
      : "=f"(r.x), "=f"(r.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}
// (a.x hi + a.x lo, a.y hi + a.y lo), the compensated real scaling below
__device__ __forceinline__ float2 cscale2_f32x2(float2 a, float hi, float lo)
{
  float2 r;
  asm("{\n\t.reg .b64 ra, rh, rl, rt, rd;\n\tmov.b64 ra, {%2, %3};\n\t"
      "mov.b64 rh, {%4, %4};\n\tmov.b64 rl, {%5, %5};\n\t"
      "mul.rn.f32x2 rt, ra, rl;\n\tfma.rn.f32x2 rd, ra, rh, rt;\n\tmov.b64 {%0, %1}, rd;\n\t}"
      : "=f"(r.x), "=f"(r.y) : "f"(a.x), "f"(a.y), "f"(hi), "f"(lo));
  return r;
}
#define QD_F32X2 1
#endif
template <typename C> __device__ __forceinline__ C cmul(C a, C b)
{ return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
template <typename C> __device__ __forceinline__ C cconj(C a) { return mk(a.x, -a.y); }
template <typename C, typename S> __device__ __forceinline__ C cscale(C a, S s)
{ return mk(a.x * s, a.y * s); }
// multiply by +i (sgn > 0) or -i (sgn < 0)
template <typename C> __device__ __forceinline__ C cmul_i(C a, int sgn)
{ return sgn > 0 ? mk(-a.y, a.x) : mk(a.y, -a.x); }

__device__ __forceinline__ float2 to_c(double2 a) { return make_float2((float)a.x, (float)a.y); }
__device__ __forceinline__ double2 to_z(float2 a) { return make_double2(a.x, a.y); }
__device__ __forceinline__ double2 to_z(double2 a) { return a; }
template <typename C> __device__ __forceinline__ C from_z(double2 a);
template <> __device__ __forceinline__ float2 from_z<float2>(double2 a) { return to_c(a); }
template <> __device__ __forceinline__ double2 from_z<double2>(double2 a) { return a; }

// exp(2 pi i * turns) in FP32 from a phase given in turns (|turns| <= ~1).
__device__ __forceinline__ float2 expi_turns(float turns)
{
  float s, c;
  sincospif(2.0f * turns, &s, &c);
  return make_float2(c, s);
}

// ---------------------------------------------------------------------------
// Small DFTs in registers.  sgn = -1 forward (exp(-2 pi i qm/R)), +1 inverse.
// ---------------------------------------------------------------------------
template <int RAD, typename C> struct SmallDFT;

template <typename C> struct SmallDFT<2, C> {
  static __device__ __forceinline__ void run(C *v, int, const C *, int)
  {
    C a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};

template <typename C> struct SmallDFT<4, C> {
  static __device__ __forceinline__ void run(C *v, int sgn, const C *, int)
  {
    C a = v[0], b = v[1], c = v[2], d = v[3];
    C s0 = cadd(a, c), s1 = csub(a, c), s2 = cadd(b, d), s3 = cmul_i(csub(b, d), sgn);
    v[0] = cadd(s0, s2);
    v[2] = csub(s0, s2);
    v[1] = cadd(s1, s3);
    v[3] = csub(s1, s3);
  }
};

// Irrational butterfly constants as value + residual.  A float constant alone
// would scale some outputs of every butterfly by a fixed 1 - O(1e-8); applied
// at every stage of every step that is a systematic norm drift, so the FP32
// butterflies multiply by hi + lo (residual ~1e-15).
template <typename R> struct Konst;
template <> struct Konst<float> {
  static constexpr float rsqrt2_hi = 0.70710677f, rsqrt2_lo = 1.2101617e-8f;
  static constexpr float sqrt3h_hi = 0.8660254f, sqrt3h_lo = 1.5543624e-8f;
};
template <> struct Konst<double> {
  static constexpr double rsqrt2_hi = 0.70710678118654752440, rsqrt2_lo = 0.0;
  static constexpr double sqrt3h_hi = 0.86602540378443864676, sqrt3h_lo = 0.0;
};
template <typename C, typename R> __device__ __forceinline__ C cscale2(C a, R hi, R lo)
{ return mk(fma(a.x, hi, a.x * lo), fma(a.y, hi, a.y * lo)); }
#ifdef QD_F32X2
__device__ __forceinline__ float2 cscale2(float2 a, float hi, float lo) { return cscale2_f32x2(a, hi, lo); }
#endif

template <typename C> struct SmallDFT<8, C> {
  static __device__ __forceinline__ void run(C *v, int sgn, const C *, int)
  {
    typedef decltype(v[0].x) R;
    C e[4] = {v[0], v[2], v[4], v[6]};
    C o[4] = {v[1], v[3], v[5], v[7]};
    SmallDFT<4, C>::run(e, sgn, nullptr, 0);
    SmallDFT<4, C>::run(o, sgn, nullptr, 0);
    // w8^m = exp(sgn 2 pi i m / 8):  w8 = (1 + sgn i)/sqrt2, w8^3 = (-1 + sgn i)/sqrt2
    const R hh = Konst<R>::rsqrt2_hi, hl = Konst<R>::rsqrt2_lo;
    C t1 = cscale2(cadd(o[1], cmul_i(o[1], sgn)), hh, hl);
    C t2 = cmul_i(o[2], sgn);
    C t3 = cscale2(csub(cmul_i(o[3], sgn), o[3]), hh, hl);
    v[0] = cadd(e[0], o[0]); v[4] = csub(e[0], o[0]);
    v[1] = cadd(e[1], t1);   v[5] = csub(e[1], t1);
    v[2] = cadd(e[2], t2);   v[6] = csub(e[2], t2);
    v[3] = cadd(e[3], t3);   v[7] = csub(e[3], t3);
  }
};

template <typename C> struct SmallDFT<3, C> {
  static __device__ __forceinline__ void run(C *v, int sgn, const C *, int)
  {
    typedef decltype(v[0].x) R;
    C a = v[0], b = v[1], c = v[2];
    C s = cadd(b, c);
    C t = mk(a.x - (R)0.5 * s.x, a.y - (R)0.5 * s.y);
    C u = cmul_i(cscale2(csub(b, c), Konst<R>::sqrt3h_hi, Konst<R>::sqrt3h_lo), sgn);
    v[0] = cadd(a, s);
    v[1] = cadd(t, u);
    v[2] = csub(t, u);
  }
};

// Generic radix from the n-point root table tw[k] = exp(-2 pi i k / n).
template <int RAD, typename C> struct SmallDFTGeneric {
  static __device__ __forceinline__ void run(C *v, int sgn, const C *tw, int n)
  {
    C out[RAD];
    const int st = n / RAD;
#pragma unroll
    for (int m = 0; m < RAD; m++) {
      C acc = v[0];
#pragma unroll
      for (int q = 1; q < RAD; q++) {
        C w = tw[((q * m) % RAD) * st];
        if (sgn > 0) w = cconj(w);
        acc = cadd(acc, cmul(v[q], w));
      }
      out[m] = acc;
    }
#pragma unroll
    for (int m = 0; m < RAD; m++) v[m] = out[m];
  }
};
template <typename C> struct SmallDFT<5, C> : SmallDFTGeneric<5, C> {};

// ---------------------------------------------------------------------------
// One Stockham stage over many lines held in shared memory.
//   n        line length;   Ns  product of the radices of earlier stages
//   line l, element e at  base[l * lstride + e * estride]
//   lines_fast: consecutive threads walk lines (columns) instead of elements
// Reads src, writes dst (distinct buffers).  tw: n roots exp(-2 pi i k/n).
// ---------------------------------------------------------------------------
template <int RAD, typename C>
__device__ __forceinline__ void stockham_stage(const C *__restrict__ src, C *__restrict__ dst,
                                               int n, int Ns, int nlines, int lstride,
                                               int estride, bool lines_fast,
                                               const C *__restrict__ tw, int sgn)
{
  const int nb = n / RAD;
  const int total = nb * nlines;
  const int tstep = n / (Ns * RAD);
  for (int b = threadIdx.x; b < total; b += blockDim.x) {
    int line, j;
    if (lines_fast) { line = b % nlines; j = b / nlines; }
    else            { line = b / nb;     j = b % nb; }
    const C *s = src + line * lstride;
    C *d = dst + line * lstride;
    C v[RAD];
#pragma unroll
    for (int r = 0; r < RAD; r++) v[r] = s[(j + r * nb) * estride];
    const int k = j % Ns;
    if (Ns > 1) {
#pragma unroll
      for (int r = 1; r < RAD; r++) {
        C w = tw[r * k * tstep];
        if (sgn > 0) w = cconj(w);
        v[r] = cmul(v[r], w);
      }
    }
    SmallDFT<RAD, C>::run(v, sgn, tw, n);
    const int o = (j / Ns) * Ns * RAD + k;
#pragma unroll
    for (int r = 0; r < RAD; r++) d[(o + r * Ns) * estride] = v[r];
  }
}

struct FftPlan {
  int n;
  int nst;
  int rad[16];
};

// Full 1-D FFT of all lines: ping-pong between bufA and bufB.  Returns the
// buffer that holds the result.  All threads of the block must call it.
template <typename C>
__device__ C *smem_fft_lines(C *bufA, C *bufB, const FftPlan &pl, int nlines, int lstride,
                             int estride, bool lines_fast, const C *tw, int sgn)
{
  C *src = bufA, *dst = bufB;
  int Ns = 1;
  for (int s = 0; s < pl.nst; s++) {
    const int R = pl.rad[s];
    switch (R) {
      case 2: stockham_stage<2>(src, dst, pl.n, Ns, nlines, lstride, estride, lines_fast, tw, sgn); break;
      case 3: stockham_stage<3>(src, dst, pl.n, Ns, nlines, lstride, estride, lines_fast, tw, sgn); break;
      case 4: stockham_stage<4>(src, dst, pl.n, Ns, nlines, lstride, estride, lines_fast, tw, sgn); break;
      case 5: stockham_stage<5>(src, dst, pl.n, Ns, nlines, lstride, estride, lines_fast, tw, sgn); break;
      default: stockham_stage<8>(src, dst, pl.n, Ns, nlines, lstride, estride, lines_fast, tw, sgn); break;
    }
    __syncthreads();
    C *t = src; src = dst; dst = t;
    Ns *= R;
  }
  return src;
}

// Block-wide FP64 sum; result valid in thread 0.  red: >= 32 doubles of smem.
__device__ __forceinline__ double block_sum(double v, double *red)
{
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  const int nw = (blockDim.x + 31) >> 5;
  v = (threadIdx.x < nw) ? red[threadIdx.x] : 0.0;
  if (wid == 0)
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
