// k_slice_rf.cu -- the l-space part of one complex64 split-operator step,
//     psi_l <- Rot(dt/2) IFFT2 [exp(-i(T1+T2)dt)/(n1 n2)] FFT2 Rot(dt/2) psi_l
// (evolution_dt, timeEvol.C:625-635; the FFTW 2-D DFT pair of
// fftwinterface.C:70-76; phase tables timeEvol.C:465-517), one l-slice per
// CTA (or per 2- or 4-CTA cluster), with every 1-D transform done as two
// register passes.
//
// Both phases are separable in (R, r): Rot(dt/2) = D1(i) D2(j) with
// D1 = exp(-i l(l+1) I_R(i) dt/2), D2 likewise with I_r(j), and the kinetic
// phase is K1(k_i) K2(k_j).  A diagonal factor in i commutes with any
// operator along j and vice versa, so the slice operator is the product of
// a row operator and a column operator,
//     [D1 IFFT_R K1 FFT_R D1] (each row j)  x  [D2 IFFT_r K2 FFT_r D2] (each column i),
// which is applied in that order: the row operator works on whole rows, the
// column operator on whole columns, and the slice goes back to global memory
// straight from the column passes.  The arithmetic is that of the reference's
// 2-D transform pair, regrouped (rounding differs at the 1e-7 level).
//
// A length N = A*B transform (n = a + A b, k = c + B d) is
//   pass 1, one item per a:  B-point DFT over b in registers, times W_N^{a c}
//   pass 2, one item per c:  A-point DFT over a in registers -> X[c + B d]
// and its inverse mirrors it (an A-point inverse DFT over d per c, times
// W_N^{-a c}, then a B-point inverse DFT over c per a).  Pass 2 of the forward
// transform, the phase and pass 1 of the inverse share one item, so each 1-D
// operator costs three register passes and two shared-memory round trips.
// The slice lives in shared memory in ONE padded layout, every pass works in
// place, and five barriers separate the six passes:
//   Pa  global -> regs: D1, row pass 1 (B1-pt), twiddle               -> smem
//   Pb  row pass 2 (A1-pt), K1, inverse row pass 1 (A1-pt)            in place
//   Pc  twiddle, inverse row pass 2 (B1-pt), D1                       in place
//   Pd  D2, column pass 1 (B2-pt), twiddle                            in place
//   Pe  column pass 2 (A2-pt), K2/(n1 n2), inverse column pass 1, tw. in place
//   Pf  inverse column pass 2 (B2-pt), D2                             -> global
// Row layout: element i of a row sits at slot i % A1 of block i / A1, slot s
// of block c at s + (A1+1) c; row stride RS = N1 + B1 (= 8 mod 16 complex).
// Between Pa and Pc the row holds its transform at slot d of block c
// (frequency c + B1 d).  With this padding every warp access of every pass
// touches each shared-memory bank at most twice (the minimum for 8-byte
// elements), and global loads and stores are whole 64- or 128-byte segments.
//
// The phase tables (rc1[l] and rc2[l], kc1, kc2) and the N2-point roots are
// staged in shared memory by the prologue, which runs before the previous
// kernel's results are waited on.
//
// Energy steps (LineParams::esum): Pb, Pe and Pf also sum, in FP64, the
// kinetic energy from the row and column transforms (Parseval along the other
// dimension) and the rotational energy of the step's final l-space values.
//
// A slice may also run on a 2-CTA cluster (for small batches, where one CTA
// per slice leaves most SMs idle) or, at 256 x 192 (384 KB), on a 4-CTA
// cluster: each CTA then keeps 1/CL of the rows for the row passes and 1/CL
// of the columns, over all rows, for the column passes.  The one transpose
// between them is folded into the last row pass, which stores each result
// into the CTA whose columns it belongs to (rounds of rows between cluster
// barriers), so each CTA holds only its own rows (101 KB at 256 x 192, where
// two clusters' CTAs share an SM).
//
// The 6-, 12-, 16-, 24- and 32-point DFTs are P x Q compositions whose
// internal twiddles are compensated constants (value + residual), like the
// radix-8 and radix-3 butterflies, so no fixed-point rounding bias enters
// the norm.
#include <cstdlib>
#include "qd_kernels.h"

namespace {

// ---- compile-time twiddles exp(SGN 2 pi i E / N) --------------------------
// cos(2 pi a / 96) as (magnitude code, sign); a in [0, 96), a multiple of 3 or 4.
// codes: 0 -> 0, 1 -> 1, 2 -> 1/2, 3 -> 1/sqrt2, 4 -> sqrt3/2, 5 -> cos(pi/8),
// 6 -> sin(pi/8), 7 -> cos(pi/16), 8 -> cos(3pi/16), 9 -> sin(3pi/16),
// 10 -> sin(pi/16), 11 -> cos(pi/12), 12 -> sin(pi/12)
__host__ __device__ constexpr int kcode(int a)
{
  const int r = a % 48 <= 24 ? a % 48 : 48 - a % 48;    // |cos| is even in a and 48-periodic
  return r == 0 ? 1 : r == 3 ? 7 : r == 4 ? 11 : r == 6 ? 5 : r == 8 ? 4 : r == 9 ? 8
       : r == 12 ? 3 : r == 15 ? 9 : r == 16 ? 2 : r == 18 ? 6 : r == 20 ? 12 : r == 21 ? 10
       : r == 24 ? 0 : -1;
}
__host__ __device__ constexpr int ksign(int a)
{
  return (a % 96 > 24 && a % 96 < 72) ? -1 : 1;
}

template <int CODE> __device__ __forceinline__ float kmag(float x)
{
  if constexpr (CODE == 1) return x;
  else if constexpr (CODE == 2) return 0.5f * x;
  else if constexpr (CODE == 3) return fmaf(x, 7.07106769e-01f, x * 1.21016175e-08f);
  else if constexpr (CODE == 4) return fmaf(x, 8.66025388e-01f, x * 1.55436251e-08f);
  else if constexpr (CODE == 5) return fmaf(x, 9.23879504e-01f, x * 2.83074897e-08f);
  else if constexpr (CODE == 6) return fmaf(x, 3.82683426e-01f, x * 6.22335072e-09f);
  else if constexpr (CODE == 7) return fmaf(x, 9.80785251e-01f, x * 2.97394731e-08f);
  else if constexpr (CODE == 8) return fmaf(x, 8.31469595e-01f, x * 1.68702634e-08f);
  else if constexpr (CODE == 9) return fmaf(x, 5.55570245e-01f, x * -1.17695214e-08f);
  else if constexpr (CODE == 10) return fmaf(x, 1.95090324e-01f, x * -1.67047143e-09f);
  else if constexpr (CODE == 11) return fmaf(x, 9.65925813e-01f, x * 1.35678162e-08f);
  else if constexpr (CODE == 12) return fmaf(x, 2.58819044e-01f, x * 1.46619872e-09f);
  else return 0.f;
}

// x * cos(2 pi A / 96)
template <int A> __device__ __forceinline__ float kcos(float x)
{
  static_assert(kcode(A) >= 0, "angle not in the table");
  const float v = kmag<kcode(A)>(x);
  return ksign(A) < 0 ? -v : v;
}

#ifdef QD_F32X2
// z * |cos(2 pi A / 96)| for both parts of z (the sign is the caller's)
template <int CODE> __device__ __forceinline__ float2 kmag2(float2 z)
{
  if constexpr (CODE == 1) return z;
  else if constexpr (CODE == 2) return make_float2(0.5f * z.x, 0.5f * z.y);
  else if constexpr (CODE == 3) return cscale2_f32x2(z, 7.07106769e-01f, 1.21016175e-08f);
  else if constexpr (CODE == 4) return cscale2_f32x2(z, 8.66025388e-01f, 1.55436251e-08f);
  else if constexpr (CODE == 5) return cscale2_f32x2(z, 9.23879504e-01f, 2.83074897e-08f);
  else if constexpr (CODE == 6) return cscale2_f32x2(z, 3.82683426e-01f, 6.22335072e-09f);
  else if constexpr (CODE == 7) return cscale2_f32x2(z, 9.80785251e-01f, 2.97394731e-08f);
  else if constexpr (CODE == 8) return cscale2_f32x2(z, 8.31469595e-01f, 1.68702634e-08f);
  else if constexpr (CODE == 9) return cscale2_f32x2(z, 5.55570245e-01f, -1.17695214e-08f);
  else if constexpr (CODE == 10) return cscale2_f32x2(z, 1.95090324e-01f, -1.67047143e-09f);
  else if constexpr (CODE == 11) return cscale2_f32x2(z, 9.65925813e-01f, 1.35678162e-08f);
  else if constexpr (CODE == 12) return cscale2_f32x2(z, 2.58819044e-01f, 1.46619872e-09f);
  else return make_float2(0.f, 0.f);
}
#endif

template <int N, int E, int SGN> __device__ __forceinline__ float2 twk(float2 z)
{
  static_assert(96 % N == 0, "N must divide 96");
  constexpr int a = (E % N) * (96 / N);
  constexpr int as = (a + 72) % 96;                     // sin(t) = cos(t - pi/2)
  if constexpr (a == 0) {
    return z;
  } else {
    float re, im;
    if constexpr (kcode(as) == 0) {                     // sin = 0
      re = kcos<a>(z.x);
      im = kcos<a>(z.y);
    } else if constexpr (kcode(a) == 0) {               // cos = 0
      re = SGN > 0 ? -kcos<as>(z.y) : kcos<as>(z.y);
      im = SGN > 0 ? kcos<as>(z.x) : -kcos<as>(z.x);
    } else {
#ifdef QD_F32X2
      // (c x, c y) and (s x, s y) as paired products, then the cross sums
      const float2 C = kmag2<kcode(a)>(z), Sn = kmag2<kcode(as)>(z);
      const float cx = ksign(a) < 0 ? -C.x : C.x, cy = ksign(a) < 0 ? -C.y : C.y;
      const float sx = ksign(as) < 0 ? -Sn.x : Sn.x, sy = ksign(as) < 0 ? -Sn.y : Sn.y;
      re = SGN > 0 ? cx - sy : cx + sy;
      im = SGN > 0 ? sx + cy : cy - sx;
#else
      re = SGN > 0 ? kcos<a>(z.x) - kcos<as>(z.y) : kcos<a>(z.x) + kcos<as>(z.y);
      im = SGN > 0 ? kcos<as>(z.x) + kcos<a>(z.y) : kcos<a>(z.y) - kcos<as>(z.x);
#endif
    }
    return make_float2(re, im);
  }
}

// ---- DFTs in registers, natural order in and out --------------------------
template <int N, int SGN> struct Dft;
template <int SGN> struct Dft<2, SGN> {
  static __device__ __forceinline__ void run(float2 *v) { SmallDFT<2, float2>::run(v, SGN, nullptr, 0); }
};
template <int SGN> struct Dft<3, SGN> {
  static __device__ __forceinline__ void run(float2 *v) { SmallDFT<3, float2>::run(v, SGN, nullptr, 0); }
};
template <int SGN> struct Dft<4, SGN> {
  static __device__ __forceinline__ void run(float2 *v) { SmallDFT<4, float2>::run(v, SGN, nullptr, 0); }
};
template <int SGN> struct Dft<8, SGN> {
  static __device__ __forceinline__ void run(float2 *v) { SmallDFT<8, float2>::run(v, SGN, nullptr, 0); }
};

// N = P Q: n = p + P q, Q-point DFTs over q, twiddles W_N^{p c}, P-point
// DFTs over p, X[c + Q d]
template <int N, int P, int Q, int SGN> struct DftPxQ {
  template <int PP, int C> static __device__ __forceinline__ void tw(float2 (&u)[P][Q])
  {
    if constexpr (C < Q) {
      u[PP][C] = twk<N, PP * C, SGN>(u[PP][C]);
      tw<PP, C + 1>(u);
    } else if constexpr (PP + 1 < P) {
      tw<PP + 1, 0>(u);
    }
  }
  static __device__ __forceinline__ void run(float2 *v)
  {
    float2 u[P][Q];
#pragma unroll
    for (int p = 0; p < P; p++) {
#pragma unroll
      for (int q = 0; q < Q; q++) u[p][q] = v[p + P * q];
      Dft<Q, SGN>::run(u[p]);
    }
    tw<1, 1>(u);
#pragma unroll
    for (int c = 0; c < Q; c++) {
      float2 s[P];
#pragma unroll
      for (int p = 0; p < P; p++) s[p] = u[p][c];
      Dft<P, SGN>::run(s);
#pragma unroll
      for (int d = 0; d < P; d++) v[c + Q * d] = s[d];
    }
  }
};
template <int SGN> struct Dft<6, SGN> {
  static __device__ __forceinline__ void run(float2 *v) { DftPxQ<6, 2, 3, SGN>::run(v); }
};
template <int SGN> struct Dft<12, SGN> {
  static __device__ __forceinline__ void run(float2 *v) { DftPxQ<12, 4, 3, SGN>::run(v); }
};
template <int SGN> struct Dft<16, SGN> {
  static __device__ __forceinline__ void run(float2 *v) { DftPxQ<16, 4, 4, SGN>::run(v); }
};
template <int SGN> struct Dft<24, SGN> {
  static __device__ __forceinline__ void run(float2 *v) { DftPxQ<24, 4, 6, SGN>::run(v); }
};
template <int SGN> struct Dft<32, SGN> {
  static __device__ __forceinline__ void run(float2 *v) { DftPxQ<32, 4, 8, SGN>::run(v); }
};

// A1X: row pass 2 radix (0: the default of the size, B1 = 8; 16 for N1 = 256
// gives B1 = 16, i.e. twice the row-pass-2 items at half their registers)
template <int N1, int N2, int NT, int CL, int A1X = 0> struct RfShape {
  static constexpr int A1 = A1X ? A1X : N1 == 64 ? 8 : N1 == 256 ? 32 : 16;   // row pass 2 radix
  static constexpr int B1 = N1 / A1;
  static constexpr int A2 = N2 / 8;                   // column pass 2 radix (B2 = 8)
  static constexpr int B2 = 8;
  static constexpr int RS = N1 + B1;                  // padded row stride (complex)
  static constexpr int HR = N2 / CL;                  // rows held by one CTA
  static constexpr int HW = RS / CL;                  // column part width: B1 / CL whole blocks
  static constexpr int BPO = B2 / CL;                 // column-pass row groups per CTA's rows
  // CL > 1: the transpose moves row parts between the CTAs' row arrays in
  // place (pc_swap), so a CTA holds only its own rows
  static constexpr int P1_UNROLL = 2;                // row items per thread loaded together
  // own rows [HR][RS]; rc1[l], kc1 (N1 each), W_N2, kc2, rc2[l] (N2 each)
  static constexpr size_t TABLES = 2 * N1 + 3 * N2;
  static constexpr size_t SMEM = sizeof(float2) * ((size_t)HR * RS + TABLES);
  // 8 B1 blocks of A1 + 1 slots with RS = 8 mod 16, or 16 blocks with RS = 0
  // mod 16: either way a warp's access of any pass touches each bank pair twice
  static_assert((B1 == 8 && RS % 16 == 8) || (B1 == 16 && RS % 16 == 0), "row layout");
  static_assert(NT % A1 == 0 && NT % B1 == 0, "per-thread constant row index");
  static_assert(CL == 1 || ((CL == 2 || CL == 4) && B1 % CL == 0 && HR == BPO * A2 &&
                            HW == (B1 / CL) * (A1 + 1)),
                "cluster split: whole row blocks per column part, whole column row groups per CTA");
};

__device__ __forceinline__ uint32_t smem_addr(const void *p)
{ return (uint32_t)__cvta_generic_to_shared(p); }
// the same shared-memory offset in CTA `rank` of the cluster
__device__ __forceinline__ uint32_t peer_addr(uint32_t a, uint32_t rank)
{
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
  return r;
}
__device__ __forceinline__ void cluster_arrive_release()
{ asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory"); }
__device__ __forceinline__ void cluster_wait()
{ asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory"); }
// st.shared::cluster of 8 bytes (a mapa address)
__device__ __forceinline__ void st_peer2(uint32_t a, float2 v)
{
  asm volatile("st.shared::cluster.v2.f32 [%0], {%1, %2};" :: "r"(a), "f"(v.x), "f"(v.y) : "memory");
}

// Pc fused with the in-place transpose of a CL-CTA slice.  In rounds of whole
// rows, one item (j, a) per thread: the thread loads slot a of every block of
// row j, arrives on the cluster barrier once the values are in its registers,
// runs the inverse row pass (W^{-a c}, B1-point inverse DFT over c, D1) while
// the other CTAs arrive, waits, and stores each result where the column passes
// read it: block b of row j lies in column part o = b / (B1 / CL), which CTA o
// holds as row part `rank` of its row j, in CTA o's column part.  Every CTA has read a round's rows before any CTA writes into them,
// the rounds' rows are disjoint, and the closing barrier (release, acquire)
// makes every store visible to the column passes.
template <int A1, int B1, int RS, int HR, int HW, int NT, int CL>
__device__ __forceinline__ void pc_swap(float2 *R, const float2 *r1, const float2 *tw1, int rank,
                                        int tid)
{
  constexpr int BPP = B1 / CL;                        // row blocks per column part
  constexpr int NRF = HR * A1 / NT;                   // rounds: one item per thread each
  constexpr int RPR = HR / NRF;                       // rows per round
  static_assert(NRF >= 1 && NRF * NT == HR * A1 && HR % NRF == 0 && NT % A1 == 0,
                "one item per thread and round, whole rows per round");
  static_assert(HW == BPP * (A1 + 1), "column parts of whole row blocks");
  const int a = tid % A1;
  float2 w[B1];
#pragma unroll
  for (int c = 0; c < B1; c++) w[c] = cconj(__ldg(tw1 + a * c));
  uint32_t rb[CL];                                    // the row array in each CTA of the cluster
#pragma unroll
  for (int o = 0; o < CL; o++) rb[o] = peer_addr(smem_addr(R), (uint32_t)o);
  __shared__ uint32_t sink;                           // a store that reads every loaded value
#pragma unroll 1
  for (int r = 0; r < NRF; r++) {
    const int j = r * RPR + tid / A1;
    float2 v[B1];
    uint32_t dep = 0;
#pragma unroll
    for (int c = 0; c < B1; c++) {
      v[c] = R[j * RS + a + (A1 + 1) * c];
      dep |= __float_as_uint(v[c].x) | __float_as_uint(v[c].y);
    }
    asm volatile("st.shared.u32 [%0], %1;\n\tbarrier.cluster.arrive.relaxed.aligned;"
                 :: "r"(smem_addr(&sink)), "r"(dep) : "memory");
#pragma unroll
    for (int c = 1; c < B1; c++) v[c] = cmul(v[c], w[c]);
    Dft<B1, +1>::run(v);
#pragma unroll
    for (int b = 0; b < B1; b++) v[b] = cmul(v[b], r1[a + A1 * b]);
    cluster_wait();
#pragma unroll
    for (int b = 0; b < B1; b++) {
      const int o = b / BPP;
      st_peer2(rb[o] + (uint32_t)sizeof(float2) * (j * RS + HW * rank + a + (A1 + 1) * (b - o * BPP)),
               v[b]);
    }
  }
  cluster_arrive_release();
  cluster_wait();
}

// CL = 2 or 4: a CL-CTA thread-block cluster per slice.  CTA `rank` runs
// the row passes on rows [rank HR, (rank+1) HR) and the column passes on
// column part `rank` (row blocks rank B1/CL .. (rank+1) B1/CL - 1, columns
// rank N1/CL .. (rank+1) N1/CL - 1) over all N2 rows.  Pc stores its results
// into the CTA that holds their column part (pc_swap), after which row part o
// of the row array holds CTA o's rows in this CTA's column part; every load
// and store of the other passes is local.  CL = 1 keeps the slice in one array
// in place.
template <int N1, int N2, int NT, int CL, int A1X>
__global__ void __launch_bounds__(NT, 512 / NT) k_slice_rf(LineParams p)
{
  using Sh = RfShape<N1, N2, NT, CL, A1X>;
  constexpr int A1 = Sh::A1, B1 = Sh::B1, A2 = Sh::A2, B2 = Sh::B2, RS = Sh::RS;
  constexpr int HR = Sh::HR, HW = Sh::HW;
  extern __shared__ float4 smem4[];
  float2 *R = reinterpret_cast<float2 *>(smem4);    // own rows [HR][RS]
  float2 *r1 = R + HR * RS;                          // rc1[l][0..N1)
  float2 *k1 = r1 + N1;                              // kc1
  float2 *t2 = k1 + N1;                              // W_N2^k, k < N2
  float2 *k2 = t2 + N2;                              // kc2
  float2 *r2 = k2 + N2;                              // rc2[l][0..N2)
  __shared__ double red[32];                         // energy steps: block sums
  const int tid = threadIdx.x;
  pdl_trigger();
  if ((int)blockIdx.x >= p.nruns * p.nl * CL) {      // extra CTAs: flux preparation
    pdl_wait();
    const int q = ((int)blockIdx.x - p.nruns * p.nl * CL) * NT + tid;
    if (q < p.flux.nruns * p.flux.nth * p.flux.n1) flux_point<float2>(p.flux, q);
    return;
  }
  int rank = 0;
  if constexpr (CL > 1) asm("mov.u32 %0, %%cluster_ctarank;" : "=r"(rank));
  const int sl = blockIdx.x / CL, l = rot_row(p, sl);   // slice = run * nl + l; l = table row
  const int j0 = rank * HR, q0 = rank * (N1 / CL);
  float2 *g = reinterpret_cast<float2 *>(p.lpsi) + (long)sl * (N1 * N2);
  const float2 *tw1 = reinterpret_cast<const float2 *>(p.tw1);
  const float2 *tw2 = reinterpret_cast<const float2 *>(p.tw2);
  for (int e = tid; e < N1; e += NT) {
    r1[e] = __ldg(p.rc1 + l * N1 + e);
    k1[e] = __ldg(p.kc1 + e);
  }
  for (int e = tid; e < N2; e += NT) {
    t2[e] = __ldg(tw2 + e);
    k2[e] = __ldg(p.kc2 + e);
    r2[e] = __ldg(p.rc2 + l * N2 + e);
  }
  pdl_wait();                                        // psi_l: the column pass's output
  __syncthreads();
  // energy step: this thread's shares of sum_k T1 |row FFT|^2, of sum T2 |column
  // FFT|^2 and of sum (I1 + I2) |psi_l|^2 (the kinetic sums before their phases,
  // whose moduli are one)
  const bool en = p.esum != nullptr;
  double e_k1 = 0.0, e_k2 = 0.0, e_r = 0.0;

  // ---- the row operator D1 IFFT_R K1 FFT_R D1 on this CTA's rows ------------------
  // Pa: items (j, a): elements i = a + A1 b from global, D1, B1-point DFT over
  // b, W^{a c} -> slot a of block c
  {
    const int a = tid % A1;
    float2 w[B1];
#pragma unroll
    for (int c = 0; c < B1; c++) w[c] = __ldg(tw1 + a * c);
#pragma unroll (Sh::P1_UNROLL)
    for (int e = tid; e < HR * A1; e += NT) {
      const int j = e / A1, jg = j0 + j;
      float2 v[B1];
#pragma unroll
      for (int b = 0; b < B1; b++) v[b] = g[jg * N1 + a + A1 * b];
#pragma unroll
      for (int b = 0; b < B1; b++) v[b] = cmul(v[b], r1[a + A1 * b]);
      Dft<B1, -1>::run(v);
#pragma unroll
      for (int c = 0; c < B1; c++) R[j * RS + a + (A1 + 1) * c] = c ? cmul(v[c], w[c]) : v[c];
    }
  }
  __syncthreads();
  // Pb: items (j, c): the A1-point DFT over the slots a of block c gives
  // frequency c + B1 d at d; K1; the A1-point inverse DFT over d gives slot a
  for (int e = tid; e < HR * B1; e += NT) {
    const int j = e / B1, c = e % B1;
    float2 *blk = R + j * RS + (A1 + 1) * c;
    float2 v[A1];
#pragma unroll
    for (int a = 0; a < A1; a++) v[a] = blk[a];
    Dft<A1, -1>::run(v);
    if (en) {
#pragma unroll
      for (int d = 0; d < A1; d++)
        e_k1 += (double)(v[d].x * v[d].x + v[d].y * v[d].y) * __ldg(p.T1 + c + B1 * d);
    }
#pragma unroll
    for (int d = 0; d < A1; d++) v[d] = cmul(v[d], k1[c + B1 * d]);
    Dft<A1, +1>::run(v);
#pragma unroll
    for (int a = 0; a < A1; a++) blk[a] = v[a];
  }
  __syncthreads();
  // Pc: items (j, a): slot a of every block c, W^{-a c}, B1-point inverse DFT
  // over c -> element i = a + A1 b, D1 -> slot a of block b (the same slots);
  // CL > 1: fused with the transpose (pc_swap)
  if constexpr (CL == 1) {
    const int a = tid % A1;
    float2 w[B1];
#pragma unroll
    for (int c = 0; c < B1; c++) w[c] = cconj(__ldg(tw1 + a * c));
#pragma unroll 2
    for (int e = tid; e < HR * A1; e += NT) {
      const int j = e / A1;
      float2 v[B1];
#pragma unroll
      for (int c = 0; c < B1; c++) v[c] = R[j * RS + a + (A1 + 1) * c];
#pragma unroll
      for (int c = 1; c < B1; c++) v[c] = cmul(v[c], w[c]);
      Dft<B1, +1>::run(v);
#pragma unroll
      for (int b = 0; b < B1; b++) R[j * RS + a + (A1 + 1) * b] = cmul(v[b], r1[a + A1 * b]);
    }
    __syncthreads();
  } else {
    pc_swap<A1, B1, RS, HR, HW, NT, CL>(R, r1, tw1, rank, tid);
  }

  // ---- the column operator D2 IFFT_r K2 FFT_r D2 on this CTA's columns ------------
  // column counter qq: column i = q0 + qq at offset pcol(qq) of this CTA's
  // part; row A2 b + r (b < B2) is held by CTA b / BPO, as its row A2 (b % BPO) + r
  constexpr int BPO = Sh::BPO;
  auto pcol = [](int qq) { return (qq % A1) + (A1 + 1) * (qq / A1); };
  auto at = [&](int b, int inner, int qq) -> float2 & {
    return R[(inner + A2 * (b % BPO)) * RS + HW * (b / BPO) + pcol(qq)];
  };
  constexpr int QC = N1 / CL;
  // Pd: items (q, a'): rows a' + A2 b, D2, B2-point DFT over b, W^{a' c} -> rows a' + A2 c
  for (int e = tid; e < QC * A2; e += NT) {
    const int qq = e % QC, ap = e / QC;
    float2 v[B2];
#pragma unroll
    for (int b = 0; b < B2; b++) v[b] = cmul(at(b, ap, qq), r2[ap + A2 * b]);
    Dft<B2, -1>::run(v);
#pragma unroll
    for (int c = 0; c < B2; c++) at(c, ap, qq) = c ? cmul(v[c], t2[ap * c]) : v[c];
  }
  __syncthreads();
  // Pe: items (q, c'): rows a' + A2 c'; forward pass 2, K2 / (n1 n2), inverse pass 1
  for (int e = tid; e < QC * B2; e += NT) {
    const int qq = e % QC, cp = e / QC;
    float2 *col = R + A2 * (cp % BPO) * RS + HW * (cp / BPO) + pcol(qq);
    constexpr int cst = RS;
    float2 v[A2];
#pragma unroll
    for (int a = 0; a < A2; a++) v[a] = col[a * cst];
    Dft<A2, -1>::run(v);
    if (en) {
#pragma unroll
      for (int d = 0; d < A2; d++)
        e_k2 += (double)(v[d].x * v[d].x + v[d].y * v[d].y) * __ldg(p.T2 + cp + B2 * d);
    }
#pragma unroll
    for (int d = 0; d < A2; d++)
      v[d] = cmul(v[d], cscale2(k2[cp + B2 * d], p.kscale, p.kscale_lo));
    Dft<A2, +1>::run(v);
#pragma unroll
    for (int cc = 0; cc < A2; cc++) col[cc * cst] = cc ? cmul(v[cc], cconj(t2[cp * cc])) : v[cc];
  }
  __syncthreads();
  // Pf: items (q, c''): rows c'' + A2 a -> natural rows j = c'' + A2 d, D2 -> global
#pragma unroll 2
  for (int e = tid; e < QC * A2; e += NT) {
    const int qq = e % QC, cc = e / QC;
    float2 v[B2];
#pragma unroll
    for (int a = 0; a < B2; a++) v[a] = at(a, cc, qq);
    Dft<B2, +1>::run(v);
#pragma unroll
    for (int d = 0; d < B2; d++) {
      const int j = cc + A2 * d;
      g[j * N1 + q0 + qq] = cmul(v[d], r2[j]);
    }
    if (en) {
      const double i1 = __ldg(p.I1 + q0 + qq);
#pragma unroll
      for (int d = 0; d < B2; d++)
        e_r += (double)(v[d].x * v[d].x + v[d].y * v[d].y) * (i1 + __ldg(p.I2 + cc + A2 * d));
    }
  }
  if (en) {
    // E_kin (dr1 dr2 applied on the host) = [n2 S1 + S2 / n1] / (n1 n2): S1 sums
    // T1 over the row transforms of D1 psi, S2 sums T2 over the column transforms
    // of the row operator's output, which carries the factor n1 of the
    // unnormalised row transform pair (Parseval along the other dimension)
    const int run = sl / p.nl, ll = sl - run * p.nl;
    const double wl = p.orth ? 1.0 : 1.0 / (ll + 0.5);
    const double jj = (double)l;                     // rotational quantum number j = K + l
    const double ek = block_sum(e_k1 / N1 + e_k2 / ((double)N1 * N1 * N2), red);
    if (tid == 0) atomicAdd(p.esum + 3 * run, ek * wl);
    const double er = block_sum(e_r, red);
    if (tid == 0) atomicAdd(p.esum + 3 * run + 1, er * jj * (jj + 1.0) * wl);
  }
  // (no CTA touches a peer's memory after the transpose's closing barrier)
}

template <int N1, int N2, int NT, int CL, int A1X = 0>
cudaError_t launch_rf(const LineParams &p, cudaStream_t s)
{
  constexpr size_t sm = RfShape<N1, N2, NT, CL, A1X>::SMEM;
  cudaError_t e = cudaFuncSetAttribute(k_slice_rf<N1, N2, NT, CL, A1X>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(p.nruns * p.nl * CL + p.flux_ctas));
  cfg.blockDim = dim3(NT);
  cfg.dynamicSmemBytes = sm;
  cfg.stream = s;
  cudaLaunchAttribute attr[2];
  int na = 0;
  if (CL > 1) {
    attr[na].id = cudaLaunchAttributeClusterDimension;
    attr[na].val.clusterDim.x = CL;
    attr[na].val.clusterDim.y = 1;
    attr[na].val.clusterDim.z = 1;
    na++;
  }
  if (pdl_enabled()) {
    attr[na].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[na].val.programmaticStreamSerializationAllowed = 1;
    na++;
  }
  cfg.attrs = attr;
  cfg.numAttrs = na;
  cudaLaunchKernelEx(&cfg, k_slice_rf<N1, N2, NT, CL, A1X>, p);
  return cudaGetLastError();
}

}  // namespace

int slice_rf_threads(int n1, int n2, int cl)
{
  if (cl == 1) {
    if (n1 == 64 && n2 == 64) return 256;
    if (n1 == 128 && n2 == 96) return 256;
    if (n1 == 128 && n2 == 128) return 512;
  } else if (cl == 2) {
    if (n1 == 128 && n2 == 96) return 256;
    if (n1 == 128 && n2 == 128) return 512;
  } else if (cl == 4) {
    if (n1 == 256 && n2 == 192) return 256;   // 128 x 96 and 128 x 128 run faster on CL <= 2
  }
  return 0;
}

cudaError_t launch_slice_rf(const LineParams &p, int cl, cudaStream_t s)
{
  if (cl == 1) {
    if (p.n1 == 64 && p.n2 == 64) return launch_rf<64, 64, 256, 1>(p, s);
    if (p.n1 == 128 && p.n2 == 96) return launch_rf<128, 96, 256, 1>(p, s);
    if (p.n1 == 128 && p.n2 == 128) return launch_rf<128, 128, 512, 1>(p, s);
  } else if (cl == 2) {
    if (p.n1 == 128 && p.n2 == 96) return launch_rf<128, 96, 256, 2>(p, s);
    if (p.n1 == 128 && p.n2 == 128) return launch_rf<128, 128, 512, 2>(p, s);
  } else if (cl == 4) {
    if (p.n1 == 256 && p.n2 == 192) return launch_rf<256, 192, 256, 4>(p, s);
  }
  return cudaErrorInvalidValue;
}

// the 4-CTA kernel with 16 x 16 row transforms (built for 256 x 192)
bool slice_rf_wide_ok(int n1, int n2) { return n1 == 256 && n2 == 192; }
cudaError_t launch_slice_rf_wide(const LineParams &p, cudaStream_t s)
{
  if (p.n1 == 256 && p.n2 == 192) return launch_rf<256, 192, 256, 4, 16>(p, s);
  return cudaErrorInvalidValue;
}

bool pdl_enabled()
{
  static const bool on = [] {
    const char *e = getenv("QD_PDL");
    return !(e && e[0] == '0');
  }();
  return on;
}
