// k_column_tc.cu -- the column pass of the complex64 propagation on the
// 5th-generation tensor cores (tcgen05, kind::f16, accumulators in TMEM).
//
// Same work as k_column.cu (B, dump, flux rows, norm, V, F; see there for the
// reference functions), with both Legendre contractions as back-to-back
// GEMMs per tile of 64 grid columns (S = n_l, n_theta padded to 16):
//   GEMM1  D[128 x S] = A1[128 x S] * Q^T      A1 = psi'_l tile (K = l)
//   theta-space ops on D (tcgen05.ld -> registers) -> A2 (TMEM)
//   GEMM2  D[128 x S] = A2[128 x S] * Q        (K = k)
// with Q[k][l] = sqrt(w_k) sqrt(l+1/2) P_l(x_k) (and its orthonormal
// completion to n_theta orders, for the output norm).  The 128 GEMM rows are
// the real and imaginary parts of the 64 complex points (row 2p = Re,
// 2p+1 = Im), so the complex-by-real transform is one real GEMM.
//
// FP32 accuracy from FP16 units by split products (3xFP16):
//   A*B ~ Ahi*Bhi + Ahi*Blo + Alo*Bhi,  Ahi = fp16(A), Alo = fp16(A - Ahi),
// the same 11-bit significands as a TF32 split at twice the TF32 MMA rate.
// FP16's narrow exponent range is handled by exact power-of-two scales: Q is
// stored times 2^12 (its entries are at most 1, so the low parts stay normal),
// and each complex point's row pair is scaled by 2^(13-e) with 2^e >= the
// point's norm, so every scaled entry is at most 2^13 and entries down to
// 2^-27 of the point's norm keep 11 bits.  The scales are undone on the FP32
// accumulator outputs, folded into multiplications the epilogue does anyway.
//
// Data placement: the A operands live in tensor memory (written by the
// threads with tcgen05.st, two FP16 values per 32-bit column; each thread owns
// one TMEM lane = one GEMM row and a quarter of its K range), the constant Q
// image pair (hi | lo) in shared memory, the accumulator in TMEM.  One image
// serves both GEMMs: stored with rows k and 64 orders l per 128-byte swizzled
// row, it is the K-major operand of GEMM1 and the MN-major operand of GEMM2.
// The tile's exp(-i V dt) values are staged into shared memory by
// asynchronous copies issued while the previous tile finishes.  512 threads
// per CTA.  S <= 64: two CTAs per SM overlap each other's load / MMA /
// epilogue phases; S = 96, 128 (n_theta up to 128): one CTA per SM, which
// issues the next tile's GEMM1 as soon as the current tile's GEMM2 output is
// in registers.
//
// Norm of each grid column.  The tensor-core FP32 accumulation rounds toward
// smaller magnitudes (measured ~1e-7 per GEMM), which compounded over 1e4
// steps would shrink the wavepacket by ~1%.  Both transforms are exact
// isometries per grid column in the quadrature norms -- B (l -> theta)
// whenever n_l <= n_theta (Gauss quadrature is exact to degree 2 n_theta - 1),
// F (theta -> l) when its output is taken over all n_theta orders -- so each
// column's output is rescaled to the exactly known norm
//   sum_k w_k |psi_theta|^2 = sum_l |psi_l|^2/(l+1/2)
// (times the absorber squared).  The state is kept in the orthonormal basis
// psi'_l = psi_l/sqrt(l+1/2), where these norms are plain sums of squares.
// For n_l < n_theta, GEMM2 also forms the orders n_l..n_theta-1 (the
// completion columns of Q) for the norm only; they are not stored.  This
// fixes the magnitude only; shape and phase stay as computed.
//
// One thread issues the MMAs; completion arrives on an mbarrier through
// tcgen05.commit.  Every wait is bounded: on timeout the CTA records an error
// in the status word, releases its TMEM and returns.
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>
#include <cuda_fp16.h>
#include "qd.h"
#include "qd_tc.h"

namespace {

constexpr int TPTS = 64;          // complex grid points per tile
constexpr int MROWS = 128;        // GEMM rows per tile
// threads per CTA (a multiple of 128: NG column groups of four warps).  1024
// threads at S = 128 (64 registers, 16 columns per thread) measured 33 % slower.
__host__ __device__ constexpr int nthreads(int) { return 512; }
constexpr int MAXS = 128;         // max padded n_l / n_theta handled here
constexpr int B_LOG2 = 12;        // Q is stored times 2^12
constexpr int A_LOG2 = 13;        // scaled A entries are at most 2^13
// per-size resources: TMEM columns of each A half (S/2 packed columns,
// rounded up to 16), the allocation (Ahi | Alo | D, a power of two), CTAs per SM
__host__ __device__ constexpr int a_cols(int S) { return (S / 2 + 15) / 16 * 16; }
__host__ __device__ constexpr uint32_t tmem_cols(int S)
{
  return 2 * a_cols(S) + S <= 64 ? 64u : 2 * a_cols(S) + S <= 128 ? 128u : 256u;
}
__host__ __device__ constexpr int ctas_per_sm(int S) { return S <= 64 ? 2 : 1; }
// bytes of one operand image (hi or lo): 128-byte rows of 64 orders, S rows
// per 64-order block
__host__ __device__ constexpr int image_bytes(int S) { return (S + 63) / 64 * S * 128; }
constexpr long WAIT_LIMIT = 1L << 22;   // mbarrier polls before giving up


// byte offset of 16-bit element (r, c) of an operand image of R rows, 64
// columns per 128-byte swizzled row (16-byte chunk index XOR row mod 8)
__host__ __device__ __forceinline__ uint32_t sw128_off16(int r, int c, int R)
{
  const int a = c >> 6, ch = (c & 63) >> 3;
  return (uint32_t)(a * R * 128 + r * 128 + ((ch ^ (r & 7)) << 4) + ((c & 7) << 1));
}

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
  return (uint32_t)__cvta_generic_to_shared(p);
}

// 2^k for integer k in [-126, 127]
__host__ __device__ __forceinline__ float exp2i(int k)
{
#ifdef __CUDA_ARCH__
  return __int_as_float((k + 127) << 23);
#else
  return std::ldexp(1.0f, k);
#endif
}

// e with sqrt(n) <= 2^e for a point norm n >= 0 (from n's exponent field;
// clamped so that every scale below stays a normal FP32 number)
__device__ __forceinline__ int norm_exp(float n)
{
  const int eb = (__float_as_int(n) >> 23) & 0xff;
  const int e = eb == 0 ? -60 : (eb - 125) >> 1;
  return e < -60 ? -60 : e > 60 ? 60 : e;
}

// shared-memory matrix descriptors, 128-byte swizzle (sm100 format):
// K-major (GEMM1: 8-row groups 1024 B apart, K inside the row) and MN-major
// (GEMM2: K rows 128 B apart in 8-row groups 1024 B apart, 64-element MN
// blocks lbo bytes apart)
__device__ __forceinline__ uint64_t desc_common(uint32_t saddr)
{
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3fffu);          // start address
  d |= (uint64_t)(1024u >> 4) << 32;                // SBO: 8 rows x 128 B
  d |= (uint64_t)1u << 46;                          // descriptor version (sm100)
  d |= (uint64_t)2u << 61;                          // SWIZZLE_128B
  return d;
}
__device__ __forceinline__ uint64_t make_desc_k(uint32_t saddr)
{
  return desc_common(saddr) | ((uint64_t)1u << 16);            // LBO unused (1)
}
__device__ __forceinline__ uint64_t make_desc_mn(uint32_t saddr, uint32_t lbo)
{
  return desc_common(saddr) | ((uint64_t)((lbo >> 4) & 0x3fffu) << 16);
}

// kind::f16 instruction descriptor: D f32, A/B f16, A K-major, B K- or
// MN-major, M = 128, N
__host__ __device__ constexpr uint32_t make_idesc(int N, bool b_mn)
{
  return (1u << 4) | (0u << 7) | (0u << 10) | ((b_mn ? 1u : 0u) << 16) |
         ((uint32_t)(N >> 3) << 17) | ((uint32_t)(MROWS >> 4) << 24);
}

__device__ __forceinline__ void mma_commit(uint32_t mbar)
{
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               :: "r"(mbar) : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t phase)
{
  for (long it = 0; it < WAIT_LIMIT; it++) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok) : "r"(mbar), "r"(phase) : "memory");
    if (ok) return true;
  }
  return false;
}

__device__ __forceinline__ void cp16_zfill(void *dst, const void *src, bool valid)
{
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;"
               :: "r"(smem_u32(dst)), "l"(src), "r"(valid ? 16 : 0) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

struct TcDev {
  const float4 *mats;    // image sets (Q hi|lo), set_bytes apart
  uint32_t set_bytes;
  const int *run_set;    // image set of each run (null: set 0)
  const int *run_order;  // tile order: virtual run v is run_order[v], runs of a set adjacent
  const int *run_nl;     // orders stored per run (null: n_l)
  int *status;           // device status word (0 = ok)
  int renorm;            // per-column isometry rescaling on
  int nnorm;             // orders l < nnorm enter the GEMM2 output norm
  // x / tiles-per-run and x / n1 as (x * m) >> 40, m = floor(2^40 / d) + 1:
  // exact while x * d < 2^40 (checked at launch)
  uint64_t m_tpr, m_n1;
};


// tcgen05.st of 2 / 4 consecutive 32-bit columns of this thread's lane
__device__ __forceinline__ void tmem_st2(uint32_t taddr, uint32_t a, uint32_t b)
{
  asm volatile("tcgen05.st.sync.aligned.32x32b.x2.b32 [%0], {%1,%2};"
               :: "r"(taddr), "r"(a), "r"(b) : "memory");
}
__device__ __forceinline__ void tmem_st4(uint32_t taddr, uint32_t a, uint32_t b, uint32_t c,
                                         uint32_t d)
{
  asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1,%2,%3,%4};"
               :: "r"(taddr), "r"(a), "r"(b), "r"(c), "r"(d) : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// tcgen05.ld of this thread's H consecutive columns: all loads issued, then
// one wait; the wait names the destination registers, so no use of them can
// be scheduled before it
template <int H>
__device__ __forceinline__ void tmem_ld_all(uint32_t taddr, float (&v)[H])
{
  static_assert(H % 4 == 0, "whole x4 loads");
  uint32_t r[H];
#pragma unroll
  for (int u = 0; u < H; u += 4)
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r[u]), "=r"(r[u + 1]), "=r"(r[u + 2]), "=r"(r[u + 3]) : "r"(taddr + u));
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]) :: "memory");
#pragma unroll
  for (int u = 4; u < H; u += 4)
    asm volatile("" : "+r"(r[u]), "+r"(r[u + 1]), "+r"(r[u + 2]), "+r"(r[u + 3]));
#pragma unroll
  for (int u = 0; u < H; u++) v[u] = __uint_as_float(r[u]);
}

// hi and lo FP16 parts of two values, each pair packed into one 32-bit
// column (the even K index in the low half)
__device__ __forceinline__ void split2(float x0, float x1, uint32_t &hi, uint32_t &lo)
{
  const __half2 h = __floats2half2_rn(x0, x1);
  const float2 b = __half22float2(h);
  const __half2 l = __floats2half2_rn(x0 - b.x, x1 - b.y);
  hi = *reinterpret_cast<const uint32_t *>(&h);
  lo = *reinterpret_cast<const uint32_t *>(&l);
}

// the split of 4 values (K indices k..k+3, k % 4 == 0) into the Ahi and Alo
// TMEM columns k/2, k/2+1
__device__ __forceinline__ void put4_tmem(uint32_t ahi, uint32_t alo, float x0, float x1,
                                          float x2, float x3)
{
  uint32_t h0, l0, h1, l1;
  split2(x0, x1, h0, l0);
  split2(x2, x3, h1, l1);
  tmem_st2(ahi, h0, h1);
  tmem_st2(alo, l0, l1);
}

// the split of a thread's H values (K indices c0..c0+H-1) times the point
// scale sa into its Ahi / Alo columns
template <int H>
__device__ __forceinline__ void put_row(uint32_t my_hi, uint32_t my_lo, const float (&v)[H],
                                        float sa)
{
  if constexpr (H % 8 == 0) {
#pragma unroll
    for (int u = 0; u < H; u += 8) {
      uint32_t h[4], l[4];
#pragma unroll
      for (int x = 0; x < 4; x++) split2(v[u + 2 * x] * sa, v[u + 2 * x + 1] * sa, h[x], l[x]);
      tmem_st4(my_hi + u / 2, h[0], h[1], h[2], h[3]);
      tmem_st4(my_lo + u / 2, l[0], l[1], l[2], l[3]);
    }
  } else {
#pragma unroll
    for (int u = 0; u < H; u += 4)
      put4_tmem(my_hi + u / 2, my_lo + u / 2, v[u] * sa, v[u + 1] * sa, v[u + 2] * sa,
                v[u + 3] * sa);
  }
}

__device__ __forceinline__ void mma_f16_ts(uint32_t dtmem, uint32_t atmem, uint64_t bdesc,
                                           uint32_t idesc, uint32_t accumulate)
{
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}\n"
      :
      : "r"(dtmem), "r"(atmem), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

// D = A * B over K = S, A in TMEM columns [ahi, ahi+S/2) and [alo, alo+S/2)
// (packed FP16 pairs), B the image pair at b (hi | lo, image_bytes(S) apart):
// GEMM1 (MN = false) reads it K-major, GEMM2 (MN = true) MN-major.  The small
// split terms first, the main one last.
// desc0: the descriptor of the hi image at its first K slice (make_desc_k or
// make_desc_mn of its address); the others differ only in the start-address
// field (address / 16, 14 bits: shared-memory offsets stay below 256 KB, so
// adding to it never carries out)
template <int S, bool MN>
__device__ __forceinline__ void gemm_split_ts(uint32_t dtmem, uint32_t ahi, uint32_t alo,
                                              uint64_t desc0)
{
  constexpr uint32_t idesc = make_idesc(S, MN);
  constexpr int BB = image_bytes(S);
#pragma unroll 1
  for (int term = 0; term < 3; term++) {
    // term 0: Ahi*Blo, 1: Alo*Bhi, 2: Ahi*Bhi
    const uint32_t a = term == 1 ? alo : ahi;
    const uint64_t dt = desc0 + (term == 0 ? (uint64_t)(BB >> 4) : 0ull);
#pragma unroll
    for (int kk = 0; kk < S; kk += 16) {
      const uint32_t off = MN ? (uint32_t)kk * 128u
                              : (uint32_t)((kk >> 6) * S * 128 + ((kk & 63) >> 4) * 32);
      mma_f16_ts(dtmem, a + kk / 2, dt + (off >> 4), idesc, (term | kk) ? 1u : 0u);
    }
  }
}

// column groups (warps w, w+4, ... share a TMEM lane quarter)
__host__ __device__ constexpr int ngroups(int S) { return nthreads(S) / 128; }

// EX: exact shape -- n_l = n_theta = S, n12 and n1 multiples of the tile, so
// every point and column of a tile is valid and a tile lies in one grid row j.
//
// Orthonormal representation.  The l-space state is kept as
// psi'_l = psi_l / sqrt(l+1/2) and theta values as sqrt(w_k) psi(theta_k), so
// both transforms use the same matrix Q (B: D1 = Q psi', F: psi' = Q^T A2)
// and every norm is a plain sum of squares.
// Renormalisation.  The column output is rescaled to the norm the exact
// transform pair would give, dd^2 * sum_l |psi'_l|^2 per grid column (dd =
// absorber); the theta-space intermediate needs its own scale only where it
// leaves the kernel (flux rows, psi_z, energies, the last step of a call: the
// "slow" tiles), elsewhere GEMM2 runs on V * D1 as it comes out of GEMM1 and
// one factor dd sqrt(n_l / n_out) at the store does both.
// Scales.  A point with l-space norm n_l gets the A scale 2^(13-e), 2^e >=
// sqrt(n_l) (the exponent pe below); GEMM1's output is then 2^(25-e) times
// the theta values, so the fast tiles form A2 = 2^-12 * V * D1 (the same
// scale 2^(13-e), as the transform preserves the norm), and the rescalings
// to a known norm above are scale-free.
// MS: runs of the batch have different angular bases (image sets, orders stored)
template <int S, int MODE, bool EX, bool MS>
__global__ void __launch_bounds__(nthreads(S), ctas_per_sm(S)) k_column_tc(ColumnParams p, TcDev t)
{
  constexpr int NTHREADS = nthreads(S), NG = ngroups(S);
  constexpr int mode = MODE;
  constexpr int H = S / NG;                    // K columns per thread (one group)
  constexpr int BB = image_bytes(S);
  constexpr int AC = a_cols(S);
  constexpr uint32_t TMEM_COLS = tmem_cols(S);
  static_assert(H % 4 == 0, "column group must be a multiple of 4");
  extern __shared__ unsigned char smem_raw[];
  const uint32_t base_u = smem_u32(smem_raw);
  unsigned char *base = smem_raw + ((1024u - (base_u & 1023u)) & 1023u);
  unsigned char *Bq = base;                     // Q image pair: hi | lo
  uint64_t *mbar = reinterpret_cast<uint64_t *>(base + 2 * BB);
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(mbar + 4);
  float *xch = reinterpret_cast<float *>(mbar + 4 + 32);  // [4 exchanges][NG][TPTS]
  float *sw = xch + 4 * NG * TPTS;                        // [S] sqrt(w_k), 0 beyond n_theta
  float *rsw = sw + S;                                    // [S] 1/sqrt(w_k)
  float2 *evs = reinterpret_cast<float2 *>(rsw + S);      // [S][TPTS] exp(-i V dt) of a tile

  pdl_trigger();
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int row = (warp & 3) * 32 + lane;        // TMEM lane == GEMM row
  const int grp = warp >> 2;                     // column group
  const int c0 = grp * H;                        // first K/N column of this thread
  const int pt = row >> 1;                       // complex point within tile
  const bool is_im = row & 1;
  const int comp = is_im ? 1 : 0;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(smem_u32(tmem_slot)), "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  // tiles are strided over the CTAs (neighbouring CTAs read neighbouring
  // columns); tile t belongs to virtual run t / tpr, and runs that share an
  // angular set are adjacent in that order, so a CTA reloads its operand
  // images at most (sets - 1) times
  const int n12 = (int)p.n12, n1 = p.n1;
  const int tpr = (n12 + TPTS - 1) / TPTS;      // tiles per run
  const int ntiles = tpr * p.nruns;
  const int tbeg = blockIdx.x, tend = ntiles;
#define QD_DIV(x, m) ((int)(((uint64_t)(uint32_t)(x) * (m)) >> 40))
#define QD_RUN_OF(tl) (MS && t.run_order ? t.run_order[QD_DIV(tl, t.m_tpr)] : QD_DIV(tl, t.m_tpr))
  const uint32_t mb3 = smem_u32(&mbar[3]);      // completion of the image copy
  // the image pair of set `st` (2 x BB bytes, a multiple of 16) by bulk
  // asynchronous copies from this GPU's global memory into this CTA's shared
  // memory, completing on mbar[3]
#define QD_LOAD_IMAGES(st)                                                             \
  do {                                                                                 \
    const uint32_t total = 2 * BB, chunk = 16384;                                      \
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"              \
                 :: "r"(mb3), "r"(total) : "memory");                                  \
    const char *src = reinterpret_cast<const char *>(t.mats) + (size_t)(st) * t.set_bytes; \
    for (uint32_t off = 0; off < total; off += chunk) {                                \
      const uint32_t n = total - off < chunk ? total - off : chunk;                    \
      asm volatile(                                                                    \
          "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" \
          :: "r"(smem_u32(Bq) + off), "l"(src + off), "r"(n), "r"(mb3) : "memory");    \
    }                                                                                  \
  } while (0)
#define QD_SET_OF(tl) (MS && t.run_set ? t.run_set[QD_RUN_OF(tl)] : 0)
  int loaded = tbeg < tend ? QD_SET_OF(tbeg) : 0;   // image set in smem
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&mbar[0])));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&mbar[1])));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(mb3));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    QD_LOAD_IMAGES(loaded);
  }
  static_assert(S <= NTHREADS, "one quadrature weight per thread");
  const double wq = tid < S && tid < p.nth ? p.w[tid] : 0.0;   // in flight during what follows
  // 32-bit tile arithmetic: the host checks n12 * n_l * 2 * n_runs < 2^31
  const int nl = p.nl, nth = p.nth;
  const int stride = 2 * n12;                   // floats between orders l (or k) of a point
  const float *lsrc = reinterpret_cast<const float *>(p.lpsi);
  float *ldst = reinterpret_cast<float *>(p.lpsi);
  float *surf = reinterpret_cast<float *>(p.surf);
  double *psiz = reinterpret_cast<double *>(p.psi_z);
  const float2 *expv = p.expV32;
  const float ysg = is_im ? 1.f : -1.f;         // V z: mine e.x + ysg other e.y

  float a[H];
#define QD_PREFETCH_A(tl)                                                            \
  do {                                                                               \
    const int rr = (tl) < tend ? QD_RUN_OF(tl) : 0;                                  \
    const int qq = ((tl) - QD_DIV(tl, t.m_tpr) * tpr) * TPTS + pt;                   \
    const bool ok = EX || ((tl) < tend && qq < n12);                                 \
    const float *src = lsrc + (size_t)rr * nl * stride + (size_t)c0 * stride + 2 * qq + comp; \
    _Pragma("unroll") for (int u = 0; u < H; u++) {                                  \
      if (EX) a[u] = (tl) < tend ? src[u * stride] : 0.f;                             \
      else a[u] = (ok && c0 + u < nl) ? src[u * stride] : 0.f;                       \
    }                                                                                \
  } while (0)
  // exp(-i V dt) of tile tl into evs, 16-byte asynchronous copies (zero-filled
  // past n_theta and past the grid; n12 is even, so a copy never straddles it).
  // (One bulk copy per theta row, issued by one warp and waited on through an
  // mbarrier by every thread, measured 25 % slower on the C4 column pass.)
#define QD_STAGE_EV(tl)                                                              \
  do {                                                                               \
    if ((tl) < tend) {                                                               \
      const int rr = QD_RUN_OF(tl), qb = ((tl) - QD_DIV(tl, t.m_tpr) * tpr) * TPTS; \
      const float2 *eb = expv + (size_t)rr * p.vrun + qb;                            \
      for (int x = tid; x < S * (TPTS / 2); x += NTHREADS) {                         \
        const int k = x / (TPTS / 2), c2 = 2 * (x % (TPTS / 2));                     \
        const bool okv = EX || (k < nth && qb + c2 < n12);                           \
        cp16_zfill(&evs[k * TPTS + c2], okv ? eb + (size_t)k * n12 + c2 : expv, okv); \
      }                                                                              \
    }                                                                                \
    asm volatile("cp.async.commit_group;" ::: "memory");                             \
  } while (0)
  if (mode == COL_MID) QD_STAGE_EV(tbeg);      // exp(-iVdt): set up before this launch
  pdl_wait();                                   // psi_l, psi_z, flux rows: the previous grid's
  if (mode != COL_HEAD) QD_PREFETCH_A(tbeg);
  // the prologue's loads (images, exp(-iVdt), psi_l, weights) are all in
  // flight before anything waits on one of them
  if (tid < S) {
    sw[tid] = (float)sqrt(wq);
    rsw[tid] = wq > 0.0 ? (float)(1.0 / sqrt(wq)) : 0.f;
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const uint32_t lane_base = ((uint32_t)((warp & 3) * 32)) << 16;
  const uint32_t Ahi = tmem, Alo = tmem + AC, D = tmem + 2 * AC;     // column bases
  const uint32_t my_hi = Ahi + lane_base + c0 / 2, my_lo = Alo + lane_base + c0 / 2;
  const uint32_t my_d = D + lane_base + c0;
  const uint32_t mb1 = smem_u32(&mbar[0]), mb2 = smem_u32(&mbar[1]);
  const uint32_t bq = smem_u32(Bq);
  const uint64_t dk0 = make_desc_k(bq), dmn0 = make_desc_mn(bq, (uint32_t)S * 128u);
  uint32_t ph1 = 0, ph2 = 0, ph3 = 1;
  // every thread observes each mbarrier completion itself before it reads
  // what the asynchronous operation wrote
  bool failed = __syncthreads_or(!mbar_wait(mb3, 0));
  // MID: the tile's A1 is already in TMEM and its GEMM1 issued -- done at the
  // end of the previous tile, as soon as that tile's GEMM2 output was in
  // registers, so that GEMM1 runs under the previous tile's stores
  bool a_ready = false;
  float n_l_next = 0.f;                         // l-space point norm of that next tile

  for (int tile = tbeg; tile < tend && !failed; tile += gridDim.x) {
    const int run = QD_RUN_OF(tile);
    int nlr = nl;                               // orders stored for this run
    if constexpr (MS) {
      const int set = t.run_set ? t.run_set[run] : 0;
      if (!a_ready && set != loaded) {          // another angular basis
        if (tid == 0) QD_LOAD_IMAGES(set);      // earlier MMAs have all completed
        if (__syncthreads_or(!mbar_wait(mb3, ph3))) { failed = true; break; }
        ph3 ^= 1;
        loaded = set;
      }
      if (t.run_nl) nlr = t.run_nl[run];
    }
    const int q0 = (tile - QD_DIV(tile, t.m_tpr) * tpr) * TPTS;
    const int q = q0 + pt;
    const bool qok = EX || q < n12;
    int j, i;
    if (EX) { j = QD_DIV(q0, t.m_n1); i = q0 - j * n1 + pt; }
    else { j = qok ? QD_DIV(q, t.m_n1) : 0; i = qok ? q - j * n1 : 0; }
    const size_t voff = (size_t)run * p.vrun;
    const float ddv = (mode != COL_HEAD && p.d1 && qok) ? (float)(p.d1[i] * p.d2[j]) : 1.f;
    const bool frow = mode != COL_HEAD && p.do_flux && qok && j >= p.surf_j0 &&
                      j < p.surf_j0 + p.surf_nrows;
    // slow tiles form the true theta-space state: every tile of a launch that
    // outputs theta values, and the tiles with a point on a flux row (a
    // whole-tile test, as the branch holds barriers; EX: a tile lies in one row)
    bool tile_frow = frow;
    if (!EX && mode != COL_HEAD && p.do_flux) {
      const int ja = QD_DIV(q0, t.m_n1), jb = QD_DIV(min(q0 + TPTS, n12) - 1, t.m_n1);
      tile_frow = jb >= p.surf_j0 && ja < p.surf_j0 + p.surf_nrows;
    }
    const bool slow = mode == COL_TAIL || !t.renorm || p.out_z || tile_frow || p.esum;
    float n_l = 0.f, sc = 1.f;
    int pe = 0;                                 // the point's scale exponent
    // GEMM1 output (theta values) of this thread; with one CTA per SM (128
    // registers) a slow tile keeps its first TMEM read for the theta-space work
    constexpr bool KEEP = ctas_per_sm(S) == 1;
    float dv[H];

    if (mode != COL_HEAD) {
      // ---- A1 = psi'_l tile into TMEM (scaled by its point norm), GEMM1 ---------------
      if (!a_ready) {
        float nl_part = 0.f;
#pragma unroll
        for (int u = 0; u < H; u++) nl_part = fmaf(a[u], a[u], nl_part);
        nl_part += __shfl_xor_sync(0xffffffffu, nl_part, 1);
        if (!is_im) xch[grp * TPTS + pt] = nl_part;
        if (mode == COL_MID) asm volatile("cp.async.wait_group 0;" ::: "memory");   // evs
        __syncthreads();
#pragma unroll
        for (int g = 0; g < NG; g++) n_l += xch[g * TPTS + pt];
        pe = norm_exp(n_l);
        put_row<H>(my_hi, my_lo, a, exp2i(A_LOG2 - pe));
        tmem_wait_st();
        tc_fence_before();
        __syncthreads();
        if (tid == 0) {
          tc_fence_after();
          gemm_split_ts<S, false>(D, Ahi, Alo, dk0);
          mma_commit(mb1);
        }
        // TAIL: this tile's values are in TMEM, so the next tile's loads can
        // fly during its GEMM and theta-space work
        if (mode == COL_TAIL) QD_PREFETCH_A(tile + (int)gridDim.x);
      } else {
        n_l = n_l_next;
        pe = norm_exp(n_l);
      }
      a_ready = false;
      if (__syncthreads_or(!mbar_wait(mb1, ph1))) { failed = true; break; }
      ph1 ^= 1;
      tc_fence_after();
      if (slow) {                               // theta norm of GEMM1 -> isometry scale
        float nt_part = 0.f, dn[H];
        float (&dl)[H] = KEEP ? dv : dn;
        tmem_ld_all<H>(my_d, dl);
#pragma unroll
        for (int u = 0; u < H; u++) nt_part = fmaf(dl[u], dl[u], nt_part);
        nt_part += __shfl_xor_sync(0xffffffffu, nt_part, 1);
        if (!is_im) xch[NG * TPTS + grp * TPTS + pt] = nt_part;
        __syncthreads();
        float n_t = 0.f;
#pragma unroll
        for (int g = 0; g < NG; g++) n_t += xch[NG * TPTS + g * TPTS + pt];
        // to the exact norm n_l (scale-free), or just undo the scales
        sc = t.renorm ? (n_t > 0.f ? sqrtf(n_l / n_t) : 1.f) : exp2i(pe - A_LOG2 - B_LOG2);
      }
    }

    // ---- theta-space operations, A2 into TMEM ----------------------------------------
    float tsum = 0.f;                           // this thread's share of sum_k |theta'_k|^2
    const float sin_ = sc * ddv;                // slow tiles: true theta values
    double *zrow = (mode != COL_HEAD && p.out_z) ? psiz + 2 * ((size_t)run * nth * n12 + q) + comp
                                                 : nullptr;
    float *srow = frow ? surf + 2 * (((size_t)run * p.surf_nrows + (j - p.surf_j0)) * nth * n1 + i) + comp
                       : nullptr;
    if (mode != COL_HEAD) {
      if (!(KEEP && slow)) tmem_ld_all<H>(my_d, dv);
      if (slow) {                               // whole-tile branch: the fast tiles skip it
        if (p.esum) {                           // potential energy, before the absorber
          double ep = 0.0;
#pragma unroll
          for (int u = 0; u < H; u++) {
            const int k = c0 + u;
            if (EX || (qok && k < nth)) {
              const float x = dv[u] * sc;
              ep += (double)(x * x) * p.pot[voff + (size_t)k * n12 + q];
            }
          }
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) ep += __shfl_xor_sync(0xffffffffu, ep, o);
          if (lane == 0) atomicAdd(p.esum + 3 * run + 2, ep);
        }
#pragma unroll
        for (int u = 0; u < H; u++) {
          const int k = c0 + u;
          dv[u] *= sin_;
          tsum = fmaf(dv[u], dv[u], tsum);
          if (EX || (qok && k < nth)) {
            if (srow) srow[(size_t)2 * k * n1] = dv[u] * rsw[k];
            if (zrow) zrow[(size_t)2 * k * n12] = dv[u] * rsw[k];
          }
        }
      }
    }
    if (mode == COL_MID) {                      // V z, into TMEM at the point's scale
#pragma unroll
      for (int u = 0; u < H; u++) {
        const float other = __shfl_xor_sync(0xffffffffu, dv[u], 1);
        const float2 e = evs[(c0 + u) * TPTS + pt];
        dv[u] = fmaf(other * ysg, e.y, dv[u] * e.x);
      }
      put_row<H>(my_hi, my_lo, dv, slow ? exp2i(A_LOG2 - pe) : exp2i(-B_LOG2));
    } else if (mode == COL_HEAD) {              // psi_z -> theta' values
      // eight values' loads are issued before their arithmetic, so that their
      // latencies overlap
      // (four at two CTAs per SM: eight would spill at their 64 registers)
      constexpr int GV = H % 8 == 0 && ctas_per_sm(S) == 1 ? 8 : 4;   // H is a multiple of 4
      const double2 *zr = p.psi_z + (size_t)run * nth * n12 + q;
      const float2 *fr = expv + voff + q;
#pragma unroll
      for (int u0 = 0; u0 < H; u0 += GV) {
        double2 z[GV];
        float2 fv[GV];
        double wv[GV];
#pragma unroll
        for (int v = 0; v < GV; v++) {
          const int k = c0 + u0 + v;
          const bool ok = qok && k < nth;
          z[v] = ok ? __ldg(zr + (size_t)k * n12) : make_double2(0.0, 0.0);
          fv[v] = ok ? __ldg(fr + (size_t)k * n12) : make_float2(1.f, 0.f);
          wv[v] = ok ? __ldg(p.w + k) : 0.0;
        }
#pragma unroll
        for (int v = 0; v < GV; v++) {
          // exp(-i V dt) from the step's own complex64 table; the first step of
          // a run takes its principal square root (psi / sqrt(v) * v), by the
          // half-angle formulas in the form without cancellation
          float2 f = fv[v];
          if (p.prestep) {
            if (f.x >= 0.f) {
              const float ch = sqrtf(0.5f * (1.f + f.x));
              f = make_float2(ch, f.y / (2.f * ch));
            } else {
              const float sh = copysignf(sqrtf(0.5f * (1.f - f.x)), f.y);
              f = make_float2(f.y / (2.f * sh), sh);
            }
          }
          const double2 zz = z[v];
          const float val = (float)((is_im ? zz.x * f.y + zz.y * f.x : zz.x * f.x - zz.y * f.y) *
                                    sqrt(wv[v]));
          dv[u0 + v] = val;
          tsum = fmaf(val, val, tsum);
        }
      }
    }
    // target norm of the column output (and the step norm of the point)
    float target;
    if (slow || mode == COL_HEAD) {
      tsum += __shfl_xor_sync(0xffffffffu, tsum, 1);
      if (!is_im) xch[2 * NG * TPTS + grp * TPTS + pt] = tsum;
    }
    if (mode == COL_MID) tmem_wait_st();
    tc_fence_before();
    __syncthreads();
    if (slow || mode == COL_HEAD) {
      target = 0.f;
#pragma unroll
      for (int g = 0; g < NG; g++) target += xch[2 * NG * TPTS + g * TPTS + pt];
    } else {
      target = ddv * ddv * n_l;
    }
    if (mode == COL_HEAD) {                     // A2 at the scale of the point's norm
      pe = norm_exp(target);
      put_row<H>(my_hi, my_lo, dv, exp2i(A_LOG2 - pe));
      tmem_wait_st();
      tc_fence_before();
      __syncthreads();
    }
    if (p.norm_out && mode != COL_HEAD) {       // this tile's share of its run's norm
      double s = (grp == 0 && !is_im && qok) ? (double)target : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if (grp == 0 && lane == 0) atomicAdd(p.norm_out + run, s);
    }
    if (mode == COL_TAIL) continue;            // the next tile's loads were issued after GEMM1
    // ---- GEMM2: psi' = Q^T A2 ------------------------------------------------------------
    if (tid == 0) {
      tc_fence_after();
      gemm_split_ts<S, true>(D, Ahi, Alo, dmn0);
      mma_commit(mb2);
    }
    if (mode == COL_MID) QD_STAGE_EV(tile + (int)gridDim.x);   // evs is free again
    if (mode != COL_HEAD) QD_PREFETCH_A(tile + (int)gridDim.x);   // next tile's loads fly during GEMM2
    if (__syncthreads_or(!mbar_wait(mb2, ph2))) { failed = true; break; }
    ph2 ^= 1;
    tc_fence_after();
    float no_part = 0.f, ov[H];
    tmem_ld_all<H>(my_d, ov);
#pragma unroll
    for (int u = 0; u < H; u++) {
      if (EX) no_part = fmaf(ov[u], ov[u], no_part);
      else no_part += c0 + u < t.nnorm ? ov[u] * ov[u] : 0.f;
    }
    no_part += __shfl_xor_sync(0xffffffffu, no_part, 1);
    if (!is_im) xch[3 * NG * TPTS + grp * TPTS + pt] = no_part;
    // the next tile's A1 into TMEM and its GEMM1, while this tile finishes
    // (GEMM2 has completed, so its A2 is free, and this thread's D is in ov)
    const int nxt = tile + (int)gridDim.x;
    const bool ahead = mode == COL_MID && nxt < tend;
    if (ahead) {
      if constexpr (MS) {
        const int set = t.run_set ? t.run_set[QD_RUN_OF(nxt)] : 0;
        if (set != loaded) {                    // no MMA reads the images now
          if (tid == 0) QD_LOAD_IMAGES(set);
          if (__syncthreads_or(!mbar_wait(mb3, ph3))) { failed = true; break; }
          ph3 ^= 1;
          loaded = set;
        }
      }
      float nl_part = 0.f;
#pragma unroll
      for (int u = 0; u < H; u++) nl_part = fmaf(a[u], a[u], nl_part);
      nl_part += __shfl_xor_sync(0xffffffffu, nl_part, 1);
      if (!is_im) xch[grp * TPTS + pt] = nl_part;
    }
    if (ahead) asm volatile("cp.async.wait_group 0;" ::: "memory");   // the next tile's evs
    tc_fence_before();
    __syncthreads();
    float n_o = 0.f;
#pragma unroll
    for (int g = 0; g < NG; g++) n_o += xch[3 * NG * TPTS + g * TPTS + pt];
    if (ahead) {
      n_l_next = 0.f;
#pragma unroll
      for (int g = 0; g < NG; g++) n_l_next += xch[g * TPTS + pt];
      put_row<H>(my_hi, my_lo, a, exp2i(A_LOG2 - norm_exp(n_l_next)));
      tmem_wait_st();
      tc_fence_before();
      __syncthreads();
      if (tid == 0) {
        tc_fence_after();
        gemm_split_ts<S, false>(D, Ahi, Alo, dk0);
        mma_commit(mb1);
      }
    }
    a_ready = ahead;
    float so;
    if (t.renorm) so = n_o > 0.f ? sqrtf(target / n_o) : 1.f;
    else so = ((slow || mode == COL_HEAD) ? 1.f : ddv) * exp2i(pe - A_LOG2 - B_LOG2);
    float *dst = ldst + (size_t)run * nl * stride + (size_t)c0 * stride + 2 * q + comp;
    if (EX && (!MS || c0 + H <= nlr)) {         // every order of this column group is stored
#pragma unroll
      for (int u = 0; u < H; u++) dst[u * stride] = ov[u] * so;
    } else {
#pragma unroll
      for (int u = 0; u < H; u++)
        if ((EX || qok) && c0 + u < nlr) dst[u * stride] = ov[u] * so;
    }
    tc_fence_before();
  }
#undef QD_PREFETCH_A
#undef QD_STAGE_EV
#undef QD_LOAD_IMAGES
#undef QD_SET_OF
#undef QD_RUN_OF
#undef QD_DIV

  if (failed && lane == 0) atomicExch(t.status, 1);
  asm volatile("cp.async.wait_group 0;" ::: "memory");   // no copy outlives the CTA
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                 :: "r"(tmem), "r"(TMEM_COLS));
  }
}

template <int S, bool EX, bool MS> cudaError_t set_smem_attr_ex(int bytes)
{
  cudaError_t e = cudaFuncSetAttribute(k_column_tc<S, COL_HEAD, EX, MS>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_column_tc<S, COL_MID, EX, MS>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_column_tc<S, COL_TAIL, EX, MS>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  return e;
}
template <int S> cudaError_t set_smem_attr(int bytes)
{
  cudaError_t e = set_smem_attr_ex<S, false, false>(bytes);
  if (e == cudaSuccess) e = set_smem_attr_ex<S, false, true>(bytes);
  if constexpr (S == 64 || S == 128) {
    if (e == cudaSuccess) e = set_smem_attr_ex<S, true, false>(bytes);
    if (e == cudaSuccess) e = set_smem_attr_ex<S, true, true>(bytes);
  }
  return e;
}

template <int S, bool EX, bool MS>
void launch_mode_ex(int grid, int smem, cudaStream_t s, const ColumnParams &p, const TcDev &t,
                    int mode)
{
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(nthreads(S));
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl_enabled() ? 1 : 0;
  if (mode == COL_HEAD) cudaLaunchKernelEx(&cfg, k_column_tc<S, COL_HEAD, EX, MS>, p, t);
  else if (mode == COL_MID) cudaLaunchKernelEx(&cfg, k_column_tc<S, COL_MID, EX, MS>, p, t);
  else cudaLaunchKernelEx(&cfg, k_column_tc<S, COL_TAIL, EX, MS>, p, t);
}

template <int S>
void launch_mode(int grid, int smem, cudaStream_t s, const ColumnParams &p, const TcDev &t,
                 int mode)
{
  const bool ex = p.nl == S && p.nth == S && p.n12 % TPTS == 0 && p.n1 % TPTS == 0;
  const bool ms = t.run_set || t.run_nl;
  if constexpr (S == 64 || S == 128) {   // the exact-shape forms built
    if (ex && ms) { launch_mode_ex<S, true, true>(grid, smem, s, p, t, mode); return; }
    if (ex) { launch_mode_ex<S, true, false>(grid, smem, s, p, t, mode); return; }
  }
  if (ms) launch_mode_ex<S, false, true>(grid, smem, s, p, t, mode);
  else launch_mode_ex<S, false, false>(grid, smem, s, p, t, mode);
}

template <int S> constexpr int smem_bytes_for()
{
  return 1024 + 2 * image_bytes(S) + 4 * 8 + 32 * 8 + 4 * ngroups(S) * TPTS * 4 + 2 * S * 4 +
         S * TPTS * 8;   // Q image pair, barriers, exchanges, sqrt(w), 1/sqrt(w), exp(-iVdt)
}
static_assert(smem_bytes_for<128>() <= 227 * 1024 && 2 * smem_bytes_for<64>() <= 227 * 1024,
              "shared memory of the column tiles");

// the kernel sizes built: S is n_l / n_theta padded up to one of them
int kernel_size(int n)
{
  for (int s : {16, 32, 48, 64, 96, 128})
    if (n <= s) return s;
  return 0;
}

}  // namespace

int tc_plan_create(TcPlan &plan, int nth, int nl, int nsets, const double *const *leg,
                   const int *nl_set, const double *w, cudaStream_t s)
{
  const int S = kernel_size(nl > nth ? nl : nth);
  if (S == 0 || S > MAXS) return QD_ERR_UNSUPPORTED;
  // Q[k][l] = sqrt(w_k) sqrt(l+1/2) L[l][k] per angular set; the transform pair
  // is an isometry per grid column when Q has orthonormal columns, and GEMM2
  // then also forms an orthonormal completion of them (modified Gram-Schmidt
  // against the unit vectors, twice) so that its output norm is exact.  The
  // sets are independent: each is built on a host thread of its own.
  std::vector<std::vector<double>> Q(nsets), Qx(nsets);
  std::vector<double> sw(nth), sl(nl > nth ? nl : nth);
  for (int k = 0; k < nth; k++) sw[k] = std::sqrt(w[k]);
  for (size_t l = 0; l < sl.size(); l++) sl[l] = std::sqrt(l + 0.5);
  std::vector<char> set_ok(nsets, 1);
  auto build_set = [&](int t) {
    const int m = nl_set[t];
    Q[t].assign((size_t)nth * m, 0.0);
    for (int l = 0; l < m; l++)
      for (int k = 0; k < nth; k++)
        Q[t][(size_t)l * nth + k] = sw[k] * sl[l] * leg[t][l + (long)k * m];
    if (m > nth) { set_ok[t] = 0; return; }
    // the Gram matrix (symmetric: l2 >= l), four partial sums per entry
    for (int l = 0; l < m; l++) {
      const double *ql = Q[t].data() + (size_t)l * nth;
      for (int l2 = l; l2 < m; l2++) {
        const double *qm = Q[t].data() + (size_t)l2 * nth;
        double g0 = 0.0, g1 = 0.0, g2 = 0.0, g3 = 0.0;
        int k = 0;
        for (; k + 4 <= nth; k += 4) {
          g0 += ql[k] * qm[k];
          g1 += ql[k + 1] * qm[k + 1];
          g2 += ql[k + 2] * qm[k + 2];
          g3 += ql[k + 3] * qm[k + 3];
        }
        for (; k < nth; k++) g0 += ql[k] * qm[k];
        const double g = (g0 + g1) + (g2 + g3);
        if (std::fabs(g - (l == l2 ? 1.0 : 0.0)) > 1e-9) { set_ok[t] = 0; return; }
      }
    }
    std::vector<double> basis = Q[t];                // columns, each nth long
    int have = m;
    for (int c = 0; c < nth && have < nth; c++) {
      std::vector<double> v(nth, 0.0);
      v[c] = 1.0;
      for (int pass = 0; pass < 2; pass++)
        for (int b = 0; b < have; b++) {
          double d = 0.0;
          for (int k = 0; k < nth; k++) d += basis[(size_t)b * nth + k] * v[k];
          for (int k = 0; k < nth; k++) v[k] -= d * basis[(size_t)b * nth + k];
        }
      double nv = 0.0;
      for (int k = 0; k < nth; k++) nv += v[k] * v[k];
      if (nv < 1e-2) continue;
      nv = 1.0 / std::sqrt(nv);
      for (int k = 0; k < nth; k++) basis.push_back(v[k] * nv);
      have++;
    }
    if (have < nth) set_ok[t] = 0;
    Qx[t] = std::move(basis);                         // nth columns: Q, then the completion
  };
  auto each_set = [&](auto &&fn) {
    std::vector<std::thread> th;
    for (int t = 1; t < nsets; t++) th.emplace_back(fn, t);
    fn(0);
    for (auto &x : th) x.join();
  };
  each_set(build_set);
  bool renorm = true;
  for (int t = 0; t < nsets; t++) renorm = renorm && set_ok[t];
  // one image pair per set: row k (< n_theta) holds Q[k][l] times 2^12 for the
  // orders GEMM2 forms (the stored ones and, with renormalisation, the
  // completion up to n_theta), split into FP16 hi and lo parts
  const int bb = image_bytes(S);
  const size_t set_bytes = 2 * (size_t)bb;
  std::vector<unsigned char> img(set_bytes * nsets, 0);
  const double bscale = std::ldexp(1.0, B_LOG2);
  auto put = [&](unsigned char *im, int r, int c, double val) {     // hi | lo
    const double v = val * bscale;
    const __half h = __double2half(v);
    const __half l = __double2half(v - (double)__half2float(h));
    const uint32_t off = sw128_off16(r, c, S);
    std::memcpy(im + off, &h, 2);
    std::memcpy(im + bb + off, &l, 2);
  };
  each_set([&](int t) {
    unsigned char *b1 = img.data() + t * set_bytes;
    const int m = nl_set[t];
    const int cols = renorm ? nth : m;                   // output orders formed by GEMM2
    const std::vector<double> &q2 = renorm ? Qx[t] : Q[t];
    for (int k = 0; k < nth; k++)
      for (int l = 0; l < cols; l++) put(b1, k, l, q2[(size_t)l * nth + k]);
  });
  // from the device's stream-ordered pool, like the handle's other buffers;
  // a copy from pageable memory has read `img` when it returns
  void *d = nullptr;
  if (cudaMallocAsync(&d, img.size() + sizeof(int), s) != cudaSuccess) {
    cudaGetLastError();
    return QD_ERR_NOMEM;
  }
  if (cudaMemcpyAsync(d, img.data(), img.size(), cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemsetAsync((char *)d + img.size(), 0, sizeof(int), s) != cudaSuccess) {
    cudaFreeAsync(d, s);
    return QD_ERR_CUDA;
  }
  plan.nth = nth; plan.nl = nl; plan.S = S; plan.renorm = renorm ? 1 : 0;
  plan.nsets = nsets;
  plan.set_bytes = set_bytes;
  plan.mats = d;
  plan.mats_bytes = img.size();
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  plan.grid = ctas_per_sm(S) * sms;   // two CTAs per SM where shared memory and TMEM allow
  cudaError_t e = cudaSuccess;
  switch (S) {
    case 16: plan.smem_bytes = smem_bytes_for<16>();
      e = set_smem_attr<16>(plan.smem_bytes); break;
    case 32: plan.smem_bytes = smem_bytes_for<32>();
      e = set_smem_attr<32>(plan.smem_bytes); break;
    case 48: plan.smem_bytes = smem_bytes_for<48>();
      e = set_smem_attr<48>(plan.smem_bytes); break;
    case 96: plan.smem_bytes = smem_bytes_for<96>();
      e = set_smem_attr<96>(plan.smem_bytes); break;
    case 128: plan.smem_bytes = smem_bytes_for<128>();
      e = set_smem_attr<128>(plan.smem_bytes); break;
    default: plan.smem_bytes = smem_bytes_for<64>();
      e = set_smem_attr<64>(plan.smem_bytes); break;
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    cudaFreeAsync(d, s);
    plan.mats = nullptr;
    return QD_ERR_UNSUPPORTED;
  }
  return QD_OK;
}

void tc_plan_destroy(TcPlan &plan, cudaStream_t s)
{
  if (plan.mats) cudaFreeAsync(plan.mats, s);
  plan.mats = nullptr;
}

int *tc_status_ptr(const TcPlan &plan)
{
  return reinterpret_cast<int *>(static_cast<char *>(plan.mats) + plan.mats_bytes);
}

cudaError_t launch_column_tc(const TcPlan &plan, const ColumnParams &p, int mode,
                             cudaStream_t s)
{
  TcDev t;
  t.mats = reinterpret_cast<const float4 *>(plan.mats);
  t.set_bytes = (uint32_t)plan.set_bytes;
  t.run_set = p.run_set;
  t.run_order = p.run_order;
  t.run_nl = p.run_nl;
  t.status = tc_status_ptr(plan);
  t.renorm = plan.renorm;
  t.nnorm = plan.nth < plan.S ? plan.nth : plan.S;
  const long tpr = (p.n12 + TPTS - 1) / TPTS;
  const long ntiles = tpr * p.nruns;                          // tiles of all runs
  const int grid = (int)(ntiles < plan.grid ? ntiles : plan.grid);
  if ((uint64_t)(ntiles + grid) * (uint64_t)tpr >= (1ull << 40) ||
      (uint64_t)p.n12 * (uint64_t)p.n1 >= (1ull << 40))
    return cudaErrorInvalidValue;                              // tile arithmetic range
  t.m_tpr = (1ull << 40) / (uint64_t)tpr + 1;
  t.m_n1 = (1ull << 40) / (uint64_t)p.n1 + 1;
  switch (plan.S) {
    case 16: launch_mode<16>(grid, plan.smem_bytes, s, p, t, mode); break;
    case 32: launch_mode<32>(grid, plan.smem_bytes, s, p, t, mode); break;
    case 48: launch_mode<48>(grid, plan.smem_bytes, s, p, t, mode); break;
    case 96: launch_mode<96>(grid, plan.smem_bytes, s, p, t, mode); break;
    case 128: launch_mode<128>(grid, plan.smem_bytes, s, p, t, mode); break;
    default: launch_mode<64>(grid, plan.smem_bytes, s, p, t, mode); break;
  }
  return cudaGetLastError();
}
