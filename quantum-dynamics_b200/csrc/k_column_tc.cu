// k_column_tc.cu -- the column pass of the complex64 propagation on the
// 5th-generation tensor cores (tcgen05, kind::tf32, accumulators in TMEM).
//
// Same work as k_column.cu (B, dump, flux rows, norm, V, F; see there for the
// reference functions), with both Legendre contractions as back-to-back
// GEMMs per tile of 64 grid columns (S = n_l, n_theta padded to 16):
//   GEMM1  D1[128 x S] = A1[128 x S] * B1[S x S]    A1 = psi_l tile, B1[l][k] = P_l(x_k)
//   theta-space ops on D1 (tcgen05.ld -> registers)  -> A2 (smem)
//   GEMM2  D2[128 x S] = A2[128 x S] * B2[S x S]    B2[k][l] = (l+1/2) w_k P_l(x_k)
// The 128 GEMM rows are the real and imaginary parts of the 64 complex
// points (row 2p = Re, 2p+1 = Im), so the complex-by-real transform is one
// real GEMM.  FP32 accuracy from TF32 units by split products
//   A*B ~ Ahi*(Bhi + Bmid + Blo) + Alo*Bhi,   A = Ahi + Alo,  Ahi = tf32(A),
// with the constant Legendre matrices carried to ~2^-33 in three TF32 terms.
//
// Norm of each grid column.  The tensor-core FP32 accumulation rounds toward
// smaller magnitudes (measured ~1e-7 per GEMM), which compounded over 1e4
// steps would shrink the wavepacket by ~1%.  Both transforms are exact
// isometries per grid column in the quadrature norms -- B (l -> theta)
// whenever n_l <= n_theta (Gauss quadrature is exact to degree 2 n_theta - 1),
// F (theta -> l) when its output is taken over all n_theta orders -- so each
// column's output is rescaled to the exactly known input norm:
//   sum_k w_k |psi_theta|^2 = sum_l |psi_l|^2/(l+1/2).
// For n_l < n_theta, GEMM2 also forms the orders n_l..n_theta-1 (rows from the
// same three-term recurrence) for the norm only; they are not stored.  This
// fixes the magnitude only; shape and phase stay as computed.
//
// Operands sit in shared memory in the K-major 128-byte-swizzled layout that
// the UMMA smem descriptor describes; B1/B2 images are built once on the
// host (FP64 -> hi/mid/lo) and copied into every CTA.  One thread issues the
// MMAs; completion arrives on an mbarrier through tcgen05.commit.  Global
// loads of the next tile are issued while the MMAs of the current one run.
// Every wait is bounded: on timeout the CTA records an error in the status
// word, releases its TMEM and returns.
#include <cmath>
#include <cstring>
#include <vector>
#include "qd.h"
#include "qd_tc.h"

namespace {

constexpr int TPTS = 64;          // complex grid points per tile
constexpr int MROWS = 128;        // GEMM rows per tile
constexpr int NTHREADS = 256;
constexpr int MAXS = 64;          // max padded n_l / n_theta handled here
constexpr uint32_t TMEM_COLS = 128;
constexpr long WAIT_LIMIT = 1L << 22;   // mbarrier polls before giving up

__host__ __device__ constexpr int pad16(int x) { return (x + 15) & ~15; }

// byte offset of element (r, k) in a K-major SW128 operand of R rows
__host__ __device__ __forceinline__ uint32_t sw128_off(int r, int k, int R)
{
  const int a = k >> 5, c = (k & 31) >> 2;
  return (uint32_t)(a * R * 128 + r * 128 + ((c ^ (r & 7)) << 4) + ((k & 3) << 2));
}

// host: round to TF32 (nearest even on the 13 dropped bits)
float tf32_round_host(float x)
{
  uint32_t b;
  std::memcpy(&b, &x, 4);
  if ((b & 0x7f800000u) != 0x7f800000u) {
    b += 0xfffu + ((b >> 13) & 1u);
    b &= 0xffffe000u;
  }
  float y;
  std::memcpy(&y, &b, 4);
  return y;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ float tf32_rna(float x)
{
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

__device__ __forceinline__ uint64_t make_desc(uint32_t saddr)
{
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3fffu);          // start address
  d |= (uint64_t)1u << 16;                          // LBO (unused for SW128 K-major)
  d |= (uint64_t)(1024u >> 4) << 32;                // SBO: 8 rows x 128 B
  d |= (uint64_t)1u << 46;                          // descriptor version (sm100)
  d |= (uint64_t)2u << 61;                          // SWIZZLE_128B
  return d;
}

// kind::tf32 instruction descriptor: D f32, A/B tf32, both K-major, M=128, N
__host__ __device__ constexpr uint32_t make_idesc(int N)
{
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(MROWS >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t dtmem, uint64_t adesc, uint64_t bdesc,
                                         uint32_t idesc, uint32_t accumulate)
{
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n"
      :
      : "r"(dtmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
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

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float *v)
{
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                 "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 8; i++) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void fence_async_smem()
{
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

struct TcDev {
  const float4 *mats;    // B1 hi|mid|lo, B2 hi|mid|lo images
  int *status;           // device status word (0 = ok)
  int renorm;            // per-column isometry rescaling on
};

// 4 consecutive K values (hi and lo parts) of row r at k0 (k0 % 4 == 0)
__device__ __forceinline__ void put4(unsigned char *Ahi, unsigned char *Alo, int r, int k0,
                                     const float *x)
{
  const float h0 = tf32_rna(x[0]), h1 = tf32_rna(x[1]), h2 = tf32_rna(x[2]), h3 = tf32_rna(x[3]);
  const uint32_t off = sw128_off(r, k0, MROWS);
  *reinterpret_cast<float4 *>(Ahi + off) = make_float4(h0, h1, h2, h3);
  *reinterpret_cast<float4 *>(Alo + off) = make_float4(
      tf32_rna(x[0] - h0), tf32_rna(x[1] - h1), tf32_rna(x[2] - h2), tf32_rna(x[3] - h3));
}

// D = A * B over K = S: the small split terms first, the main term last
template <int S>
__device__ __forceinline__ void gemm_split(uint32_t dtmem, uint32_t a_hi, uint32_t a_lo,
                                           uint32_t b, int b_bytes)
{
  constexpr uint32_t idesc = make_idesc(S);
#pragma unroll
  for (int term = 0; term < 4; term++) {
#pragma unroll
    for (int kk = 0; kk < S; kk += 8) {
      const uint32_t aoff = (uint32_t)((kk >> 5) * MROWS * 128 + ((kk & 31) >> 3) * 32);
      const uint32_t boff = (uint32_t)((kk >> 5) * S * 128 + ((kk & 31) >> 3) * 32);
      // term 0: Ahi*Blo, 1: Ahi*Bmid, 2: Alo*Bhi, 3: Ahi*Bhi
      const uint32_t a = (term == 2 ? a_lo : a_hi) + aoff;
      const uint32_t bb = b + (term == 0 ? 2 * b_bytes : term == 1 ? b_bytes : 0) + boff;
      mma_tf32(dtmem, make_desc(a), make_desc(bb), idesc, (term | kk) ? 1u : 0u);
    }
  }
}

// sum over the four threads that hold one complex point (Re/Im rows x two
// column halves); `slot` is a [2][TPTS] smem array; includes a CTA barrier
__device__ __forceinline__ float point_sum(float part, float *slot, int half, int pt, bool is_im)
{
  part += __shfl_xor_sync(0xffffffffu, part, 1);
  if (!is_im) slot[half * TPTS + pt] = part;
  __syncthreads();
  return slot[pt] + slot[TPTS + pt];
}

template <int S>
__global__ void __launch_bounds__(NTHREADS, 1) k_column_tc(ColumnParams p, TcDev t, int mode)
{
  constexpr int H = S / 2;                     // K columns per thread (one half)
  constexpr int NKA = (S + 31) / 32;           // 128-byte swizzle atoms along K
  constexpr int A_BYTES = NKA * MROWS * 128;
  constexpr int B_BYTES = NKA * S * 128;
  extern __shared__ unsigned char smem_raw[];
  const uint32_t base_u = smem_u32(smem_raw);
  unsigned char *base = smem_raw + ((1024u - (base_u & 1023u)) & 1023u);
  unsigned char *Ahi = base;
  unsigned char *Alo = Ahi + A_BYTES;
  unsigned char *B1 = Alo + A_BYTES;            // hi | mid | lo
  unsigned char *B2 = B1 + 3 * B_BYTES;
  uint64_t *mbar = reinterpret_cast<uint64_t *>(B2 + 3 * B_BYTES);
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(mbar + 2);
  double *red = reinterpret_cast<double *>(mbar + 4);
  float *xch = reinterpret_cast<float *>(red + 32);      // [4][2][TPTS]

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int row = (warp & 3) * 32 + lane;        // TMEM lane == GEMM row
  const int half = warp >> 2;                    // column half handled
  const int c0 = half * H;                       // first K/N column of this thread
  const int pt = row >> 1;                       // complex point within tile
  const bool is_im = row & 1;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(smem_u32(tmem_slot)), "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&mbar[0])));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&mbar[1])));
  }
  {
    constexpr int n16 = 6 * B_BYTES / 16;
    float4 *dst = reinterpret_cast<float4 *>(B1);
    for (int i = tid; i < n16; i += NTHREADS) dst[i] = t.mats[i];
  }
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const uint32_t lane_base = ((uint32_t)((warp & 3) * 32)) << 16;
  const uint32_t d1 = tmem + lane_base + c0, d2 = tmem + lane_base + 64 + c0;
  const uint32_t mb1 = smem_u32(&mbar[0]), mb2 = smem_u32(&mbar[1]);
  uint32_t ph1 = 0, ph2 = 0;
  bool failed = false;

  float2 *surf = reinterpret_cast<float2 *>(p.surf);
  const float *lsrc = reinterpret_cast<const float *>(p.lpsi);
  float *ldst = reinterpret_cast<float *>(p.lpsi);
  const long ntiles = (p.n12 + TPTS - 1) / TPTS;
  const int comp = is_im ? 1 : 0;
  const int nnorm = p.nth < S ? p.nth : S;        // orders that enter the GEMM2 norm
  double nsum = 0.0;

  float a[H], vt[H];
  auto prefetch = [&](long tl) {
    const long qq = tl * TPTS + pt;
    const bool ok = tl < ntiles && qq < p.n12;
    if (mode != COL_HEAD) {
#pragma unroll
      for (int u = 0; u < H; u++) {
        const int l = c0 + u;
        a[u] = (ok && l < p.nl) ? __ldg(lsrc + 2 * ((long)l * p.n12 + qq) + comp) : 0.f;
      }
    }
    if (mode == COL_MID) {
#pragma unroll
      for (int u = 0; u < H; u++) {
        const int k = c0 + u;
        vt[u] = (ok && k < p.nth) ? __ldg(p.vturn + (long)k * p.n12 + qq) : 0.f;
      }
    }
  };
  prefetch(blockIdx.x);

  for (long tile = blockIdx.x; tile < ntiles && !failed; tile += gridDim.x) {
    const long q = tile * TPTS + pt;
    const bool qok = q < p.n12;
    const int j = qok ? (int)(q / p.n1) : 0, i = qok ? (int)(q % p.n1) : 0;
    float v[H];

    if (mode != COL_HEAD) {
      // ---- A1 = psi_l tile (row = Re/Im of a point, K = l) and its l-space norm
      float nl_part = 0.f;
#pragma unroll
      for (int u = 0; u < H; u += 4) put4(Ahi, Alo, row, c0 + u, a + u);
#pragma unroll
      for (int u = 0; u < H; u++) nl_part += a[u] * a[u] * __frcp_rn((float)(c0 + u) + 0.5f);
      fence_async_smem();
      tc_fence_before();
      __syncthreads();
      if (tid == 0) {
        tc_fence_after();
        gemm_split<S>(tmem, smem_u32(Ahi), smem_u32(Alo), smem_u32(B1), B_BYTES);
        mma_commit(mb1);
      }
      nl_part += __shfl_xor_sync(0xffffffffu, nl_part, 1);
      if (!is_im) xch[half * TPTS + pt] = nl_part;
      if (__syncthreads_or(!mbar_wait(mb1, ph1))) { failed = true; break; }
      ph1 ^= 1;
      tc_fence_after();
      const float n_l = xch[pt] + xch[TPTS + pt];
#pragma unroll
      for (int u = 0; u < H; u += 8) tmem_ld8(d1 + u, v + u);
      float nt_part = 0.f;
#pragma unroll
      for (int u = 0; u < H; u++)
        if (c0 + u < p.nth) nt_part += __ldg(p.w + c0 + u) * v[u] * v[u];
      const float n_t = point_sum(nt_part, xch + 2 * TPTS, half, pt, is_im);
      const float sc = (t.renorm && n_t > 0.f) ? sqrtf(n_l / n_t) : 1.f;
#pragma unroll
      for (int u = 0; u < H; u++) v[u] *= sc;
    } else {
#pragma unroll
      for (int u = 0; u < H; u++) {
        const int k = c0 + u;
        float val = 0.f;
        if (qok && k < p.nth) {
          const long g = (long)k * p.n12 + q;
          const double2 z = p.psi_z[g];
          double s, c;
          sincos(p.dt * p.pot[g], &s, &c);        // exp(-i V dt) = (c, -s)
          double2 f = make_double2(c, -s);
          if (p.prestep) {                       // psi / sqrt(v) * v = psi * sqrt(v)
            double sh, ch;
            sincos(0.5 * atan2(-s, c), &sh, &ch);
            f = make_double2(ch, sh);
          }
          val = (float)(is_im ? z.x * f.y + z.y * f.x : z.x * f.x - z.y * f.y);
        }
        v[u] = val;
      }
    }

    // ---- theta-space operations --------------------------------------------------
    float nt2_part = 0.f;
    if (mode != COL_HEAD) {
      const float dd = (p.d1 && qok) ? (float)(p.d1[i] * p.d2[j]) : 1.f;
      const bool flux_row = p.do_flux && qok && j >= p.surf_j0 && j < p.surf_j0 + p.surf_nrows;
#pragma unroll
      for (int u = 0; u < H; u++) {
        const int k = c0 + u;
        const float mine = v[u] * dd;
        const float other = __shfl_xor_sync(0xffffffffu, mine, 1);
        float re = is_im ? other : mine, im = is_im ? mine : other;
        if (qok && k < p.nth) {
          if (!is_im) {
            const long g = (long)k * p.n12 + q;
            if (flux_row) surf[((long)(j - p.surf_j0) * p.nth + k) * p.n1 + i] = make_float2(re, im);
            if (p.norm_out) nsum += __ldg(p.w + k) * ((double)re * re + (double)im * im);
            if (p.out_z) p.psi_z[g] = make_double2(re, im);
          }
          if (mode == COL_MID) {
            float sn, cs;
            sincospif(2.0f * vt[u], &sn, &cs);
            const float nr = re * cs - im * sn, ni = re * sn + im * cs;
            re = nr;
            im = ni;
          }
        }
        v[u] = is_im ? im : re;
      }
    }
    if (mode == COL_TAIL) {
      prefetch(tile + gridDim.x);
      tc_fence_before();
      __syncthreads();
      continue;
    }
#pragma unroll
    for (int u = 0; u < H; u++)
      if (c0 + u < p.nth) nt2_part += __ldg(p.w + c0 + u) * v[u] * v[u];

    // ---- GEMM2: D2 = A2 * B2 ------------------------------------------------------
#pragma unroll
    for (int u = 0; u < H; u += 4) put4(Ahi, Alo, row, c0 + u, v + u);
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      gemm_split<S>(tmem + 64, smem_u32(Ahi), smem_u32(Alo), smem_u32(B2), B_BYTES);
      mma_commit(mb2);
    }
    nt2_part += __shfl_xor_sync(0xffffffffu, nt2_part, 1);
    if (!is_im) xch[4 * TPTS + half * TPTS + pt] = nt2_part;
    prefetch(tile + gridDim.x);                  // next tile's loads fly during the MMA
    if (__syncthreads_or(!mbar_wait(mb2, ph2))) { failed = true; break; }
    ph2 ^= 1;
    tc_fence_after();
    const float n_t2 = xch[4 * TPTS + pt] + xch[5 * TPTS + pt];
#pragma unroll
    for (int u = 0; u < H; u += 8) tmem_ld8(d2 + u, v + u);
    float no_part = 0.f;
#pragma unroll
    for (int u = 0; u < H; u++)
      if (c0 + u < nnorm) no_part += v[u] * v[u] * __frcp_rn((float)(c0 + u) + 0.5f);
    const float n_o = point_sum(no_part, xch + 6 * TPTS, half, pt, is_im);
    const float sc2 = (t.renorm && n_o > 0.f) ? sqrtf(n_t2 / n_o) : 1.f;
#pragma unroll
    for (int u = 0; u < H; u++) {
      const int l = c0 + u;
      if (qok && l < p.nl) ldst[2 * ((long)l * p.n12 + q) + comp] = v[u] * sc2;
    }
    tc_fence_before();
    __syncthreads();
  }

  if (failed && lane == 0) atomicExch(t.status, 1);
  if (p.norm_out) {
    const double s = block_sum(nsum, red);
    if (tid == 0) atomicAdd(p.norm_out, s);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                 :: "r"(tmem), "r"(TMEM_COLS));
  }
}

template <int S> constexpr int smem_bytes_for()
{
  return 1024 + 2 * ((S + 31) / 32) * MROWS * 128 + 6 * ((S + 31) / 32) * S * 128 + 4 * 8 +
         32 * 8 + 8 * TPTS * 4;
}

// P_l(x_k) for l = 0..lmax by the recurrence of LegendreP2.m:9-21 (FP64)
std::vector<double> legendre_rows(int nth, int lmax, const double *x)
{
  std::vector<double> P((size_t)nth * (lmax + 1));
  for (int k = 0; k < nth; k++) {
    double p0 = 1.0, p1 = x[k];
    P[(size_t)k * (lmax + 1)] = 1.0;
    if (lmax >= 1) P[(size_t)k * (lmax + 1) + 1] = x[k];
    for (int l = 2; l <= lmax; l++) {
      const double p2 = (2.0 - 1.0 / l) * x[k] * p1 - (1.0 - 1.0 / l) * p0;
      P[(size_t)k * (lmax + 1) + l] = p2;
      p0 = p1;
      p1 = p2;
    }
  }
  return P;
}

}  // namespace

int tc_plan_create(TcPlan &plan, int nth, int nl, const double *legendre, const double *w,
                   const double *x, cudaStream_t s)
{
  const int S = pad16(nl > nth ? nl : nth);
  if (S > MAXS) return QD_ERR_UNSUPPORTED;
  // Extra orders l = n_l .. n_theta-1 for the GEMM2 norm, and a check that the
  // quadrature makes the transform pair an isometry (else no rescaling).
  bool renorm = nl <= nth;
  std::vector<double> Pext;
  if (renorm) {
    Pext = legendre_rows(nth, nth - 1, x);
    for (int k = 0; k < nth && renorm; k++)
      for (int l = 0; l < nl; l++)
        if (std::fabs(Pext[(size_t)k * nth + l] - legendre[l + (long)k * nl]) >
            1e-10 * (1.0 + std::fabs(legendre[l + (long)k * nl]))) {
          renorm = false;
          break;
        }
    for (int l = 0; l < nth && renorm; l++)
      for (int l2 = 0; l2 < nth; l2++) {
        double g = 0.0;
        for (int k = 0; k < nth; k++)
          g += w[k] * Pext[(size_t)k * nth + l] * Pext[(size_t)k * nth + l2];
        g *= (l2 + 0.5);
        if (std::fabs(g - (l == l2 ? 1.0 : 0.0)) > 1e-9) { renorm = false; break; }
      }
  }
  const int nka = (S + 31) / 32;
  const int bb = nka * S * 128;
  std::vector<unsigned char> img(6 * (size_t)bb, 0);
  unsigned char *b1 = img.data(), *b2 = b1 + 3 * bb;
  auto put = [&](unsigned char *img3, int r, int k, double val) {
    const float h = tf32_round_host((float)val);
    const double r1 = val - (double)h;
    const float m = tf32_round_host((float)r1);
    const float l = tf32_round_host((float)(r1 - (double)m));
    const uint32_t off = sw128_off(r, k, S);
    std::memcpy(img3 + off, &h, 4);
    std::memcpy(img3 + bb + off, &m, 4);
    std::memcpy(img3 + 2 * bb + off, &l, 4);
  };
  const int lrows = renorm ? nth : nl;          // orders formed by GEMM2
  for (int k = 0; k < nth; k++) {
    for (int l = 0; l < nl; l++) put(b1, k, l, legendre[l + (long)k * nl]);   // B1: row k, K = l
    for (int l = 0; l < lrows; l++) {
      const double P = l < nl ? legendre[l + (long)k * nl] : Pext[(size_t)k * nth + l];
      put(b2, l, k, (l + 0.5) * w[k] * P);                                     // B2: row l, K = k
    }
  }
  void *d = nullptr;
  if (cudaMalloc(&d, img.size() + sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    return QD_ERR_NOMEM;
  }
  if (cudaMemcpyAsync(d, img.data(), img.size(), cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemsetAsync((char *)d + img.size(), 0, sizeof(int), s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess) {
    cudaFree(d);
    return QD_ERR_CUDA;
  }
  plan.nth = nth; plan.nl = nl; plan.S = S; plan.renorm = renorm ? 1 : 0;
  plan.mats = d;
  plan.mats_bytes = img.size();
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  plan.grid = sms;
  cudaError_t e = cudaSuccess;
  switch (S) {
    case 16: plan.smem_bytes = smem_bytes_for<16>();
      e = cudaFuncSetAttribute(k_column_tc<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, plan.smem_bytes); break;
    case 32: plan.smem_bytes = smem_bytes_for<32>();
      e = cudaFuncSetAttribute(k_column_tc<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, plan.smem_bytes); break;
    case 48: plan.smem_bytes = smem_bytes_for<48>();
      e = cudaFuncSetAttribute(k_column_tc<48>, cudaFuncAttributeMaxDynamicSharedMemorySize, plan.smem_bytes); break;
    default: plan.smem_bytes = smem_bytes_for<64>();
      e = cudaFuncSetAttribute(k_column_tc<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, plan.smem_bytes); break;
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    cudaFree(d);
    plan.mats = nullptr;
    return QD_ERR_UNSUPPORTED;
  }
  return QD_OK;
}

void tc_plan_destroy(TcPlan &plan)
{
  if (plan.mats) cudaFree(plan.mats);
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
  t.status = tc_status_ptr(plan);
  t.renorm = plan.renorm;
  const long ntiles = (p.n12 + TPTS - 1) / TPTS;
  const int grid = (int)(ntiles < plan.grid ? ntiles : plan.grid);
  switch (plan.S) {
    case 16: k_column_tc<16><<<grid, NTHREADS, plan.smem_bytes, s>>>(p, t, mode); break;
    case 32: k_column_tc<32><<<grid, NTHREADS, plan.smem_bytes, s>>>(p, t, mode); break;
    case 48: k_column_tc<48><<<grid, NTHREADS, plan.smem_bytes, s>>>(p, t, mode); break;
    default: k_column_tc<64><<<grid, NTHREADS, plan.smem_bytes, s>>>(p, t, mode); break;
  }
  return cudaGetLastError();
}
