// k_mlp.cu -- a small permutation-symmetric MLP surrogate of a triatomic
// potential energy surface, trained and evaluated by this library's own
// kernels.  No counterpart in the reference, which calls its PES routines
// (Fortran/MEX, e.g. FH2/HSW/HSWMex.C) at every grid point; the plain PES
// stays the judge of the surrogate (|dV| on the grid, |dP(E)|) and its
// fallback.
//
// Network: features of the internuclear distances (atom 1 + diatom 2 3),
//   p_ij = exp(-r_ij / 1.5 bohr),  f = (p23, p12 + p13, p12 p13),
// invariant under exchanging atoms 2 and 3, standardised; then four dense
// layers of width 64 with SiLU, and a linear scalar output (standardised V).
// Weights: FP32 master copies for Adam, and an FP32 copy (wq) that every
// forward and backward product reads, FP32 accumulation.  (Products on
// BF16-rounded weights left 5.3 meV RMS on the C1 grid against 3.0 meV with
// FP32 weights, same training.)
//
// Training kernels over a minibatch of n samples (activations [n][64] in
// global memory, L2-resident): dense forward (Z = A W^T + b, A' = SiLU(Z)),
// output layer and loss, backward through the output, backward data
// (D_prev = (D W) * SiLU'(Z_prev)), weight gradients (G = D^T A_prev, summed
// over the batch in registers per CTA, then one atomic add per entry), Adam.
// Inference: one fused kernel per tile of 64 points (features from the
// Jacobi geometry, all layers in shared memory).
#include <cmath>
#include <cstring>
#include <vector>
#include "qd_err.h"

namespace {

constexpr int W = 64;                   // hidden width
constexpr int NF = 3;                   // features
constexpr int NL = 4;                   // hidden layers
// parameter layout (floats): W1[64][3] b1[64] | W2[64][64] b2 | W3 | W4 | Wo[64] bo
constexpr int layer_off(int l) { return l == 0 ? 0 : W * NF + W + (l - 1) * (W * W + W); }
constexpr int OFF_WO = layer_off(NL), OFF_BO = OFF_WO + W;
constexpr int NPARAM = OFF_BO + 1;
constexpr float FEAT_SCALE = 1.5f;      // bohr

__device__ __forceinline__ float silu(float z) { return z / (1.f + __expf(-z)); }
__device__ __forceinline__ float dsilu(float z)
{
  const float s = 1.f / (1.f + __expf(-z));
  return s * (1.f + z * (1.f - s));
}

struct Norm {
  float fmean[NF], fstd[NF];            // feature standardisation
  float vmean, vstd;                    // target standardisation
};

__device__ __forceinline__ void features(float r12, float r23, float r13, const Norm &nm, float *f)
{
  const float p12 = __expf(-r12 / FEAT_SCALE), p23 = __expf(-r23 / FEAT_SCALE),
              p13 = __expf(-r13 / FEAT_SCALE);
  f[0] = (p23 - nm.fmean[0]) / nm.fstd[0];
  f[1] = (p12 + p13 - nm.fmean[1]) / nm.fstd[1];
  f[2] = (p12 * p13 - nm.fmean[2]) / nm.fstd[2];
}

__global__ void k_features(int n, const double *r12, const double *r23, const double *r13,
                           Norm nm, float *F)
{
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    float f[NF];
    features((float)r12[s], (float)r23[s], (float)r13[s], nm, f);
    for (int c = 0; c < NF; c++) F[(long)s * NF + c] = f[c];
  }
}

// Z[s][o] = sum_k A[s][k] Wt[o][k] + b[o], A'[s][o] = SiLU(Z).  CTA: 64 samples x
// 64 outputs, 256 threads with 4 x 4 outputs each (rows tr + 16 i, cols tc + 16 j).
__global__ void __launch_bounds__(256) k_dense_fwd(int n, int K, const float *A, const float *Wt,
                                                   const float *b, float *Z, float *Aout)
{
  __shared__ float As[64][W + 1], Ws[W][W + 1];
  const int tid = threadIdx.x, tr = tid >> 4, tc = tid & 15, s0 = blockIdx.x * 64;
  for (int x = tid; x < 64 * K; x += 256) {
    const int r = x / K, k = x % K;
    As[r][k] = s0 + r < n ? A[(long)(s0 + r) * K + k] : 0.f;
    Ws[r][k] = Wt[r * K + k];
  }
  __syncthreads();
  float acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) acc[i][j] = b[tc + 16 * j];
  for (int k = 0; k < K; k++) {
    float a[4], w[4];
#pragma unroll
    for (int i = 0; i < 4; i++) a[i] = As[tr + 16 * i][k];
#pragma unroll
    for (int j = 0; j < 4; j++) w[j] = Ws[tc + 16 * j][k];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
      for (int j = 0; j < 4; j++) acc[i][j] = fmaf(a[i], w[j], acc[i][j]);
  }
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const int s = s0 + tr + 16 * i;
    if (s >= n) continue;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      Z[(long)s * W + tc + 16 * j] = acc[i][j];
      Aout[(long)s * W + tc + 16 * j] = silu(acc[i][j]);
    }
  }
}

// output layer, loss and its gradient: y = A4 . wo + bo, e = 2 (y - t) / n_total,
// D4[s][k] = e wo[k] SiLU'(Z4[s][k]); the loss sum goes to *loss
__global__ void __launch_bounds__(256) k_out_loss(int n, float inv_total, const float *A4,
                                                  const float *Z4, const float *wo, const float *bo,
                                                  const float *target, float *y, float *D4,
                                                  float *loss)
{
  __shared__ float red[8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int s = blockIdx.x * 8 + warp;            // one warp per sample
  float l2 = 0.f;
  if (s < n) {
    float acc = A4[(long)s * W + lane] * wo[lane] + A4[(long)s * W + lane + 32] * wo[lane + 32];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    const float yp = acc + bo[0];
    const float d = yp - (target ? target[s] : 0.f);
    if (lane == 0) {
      if (y) y[s] = yp;
      l2 = d * d;
    }
    if (D4) {
      const float e = 2.f * d * inv_total;
      D4[(long)s * W + lane] = e * wo[lane] * dsilu(Z4[(long)s * W + lane]);
      D4[(long)s * W + lane + 32] = e * wo[lane + 32] * dsilu(Z4[(long)s * W + lane + 32]);
    }
  }
  if (lane == 0) red[warp] = l2;
  __syncthreads();
  if (threadIdx.x == 0 && loss) {
    float t = 0.f;
    for (int w = 0; w < 8; w++) t += red[w];
    atomicAdd(loss, t);
  }
}

// Dp[s][k] = (sum_o D[s][o] Wt[o][k]) * SiLU'(Zp[s][k]) for the layer below (K = 64)
__global__ void __launch_bounds__(256) k_dense_bwd_data(int n, const float *D, const float *Wt,
                                                        const float *Zp, float *Dp)
{
  __shared__ float Ds[64][W + 1], Ws[W][W + 1];
  const int tid = threadIdx.x, tr = tid >> 4, tc = tid & 15, s0 = blockIdx.x * 64;
  for (int x = tid; x < 64 * W; x += 256) {
    const int r = x / W, k = x % W;
    Ds[r][k] = s0 + r < n ? D[(long)(s0 + r) * W + k] : 0.f;
    Ws[r][k] = Wt[r * W + k];
  }
  __syncthreads();
  float acc[4][4] = {};
  for (int o = 0; o < W; o++) {
    float d[4], w[4];
#pragma unroll
    for (int i = 0; i < 4; i++) d[i] = Ds[tr + 16 * i][o];
#pragma unroll
    for (int j = 0; j < 4; j++) w[j] = Ws[o][tc + 16 * j];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
      for (int j = 0; j < 4; j++) acc[i][j] = fmaf(d[i], w[j], acc[i][j]);
  }
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const int s = s0 + tr + 16 * i;
    if (s >= n) continue;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const long q = (long)s * W + tc + 16 * j;
      Dp[q] = acc[i][j] * dsilu(Zp[q]);
    }
  }
}

// G[o][k] += sum_s D[s][o] Ap[s][k], gb[o] += sum_s D[s][o] over this CTA's
// chunk of samples (K <= 64; Ap = features for the first layer, then A)
constexpr int GCHUNK = 512;
__global__ void __launch_bounds__(256) k_dense_bwd_weight(int n, int K, const float *D,
                                                          const float *Ap, float *G, float *gb)
{
  __shared__ float Ds[64][W + 1], As[64][W + 1];
  const int tid = threadIdx.x, tr = tid >> 4, tc = tid & 15;
  float acc[4][4] = {};
  float accb[4] = {};
  const int sb = blockIdx.x * GCHUNK, se = min(n, sb + GCHUNK);
  for (int s0 = sb; s0 < se; s0 += 64) {
    for (int x = tid; x < 64 * W; x += 256) {
      const int r = x / W, c = x % W;
      const bool ok = s0 + r < se;
      Ds[r][c] = ok ? D[(long)(s0 + r) * W + c] : 0.f;
      As[r][c] = (ok && c < K) ? Ap[(long)(s0 + r) * K + c] : 0.f;
    }
    __syncthreads();
    for (int r = 0; r < 64; r++) {
      float d[4], a[4];
#pragma unroll
      for (int i = 0; i < 4; i++) d[i] = Ds[r][tr + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; j++) a[j] = As[r][tc + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; i++) {
        if (tc == 0) accb[i] += d[i];
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = fmaf(d[i], a[j], acc[i][j]);
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const int o = tr + 16 * i;
    if (tc == 0) atomicAdd(gb + o, accb[i]);
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int k = tc + 16 * j;
      if (k < K) atomicAdd(G + o * K + k, acc[i][j]);
    }
  }
}

// output-layer gradients: gwo[k] = sum_s e_s A4[s][k] with e_s = D4 / (wo SiLU')
// recomputed from y and the targets; done as G = E^T A4 with E the scalar errors
__global__ void __launch_bounds__(256) k_out_grad(int n, float inv_total, const float *A4,
                                                  const float *y, const float *target, float *gwo,
                                                  float *gbo)
{
  __shared__ float red[W][9];
  const int k = threadIdx.x & 63, part = threadIdx.x >> 6;   // 4 parts of the chunk
  float acc = 0.f, accb = 0.f;
  const int sb = blockIdx.x * GCHUNK, se = min(n, sb + GCHUNK);
  for (int s = sb + part; s < se; s += 4) {
    const float e = 2.f * (y[s] - target[s]) * inv_total;
    acc = fmaf(e, A4[(long)s * W + k], acc);
    if (k == 0) accb += e;
  }
  red[k][part] = acc;
  red[k][4 + part] = accb;
  __syncthreads();
  if (threadIdx.x < W) {
    const float t = red[k][0] + red[k][1] + red[k][2] + red[k][3];
    atomicAdd(gwo + k, t);
    if (k == 0) atomicAdd(gbo, red[0][4] + red[0][5] + red[0][6] + red[0][7]);
  }
}

// Adam on the FP32 masters; their copies feed the products
__global__ void k_adam(int np, float *w, float *wq, const float *g, float *m, float *v, float lr,
                       float b1, float b2, float eps, float c1, float c2)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi, vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    wq[i] = wi;
  }
}

__global__ void k_copy_weights(int np, const float *w, float *wq)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x)
    wq[i] = w[i];
}

// Fused inference on the Jacobi grid (H3/H3PESJacobi.m:5-27 geometry): per
// tile of 64 points, features, four SiLU layers and the output in shared
// memory; V = vmax where a distance <= rmin, else min(V_mlp, vmax) if cap.
struct GridArgs {
  int n1, n2, nth;
  const double *R, *r, *x;
  double f2, f3, vmax, rmin;
  int cap;
};
// every layer's weights stay in shared memory for the whole launch (loaded
// once per CTA), activations of 64 points at a time in place
constexpr int WS = W + 1;                                  // padded weight / activation row
constexpr size_t GRID_SMEM = sizeof(float) * ((size_t)NL * W * WS + 64 * WS + 64 * NF) + 64;
__global__ void __launch_bounds__(256) k_mlp_grid(GridArgs g, Norm nm, const float *wq,
                                                  double *pot, long npts, const double *r12p,
                                                  const double *r23p, const double *r13p)
{
  extern __shared__ float4 grid_sm4[];
  float *sm = reinterpret_cast<float *>(grid_sm4);
  float (*Wsm)[W][WS] = reinterpret_cast<float (*)[W][WS]>(sm);            // [NL][W][WS]
  float (*H)[WS] = reinterpret_cast<float (*)[WS]>(sm + NL * W * WS);      // [64][WS]
  float (*feat)[NF] = reinterpret_cast<float (*)[NF]>(sm + NL * W * WS + 64 * WS);
  unsigned char *mask = reinterpret_cast<unsigned char *>(sm + NL * W * WS + 64 * WS + 64 * NF);
  const int tid = threadIdx.x, tr = tid >> 4, tc = tid & 15;
  for (int l = 0; l < NL; l++) {
    const int K = l == 0 ? NF : W;
    const float *Wl = wq + layer_off(l);
    for (int x = tid; x < W * K; x += 256) Wsm[l][x / K][x % K] = Wl[x];
  }
  for (long base = (long)blockIdx.x * 64; base < npts; base += (long)gridDim.x * 64) {
    if (tid < 64) {
      const long q = base + tid;
      float f[NF] = {0.f, 0.f, 0.f};
      unsigned char ok = 0;
      if (q < npts) {
        double r12, r23, r13;
        if (r12p) {
          r12 = r12p[q]; r23 = r23p[q]; r13 = r13p[q];
          ok = 1;
        } else {
          const int i = (int)(q % g.n1), j = (int)((q / g.n1) % g.n2), k = (int)(q / ((long)g.n1 * g.n2));
          const double Rv = g.R[i], rv = g.r[j], c = g.x[k];
          const double a = g.f2 * rv, b = g.f3 * rv;
          r23 = rv;
          r12 = sqrt(a * a + Rv * Rv - 2.0 * g.f2 * rv * Rv * c);
          r13 = sqrt(b * b + Rv * Rv + 2.0 * g.f3 * rv * Rv * c);
          ok = (r12 > g.rmin && r13 > g.rmin && r23 > g.rmin) ? 1 : 0;
        }
        features((float)r12, (float)r23, (float)r13, nm, f);
      }
      for (int c = 0; c < NF; c++) feat[tid][c] = f[c];
      mask[tid] = ok;
    }
    __syncthreads();                      // features (and, first time, the weights) in place
    for (int l = 0; l < NL; l++) {
      const int K = l == 0 ? NF : W;
      const float *bl = wq + layer_off(l) + W * K;
      float acc[4][4];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = bl[tc + 16 * j];
      for (int k = 0; k < K; k++) {
        float a[4], w[4];
#pragma unroll
        for (int i = 0; i < 4; i++) a[i] = l == 0 ? feat[tr + 16 * i][k] : H[tr + 16 * i][k];
#pragma unroll
        for (int j = 0; j < 4; j++) w[j] = Wsm[l][tc + 16 * j][k];
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
          for (int j = 0; j < 4; j++) acc[i][j] = fmaf(a[i], w[j], acc[i][j]);
      }
      __syncthreads();                    // every read of H is done
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) H[tr + 16 * i][tc + 16 * j] = silu(acc[i][j]);
      __syncthreads();
    }
    // output: one warp per 8 points
    const int lane = tid & 31, warp = tid >> 5;
    for (int pnt = warp; pnt < 64; pnt += 8) {
      float acc = H[pnt][lane] * wq[OFF_WO + lane] + H[pnt][lane + 32] * wq[OFF_WO + lane + 32];
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
      const long q = base + pnt;
      if (lane == 0 && q < npts) {
        double v = (double)(acc + wq[OFF_BO]) * nm.vstd + nm.vmean;
        if (!r12p) {
          if (!mask[pnt]) v = g.vmax;
          else if (g.cap) v = fmin(v, g.vmax);
        }
        pot[q] = v;
      }
    }
    __syncthreads();
  }
}

cudaError_t launch_mlp_grid(long blocks, const GridArgs &g, const Norm &nm, const float *wq,
                            double *pot, long npts, const double *r12p, const double *r23p,
                            const double *r13p)
{
  static const cudaError_t attr = cudaFuncSetAttribute(
      k_mlp_grid, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)GRID_SMEM);
  if (attr != cudaSuccess) return attr;
  k_mlp_grid<<<(unsigned)(blocks < 148 * 2 ? blocks : 148 * 2), 256, GRID_SMEM>>>(
      g, nm, wq, pot, npts, r12p, r23p, r13p);
  qd_count_launches(1);
  return cudaGetLastError();
}

}  // namespace

// ---- host side -----------------------------------------------------------

struct qd_mlp {
  Norm norm{};
  std::vector<float> w;                 // FP32 masters (host copy)
  float *d_w = nullptr, *d_wq = nullptr, *d_m = nullptr, *d_v = nullptr, *d_g = nullptr;
  long step = 0;
  ~qd_mlp()
  {
    for (float *p : {d_w, d_wq, d_m, d_v, d_g}) cudaFree(p);
  }
};

namespace {

// splitmix64 + Box-Muller free uniform init (He-uniform per layer), seeded
uint64_t mix(uint64_t &s)
{
  uint64_t z = (s += 0x9e3779b97f4a7c15ull);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

void host_features(double r12, double r23, double r13, double *f)
{
  const double p12 = std::exp(-r12 / FEAT_SCALE), p23 = std::exp(-r23 / FEAT_SCALE),
               p13 = std::exp(-r13 / FEAT_SCALE);
  f[0] = p23;
  f[1] = p12 + p13;
  f[2] = p12 * p13;
}

int upload_params(qd_mlp *m)
{
  QD_CU(cudaMemcpy(m->d_w, m->w.data(), sizeof(float) * NPARAM, cudaMemcpyHostToDevice));
  k_copy_weights<<<(NPARAM + 255) / 256, 256>>>(NPARAM, m->d_w, m->d_wq);
  qd_count_launches(1);
  QD_CU(cudaGetLastError());
  return QD_OK;
}

}  // namespace

extern "C" {

int qd_mlp_create(qd_mlp **out, uint64_t seed)
{
  if (!out) return qd_errf(QD_ERR_INVALID, "NULL argument");
  qd_mlp *m = new qd_mlp();
  m->w.assign(NPARAM, 0.f);
  uint64_t s = seed;
  for (int l = 0; l <= NL; l++) {
    const int K = l == 0 ? NF : W, nout = l == NL ? 1 : W;
    const int off = l == NL ? OFF_WO : layer_off(l);
    const double a = std::sqrt(6.0 / K);
    for (int x = 0; x < nout * K; x++)
      m->w[off + x] = (float)(a * (2.0 * (double)(mix(s) >> 11) / 9007199254740992.0 - 1.0));
  }
  for (int c = 0; c < NF; c++) { m->norm.fmean[c] = 0.f; m->norm.fstd[c] = 1.f; }
  m->norm.vmean = 0.f;
  m->norm.vstd = 1.f;
  for (float **p : {&m->d_w, &m->d_wq, &m->d_m, &m->d_v, &m->d_g})
    if (cudaMalloc(p, sizeof(float) * NPARAM) != cudaSuccess) {
      cudaGetLastError();
      delete m;
      return qd_errf(QD_ERR_NOMEM, "qd_mlp_create: cudaMalloc failed");
    }
  cudaMemset(m->d_m, 0, sizeof(float) * NPARAM);
  cudaMemset(m->d_v, 0, sizeof(float) * NPARAM);
  int rc = upload_params(m);
  if (rc != QD_OK) { delete m; return rc; }
  *out = m;
  return QD_OK;
}

int qd_mlp_destroy(qd_mlp *m)
{
  delete m;
  return QD_OK;
}

int32_t qd_mlp_n_params(void) { return NPARAM; }

int qd_mlp_get_params(qd_mlp *m, float *w_out, float norm_out[8])
{
  if (!m || !w_out) return qd_errf(QD_ERR_INVALID, "NULL argument");
  QD_CU(cudaMemcpy(w_out, m->d_w, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost));
  if (norm_out) {
    for (int c = 0; c < NF; c++) { norm_out[c] = m->norm.fmean[c]; norm_out[NF + c] = m->norm.fstd[c]; }
    norm_out[6] = m->norm.vmean;
    norm_out[7] = m->norm.vstd;
  }
  return QD_OK;
}

int qd_mlp_set_params(qd_mlp *m, const float *w, const float norm[8])
{
  if (!m || !w) return qd_errf(QD_ERR_INVALID, "NULL argument");
  m->w.assign(w, w + NPARAM);
  if (norm) {
    for (int c = 0; c < NF; c++) { m->norm.fmean[c] = norm[c]; m->norm.fstd[c] = norm[NF + c]; }
    m->norm.vmean = norm[6];
    m->norm.vstd = norm[7];
  }
  return upload_params(m);
}

// standardisation of features and targets from a training set (host, FP64)
int qd_mlp_fit_normalisation(qd_mlp *m, int64_t n, const double *r12, const double *r23,
                             const double *r13, const double *V)
{
  if (!m || n < 2 || !r12 || !r23 || !r13 || !V) return qd_errf(QD_ERR_INVALID, "bad argument");
  double s[NF] = {}, s2[NF] = {}, sv = 0.0, sv2 = 0.0;
  for (int64_t i = 0; i < n; i++) {
    double f[NF];
    host_features(r12[i], r23[i], r13[i], f);
    for (int c = 0; c < NF; c++) { s[c] += f[c]; s2[c] += f[c] * f[c]; }
    sv += V[i];
    sv2 += V[i] * V[i];
  }
  for (int c = 0; c < NF; c++) {
    const double mu = s[c] / n, var = s2[c] / n - mu * mu;
    m->norm.fmean[c] = (float)mu;
    m->norm.fstd[c] = (float)std::sqrt(var > 1e-30 ? var : 1e-30);
  }
  const double mu = sv / n, var = sv2 / n - mu * mu;
  m->norm.vmean = (float)mu;
  m->norm.vstd = (float)std::sqrt(var > 1e-30 ? var : 1e-30);
  return QD_OK;
}

// Loss (mean squared error of the standardised V) and, if grad_out, its
// gradient with respect to the FP32 parameters, for n samples in one batch.
// With train_steps > 0 instead: that many Adam steps over the data in
// minibatches of `batch` samples (in order, wrapping), learning rate lr
// decaying geometrically to lr_end; loss_out gets the last epoch's mean loss.
int qd_mlp_train(qd_mlp *m, int64_t n, const double *r12, const double *r23, const double *r13,
                 const double *V, int32_t train_steps, int32_t batch, double lr, double lr_end,
                 float *grad_out, double *loss_out)
{
  if (!m || n < 1 || !r12 || !r23 || !r13 || !V || batch < 1)
    return qd_errf(QD_ERR_INVALID, "qd_mlp_train: bad argument");
  const int B = (int)(train_steps > 0 ? (batch < n ? batch : n) : n);
  // device data: features and standardised targets for all n samples
  double *dr = nullptr;
  float *buf = nullptr;
  QD_CU(cudaMalloc(&dr, sizeof(double) * 3 * n));
  const size_t act = (size_t)B * W;
  const size_t nbuf = (size_t)n * NF + n + (size_t)B * NF + 2 * NL * act + 2 * act + B + 1;
  cudaError_t e = cudaMalloc(&buf, sizeof(float) * nbuf);
  if (e != cudaSuccess) { cudaFree(dr); return qd_errf(QD_ERR_NOMEM, "qd_mlp_train: cudaMalloc"); }
  float *F = buf, *T = F + (size_t)n * NF, *FB = T + n;
  float *Z = FB + (size_t)B * NF, *A = Z + NL * act;          // [NL][B][64] each
  float *D = A + NL * act, *D2 = D + act, *Y = D2 + act, *loss = Y + B;
  std::vector<float> tgt(n);
  for (int64_t i = 0; i < n; i++) tgt[i] = (float)((V[i] - m->norm.vmean) / m->norm.vstd);
  int rc = QD_OK;
  auto fail = [&](cudaError_t x) {
    rc = qd_errf(QD_ERR_CUDA, "qd_mlp_train: %s", cudaGetErrorString(x));
  };
  if ((e = cudaMemcpy(dr, r12, sizeof(double) * n, cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemcpy(dr + n, r23, sizeof(double) * n, cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemcpy(dr + 2 * n, r13, sizeof(double) * n, cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemcpy(T, tgt.data(), sizeof(float) * n, cudaMemcpyHostToDevice)) != cudaSuccess)
    fail(e);
  if (rc == QD_OK) {
    k_features<<<(int)((n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096), 256>>>(
        (int)n, dr, dr + n, dr + 2 * n, m->norm, F);
    qd_count_launches(1);
  }
  // one forward + backward over samples [s0, s0 + b): gradient into d_g
  auto pass = [&](int64_t s0, int b, float inv_total, bool grads) -> cudaError_t {
    const float *Fb = F + s0 * NF;
    const float *tb = T + s0;
    const int g64 = (b + 63) / 64, gch = (b + GCHUNK - 1) / GCHUNK;
    for (int l = 0; l < NL; l++) {
      const int K = l == 0 ? NF : W;
      const float *in = l == 0 ? Fb : A + (l - 1) * act;
      k_dense_fwd<<<g64, 256>>>(b, K, in, m->d_wq + layer_off(l), m->d_wq + layer_off(l) + W * K,
                                Z + l * act, A + l * act);
    }
    k_out_loss<<<(b + 7) / 8, 256>>>(b, inv_total, A + (NL - 1) * act, Z + (NL - 1) * act,
                                     m->d_wq + OFF_WO, m->d_wq + OFF_BO, tb, Y,
                                     grads ? D : nullptr, loss);
    qd_count_launches(NL + 1);
    if (!grads) return cudaGetLastError();
    k_out_grad<<<gch, 256>>>(b, inv_total, A + (NL - 1) * act, Y, tb, m->d_g + OFF_WO,
                             m->d_g + OFF_BO);
    float *Dc = D, *Dn = D2;
    for (int l = NL - 1; l >= 0; l--) {
      const int K = l == 0 ? NF : W;
      const float *in = l == 0 ? Fb : A + (l - 1) * act;
      k_dense_bwd_weight<<<gch, 256>>>(b, K, Dc, in, m->d_g + layer_off(l),
                                       m->d_g + layer_off(l) + W * K);
      if (l > 0) {
        k_dense_bwd_data<<<g64, 256>>>(b, Dc, m->d_wq + layer_off(l), Z + (l - 1) * act, Dn);
        float *t = Dc; Dc = Dn; Dn = t;
      }
    }
    qd_count_launches(1 + NL + (NL - 1));
    return cudaGetLastError();
  };
  if (rc == QD_OK && train_steps <= 0) {                      // gradient / loss only
    cudaMemset(m->d_g, 0, sizeof(float) * NPARAM);
    cudaMemset(loss, 0, sizeof(float));
    if ((e = pass(0, (int)n, 1.f / (float)n, grad_out != nullptr)) != cudaSuccess) fail(e);
    float l = 0.f;
    if (rc == QD_OK && (e = cudaMemcpy(&l, loss, sizeof(float), cudaMemcpyDeviceToHost)) != cudaSuccess)
      fail(e);
    if (rc == QD_OK && grad_out &&
        (e = cudaMemcpy(grad_out, m->d_g, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost)) != cudaSuccess)
      fail(e);
    if (loss_out) *loss_out = l / (double)n;
  } else if (rc == QD_OK) {
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const double decay = train_steps > 1 ? std::pow(lr_end / lr, 1.0 / (train_steps - 1)) : 1.0;
    double lr_t = lr, epoch_loss = 0.0;
    int64_t s0 = 0, seen = 0;
    cudaMemset(loss, 0, sizeof(float));
    for (int st = 0; st < train_steps && rc == QD_OK; st++) {
      const int b = (int)(s0 + B <= n ? B : n - s0);
      cudaMemset(m->d_g, 0, sizeof(float) * NPARAM);
      if ((e = pass(s0, b, 1.f / (float)b, true)) != cudaSuccess) { fail(e); break; }
      m->step++;
      const float c1 = 1.f - std::pow(b1, (float)m->step), c2 = 1.f - std::pow(b2, (float)m->step);
      k_adam<<<(NPARAM + 255) / 256, 256>>>(NPARAM, m->d_w, m->d_wq, m->d_g, m->d_m, m->d_v,
                                            (float)lr_t, b1, b2, eps, c1, c2);
      qd_count_launches(1);
      lr_t *= decay;
      s0 += b;
      seen += b;
      if (s0 >= n) {                                          // end of an epoch
        float l = 0.f;
        cudaMemcpy(&l, loss, sizeof(float), cudaMemcpyDeviceToHost);
        epoch_loss = l / (double)seen;
        cudaMemset(loss, 0, sizeof(float));
        s0 = 0;
        seen = 0;
      }
    }
    if (rc == QD_OK && (e = cudaDeviceSynchronize()) != cudaSuccess) fail(e);
    if (seen > 0 && rc == QD_OK) {
      float l = 0.f;
      cudaMemcpy(&l, loss, sizeof(float), cudaMemcpyDeviceToHost);
      epoch_loss = l / (double)seen;
    }
    if (loss_out) *loss_out = epoch_loss;
    if (rc == QD_OK)
      cudaMemcpy(m->w.data(), m->d_w, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost);
  }
  cudaFree(dr);
  cudaFree(buf);
  return rc;
}

// V (hartree) at n geometries (r12, r23, r13 in bohr)
int qd_mlp_eval(qd_mlp *m, int64_t n, const double *r12, const double *r23, const double *r13,
                double *V_out)
{
  if (!m || n < 1 || !r12 || !r23 || !r13 || !V_out) return qd_errf(QD_ERR_INVALID, "bad argument");
  double *d = nullptr;
  QD_CU(cudaMalloc(&d, sizeof(double) * 4 * n));
  cudaError_t e = cudaMemcpy(d, r12, sizeof(double) * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + n, r23, sizeof(double) * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + 2 * n, r13, sizeof(double) * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    GridArgs g{};
    const long blocks = (n + 63) / 64;
    e = launch_mlp_grid(blocks, g, m->norm, m->d_wq, d + 3 * n, n, d, d + n, d + 2 * n);
  }
  if (e == cudaSuccess) e = cudaMemcpy(V_out, d + 3 * n, sizeof(double) * n, cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return qd_errf(QD_ERR_CUDA, "qd_mlp_eval: %s", cudaGetErrorString(e));
  return QD_OK;
}

// the surrogate on the Jacobi grid, the layout and masking of qd_potential_jacobi
int qd_mlp_potential(qd_mlp *m, const qd_radial *R, const qd_radial *r, const qd_angle *theta,
                     const double masses[3], double vmax, double rmin, int32_t cap, double *pot_out)
{
  if (!m || !R || !r || !theta || !masses || !pot_out || !R->r || !r->r || !theta->x)
    return qd_errf(QD_ERR_INVALID, "NULL argument");
  if (R->n < 1 || r->n < 1 || theta->n < 1 || !(masses[1] + masses[2] > 0))
    return qd_errf(QD_ERR_INVALID, "bad grid or masses");
  GridArgs g{};
  g.n1 = R->n; g.n2 = r->n; g.nth = theta->n;
  g.f2 = masses[2] / (masses[1] + masses[2]);
  g.f3 = 1.0 - g.f2;
  g.vmax = vmax; g.rmin = rmin; g.cap = cap ? 1 : 0;
  const long n = (long)g.n1 * g.n2 * g.nth;
  double *d = nullptr;
  QD_CU(cudaMalloc(&d, sizeof(double) * ((size_t)n + g.n1 + g.n2 + g.nth)));
  double *dR = d + n, *dr = dR + g.n1, *dx = dr + g.n2;
  cudaError_t e = cudaMemcpy(dR, R->r, sizeof(double) * g.n1, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dr, r->r, sizeof(double) * g.n2, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dx, theta->x, sizeof(double) * g.nth, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    g.R = dR; g.r = dr; g.x = dx;
    const long blocks = (n + 63) / 64;
    e = launch_mlp_grid(blocks, g, m->norm, m->d_wq, d, n, nullptr, nullptr, nullptr);
  }
  if (e == cudaSuccess) e = cudaMemcpy(pot_out, d, sizeof(double) * n, cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return qd_errf(QD_ERR_CUDA, "qd_mlp_potential: %s", cudaGetErrorString(e));
  return QD_OK;
}

}  // extern "C"
