// k_flux.cu -- flux through the dividing surface r = r_s and P(E).
//
//   k_flux_prep    psi_s(i,k) and d psi_s/dr by the central differences of
//                  Gradient3.F:31-167 (3..11 points, same coefficient order),
//                  from the surface rows captured by the column pass; stored
//                  in FP64 in a history ring (one slot per step).
//   k_flux_phase   the factors dt e^{iE t} of a chunk of steps (the e^{iEt}
//                  recurrence of timeEvol.C:807-817 evaluated directly, FP64)
//   k_flux_gemm    phi_E += sum_t dt e^{iE t} psi_s(t), dphi_E likewise
//                  (PsiTimeToPsiEnergyOnSurface, CRPAux.F:4-31): a
//                  register-tiled complex FP64 GEMM over the chunk.
//   k_crp          P(E) = Im(sum_k w_k sum_i conj(phi) dphi) / eta^2 dr1/mu2
//                  (CalculateCRP, CRPAux.F:34-66), warp-shuffle reduction.
#include "qd_kernels.h"

namespace {

template <typename R>
__global__ void k_flux_prep(FluxParams p)
{
  typedef typename Cplx<R>::T C;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < p.nruns * p.nth * p.n1) flux_point<C>(p, q);
}

constexpr int TMAX = FLUX_CHUNK;   // max steps per chunk

// phase[run][e][t] = dt e^{i E_e (t0 + t + 1) dt} of this chunk, FP64
__global__ void __launch_bounds__(256) k_flux_phase(AccumParams p)
{
  const int n = p.nruns * p.ne * p.nt;
  for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < n; x += gridDim.x * blockDim.x) {
    const int t = x % p.nt, re = x / p.nt;                 // re = run * ne + e
    double sn, cs;
    sincos(p.energies[re] * p.dt * (double)(p.t0 + t + 1), &sn, &cs);
    p.phase[(size_t)re * TMAX + t] = make_double2(p.dt * cs, p.dt * sn);
  }
}

// phi[e][q] += sum_t phase[e][t] psi_s[t][q] (and dphi with the gradient), a
// complex FP64 GEMM per run.  CTA tile: GE energies x GQ surface points x
// {psi_s, d psi_s}; each thread owns 4 energies x 4 columns (2 points x 2
// fields) in registers, GE / 4 x 16 threads.  KT steps of phases and history
// are staged in shared memory by asynchronous copies into two buffers, so the
// next KT steps load while the current ones are multiplied; the history is
// read from HBM once per energy tile.  The variant (GE, KT) is picked per
// shape by the autotuner.
constexpr int GQ = 32;

__device__ __forceinline__ void cp16(void *dst, const void *src, bool valid)
{
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  const int n = valid ? 16 : 0;                 // 0: fill the 16 bytes with zeros
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;" :: "r"(d), "l"(src), "r"(n)
               : "memory");
}

template <int GE, int KT>
__global__ void __launch_bounds__(GE * 4) k_flux_gemm(AccumParams p)
{
  constexpr int NT = GE * 4;                    // threads: GE / 4 energy groups x 16
  __shared__ double2 As[2][GE][KT + 1];         // phases (padded rows)
  __shared__ double2 Bs[2][KT][2 * GQ];         // cols 0..GQ-1 psi_s, GQ..2GQ-1 gradient
  const int tid = threadIdx.x;
  const int te = tid >> 4, tc = tid & 15;       // GE/4 energy groups x 16 column groups
  const int e0 = blockIdx.x * GE, q0 = blockIdx.y * GQ, run = blockIdx.z;
  const double2 *ph = p.phase + ((size_t)run * p.ne) * TMAX;
  auto stage = [&](int buf, int t0) {
    for (int x = tid; x < GE * KT; x += NT) {
      const int e = x / KT, t = x % KT;
      const bool ok = e0 + e < p.ne && t0 + t < p.nt;
      cp16(&As[buf][e][t], ok ? ph + (size_t)(e0 + e) * TMAX + t0 + t : ph, ok);
    }
    for (int x = tid; x < KT * 2 * GQ; x += NT) {
      const int t = x / (2 * GQ), c = x % (2 * GQ), q = q0 + (c % GQ);
      const bool ok = t0 + t < p.nt && q < p.nq;
      const size_t o = ok ? ((size_t)(t0 + t) * p.nruns + run) * p.nq + q : 0;
      cp16(&Bs[buf][t][c], (c < GQ ? p.ring_psi : p.ring_g) + o, ok);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  double2 acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) acc[i][j] = make_double2(0.0, 0.0);
  const int nchunk = (p.nt + KT - 1) / KT;
  stage(0, 0);
  for (int ch = 0; ch < nchunk; ch++) {
    const int buf = ch & 1;
    if (ch + 1 < nchunk) {
      stage(buf ^ 1, (ch + 1) * KT);
      asm volatile("cp.async.wait_group 1;" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    }
    __syncthreads();
#pragma unroll 2
    for (int k = 0; k < KT; k++) {             // rows past nt were zero-filled
      double2 a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; i++) a[i] = As[buf][te + (GE / 4) * i][k];
#pragma unroll
      for (int j = 0; j < 4; j++) b[j] = Bs[buf][k][tc + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) {
          acc[i][j].x = fma(a[i].x, b[j].x, fma(-a[i].y, b[j].y, acc[i][j].x));
          acc[i][j].y = fma(a[i].x, b[j].y, fma(a[i].y, b[j].x, acc[i][j].y));
        }
    }
    __syncthreads();                            // buffer free for the stage after next
  }
  // phi += acc, two energy rows at a time: their eight loads are all issued
  // before any of their stores (a store between two loads would make each
  // load wait for the one before, since phi and dphi may alias as far as the
  // compiler knows)
  auto at = [&](int i, int j) -> double2 * {
    const int e = e0 + te + (GE / 4) * i, c = tc + 16 * j, q = q0 + (c % GQ);
    if (e >= p.ne || q >= p.nq) return nullptr;
    return (c < GQ ? p.fai : p.dfai) + ((size_t)run * p.ne + e) * p.nq + q;
  };
  // with crp_part: this tile's share of P(E), the sum over its points of
  // w_k Im(conj(phi) dphi) of the updated values (columns j and j + 2 of a
  // thread are phi and dphi of one point; entries past n_E or past the
  // surface are zero), formed as each energy row pair is written and reduced
  // over the 16 column groups of each row at the end.  A tile of GQ points
  // spans at most two theta rows when n1 >= GQ.
  const bool want_pe = p.crp_part != nullptr;
  double wq[2] = {0.0, 0.0};
  if (want_pe) {
    const int k0 = q0 / p.n1;
#pragma unroll
    for (int j = 0; j < 2; j++) {
      const int q = q0 + tc + 16 * j;
      const int k = p.n1 >= GQ ? (q - k0 * p.n1 >= p.n1 ? k0 + 1 : k0) : q / p.n1;
      wq[j] = q < p.nq ? __ldg(p.w + k) : 0.0;
    }
  }
  double pe[4];
#pragma unroll
  for (int h = 0; h < 4; h += 2) {
#pragma unroll
    for (int i = h; i < h + 2; i++)
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const double2 *src = at(i, j);
        if (src) {
          const double2 f = *src;
          acc[i][j].x += f.x;
          acc[i][j].y += f.y;
        }
      }
#pragma unroll
    for (int i = h; i < h + 2; i++) {
#pragma unroll
      for (int j = 0; j < 4; j++) {
        double2 *dst = at(i, j);
        if (dst) *dst = acc[i][j];
      }
      pe[i] = wq[0] * (acc[i][0].x * acc[i][2].y - acc[i][0].y * acc[i][2].x) +
              wq[1] * (acc[i][1].x * acc[i][3].y - acc[i][1].y * acc[i][3].x);
    }
  }
  if (want_pe) {
#pragma unroll
    for (int i = 0; i < 4; i++) {
      double sum = pe[i];
#pragma unroll
      for (int o = 8; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
      const int e = e0 + te + (GE / 4) * i;
      if (tc == 0 && e < p.ne)
        p.crp_part[((size_t)run * p.ne + e) * gridDim.y + blockIdx.y] = sum;
    }
  }
}

// ---- chirp-z form of the accumulation, for energies on a uniform grid ------------------
// With E_e = E_0 + e dE (E_0, dE per run) and c(k) = e^{i dE dt k^2 / 2}, the
// identity e t = (e^2 + t^2 - (e - t)^2) / 2 (Bluestein's) turns the chunk's sum
// into a convolution:
//   sum_t dt e^{i E_e (u + t) dt} x_t = F_e sum_t a_t conj(c(e - t)),
//   a_t = x_t e^{i E_0 t dt} c(t),  F_e = dt e^{i E_e u dt} c(e),  u = t0 + 1,
// taken as a cyclic convolution of length CZT_N >= FLUX_CHUNK + n_E - 1:
// (a * b)_e = IFFT(FFT(a) FFT(b))_e with b_k = conj(c(k)) at k mod CZT_N for
// -(FLUX_CHUNK - 1) <= k < n_E.  Two FP64 FFTs of 512 points per surface point
// and field instead of n_E complex products per step: about 9x fewer FLOPs for
// a full chunk.  FFTs: Stockham radix 8, three passes, one warp per sequence
// (sixteen values per lane in registers between passes).

// element m of a sequence in shared memory sits at czp(m): one padding slot
// after every 8, so that the 16-byte accesses of every pass (stride 1, 8 or 64
// elements across the lanes) fall into distinct bank groups
__device__ __forceinline__ int czp(int m) { return m + (m >> 3); }
constexpr int CZ_PADN = CZT_N + CZT_N / 8;  // padded sequence length (double2)

// twiddles of the two passes that have them, laid out [i][k] so that the
// lanes of a warp (consecutive k) read consecutive entries: twf[i 8 + k] =
// w^(8 i k) (pass 2, k < 8), twf[64 + i 64 + k] = w^(i k) (pass 3, k < 64),
// w = exp(-2 pi i / 512); built from tw[m] = w^m
constexpr int CZ_TWF = 64 + 8 * 64;
__device__ __forceinline__ void build_twf(double2 *twf, const double2 *tw, int tid, int nthr)
{
  for (int x = tid; x < CZ_TWF; x += nthr) {
    const int i = x < 64 ? x >> 3 : (x - 64) >> 6, k = x < 64 ? x & 7 : (x - 64) & 63;
    twf[x] = tw[x < 64 ? 8 * i * k : i * k];
  }
}

// x (one warp's sequence in shared memory, padded) <- its DFT with
// exp(SGN 2 pi i n m / 512); twf from build_twf
template <int SGN>
__device__ __forceinline__ void warp_fft512(double2 *x, const double2 *twf, int lane)
{
#pragma unroll
  for (int s = 0, Ns = 1; s < 3; s++, Ns *= 8) {
    double2 v[2][8];
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int j = lane + 32 * h, k = j & (Ns - 1);
#pragma unroll
      for (int i = 0; i < 8; i++) {
        double2 z = x[czp(j + 64 * i)];
        if (i && k) {                       // exp(SGN 2 pi i i k / (8 Ns))
          const double2 w = twf[Ns == 8 ? i * 8 + k : 64 + i * 64 + k];
          z = cmul(z, SGN < 0 ? w : make_double2(w.x, -w.y));
        }
        v[h][i] = z;
      }
      SmallDFT<8, double2>::run(v[h], SGN, nullptr, 0);
    }
    __syncwarp();                           // every lane has read its inputs
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int j = lane + 32 * h, k = j & (Ns - 1);
      const int base = (j - k) * 8 + k;
#pragma unroll
      for (int i = 0; i < 8; i++) x[czp(base + i * Ns)] = v[h][i];
    }
    __syncwarp();
  }
}

constexpr int CZ_Q = 8;                     // surface points per tile: one warp each
constexpr int CZ_LD = CZ_PADN + 1;          // sequence row stride (double2): rows 4 banks apart

// F_e of the chunk into phase[run][e][0]
__global__ void __launch_bounds__(256) k_czt_f(AccumParams p)
{
  const int n = p.nruns * p.ne;
  for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < n; x += gridDim.x * blockDim.x) {
    const int run = x / p.ne, e = x % p.ne;
    const double u = (double)(p.t0 + 1);
    double s1, c1, s2, c2;
    sincos(p.energies[x] * p.dt * u, &s1, &c1);
    sincos(0.5 * p.czt_de[run] * p.dt * (double)e * (double)e, &s2, &c2);
    p.phase[(size_t)x * TMAX] = make_double2(p.dt * (c1 * c2 - s1 * s2), p.dt * (s1 * c2 + c1 * s2));
  }
}

// grid (tiles, 2 fields, runs), 256 threads: tiles of CZ_Q surface points
// strided over blockIdx.x; phi[e][q] += F_e IFFT(FFT(a) B)_e
__global__ void __launch_bounds__(256, 2) k_flux_czt(AccumParams p)
{
  extern __shared__ double2 czs[];
  double2 *seq = czs;                        // [CZ_Q][CZ_LD]
  double2 *tw = seq + CZ_Q * CZ_LD;          // [CZ_TWF] pass twiddles
  double2 *bh = tw + CZ_TWF;                 // [CZT_N] this run's FFT(b) / CZT_N
  double2 *gt = bh + CZT_N;                  // [TMAX]
  double2 *fe = gt + TMAX;                   // [ne], ne <= CZT_N - TMAX + 1
  const int field = blockIdx.y, run = blockIdx.z;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  build_twf(tw, p.czt_tw, tid, 256);
  for (int x = tid; x < CZT_N; x += 256) bh[x] = p.czt_b[(size_t)run * CZT_N + x];
  for (int x = tid; x < p.nt; x += 256) gt[x] = p.czt_g[(size_t)run * TMAX + x];
  for (int x = tid; x < p.ne; x += 256) fe[x] = p.phase[((size_t)run * p.ne + x) * TMAX];
  const double2 *ring = field ? p.ring_g : p.ring_psi;
  double2 *phi = field ? p.dfai : p.fai;
  const int nqb = (p.nq + CZ_Q - 1) / CZ_Q;
  const int qi = tid & 7, tl = tid >> 3;    // loads and stores: 8 points x 32 rows
  constexpr int NR = (TMAX + 31) / 32;       // history rows per thread
  double2 nx[NR];                            // this thread's history values of the tile
  auto fetch = [&](int qb) {
    const int q = qb * CZ_Q + qi;
#pragma unroll
    for (int r = 0; r < NR; r++) {
      const int t = tl + 32 * r;
      nx[r] = (qb < nqb && t < p.nt && q < p.nq) ? ring[((size_t)t * p.nruns + run) * p.nq + q]
                                                 : make_double2(0.0, 0.0);
    }
  };
  for (int qb = blockIdx.x; qb < nqb; qb += gridDim.x) {
    const int q = qb * CZ_Q + qi;
    fetch(qb);                               // (loading the next tile's during the transforms
                                             // measured no faster, with more registers)
    __syncthreads();                         // tables in, the previous tile's outputs read
#pragma unroll
    for (int r = 0; r < NR; r++) {           // a_t
      const int t = tl + 32 * r;
      if (t < TMAX) seq[qi * CZ_LD + czp(t)] = t < p.nt ? cmul(nx[r], gt[t]) : make_double2(0.0, 0.0);
    }
    for (int t = TMAX + tl; t < CZT_N; t += 32) seq[qi * CZ_LD + czp(t)] = make_double2(0.0, 0.0);
    __syncthreads();
    double2 *x = seq + warp * CZ_LD;
    warp_fft512<-1>(x, tw, lane);
    for (int m = lane; m < CZT_N; m += 32) x[czp(m)] = cmul(x[czp(m)], bh[m]);
    __syncwarp();
    warp_fft512<+1>(x, tw, lane);
    __syncthreads();
    if (q < p.nq)
      for (int e = tl; e < p.ne; e += 32) {
        const double2 z = cmul(seq[qi * CZ_LD + czp(e)], fe[e]);
        double2 *d = phi + ((size_t)run * p.ne + e) * p.nq + q;
        double2 o = *d;
        o.x += z.x;
        o.y += z.y;
        *d = o;
      }
  }
}

size_t czt_smem() { return sizeof(double2) * ((size_t)CZ_Q * CZ_LD + CZ_TWF + CZT_N + TMAX + (CZT_N - TMAX + 1)); }

// per run: g[t] = e^{i E_0 t dt} c(t), and FFT(b) / CZT_N by one warp; block 0
// also writes the twiddle table
__global__ void __launch_bounds__(64) k_czt_tables(int ne, double dt, const double *e0,
                                                   const double *de, double2 *tw, double2 *g,
                                                   double2 *b)
{
  __shared__ double2 tws[CZT_N], twf[CZ_TWF], bs[CZ_PADN];
  const int run = blockIdx.x, tid = threadIdx.x;
  for (int m = tid; m < CZT_N; m += 64) {
    double s, c;
    sincospi((double)m / (CZT_N / 2), &s, &c);
    tws[m] = make_double2(c, -s);
    if (run == 0) tw[m] = tws[m];
  }
  const double hd = 0.5 * de[run] * dt;
  for (int t = tid; t < TMAX; t += 64) {
    double s1, c1, s2, c2;
    sincos(e0[run] * dt * (double)t, &s1, &c1);
    sincos(hd * (double)t * (double)t, &s2, &c2);
    g[(size_t)run * TMAX + t] = make_double2(c1 * c2 - s1 * s2, s1 * c2 + c1 * s2);
  }
  for (int m = tid; m < CZT_N; m += 64) {
    const int k = m < ne ? m : m - CZT_N;    // k in [-(TMAX-1), ne - 1] or unused
    double2 v = make_double2(0.0, 0.0);
    if (k < ne && k > -TMAX) {
      double s, c;
      sincos(hd * (double)k * (double)k, &s, &c);
      v = make_double2(c, -s);               // conj(c(k))
    }
    bs[czp(m)] = v;
  }
  __syncthreads();
  build_twf(twf, tws, tid, 64);
  __syncthreads();
  if (tid < 32) warp_fft512<-1>(bs, twf, tid);
  __syncthreads();
  for (int m = tid; m < CZT_N; m += 64)
    b[(size_t)run * CZT_N + m] = make_double2(bs[czp(m)].x / CZT_N, bs[czp(m)].y / CZT_N);
}

__global__ void __launch_bounds__(256) k_crp(CrpParams p)
{
  __shared__ double red[32];
  const int b = blockIdx.x;                    // run * ne + e
  const long nq = (long)p.nth * p.n1;
  const double2 *f = p.fai + (long)b * nq, *df = p.dfai + (long)b * nq;
  double s = 0.0;
  for (long q = threadIdx.x; q < nq; q += blockDim.x) {
    const int k = (int)(q / p.n1);
    const double2 a = f[q], b = df[q];
    s += p.w[k] * (a.x * b.y - a.y * b.x);   // Im(conj(phi) dphi)
  }
  s = block_sum(s, red);
  if (threadIdx.x == 0) p.crp[b] = s / p.eta_sq[b] * p.dr1_mu2;
}

// P(E) from the per-tile sums of a fused accumulation, in a fixed order
__global__ void __launch_bounds__(256) k_crp_parts(CrpParams p, const double *part, int nqt)
{
  __shared__ double red[32];
  const int b = blockIdx.x;                    // run * ne + e
  const double *pp = part + (size_t)b * nqt;
  double s = 0.0;
  for (int x = threadIdx.x; x < nqt; x += blockDim.x) s += pp[x];
  s = block_sum(s, red);
  if (threadIdx.x == 0) p.crp[b] = s / p.eta_sq[b] * p.dr1_mu2;
}

template <int GE, int KT> void launch_gemm(const AccumParams &p, cudaStream_t s)
{
  dim3 grid((p.ne + GE - 1) / GE, (p.nq + GQ - 1) / GQ, p.nruns);
  k_flux_gemm<GE, KT><<<grid, GE * 4, 0, s>>>(p);
}

}  // namespace

template <typename R>
cudaError_t launch_flux_prep(const FluxParams &p, cudaStream_t s)
{
  const int nq = p.nruns * p.nth * p.n1;
  k_flux_prep<R><<<(nq + 255) / 256, 256, 0, s>>>(p);
  return cudaGetLastError();
}
template cudaError_t launch_flux_prep<float>(const FluxParams &, cudaStream_t);
template cudaError_t launch_flux_prep<double>(const FluxParams &, cudaStream_t);

int flux_variants() { return 4; }

bool flux_accum_is_czt(const AccumParams &p)
{
  return p.czt_b && p.nt >= CZT_MIN_STEPS && p.ne <= CZT_N - TMAX + 1;
}

int flux_q_tiles(int nq) { return (nq + GQ - 1) / GQ; }

cudaError_t launch_flux_accum(const AccumParams &p, cudaStream_t s)
{
  if (p.nt <= 0) return cudaSuccess;
  if (p.nt > TMAX) return cudaErrorInvalidValue;
  if (flux_accum_is_czt(p)) {                                   // chirp-z form
    static bool attr = false;
    const size_t sm = czt_smem();
    if (!attr) {
      cudaError_t e = cudaFuncSetAttribute(k_flux_czt, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)sm);
      if (e != cudaSuccess) return e;
      attr = true;
    }
    const int nf = p.nruns * p.ne;
    k_czt_f<<<(nf + 255) / 256, 256, 0, s>>>(p);
    const int nqb = (p.nq + CZ_Q - 1) / CZ_Q;
    int gx = (148 * 8 + 2 * p.nruns - 1) / (2 * p.nruns);   // about eight CTAs per SM in all
    gx = gx < 1 ? 1 : gx > nqb ? nqb : gx;
    k_flux_czt<<<dim3(gx, 2, p.nruns), 256, sm, s>>>(p);
    return cudaGetLastError();
  }
  const int n = p.nruns * p.ne * p.nt;
  k_flux_phase<<<(n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096, 256, 0, s>>>(p);
  switch (p.variant) {   // (energies per CTA, steps per staged chunk)
    case 1: launch_gemm<64, 5>(p, s); break;
    case 2: launch_gemm<32, 10>(p, s); break;
    case 3: launch_gemm<32, 15>(p, s); break;
    default: launch_gemm<64, 10>(p, s); break;
  }
  return cudaGetLastError();
}

cudaError_t launch_crp(const CrpParams &p, cudaStream_t s)
{
  k_crp<<<p.nruns * p.ne, 256, 0, s>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_crp_parts(const CrpParams &p, const double *part, int nqt, cudaStream_t s)
{
  k_crp_parts<<<p.nruns * p.ne, 256, 0, s>>>(p, part, nqt);
  return cudaGetLastError();
}

int flux_accum_launches() { return 2; }

cudaError_t launch_czt_tables(int nruns, int ne, double dt, const double *e0, const double *de,
                              double2 *tw, double2 *g, double2 *b, cudaStream_t s)
{
  if (ne < 1 || ne > CZT_N - TMAX + 1) return cudaErrorInvalidValue;
  k_czt_tables<<<nruns, 64, 0, s>>>(ne, dt, e0, de, tw, g, b);
  return cudaGetLastError();
}
