// qd_api.cu -- C ABI of the propagator (include/qd.h): validation, device
// state, the step loop and the reference-facing entry point
// qd_time_evolution (the counterpart of TimeEvolutionMexCUDA,
// common-cuda/TimeEvolutionMexCUDA.C:20-83).
//
// One step of the reference (timeEvol.C:649-685) is issued as
//   column pass  (B, dump, flux rows, norm of step n; V, F of step n+1)
//   l-space pass (Rot/2, FFT, T, IFFT, Rot/2 of step n+1)
//   flux prep    (psi_s, d psi_s/dr of step n into the FP64 history ring)
// with the E-accumulation GEMM every QD_RING steps and P(E) at the end of a
// call.  The l-space wavepacket stays on the device between calls.
#include <cuda_runtime.h>
#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <functional>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <thread>
#include <string>
#include <tuple>
#include <vector>
#include <unistd.h>
#ifdef __SSE2__
#include <emmintrin.h>
#endif
#include "qd.h"
#include "qd_kernels.h"
#include "qd_tc.h"

namespace {

thread_local std::string g_err;
std::atomic<int64_t> g_launches{0};

int set_err(int code, const char *fmt, ...)
{
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

#define CU(x)                                                                           \
  do {                                                                                  \
    cudaError_t e_ = (x);                                                               \
    if (e_ != cudaSuccess)                                                              \
      return set_err(QD_ERR_CUDA, "%s failed: %s (%s:%d)", #x, cudaGetErrorString(e_), \
                     __FILE__, __LINE__);                                               \
  } while (0)

#define TRY(x)                  \
  do {                          \
    int rc_ = (x);              \
    if (rc_ != QD_OK) return rc_; \
  } while (0)

constexpr int QD_RING = FLUX_CHUNK;   // steps per E-accumulation chunk

bool radix_plan(int n, FftPlan &pl)
{
  pl.n = n;
  pl.nst = 0;
  int m = n;
  const int pref[] = {8, 4, 2, 3, 5};
  while (m > 1) {
    bool found = false;
    for (int r : pref) {
      if (m % r == 0) {
        if (pl.nst >= 16) return false;
        pl.rad[pl.nst++] = r;
        m /= r;
        found = true;
        break;
      }
    }
    if (!found) return false;
  }
  return true;
}

// Momentum grid by the repeated additions of get_momentum_for_fftw
// (fftwinterface.C:110-125) and p^2/(2m), 1/(2 m r^2) (MatlabStructures.C:17-36).
void radial_tables(const qd_radial &c, std::vector<double> &T, std::vector<double> &I)
{
  const int n = c.n;
  T.assign(n, 0.0);
  I.assign(n, 0.0);
  const double xl = n * c.dr;
  const double two_pi_xl = 2.0 * M_PI / xl;
  const int half = n / 2;
  double p1 = 0;
  for (int i = 0; i <= half; i++) { T[i] = p1; p1 += two_pi_xl; }
  p1 = two_pi_xl * (-half + 1);
  for (int i = half + 1; i < n; i++) { T[i] = p1; p1 += two_pi_xl; }
  for (int i = 0; i < n; i++) T[i] = T[i] * T[i] / (2 * c.mass);
  const double m2 = c.mass + c.mass;
  for (int i = 0; i < n; i++) I[i] = 1.0 / (m2 * c.r[i] * c.r[i]);
}

// Host worker threads for the input checks and the staging copies: created
// once per process (up to 16, the calling thread included) and reused, so a
// 32 MiB chunk costs no thread creation.  run(fn) calls fn(t) for every
// worker t and returns when all are done; callers take turns.  In a process
// forked after the pool was made (its workers do not exist there) the calling
// thread does every part itself.
class HostPool {
 public:
  static HostPool &get()
  {
    static HostPool *p = new HostPool();   // never destroyed: workers may outlive exit
    return *p;
  }
  unsigned size() const { return (unsigned)th_.size() + 1; }
  template <typename F> void run(const F &fn)
  {
    std::lock_guard<std::mutex> turn(run_mu_);
    if (th_.empty() || getpid() != pid_) {
      for (unsigned t = 0; t < size(); t++) fn(t);
      return;
    }
    const std::function<void(unsigned)> job = fn;
    {
      std::lock_guard<std::mutex> l(m_);
      job_ = &job;
      pending_ = th_.size();
      gen_++;
    }
    cv_.notify_all();
    fn(0);
    std::unique_lock<std::mutex> l(m_);
    done_.wait(l, [&] { return pending_ == 0; });
    job_ = nullptr;
  }

 private:
  HostPool() : pid_(getpid())
  {
    const unsigned hw = std::thread::hardware_concurrency();
    const unsigned n = std::max(1u, std::min(16u, hw ? hw : 1u));
    for (unsigned t = 1; t < n; t++) th_.emplace_back([this, t] { loop(t); });
  }
  void loop(unsigned t)
  {
    uint64_t seen = 0;
    for (;;) {
      const std::function<void(unsigned)> *f;
      {
        std::unique_lock<std::mutex> l(m_);
        cv_.wait(l, [&] { return gen_ != seen; });
        seen = gen_;
        f = job_;
      }
      (*f)(t);
      std::lock_guard<std::mutex> l(m_);
      if (--pending_ == 0) done_.notify_one();
    }
  }
  std::vector<std::thread> th_;
  pid_t pid_;
  std::mutex run_mu_, m_;
  std::condition_variable cv_, done_;
  const std::function<void(unsigned)> *job_ = nullptr;
  uint64_t gen_ = 0;
  size_t pending_ = 0;
};

// Inf and NaN are the doubles whose exponent field is all ones.  The scan
// ORs that test over the words without an early exit (so it stays a stream
// of independent loads), and splits arrays of a million or more words over
// the host pool: the check reads the whole input once per call and is bound
// by host memory bandwidth.
bool finite_words(const double *a, size_t n)
{
  constexpr uint64_t E = 0x7ff0000000000000ull;
  uint64_t b0 = 0, b1 = 0, b2 = 0, b3 = 0;
  size_t i = 0;
  for (; i + 4 <= n; i += 4) {
    uint64_t u[4];
    std::memcpy(u, a + i, sizeof u);
    b0 |= (u[0] & E) == E;
    b1 |= (u[1] & E) == E;
    b2 |= (u[2] & E) == E;
    b3 |= (u[3] & E) == E;
  }
  for (; i < n; i++) {
    uint64_t u;
    std::memcpy(&u, a + i, sizeof u);
    b0 |= (u & E) == E;
  }
  return (b0 | b1 | b2 | b3) == 0;
}

bool all_finite(const double *a, size_t n)
{
  if (n < (size_t(1) << 20)) return finite_words(a, n);
  HostPool &pool = HostPool::get();
  const unsigned nt = pool.size();
  const size_t chunk = (n + nt - 1) / nt;
  std::vector<char> ok(nt, 1);
  pool.run([&](unsigned t) {
    const size_t b = std::min(n, t * chunk), e = std::min(n, b + chunk);
    if (b < e) ok[t] = finite_words(a + b, e - b);
  });
  return std::all_of(ok.begin(), ok.end(), [](char c) { return c != 0; });
}

// Makes the handle's device current for one API call and restores the
// caller's afterwards: the handle's stream and buffers belong to that device.
struct DevGuard {
  int prev = -1;
  explicit DevGuard(int dev)
  {
    if (cudaGetDevice(&prev) != cudaSuccess) { cudaGetLastError(); prev = -1; return; }
    if (prev == dev) prev = -1;
    else if (cudaSetDevice(dev) != cudaSuccess) { cudaGetLastError(); prev = -1; }
  }
  ~DevGuard()
  {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

// Copies between the caller's (pageable) arrays and the device through
// page-locked staging buffers, allocated once per process and reused: host
// threads copy one chunk at a time into a staging buffer -- checking the
// words for NaN/Inf on the way when asked, while they are in cache -- and the
// copy engine moves each chunk as soon as it is staged, so the host copy of
// chunk c overlaps the transfer of chunk c - 1.  One transfer at a time per
// process; without page-locked memory the copies fall back to plain
// cudaMemcpyAsync from the caller's arrays.
class Staging {
 public:
  static constexpr size_t CHUNK = size_t(32) << 20;   // bytes per staging buffer
  static constexpr int NBUF = 4;
  static constexpr size_t LARGE = size_t(4) << 20;    // transfers from this size on use it

  static Staging &get()
  {
    static Staging s;
    return s;
  }
  // an upload of `bytes` goes through the staging buffers, so upload() checks
  // its words while it copies them (inputs that are not staged are checked
  // before any device work)
  bool staged(size_t bytes)
  {
    std::lock_guard<std::mutex> lock(mu_);
    return bytes >= LARGE && ready();
  }
  // One host array of doubles for upload(): copied as doubles (their words
  // checked for NaN/Inf when `check`), or rounded to floats (`narrow`: always
  // checked for NaN, Inf and values beyond the FP32 range).
  struct Up {
    void *dst;            // device
    const double *src;    // host
    size_t n;             // doubles
    bool narrow = false;
    bool check = false;
  };
  // host -> device of several arrays as one stream of whole staging buffers
  // (a buffer holds the end of one array and the start of the next), so a
  // batch of mid-size arrays moves in as few chunks as its bytes need;
  // bad[i] = array i failed its check.  The staging buffers are taken in
  // turn across calls, so the host copy of one call's first chunk overlaps
  // the transfer of the previous call's last.
  cudaError_t upload(const Up *pc, int np, cudaStream_t st, std::vector<char> &bad)
  {
    bad.assign(np, 0);
    std::lock_guard<std::mutex> lock(mu_);
    if (!ready()) {
      for (int i = 0; i < np; i++) {
        if (pc[i].narrow) return cudaErrorMemoryAllocation;
        if (pc[i].check && !all_finite(pc[i].src, pc[i].n)) bad[i] = 1;
        cudaError_t e = cudaMemcpyAsync(pc[i].dst, pc[i].src, sizeof(double) * pc[i].n,
                                        cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return e;
      }
      return cudaSuccess;
    }
    int i = 0;
    size_t done = 0;                             // doubles of array i already staged
    while (i < np) {
      const int b = (int)(next_++ % NBUF);
      cudaError_t e = cudaEventSynchronize(ev_[b]);   // the buffer's last transfer is done
      if (e != cudaSuccess) return e;
      size_t co = 0;                             // bytes of the buffer in use
      while (i < np) {
        const size_t w = pc[i].narrow ? sizeof(float) : sizeof(double);
        const size_t m = std::min(pc[i].n - done, (CHUNK - co) / w);
        if (m == 0 && done < pc[i].n) break;     // the buffer is full
        char *sb = static_cast<char *>(buf_[b]) + co;
        const bool ok = pc[i].narrow ? narrow_copy(reinterpret_cast<float *>(sb), pc[i].src + done, m)
                                     : copy_scan(sb, pc[i].src + done, m * w, pc[i].check);
        if (!ok) bad[i] = 1;
        if (m > 0) {
          e = cudaMemcpyAsync(static_cast<char *>(pc[i].dst) + done * w, sb, m * w,
                              cudaMemcpyHostToDevice, st);
          if (e != cudaSuccess) return e;
        }
        done += m;
        if (done == pc[i].n) {
          i++;
          done = 0;
        }
        co = (co + m * w + 63) & ~size_t(63);    // each part starts 64-byte aligned
        if (co >= CHUNK) break;
      }
      e = cudaEventRecord(ev_[b], st);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }
  // device -> host of one array; returns once dst holds the data
  cudaError_t download(void *dst, const void *src, size_t bytes, cudaStream_t st)
  {
    const Piece one{dst, src, bytes};
    return download(&one, 1, st);
  }
  // device -> host of several arrays as one stream of chunks (a chunk may
  // span the end of one array and the start of the next), so the transfers
  // of a batch of small arrays overlap the host copies as well
  struct Piece {
    void *dst;
    const void *src;
    size_t bytes;         // device bytes
    bool widen = false;   // src holds floats, dst receives them as doubles (2 x bytes)
  };
  cudaError_t download(const Piece *pc, int np, cudaStream_t st)
  {
    std::lock_guard<std::mutex> lock(mu_);
    size_t total = 0;
    bool widen = false;
    for (int i = 0; i < np; i++) {
      total += pc[i].bytes;
      widen = widen || pc[i].widen;
    }
    if (widen && !ready()) return cudaErrorMemoryAllocation;
    if (!widen && (!ready() || (np == 1 && total < LARGE))) {
      for (int i = 0; i < np; i++) {
        cudaError_t e = cudaMemcpyAsync(pc[i].dst, pc[i].src, pc[i].bytes, cudaMemcpyDeviceToHost,
                                        st);
        if (e != cudaSuccess) return e;
      }
      return cudaStreamSynchronize(st);
    }
    const size_t nch = (total + CHUNK - 1) / CHUNK;
    // chunk c covers bytes [c*CHUNK, ...) of the concatenation; walk the pieces
    auto each_part = [&](size_t c, auto &&fn) {
      const size_t lo = c * CHUNK, hi = std::min(total, lo + CHUNK);
      size_t base = 0;
      for (int i = 0; i < np && base < hi; base += pc[i].bytes, i++) {
        const size_t a = std::max(lo, base), z = std::min(hi, base + pc[i].bytes);
        if (a < z) fn(i, a - base, a - lo, z - a);   // piece, offset in piece, in chunk, bytes
      }
    };
    auto issue = [&](size_t c) -> cudaError_t {
      const int b = (int)(c % NBUF);
      cudaError_t e = cudaEventSynchronize(ev_[b]);
      each_part(c, [&](int i, size_t po, size_t co, size_t n) {
        if (e == cudaSuccess)
          e = cudaMemcpyAsync(static_cast<char *>(buf_[b]) + co,
                              static_cast<const char *>(pc[i].src) + po, n,
                              cudaMemcpyDeviceToHost, st);
      });
      if (e == cudaSuccess) e = cudaEventRecord(ev_[b], st);
      return e;
    };
    for (size_t c = 0; c < nch && c < (size_t)NBUF - 1; c++) {
      cudaError_t e = issue(c);
      if (e != cudaSuccess) return e;
    }
    for (size_t c = 0; c < nch; c++) {
      const int b = (int)(c % NBUF);
      cudaError_t e = cudaEventSynchronize(ev_[b]);
      if (e != cudaSuccess) return e;
      each_part(c, [&](int i, size_t po, size_t co, size_t n) {
        if (pc[i].widen)
          widen_copy(static_cast<double *>(pc[i].dst) + po / sizeof(float),
                     reinterpret_cast<const float *>(static_cast<const char *>(buf_[b]) + co),
                     n / sizeof(float));
        else
          copy_scan(static_cast<char *>(pc[i].dst) + po, static_cast<const char *>(buf_[b]) + co,
                    n, false);
      });
      if (c + NBUF - 1 < nch) {
        e = issue(c + NBUF - 1);
        if (e != cudaSuccess) return e;
      }
    }
    next_ = 0;   // every buffer's event has completed
    return cudaSuccess;
  }

 private:
  Staging() = default;
  bool ready()
  {
    if (tried_) return ok_;
    tried_ = true;
    ok_ = true;
    for (int b = 0; b < NBUF && ok_; b++)
      ok_ = cudaHostAlloc(&buf_[b], CHUNK, cudaHostAllocPortable) == cudaSuccess &&
            cudaEventCreateWithFlags(&ev_[b], cudaEventDisableTiming) == cudaSuccess;
    if (ok_)
      for (int b = 0; b < NBUF && ok_; b++) ok_ = cudaEventRecord(ev_[b], 0) == cudaSuccess;
    if (!ok_) cudaGetLastError();
    return ok_;
  }
  // memcpy over the host pool, the stores streamed past the caches where the
  // destination is 16-byte aligned (no read of the destination lines); with
  // scan, also the NaN/Inf test of the copied words, on the loaded values
  static bool copy_scan(void *dst, const void *src, size_t n, bool scan)
  {
    HostPool &pool = HostPool::get();
    const unsigned nt = pool.size();
    const size_t part = (n / nt + 63) & ~size_t(63);
    std::vector<char> ok(nt, 1);
    pool.run([&](unsigned t) {
      const size_t a = std::min(n, t * part), z = t + 1 == nt ? n : std::min(n, a + part);
      if (a >= z) return;
      char *d = static_cast<char *>(dst) + a;
      const char *s = static_cast<const char *>(src) + a;
      const size_t len = z - a;
      size_t i = 0;
      uint64_t bad = 0;
#ifdef __SSE2__
      if ((reinterpret_cast<uintptr_t>(d) & 15) == 0) {
        constexpr uint64_t E = 0x7ff0000000000000ull;
        for (; i + 64 <= len; i += 64) {
          const __m128i *p = reinterpret_cast<const __m128i *>(s + i);
          const __m128i v0 = _mm_loadu_si128(p), v1 = _mm_loadu_si128(p + 1);
          const __m128i v2 = _mm_loadu_si128(p + 2), v3 = _mm_loadu_si128(p + 3);
          __m128i *q = reinterpret_cast<__m128i *>(d + i);
          _mm_stream_si128(q, v0);
          _mm_stream_si128(q + 1, v1);
          _mm_stream_si128(q + 2, v2);
          _mm_stream_si128(q + 3, v3);
          if (scan) {
            uint64_t u[8];
            std::memcpy(u, s + i, sizeof u);
            for (int k = 0; k < 8; k++) bad |= (u[k] & E) == E;
          }
        }
        _mm_sfence();
      }
#endif
      std::memcpy(d + i, s + i, len - i);
      if (scan)
        ok[t] = bad == 0 && finite_words(reinterpret_cast<const double *>(d + i), (len - i) / 8);
    });
    return std::all_of(ok.begin(), ok.end(), [](char c) { return c != 0; });
  }
  // dst[i] = (float)src[i] over the host pool; false if some src[i] is NaN,
  // Inf or beyond the FP32 range
  static bool narrow_copy(float *dst, const double *src, size_t n)
  {
    HostPool &pool = HostPool::get();
    const unsigned nt = pool.size();
    const size_t part = (n / nt + 15) & ~size_t(15);
    std::vector<char> ok(nt, 1);
    pool.run([&](unsigned t) {
      const size_t a = std::min(n, t * part), z = t + 1 == nt ? n : std::min(n, a + part);
      // |v| above FLT_MAX, Inf and NaN are the magnitudes above FLT_MAX's bits
      constexpr uint64_t MAGN = 0x7fffffffffffffffull, FMAX = 0x47efffffe0000000ull;
      uint64_t bad = 0;
      size_t i = a;
#ifdef __SSE2__
      // four values a round, streamed past the caches into the staging buffer
      // (dst + a is 16-byte aligned: a is a multiple of 16 and dst a page-locked buffer)
      for (; i + 4 <= z; i += 4) {
        const __m128d v0 = _mm_loadu_pd(src + i), v1 = _mm_loadu_pd(src + i + 2);
        _mm_stream_ps(dst + i, _mm_movelh_ps(_mm_cvtpd_ps(v0), _mm_cvtpd_ps(v1)));
        uint64_t u[4];
        std::memcpy(u, src + i, sizeof u);
        bad |= ((u[0] & MAGN) > FMAX) | ((u[1] & MAGN) > FMAX) | ((u[2] & MAGN) > FMAX) |
               ((u[3] & MAGN) > FMAX);
      }
      _mm_sfence();
#endif
      for (; i < z; i++) {
        uint64_t u;
        std::memcpy(&u, src + i, sizeof u);
        bad |= (u & MAGN) > FMAX;
        dst[i] = (float)src[i];
      }
      ok[t] = bad == 0;
    });
    return std::all_of(ok.begin(), ok.end(), [](char c) { return c != 0; });
  }
  // dst[i] = src[i] widened to double, over the host pool
  static void widen_copy(double *dst, const float *src, size_t n)
  {
    HostPool &pool = HostPool::get();
    const unsigned nt = pool.size();
    const size_t part = (n / nt + 15) & ~size_t(15);
    pool.run([&](unsigned t) {
      const size_t a = std::min(n, t * part), z = t + 1 == nt ? n : std::min(n, a + part);
      size_t i = a;
#ifdef __SSE2__
      // two values a round, streamed to the caller's array when it is 16-byte aligned
      if ((reinterpret_cast<uintptr_t>(dst + a) & 15) == 0) {
        for (; i + 2 <= z; i += 2) {
          const __m128 f = _mm_castsi128_ps(_mm_loadl_epi64(reinterpret_cast<const __m128i *>(src + i)));
          _mm_stream_pd(dst + i, _mm_cvtps_pd(f));
        }
        _mm_sfence();
      }
#endif
      for (; i < z; i++) dst[i] = (double)src[i];
    });
  }
  std::mutex mu_;
  bool tried_ = false, ok_ = false;
  void *buf_[NBUF] = {};
  cudaEvent_t ev_[NBUF] = {};
  size_t next_ = 0;               // the upload's next staging buffer (round robin)
};

}  // namespace

// error reporting for the other translation units of the library (qd_err.h)
int qd_set_error(int code, const char *msg)
{
  g_err = msg;
  return code;
}
void qd_count_launches(int n) { g_launches += n; }

struct qd_handle {
  int dev = 0;                    // the device current at creation: its stream and buffers
  bool failed = false;            // a propagation stopped on a corrupted state
  qd_data *data = nullptr;        // run 0 (holds the fields shared by the batch)
  std::vector<qd_data *> runs;    // all runs of the batch
  int nruns = 1;
  long vrun = 0;                  // per-run stride of the potential tables (0 = shared)
  int prec = QD_PREC_FP64;
  int n1 = 0, n2 = 0, nth = 0, nl = 0;      // nl: angular functions of the layout (max over runs)
  long n12 = 0;
  // angular bases: runs with equal theta.legendre share a set; a
  // centrifugal-sudden run has j = K + l
  int nsets = 1, jrows = 0;
  std::vector<int> run_set, run_k, run_nl;
  int *d_run_set = nullptr, *d_run_k = nullptr, *d_run_nl = nullptr, *d_run_order = nullptr;
  int npts = 0, h = 0, surf_j0 = 0, ne = 0;
  bool do_crp = false, have_dump = false;
  double dt = 0;
  cudaStream_t st = nullptr;
  std::vector<void *> allocs;

  double *d_pot = nullptr, *d_w = nullptr, *d_leg = nullptr, *d_P = nullptr, *d_WP = nullptr;
  float *d_P32 = nullptr, *d_WP32 = nullptr, *d_P32lo = nullptr, *d_WP32lo = nullptr;
  double *d_I1 = nullptr, *d_I2 = nullptr, *d_T1 = nullptr, *d_T2 = nullptr;
  double *d_d1 = nullptr, *d_d2 = nullptr;
  double2 *d_expV = nullptr, *d_rot = nullptr, *d_kin = nullptr;
  float2 *d_expV32 = nullptr;
  float2 *d_rc1 = nullptr, *d_rc2 = nullptr, *d_kc1 = nullptr, *d_kc2 = nullptr;
  int slice_cluster = 0;          // l-space kernel (LineParams::cluster code)
  int flux_variant = 0;           // flux-accumulation GEMM tile variant (tune_flux)
  bool psi_z_valid = false;       // d_psi_z holds the theta-space state of every run
  bool crp_valid = false;         // d_crp holds P(E) of the accumulated flux
  double2 *d_tw1_64 = nullptr, *d_tw2_64 = nullptr;
  float2 *d_tw1_32 = nullptr, *d_tw2_32 = nullptr;
  void *d_lpsi = nullptr;
  double2 *d_psi_z = nullptr;
  // complex64 handles: the theta-space state crosses the bus in complex64 (the
  // precision it is propagated in), through this buffer
  float2 *d_psi32 = nullptr;
  void *d_surf = nullptr;
  double2 *d_ring_psi = nullptr, *d_ring_g = nullptr, *d_fai = nullptr, *d_dfai = nullptr;
  double2 *d_phase = nullptr;     // chunk phase factors [run][E][FLUX_CHUNK]
  // chirp-z form of the accumulation (every run's energies on a uniform grid)
  double2 *d_czt_tw = nullptr, *d_czt_g = nullptr, *d_czt_b = nullptr;
  double *d_czt_de = nullptr;
  double *d_energies = nullptr, *d_eta = nullptr, *d_crp = nullptr;
  double *d_crp_part = nullptr;   // [run][energy][surface-point tile]: fused P(E) sums
                                  // (null: P(E) by its own pass, QD_CRP_FUSED=0)
  double *d_norms = nullptr;
  int norms_cap = 0;
  TcPlan tc;                      // tensor-core column pass (FP32), if usable
  bool use_tc = false;
  // energies inside the propagation (qd_set_energy_interval)
  int energy_every = 0;
  double *d_esum = nullptr;       // [slot][run][3] sums of the current call
  int esum_cap = 0;
  double *esum_col = nullptr;     // slot of the next column / l-space launch (null: none)
  double *esum_lines = nullptr;
  bool lines_split = false;       // this step's l-space pass on the split kernels
  std::vector<double> energy_log; // records: step, run, E_kin, E_rot, E_pot
  double2 *d_escratch = nullptr;  // on-demand energies: DFT scratch and sums
  double *d_esums3 = nullptr;

  FftPlan pl1, pl2;
  int ring_fill = 0;
  int flux_pending = -1;          // ring slot whose preparation is not yet issued
  long acc_done = 0;
  bool started = false;           // l-space state valid on the device
  bool last_finalized = true;     // flux/norm of the last step already taken
  int32_t steps = 0;
  std::vector<double> norms_host;
  bool norm_guard = true;         // every run has n_l <= n_theta: a step cannot raise the norm
  bool profiling = false;
  std::vector<double> kernel_ms;
  void *d_flush = nullptr;        // L2 flush buffer of qd_propagate_timed
  size_t flush_bytes = 0;
  std::vector<cudaEvent_t> events;
  std::vector<cudaEvent_t> prof_pool;
  std::vector<int> prof_cls;
  size_t prof_used = 0;

  // device buffers come from the device's stream-ordered memory pool, which
  // keeps freed memory (release threshold raised once per process), so that
  // creating a handle after an earlier one was destroyed reuses its memory
  // instead of paying cudaMalloc / cudaFree again
  template <typename T> int alloc(T *&p, size_t count)
  {
    void *q = nullptr;
    const size_t bytes = count * sizeof(T) > 0 ? count * sizeof(T) : 16;
    keep_pool();
    cudaError_t e = cudaMallocAsync(&q, bytes, st);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return set_err(QD_ERR_NOMEM, "cudaMallocAsync(%zu bytes) failed: %s", bytes,
                     cudaGetErrorString(e));
    }
    allocs.push_back(q);
    p = reinterpret_cast<T *>(q);
    // pooled memory holds whatever its last user left: every buffer starts
    // zeroed (unused orders of ragged runs, flux rows and rings rely on it)
    e = cudaMemsetAsync(q, 0, bytes, st);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return set_err(QD_ERR_CUDA, "cudaMemsetAsync failed: %s", cudaGetErrorString(e));
    }
    return QD_OK;
  }
  static bool keep_pool()
  {
    static const bool ok = [] {
      int dev = 0;
      cudaMemPool_t pool;
      if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetDefaultMemPool(&pool, dev) != cudaSuccess)
        return false;
      uint64_t keep = ~0ull;
      return cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep) == cudaSuccess;
    }();
    return ok;
  }
  ~qd_handle()
  {
    if (st) cudaStreamSynchronize(st);
    for (void *p : allocs) cudaFreeAsync(p, st);
    if (d_norms) cudaFreeAsync(d_norms, st);
    if (d_esum) cudaFreeAsync(d_esum, st);
    if (d_flush) cudaFreeAsync(d_flush, st);
    tc_plan_destroy(tc, st);
    if (st) cudaStreamSynchronize(st);
    for (cudaEvent_t e : events) cudaEventDestroy(e);
    for (cudaEvent_t e : prof_pool) cudaEventDestroy(e);
    if (st) cudaStreamDestroy(st);
  }
};

namespace {

int validate(const qd_data *d)
{
  if (!d) return set_err(QD_ERR_INVALID, "data is NULL");
  const int n1 = d->r1.n, n2 = d->r2.n, nth = d->theta.n, m = d->theta.m;
  if (n1 < 2 || n2 < 2 || n1 % 2 || n2 % 2)
    return set_err(QD_ERR_INVALID, "r1.n (%d) and r2.n (%d) must be even and >= 2 "
                   "(get_momentum_for_fftw requires even n)", n1, n2);
  if (nth < 1 || m < 0) return set_err(QD_ERR_INVALID, "theta.n = %d, theta.m = %d", nth, m);
  if (!d->r1.r || !d->r2.r || !d->theta.x || !d->theta.w || !d->theta.legendre || !d->pot ||
      !d->psi)
    return set_err(QD_ERR_INVALID, "a required array (r, theta.x/w/legendre, pot, psi) is NULL");
  if (!(d->r1.dr > 0) || !(d->r2.dr > 0) || !(d->r1.mass > 0) || !(d->r2.mass > 0))
    return set_err(QD_ERR_INVALID, "dr and mass must be positive");
  if (!std::isfinite(d->time.time_step) || d->time.total_steps < 0 || d->time.steps < 0)
    return set_err(QD_ERR_INVALID, "bad time struct");
  for (int i = 0; i < n1; i++)
    if (d->r1.r[i] == 0.0) return set_err(QD_ERR_INVALID, "r1.r contains 0");
  for (int i = 0; i < n2; i++)
    if (d->r2.r[i] == 0.0) return set_err(QD_ERR_INVALID, "r2.r contains 0");
  FftPlan pl;
  if (!radix_plan(n1, pl) || !radix_plan(n2, pl))
    return set_err(QD_ERR_UNSUPPORTED, "r1.n = %d, r2.n = %d: FFT sizes must be 2^a 3^b 5^c",
                   n1, n2);
  if (d->options.precision != QD_PREC_FP64 && d->options.precision != QD_PREC_FP32)
    return set_err(QD_ERR_INVALID, "options.precision = %d", d->options.precision);
  if (d->cs.K < 0 || d->cs.J < d->cs.K)
    return set_err(QD_ERR_INVALID, "centrifugal-sudden block J = %d, K = %d: need 0 <= K <= J",
                   d->cs.J, d->cs.K);
  const size_t npt = (size_t)n1 * n2 * nth;
  // arrays that the upload stages are checked while they are copied into the
  // staging buffers (create), the others here; so every input word is read once
  // for the check, and a process without a device checks them all here
  if (!Staging::get().staged(npt * sizeof(double)) && !all_finite(d->pot, npt))
    return set_err(QD_ERR_NONFINITE, "pot contains NaN/Inf");
  if (!Staging::get().staged(2 * npt * sizeof(double)) && !all_finite(d->psi, 2 * npt))
    return set_err(QD_ERR_NONFINITE, "psi contains NaN/Inf");
  if (d->CRP.calculate_CRP) {
    const qd_crp &c = d->CRP;
    if (c.n_energies < 1 || !c.energies || !c.eta_sq || !c.CRP)
      return set_err(QD_ERR_INVALID, "CRP: n_energies/energies/eta_sq/CRP");
    const int np = c.n_gradient_points;
    if (np != 3 && np != 5 && np != 7 && np != 9 && np != 11)
      return set_err(QD_ERR_INVALID, "NPoints error: n_gradient_points = %d (3,5,7,9,11)", np);
    const int hh = (np - 1) / 2, j = c.n_dividing_surface - 1;
    if (j - hh < 0 || j + hh > n2 - 1)
      return set_err(QD_ERR_INVALID,
                     "dividing surface %d with %d points reaches outside r2 (1..%d)",
                     c.n_dividing_surface, np, n2);
  }
  return QD_OK;
}

// Kernel-class profiling (qd_set_profiling): an event after each launch
// group; the span since the previous event is charged to that group.
enum { PROF_COLUMN = 0, PROF_LINES = 1, PROF_FLUX = 2, PROF_ACCUM = 3, PROF_CRP = 4, PROF_N = 5 };

int prof_mark(qd_handle *h, int cls)
{
  if (!h->profiling) return QD_OK;
  if (h->prof_used == h->prof_pool.size()) {
    cudaEvent_t e;
    CU(cudaEventCreate(&e));
    h->prof_pool.push_back(e);
  }
  cudaEvent_t e = h->prof_pool[h->prof_used++];
  CU(cudaEventRecord(e, h->st));
  h->prof_cls.push_back(cls);
  return QD_OK;
}

// After a stream sync: fold the recorded spans into per-class averages.
int prof_collect(qd_handle *h)
{
  if (!h->profiling) return QD_OK;
  double tot[PROF_N] = {0};
  int cnt[PROF_N] = {0};
  for (size_t i = 1; i < h->prof_used; i++) {
    const int c = h->prof_cls[i];
    if (c < 0) continue;
    float ms = 0.f;
    CU(cudaEventElapsedTime(&ms, h->prof_pool[i - 1], h->prof_pool[i]));
    tot[c] += ms;
    cnt[c]++;
  }
  h->kernel_ms.assign(2 * PROF_N, 0.0);
  for (int c = 0; c < PROF_N; c++) {
    h->kernel_ms[c] = cnt[c] ? tot[c] / cnt[c] : 0.0;
    h->kernel_ms[PROF_N + c] = cnt[c];
  }
  h->prof_used = 0;
  h->prof_cls.clear();
  return QD_OK;
}

FluxParams flux_params(qd_handle *h)
{
  FluxParams f{};
  f.n1 = h->n1; f.nth = h->nth; f.npts = h->npts; f.h = h->h; f.surf = h->d_surf;
  f.nruns = h->nruns;
  static const int den[] = {0, 2, 12, 60, 840, 2520};
  f.den_dx = den[h->h] * h->data->r2.dr;
  f.ring_psi = h->d_ring_psi; f.ring_g = h->d_ring_g; f.slot = h->flux_pending;
  return f;
}
int after_flux_prep(qd_handle *h);
template <typename R> int issue_flux_prep(qd_handle *h);

// Device-side status word of the tensor-core pass (bounded waits that ran
// out; the l-space kernels wait only on hardware cluster barriers).
int check_status(qd_handle *h)
{
  int st = 0;
  if (h->use_tc) {
    CU(cudaMemcpy(&st, tc_status_ptr(h->tc), sizeof(int), cudaMemcpyDeviceToHost));
    if (st) return set_err(QD_ERR_DEVICE, "tensor-core column pass: an MMA completion wait "
                           "timed out (status %d)", st);
  }
  return QD_OK;
}

ColumnParams column_params(qd_handle *h)
{
  ColumnParams p{};
  p.n1 = h->n1; p.n2 = h->n2; p.nth = h->nth; p.nl = h->nl; p.n12 = h->n12;
  p.nruns = h->nruns; p.vrun = h->vrun;
  p.lpsi = h->d_lpsi; p.psi_z = h->d_psi_z;
  p.P = h->d_P; p.WP = h->d_WP; p.P32 = h->d_P32; p.WP32 = h->d_WP32;
  p.P32lo = h->d_P32lo; p.WP32lo = h->d_WP32lo;
  p.expV = h->d_expV; p.expV32 = h->d_expV32; p.pot = h->d_pot; p.dt = h->dt;
  p.d1 = h->have_dump ? h->d_d1 : nullptr;
  p.d2 = h->have_dump ? h->d_d2 : nullptr;
  p.surf = h->d_surf; p.surf_j0 = h->surf_j0; p.surf_nrows = 2 * h->h + 1;
  p.w = h->d_w;
  p.run_set = h->d_run_set; p.set_stride = (long)h->nth * h->nl; p.run_nl = h->d_run_nl;
  p.run_order = h->d_run_order;
  return p;
}

template <typename R> int issue_column(qd_handle *h, int mode, bool flux, double *norm_out,
                                       bool out_z)
{
  ColumnParams p = column_params(h);
  p.prestep = (mode == COL_HEAD && h->steps == 0);
  p.do_flux = flux ? 1 : 0;
  p.norm_out = norm_out;
  p.out_z = out_z ? 1 : 0;
  p.esum = mode == COL_HEAD ? nullptr : h->esum_col;
  cudaError_t e;
  TRY(prof_mark(h, -1));
  if (sizeof(R) == 4 && h->use_tc) e = launch_column_tc(h->tc, p, mode, h->st);
  else e = launch_column<R>(p, mode, h->st);
  g_launches++;
  CU(e);
  TRY(prof_mark(h, PROF_COLUMN));
  if (flux) {
    // the surface rows of this step go to ring slot ring_fill; with the fused
    // slice kernel that preparation rides along in the next l-space launch
    h->flux_pending = h->ring_fill;
    if (!(sizeof(R) == 4 && h->slice_cluster > 0 && !h->lines_split) || mode == COL_TAIL)
      TRY(issue_flux_prep<R>(h));
  }
  return QD_OK;
}

AccumParams accum_params(const qd_handle *h)
{
  AccumParams a{};
  a.nq = h->nth * h->n1; a.ne = h->ne; a.nt = h->ring_fill; a.t0 = h->acc_done;
  a.nruns = h->nruns;
  a.dt = h->dt; a.energies = h->d_energies; a.ring_psi = h->d_ring_psi;
  a.ring_g = h->d_ring_g; a.fai = h->d_fai; a.dfai = h->d_dfai;
  a.phase = h->d_phase;
  a.variant = h->flux_variant;
  a.czt_tw = h->d_czt_tw; a.czt_g = h->d_czt_g; a.czt_b = h->d_czt_b; a.czt_de = h->d_czt_de;
  return a;
}

// ring bookkeeping after the flux preparation of a step has been issued
int after_flux_prep(qd_handle *h)
{
  h->flux_pending = -1;
  h->ring_fill++;
  if (h->ring_fill == QD_RING) {
    const AccumParams a = accum_params(h);
    TRY(prof_mark(h, -1));
    CU(launch_flux_accum(a, h->st));
    g_launches += flux_accum_launches();
    TRY(prof_mark(h, PROF_ACCUM));
    h->acc_done += h->ring_fill;
    h->ring_fill = 0;
  }
  return QD_OK;
}

template <typename R> int issue_flux_prep(qd_handle *h)
{
  TRY(prof_mark(h, -1));
  CU(launch_flux_prep<R>(flux_params(h), h->st));
  g_launches++;
  TRY(prof_mark(h, PROF_FLUX));
  return after_flux_prep(h);
}

LineParams line_params(qd_handle *h, bool f32)
{
  LineParams p{};
  p.n1 = h->n1; p.n2 = h->n2; p.nl = h->nl; p.n12 = h->n12; p.lpsi = h->d_lpsi;
  p.nruns = h->nruns;
  p.rot = h->d_rot; p.kin = h->d_kin;
  p.rc1 = h->d_rc1; p.rc2 = h->d_rc2; p.kc1 = h->d_kc1; p.kc2 = h->d_kc2;
  p.cluster = f32 ? h->slice_cluster : 0;
  const double ks = 1.0 / ((double)h->n1 * h->n2);
  p.kscale = (float)ks;
  p.kscale_lo = (float)(ks - (double)p.kscale);
  if (!f32) { p.tw1 = h->d_tw1_64; p.tw2 = h->d_tw2_64; }
  else { p.tw1 = h->d_tw1_32; p.tw2 = h->d_tw2_32; }
  p.pl1 = h->pl1; p.pl2 = h->pl2;
  p.run_k = h->d_run_k; p.jrows = h->jrows;
  p.T1 = h->d_T1; p.T2 = h->d_T2; p.I1 = h->d_I1; p.I2 = h->d_I2;
  p.orth = h->prec == QD_PREC_FP32 && h->use_tc ? 1 : 0;
  return p;
}

// Autotuner of the complex64 l-space pass: time the fused slice kernel with
// 1, 2 and 4 CTAs per slice, the register-FFT slice kernel on 1, 2 or 4
// CTAs per slice (where built) and the split kernels on a scratch wavepacket and keep the
// fastest; the choice is kept for later handles of the same shapes.
// QD_SLICE_CLUSTER=0|1|2|4|8|9|10|11 forces a choice (8 = the register-FFT
// kernel, 9 and 10 = the same on a 2- and a 4-CTA cluster).
int tune_slice(qd_handle *h)
{
  h->slice_cluster = 0;
  if (h->prec != QD_PREC_FP32) return QD_OK;
  const char *force = getenv("QD_SLICE_CLUSTER");
  if (force) {
    const int cl = atoi(force);
    h->slice_cluster = slice_cluster_ok(h->n1, h->n2, cl) ? cl : 0;
    return QD_OK;
  }
  // the choice depends on the shapes only: measured once per process and device
  static std::mutex mu;
  static std::map<std::tuple<int, int, int, int, int, int, int>, int> chosen;
  int dev = 0;
  cudaGetDevice(&dev);
  const auto key = std::make_tuple(dev, h->n1, h->n2, h->nl, h->nruns, h->jrows,
                                   h->d_run_k ? 1 : 0);
  {
    std::lock_guard<std::mutex> lock(mu);
    auto it = chosen.find(key);
    if (it != chosen.end()) {
      h->slice_cluster = it->second;
      return QD_OK;
    }
  }
  void *scratch = nullptr;
  const size_t sbytes = sizeof(float2) * h->n12 * h->nl * h->nruns;
  CU(cudaMallocAsync(&scratch, sbytes, h->st));
  CU(cudaMemsetAsync(scratch, 0, sbytes, h->st));
  cudaEvent_t e0, e1;
  CU(cudaEventCreate(&e0));
  CU(cudaEventCreate(&e1));
  LineParams p = line_params(h, true);
  p.lpsi = scratch;
  float best = 1e30f;
  for (int cl : {0, 1, 2, 4, SLICE_RF, SLICE_RF2, SLICE_RF4, SLICE_RF4W}) {
    if (cl > 0 && !slice_cluster_ok(h->n1, h->n2, cl)) continue;
    p.cluster = cl;
    bool ok = true;
    for (int it = 0; it < 2 && ok; it++)
      ok = (cl ? launch_slice(p, h->st) : launch_lines<float>(p, h->st)) == cudaSuccess;
    if (ok) ok = cudaEventRecord(e0, h->st) == cudaSuccess;
    for (int it = 0; it < 5 && ok; it++)
      ok = (cl ? launch_slice(p, h->st) : launch_lines<float>(p, h->st)) == cudaSuccess;
    if (ok) ok = cudaEventRecord(e1, h->st) == cudaSuccess;
    if (ok) ok = cudaStreamSynchronize(h->st) == cudaSuccess;
    float ms = 0.f;
    if (ok) ok = cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess;
    if (!ok) {                      // e.g. a cluster shape that cannot be scheduled
      cudaGetLastError();
      continue;
    }
    if (ms < best) { best = ms; h->slice_cluster = cl; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  CU(cudaFreeAsync(scratch, h->st));
  std::lock_guard<std::mutex> lock(mu);
  chosen[key] = h->slice_cluster;
  return QD_OK;
}

// Times `launch` (reps launches after one warm-up) on the handle's stream, ms
// per launch; a negative value if a launch failed.
template <typename F> float time_launches(qd_handle *h, F launch, int reps = 3)
{
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  float ms = -1.f;
  bool ok = cudaEventCreate(&e0) == cudaSuccess && cudaEventCreate(&e1) == cudaSuccess;
  ok = ok && launch() == cudaSuccess && cudaEventRecord(e0, h->st) == cudaSuccess;
  for (int i = 0; i < reps && ok; i++) ok = launch() == cudaSuccess;
  ok = ok && cudaEventRecord(e1, h->st) == cudaSuccess &&
       cudaStreamSynchronize(h->st) == cudaSuccess &&
       cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    ms = -1.f;
  } else {
    ms /= reps;
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  return ms;
}

// Autotuner of the flux-accumulation GEMM: each tile variant accumulates one
// full chunk of (still zero) history into the handle's phi_E, which is
// cleared again afterwards; the fastest is kept per shape for the process.
// QD_FLUX_VARIANT=0..3 forces a variant.
int tune_flux(qd_handle *h)
{
  h->flux_variant = 0;
  if (!h->do_crp) return QD_OK;
  if (const char *force = getenv("QD_FLUX_VARIANT")) {
    const int v = atoi(force);
    h->flux_variant = v >= 0 && v < flux_variants() ? v : 0;
    return QD_OK;
  }
  static std::mutex mu;
  static std::map<std::tuple<int, int, int, int, int>, int> chosen;
  int dev = 0;
  cudaGetDevice(&dev);
  const auto key = std::make_tuple(dev, h->n1, h->nth, h->ne, h->nruns);
  {
    std::lock_guard<std::mutex> lock(mu);
    auto it = chosen.find(key);
    if (it != chosen.end()) {
      h->flux_variant = it->second;
      return QD_OK;
    }
  }
  AccumParams a = accum_params(h);
  a.nt = QD_RING;
  a.t0 = 0;
  a.czt_b = nullptr;      // the GEMM form (with the chirp-z tables: chunks below CZT_MIN_STEPS)
  float best = 1e30f;
  for (int v = 0; v < flux_variants(); v++) {
    a.variant = v;
    const float ms = time_launches(h, [&] { return launch_flux_accum(a, h->st); });
    if (ms >= 0.f && ms < best) { best = ms; h->flux_variant = v; }
  }
  const size_t bytes = sizeof(double2) * (size_t)h->nth * h->n1 * h->ne * h->nruns;
  CU(cudaMemsetAsync(h->d_fai, 0, bytes, h->st));
  CU(cudaMemsetAsync(h->d_dfai, 0, bytes, h->st));
  std::lock_guard<std::mutex> lock(mu);
  chosen[key] = h->flux_variant;
  return QD_OK;
}

// Autotuner of the complex64 column pass: the tensor-core kernel against the
// SIMT one, both on the handle's zero l-space buffer (a zero wavepacket stays
// zero); the faster is kept per shape for the process.  QD_COLUMN_PATH forces
// the choice.
int tune_column(qd_handle *h)
{
  if (h->prec != QD_PREC_FP32 || !h->use_tc || getenv("QD_COLUMN_PATH")) return QD_OK;
  static std::mutex mu;
  static std::map<std::tuple<int, int, int, int, int, int, int>, bool> chosen;
  int dev = 0;
  cudaGetDevice(&dev);
  const auto key = std::make_tuple(dev, h->n1, h->n2, h->nth, h->nl, h->nruns, h->nsets);
  {
    std::lock_guard<std::mutex> lock(mu);
    auto it = chosen.find(key);
    if (it != chosen.end()) {
      h->use_tc = it->second;
      return QD_OK;
    }
  }
  ColumnParams p = column_params(h);
  const float tc = time_launches(h, [&] { return launch_column_tc(h->tc, p, COL_MID, h->st); });
  const float simt = time_launches(h, [&] { return launch_column<float>(p, COL_MID, h->st); });
  CU(cudaMemsetAsync(h->d_lpsi, 0, sizeof(float2) * h->n12 * h->nl * h->nruns, h->st));
  if (tc < 0.f) return set_err(QD_ERR_CUDA, "tensor-core column pass failed while tuning");
  h->use_tc = !(simt >= 0.f && simt < tc);
  std::lock_guard<std::mutex> lock(mu);
  chosen[key] = h->use_tc;
  return QD_OK;
}

template <typename R> int issue_lines(qd_handle *h)
{
  LineParams p = line_params(h, sizeof(R) == 4);
  p.esum = h->esum_lines;
  if (h->lines_split) p.cluster = 0;            // energy step on a kernel without the sums
  const bool fused_flux = p.cluster > 0 && h->flux_pending >= 0;
  if (fused_flux) {
    p.flux = flux_params(h);
    const int nq = h->nth * h->n1 * h->nruns;
    const int nt = slice_threads(h->n1, h->n2, p.cluster);
    const int ctas = (nq + nt - 1) / nt;
    const int cl = slice_ctas(p.cluster);                   // whole clusters
    p.flux_ctas = (ctas + cl - 1) / cl * cl;
  }
  TRY(prof_mark(h, -1));
  if (p.cluster > 0) {
    CU(launch_slice(p, h->st));
    g_launches++;
  } else {
    CU(launch_lines<R>(p, h->st));
    g_launches += lines_launches_per_step(h->n1, h->n2, h->prec);
  }
  TRY(prof_mark(h, PROF_LINES));
  if (fused_flux) TRY(after_flux_prep(h));
  return QD_OK;
}

int flush_accum(qd_handle *h)
{
  if (h->ring_fill == 0) return QD_OK;
  const AccumParams a = accum_params(h);
  CU(launch_flux_accum(a, h->st));
  g_launches += flux_accum_launches();
  h->acc_done += h->ring_fill;
  h->ring_fill = 0;
  return QD_OK;
}

int compute_crp(qd_handle *h)
{
  if (!h->do_crp || h->crp_valid) return QD_OK;
  // a pending partial chunk that the GEMM form accumulates also yields P(E):
  // its epilogue sums w_k Im(conj(phi) dphi) of the values it writes per tile,
  // which saves reading phi_E and dphi_E once more
  bool fused = false;
  if (h->ring_fill > 0 && h->d_crp_part) {
    AccumParams a = accum_params(h);
    if (!flux_accum_is_czt(a)) {
      a.crp_part = h->d_crp_part; a.w = h->d_w; a.n1 = h->n1;
      CU(launch_flux_accum(a, h->st));
      g_launches += flux_accum_launches();
      h->acc_done += h->ring_fill;
      h->ring_fill = 0;
      fused = true;
    }
  }
  if (!fused) TRY(flush_accum(h));
  CrpParams c{};
  c.n1 = h->n1; c.nth = h->nth; c.ne = h->ne; c.w = h->d_w; c.eta_sq = h->d_eta;
  c.nruns = h->nruns;
  c.dr1_mu2 = h->data->r1.dr / h->data->r2.mass;
  c.fai = h->d_fai; c.dfai = h->d_dfai; c.crp = h->d_crp;
  TRY(prof_mark(h, -1));
  if (fused) CU(launch_crp_parts(c, h->d_crp_part, flux_q_tiles(h->nth * h->n1), h->st));
  else CU(launch_crp(c, h->st));
  g_launches++;
  TRY(prof_mark(h, PROF_CRP));
  h->crp_valid = true;
  return QD_OK;
}

template <typename Real> int propagate(qd_handle *h, int n, size_t flush_bytes = 0,
                                   double *device_ms = nullptr)
{
  if (n <= 0) {
    if (device_ms) *device_ms = 0.0;
    return QD_OK;
  }
  const bool timed = device_ms != nullptr;
  h->psi_z_valid = false;
  h->crp_valid = false;
  if (timed) {
    while (h->events.size() < (size_t)(2 * n + 2)) {
      cudaEvent_t e;
      CU(cudaEventCreate(&e));
      h->events.push_back(e);
    }
    if (flush_bytes > h->flush_bytes) {
      if (h->d_flush) cudaFreeAsync(h->d_flush, h->st);
      h->d_flush = nullptr;
      CU(cudaMallocAsync(&h->d_flush, flush_bytes, h->st));
      h->flush_bytes = flush_bytes;
    }
  }
  const int R = h->nruns;                         // norms: [step][run]
  if (h->norms_cap < n * R) {
    if (h->d_norms) cudaFreeAsync(h->d_norms, h->st);
    h->d_norms = nullptr;
    CU(cudaMallocAsync(&h->d_norms, sizeof(double) * n * R, h->st));
    h->norms_cap = n * R;
  }
  CU(cudaMemsetAsync(h->d_norms, 0, sizeof(double) * n * R, h->st));
  // energy steps of this call: t in (steps0, steps0 + n] with t % every == 0.
  // Step t's kinetic and rotational sums come from its l-space launch, its
  // potential sum from the next column launch (B of step t), all into slot
  // t / every - steps0 / every - 1 of d_esum.
  const int every = h->energy_every, steps0 = h->steps;
  const int nslots = every > 0 ? (steps0 + n) / every - steps0 / every : 0;
  if (nslots > 0) {
    if (h->esum_cap < nslots * R * 3) {
      if (h->d_esum) cudaFreeAsync(h->d_esum, h->st);
      h->d_esum = nullptr;
      CU(cudaMallocAsync(&h->d_esum, sizeof(double) * nslots * R * 3, h->st));
      h->esum_cap = nslots * R * 3;
    }
    CU(cudaMemsetAsync(h->d_esum, 0, sizeof(double) * nslots * R * 3, h->st));
  }
  auto slot = [&](int t) -> double * {
    if (every <= 0 || t <= steps0 || t > steps0 + n || t % every) return nullptr;
    return h->d_esum + (long)(t / every - steps0 / every - 1) * R * 3;
  };
  const bool split_ok = h->prec == QD_PREC_FP64 || h->slice_cluster == 0 ||
                        slice_is_rf(h->slice_cluster);
  for (int s = 0; s < n; s++) {
    const bool redo = !h->started || (s == 0 && h->last_finalized);
    h->esum_col = redo ? nullptr : slot(h->steps);
    h->esum_lines = slot(h->steps + 1);
    h->lines_split = h->esum_lines && !split_ok;
    if (timed && flush_bytes) {       // L2 flush outside the timed spans: write, then read back
      CU(cudaMemsetAsync(h->d_flush, s & 0xff, flush_bytes, h->st));
      CU(launch_l2_read(h->d_flush, flush_bytes, h->st));
    }
    if (timed) CU(cudaEventRecord(h->events[2 * s], h->st));
    if (!h->started) {
      TRY(issue_column<Real>(h, COL_HEAD, false, nullptr, false));
      h->started = true;
    } else if (s == 0 && h->last_finalized) {
      TRY(issue_column<Real>(h, COL_MID, false, nullptr, false));
    } else {
      TRY(issue_column<Real>(h, COL_MID, h->do_crp, h->d_norms + (long)(s - 1) * R, false));
    }
    TRY(issue_lines<Real>(h));
    h->steps++;
    if (timed && s < n - 1) CU(cudaEventRecord(h->events[2 * s + 1], h->st));
  }
  h->esum_col = slot(h->steps);
  h->esum_lines = nullptr;
  h->lines_split = false;
  TRY(issue_column<Real>(h, COL_TAIL, h->do_crp, h->d_norms + (long)(n - 1) * R, false));
  h->esum_col = nullptr;
  h->last_finalized = true;
  TRY(compute_crp(h));
  if (timed) CU(cudaEventRecord(h->events[2 * n - 1], h->st));
  std::vector<double> nb((size_t)n * R), eb((size_t)nslots * R * 3);
  CU(cudaMemcpyAsync(nb.data(), h->d_norms, sizeof(double) * n * R, cudaMemcpyDeviceToHost,
                     h->st));
  if (nslots > 0)
    CU(cudaMemcpyAsync(eb.data(), h->d_esum, sizeof(double) * nslots * R * 3,
                       cudaMemcpyDeviceToHost, h->st));
  CU(cudaStreamSynchronize(h->st));
  TRY(prof_collect(h));
  TRY(check_status(h));
  if (timed) {
    double tot = 0.0;
    for (int s = 0; s < n; s++) {
      float ms = 0.f;
      CU(cudaEventElapsedTime(&ms, h->events[2 * s], h->events[2 * s + 1]));
      tot += ms;
    }
    *device_ms = tot;
  }
  // unitarity guard: with n_l <= n_theta the Legendre pair is an isometry
  // followed by a projection, so a step only loses norm (there and through
  // the absorbers), and a norm above the run's previous one by more than
  // rounding (FP64 1e-8, complex64 1e-4 relative) means a corrupted state or
  // an absorber above 1.  With more angular functions than quadrature nodes
  // the reference's transform pair itself may raise the norm: no guard.
  // All norms of the call are checked before any is recorded; a failed check
  // leaves the handle refusing further steps (its state is the corrupted one).
  const double scale = h->data->r1.dr * h->data->r2.dr;
  const double grow_tol = h->prec == QD_PREC_FP64 ? 1e-8 : 1e-4;
  const size_t have = h->norms_host.size();
  for (long s = 0; s < (long)n * R; s++) {
    const double v = nb[s] * scale;
    const int step = h->steps - n + (int)(s / R) + 1, run = (int)(s % R);
    if (!std::isfinite(v)) {
      h->failed = true;
      return set_err(QD_ERR_NONFINITE, "non-finite wavepacket norm at step %d (run %d)", step, run);
    }
    const bool has_prev = s >= R || have >= (size_t)R;
    if (h->norm_guard && has_prev) {
      // same run, one step earlier
      const double pv = s >= R ? nb[s - R] * scale : h->norms_host[have - R + run];
      if (v > pv * (1.0 + grow_tol)) {
        h->failed = true;
        return set_err(QD_ERR_NONFINITE, "wavepacket norm grew from %.17g to %.17g at step %d (run %d):"
                       " a step only loses norm, through the absorbers", pv, v, step, run);
      }
    }
  }
  for (long s = 0; s < (long)n * R; s++) h->norms_host.push_back(nb[s] * scale);
  for (int e = 0; e < nslots; e++) {
    const int t = (steps0 / every + 1 + e) * every;
    for (int r = 0; r < R; r++) {
      const double *v = &eb[((size_t)e * R + r) * 3];
      const double rec[5] = {(double)t, (double)r, v[0] * scale, v[1] * scale, v[2] * scale};
      h->energy_log.insert(h->energy_log.end(), rec, rec + 5);
    }
  }
  return QD_OK;
}

template <typename T>
int upload(qd_handle *h, T *&dst, const T *src, size_t count)
{
  TRY(h->alloc(dst, count));
  CU(cudaMemcpyAsync(dst, src, count * sizeof(T), cudaMemcpyHostToDevice, h->st));
  return QD_OK;
}

bool same(const double *a, const double *b, size_t n)
{
  if (a == b) return true;
  if (!a || !b) return false;
  return std::memcmp(a, b, n * sizeof(double)) == 0;
}

// The runs of a batch share the grid, quadrature, time step, absorbers,
// precision and flux settings; psi, pot, energies and eta_sq may differ.
int validate_batch(const qd_data *runs, int n)
{
  if (!runs || n < 1) return set_err(QD_ERR_INVALID, "need at least one run");
  for (int r = 0; r < n; r++) {
    int rc = validate(&runs[r]);
    if (rc) return set_err(rc, "run %d: %s", r, g_err.c_str());
  }
  const qd_data &a = runs[0];
  for (int r = 1; r < n; r++) {
    const qd_data &b = runs[r];
    const bool ok =
        b.r1.n == a.r1.n && b.r2.n == a.r2.n && b.r1.dr == a.r1.dr && b.r2.dr == a.r2.dr &&
        b.r1.mass == a.r1.mass && b.r2.mass == a.r2.mass && same(b.r1.r, a.r1.r, a.r1.n) &&
        same(b.r2.r, a.r2.r, a.r2.n) && b.theta.n == a.theta.n &&
        same(b.theta.x, a.theta.x, a.theta.n) && same(b.theta.w, a.theta.w, a.theta.n) &&
        b.time.time_step == a.time.time_step && b.time.steps == a.time.steps &&
        b.options.precision == a.options.precision &&
        b.options.steps_to_copy_psi_from_device_to_host ==
            a.options.steps_to_copy_psi_from_device_to_host &&
        same(b.dump1.dump, a.dump1.dump, a.r1.n) && same(b.dump2.dump, a.dump2.dump, a.r2.n) &&
        b.CRP.calculate_CRP == a.CRP.calculate_CRP &&
        (!a.CRP.calculate_CRP ||
         (b.CRP.n_dividing_surface == a.CRP.n_dividing_surface &&
          b.CRP.n_gradient_points == a.CRP.n_gradient_points &&
          b.CRP.n_energies == a.CRP.n_energies));
    if (!ok)
      return set_err(QD_ERR_INVALID, "run %d differs from run 0 in a field the batch shares "
                     "(grids, theta nodes and weights, time, options.precision and "
                     "steps_to_copy_psi_from_device_to_host, dumps, CRP settings)", r);
  }
  return QD_OK;
}

int create(const qd_data *runs, int nruns, qd_handle **out)
{
  TRY(validate_batch(runs, nruns));
  const qd_data *d = &runs[0];
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return set_err(QD_ERR_CUDA, "no CUDA device visible: the propagator has no CPU path");
  }
  qd_handle *h = new qd_handle();
  *out = h;
  CU(cudaGetDevice(&h->dev));
  h->data = const_cast<qd_data *>(d);
  h->nruns = nruns;
  for (int r = 0; r < nruns; r++) h->runs.push_back(const_cast<qd_data *>(&runs[r]));
  h->prec = d->options.precision;
  h->n1 = d->r1.n; h->n2 = d->r2.n; h->nth = d->theta.n;
  h->n12 = (long)h->n1 * h->n2;
  // angular sets: runs with the same theta.m and theta.legendre share one
  std::vector<const qd_data *> set_of;
  h->nl = 0;
  h->jrows = 0;
  bool any_k = false;
  for (int r = 0; r < nruns; r++) {
    const qd_data &a = runs[r];
    const int nlr = a.theta.m + 1;
    int sidx = -1;
    for (size_t t = 0; t < set_of.size() && sidx < 0; t++)
      if (set_of[t]->theta.m == a.theta.m &&
          same(set_of[t]->theta.legendre, a.theta.legendre, (size_t)h->nth * nlr))
        sidx = (int)t;
    if (sidx < 0) {
      sidx = (int)set_of.size();
      set_of.push_back(&a);
    }
    h->run_set.push_back(sidx);
    h->run_k.push_back(a.cs.K);
    h->run_nl.push_back(nlr);
    h->nl = std::max(h->nl, nlr);
    h->norm_guard = h->norm_guard && nlr <= a.theta.n;
    h->jrows = std::max(h->jrows, a.cs.K + nlr);
    any_k = any_k || a.cs.K != 0;
  }
  h->nsets = (int)set_of.size();
  if ((long)h->n12 * h->nl * 2 * nruns >= (1L << 31) || (long)h->n12 * h->nth * nruns >= (1L << 31))
    return set_err(QD_ERR_UNSUPPORTED, "batch too large for 32-bit tile offsets");
  h->dt = d->time.time_step;
  h->steps = d->time.steps;
  h->have_dump = d->dump1.dump && d->dump2.dump;
  h->do_crp = d->CRP.calculate_CRP != 0;
  if (h->do_crp) {
    h->npts = d->CRP.n_gradient_points;
    h->h = (h->npts - 1) / 2;
    h->surf_j0 = d->CRP.n_dividing_surface - 1 - h->h;
    h->ne = d->CRP.n_energies;
  }
  radix_plan(h->n1, h->pl1);
  radix_plan(h->n2, h->pl2);
  CU(cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking));

  const long npt = h->n12 * h->nth;
  const bool f64 = h->prec == QD_PREC_FP64;
  // one potential table for the batch when all runs share pot, else one per run
  bool shared_pot = true;
  for (int r = 1; r < nruns && shared_pot; r++) shared_pot = same(runs[r].pot, d->pot, npt);
  const int npot = shared_pot ? 1 : nruns;
  h->vrun = shared_pot ? 0 : npt;
  TRY(h->alloc(h->d_pot, npt * npot));
  {
    // the potentials (and below the wavepackets) of all runs as one staged
    // stream; validate() has checked the arrays that are not staged
    const bool chk = Staging::get().staged(sizeof(double) * npt);
    std::vector<Staging::Up> up(npot);
    for (int r = 0; r < npot; r++) up[r] = {h->d_pot + r * npt, runs[r].pot, (size_t)npt, false, chk};
    std::vector<char> bad;
    CU(Staging::get().upload(up.data(), npot, h->st, bad));
    for (int r = 0; r < npot; r++)
      if (bad[r]) return set_err(QD_ERR_NONFINITE, "run %d: pot contains NaN/Inf", r);
  }
  TRY(upload(h, h->d_w, d->theta.w, h->nth));
  // each set's legendre matrix padded to nl functions (zero rows beyond its own)
  const size_t sstride = (size_t)h->nth * h->nl;
  std::vector<double> legpad(sstride * h->nsets, 0.0);
  std::vector<std::vector<double>> set_leg(h->nsets);
  std::vector<int> set_nl(h->nsets);
  for (int t = 0; t < h->nsets; t++) {
    const int m1 = set_of[t]->theta.m + 1;
    set_nl[t] = m1;
    set_leg[t].assign(set_of[t]->theta.legendre, set_of[t]->theta.legendre + (size_t)h->nth * m1);
    for (int k = 0; k < h->nth; k++)
      for (int l = 0; l < m1; l++)
        legpad[t * sstride + (size_t)k * h->nl + l] = set_leg[t][l + (size_t)k * m1];
  }
  TRY(upload(h, h->d_leg, legpad.data(), legpad.size()));
  TRY(h->alloc(h->d_P, sstride * h->nsets));
  TRY(h->alloc(h->d_WP, sstride * h->nsets));
  TRY(h->alloc(h->d_P32, sstride * h->nsets));
  TRY(h->alloc(h->d_WP32, sstride * h->nsets));
  TRY(h->alloc(h->d_P32lo, sstride * h->nsets));
  TRY(h->alloc(h->d_WP32lo, sstride * h->nsets));
  if (h->nsets > 1) {
    TRY(upload(h, h->d_run_set, h->run_set.data(), nruns));
    std::vector<int> order(nruns);                 // runs grouped by angular set
    for (int r = 0; r < nruns; r++) order[r] = r;
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return h->run_set[a] < h->run_set[b]; });
    TRY(upload(h, h->d_run_order, order.data(), nruns));
  }
  if (any_k) TRY(upload(h, h->d_run_k, h->run_k.data(), nruns));
  bool ragged = false;                      // some run stores fewer orders than the layout
  for (int r = 0; r < nruns; r++) ragged = ragged || h->run_nl[r] < h->nl;
  if (ragged) TRY(upload(h, h->d_run_nl, h->run_nl.data(), nruns));
  std::vector<double> T1, I1, T2, I2;
  radial_tables(d->r1, T1, I1);
  radial_tables(d->r2, T2, I2);
  TRY(upload(h, h->d_T1, T1.data(), h->n1));
  TRY(upload(h, h->d_I1, I1.data(), h->n1));
  TRY(upload(h, h->d_T2, T2.data(), h->n2));
  TRY(upload(h, h->d_I2, I2.data(), h->n2));
  if (h->have_dump) {
    TRY(upload(h, h->d_d1, d->dump1.dump, h->n1));
    TRY(upload(h, h->d_d2, d->dump2.dump, h->n2));
  }
  // FFT roots exp(-2 pi i k/n) in long double
  for (int dim = 0; dim < 2; dim++) {
    const int n = dim == 0 ? h->n1 : h->n2;
    std::vector<double2> z(n);
    std::vector<float2> f(n);
    for (int k = 0; k < n; k++) {
      const long double a = -2.0L * 3.141592653589793238462643383279502884L * k / n;
      z[k] = make_double2((double)cosl(a), (double)sinl(a));
      f[k] = make_float2((float)cosl(a), (float)sinl(a));
    }
    TRY(upload(h, dim == 0 ? h->d_tw1_64 : h->d_tw2_64, z.data(), n));
    TRY(upload(h, dim == 0 ? h->d_tw1_32 : h->d_tw2_32, f.data(), n));
  }
  for (int t = 0; t < h->nsets; t++) {
    const size_t o = t * sstride;
    CU(launch_legendre_matrices(h->nth, h->nl, nullptr, h->d_w, h->d_leg + o, h->d_P + o,
                                h->d_WP + o, h->d_P32 + o, h->d_WP32 + o, h->d_P32lo + o,
                                h->d_WP32lo + o, h->st));
    g_launches++;
  }
  if (f64) {
    TRY(h->alloc(h->d_expV, npt * npot));
    TRY(h->alloc(h->d_rot, (size_t)h->n12 * h->jrows));
    TRY(h->alloc(h->d_kin, h->n12));
    CU(launch_setup_tables_fp64(h->n1, h->n2, h->nth * npot, h->jrows, h->dt, h->d_pot, h->d_I1,
                                h->d_I2, h->d_T1, h->d_T2, h->d_expV, h->d_rot, h->d_kin,
                                h->st));
  } else {
    TRY(h->alloc(h->d_expV32, npt * npot));
    TRY(h->alloc(h->d_rc1, (size_t)h->jrows * h->n1));
    TRY(h->alloc(h->d_rc2, (size_t)h->jrows * h->n2));
    TRY(h->alloc(h->d_kc1, h->n1));
    TRY(h->alloc(h->d_kc2, h->n2));
    CU(launch_setup_tables_fp32(h->n1, h->n2, h->nth * npot, h->jrows, h->dt, h->d_pot, h->d_I1,
                                h->d_I2, h->d_T1, h->d_T2, h->d_expV32, h->d_rc1, h->d_rc2,
                                h->d_kc1, h->d_kc2, h->st));
  }
  g_launches++;
  const size_t csz = f64 ? sizeof(double2) : sizeof(float2);
  void *lp = nullptr;
  {
    unsigned char *b = nullptr;
    TRY(h->alloc(b, csz * h->n12 * h->nl * nruns));
    lp = b;
  }
  h->d_lpsi = lp;
  // orders a run does not store (n_l of its block below the batch's) stay zero:
  // the column passes read them as A entries of their contraction over l
  CU(cudaMemsetAsync(lp, 0, csz * h->n12 * h->nl * nruns, h->st));
  TRY(h->alloc(h->d_psi_z, npt * nruns));
  if (f64) {
    const bool chk = Staging::get().staged(sizeof(double2) * npt);
    std::vector<Staging::Up> up(nruns);
    for (int r = 0; r < nruns; r++)
      up[r] = {h->d_psi_z + r * npt, runs[r].psi, 2 * (size_t)npt, false, chk};
    std::vector<char> bad;
    CU(Staging::get().upload(up.data(), nruns, h->st, bad));
    for (int r = 0; r < nruns; r++)
      if (bad[r]) return set_err(QD_ERR_NONFINITE, "run %d: psi contains NaN/Inf", r);
  } else {
    // complex64 form: psi rounded to complex64 by the host threads that stage it
    // (half the bytes over the bus), then widened into the FP64 staging array
    TRY(h->alloc(h->d_psi32, npt * nruns));
    std::vector<Staging::Up> up(nruns);
    for (int r = 0; r < nruns; r++)
      up[r] = {h->d_psi32 + r * npt, runs[r].psi, 2 * (size_t)npt, true, true};
    std::vector<char> bad;
    CU(Staging::get().upload(up.data(), nruns, h->st, bad));
    for (int r = 0; r < nruns; r++)
      if (bad[r])
        return set_err(QD_ERR_NONFINITE, "run %d: psi contains NaN/Inf or values beyond the "
                       "complex64 range", r);
    CU(launch_widen_c(h->d_psi32, h->d_psi_z, (size_t)npt * nruns, h->st));
    g_launches++;
  }
  if (h->do_crp) {
    const size_t nq = (size_t)h->nth * h->n1;
    unsigned char *b = nullptr;
    TRY(h->alloc(b, csz * nq * (2 * h->h + 1) * nruns));
    h->d_surf = b;
    TRY(h->alloc(h->d_ring_psi, nq * QD_RING * nruns));
    TRY(h->alloc(h->d_ring_g, nq * QD_RING * nruns));
    TRY(h->alloc(h->d_fai, nq * h->ne * nruns));
    TRY(h->alloc(h->d_dfai, nq * h->ne * nruns));
    TRY(h->alloc(h->d_phase, (size_t)h->ne * FLUX_CHUNK * nruns));
    CU(cudaMemsetAsync(h->d_fai, 0, sizeof(double2) * nq * h->ne * nruns, h->st));
    CU(cudaMemsetAsync(h->d_dfai, 0, sizeof(double2) * nq * h->ne * nruns, h->st));
    TRY(h->alloc(h->d_energies, (size_t)h->ne * nruns));
    TRY(h->alloc(h->d_eta, (size_t)h->ne * nruns));
    for (int r = 0; r < nruns; r++) {
      CU(cudaMemcpyAsync(h->d_energies + (size_t)r * h->ne, runs[r].CRP.energies,
                         sizeof(double) * h->ne, cudaMemcpyHostToDevice, h->st));
      CU(cudaMemcpyAsync(h->d_eta + (size_t)r * h->ne, runs[r].CRP.eta_sq,
                         sizeof(double) * h->ne, cudaMemcpyHostToDevice, h->st));
    }
    TRY(h->alloc(h->d_crp, (size_t)h->ne * nruns));
    const char *cf = getenv("QD_CRP_FUSED");
    if (!(cf && cf[0] == '0'))
      TRY(h->alloc(h->d_crp_part, (size_t)h->ne * nruns * flux_q_tiles((int)nq)));
    // energies E_0 + j dE in every run (to a phase error below 1e-12 rad over a
    // chunk): the accumulation of full chunks takes the chirp-z form
    // (QD_FLUX_CZT=0 keeps the GEMM form)
    const char *cz = getenv("QD_FLUX_CZT");
    bool uniform = h->ne >= 2 && h->ne <= CZT_N - FLUX_CHUNK + 1 && !(cz && cz[0] == '0');
    std::vector<double> e0(nruns), de(nruns);
    for (int r = 0; r < nruns && uniform; r++) {
      const double *E = runs[r].CRP.energies;
      e0[r] = E[0];
      de[r] = (E[h->ne - 1] - E[0]) / (h->ne - 1);
      double dev = 0.0;
      for (int j = 0; j < h->ne; j++) dev = std::max(dev, std::fabs(E[j] - (e0[r] + j * de[r])));
      uniform = de[r] != 0.0 && dev * FLUX_CHUNK * std::fabs(h->dt) <= 1e-12;
    }
    if (uniform) {
      double *d_e0 = nullptr;
      TRY(h->alloc(h->d_czt_tw, (size_t)CZT_N));
      TRY(h->alloc(h->d_czt_g, (size_t)FLUX_CHUNK * nruns));
      TRY(h->alloc(h->d_czt_b, (size_t)CZT_N * nruns));
      TRY(h->alloc(h->d_czt_de, (size_t)nruns));
      TRY(h->alloc(d_e0, (size_t)nruns));
      CU(cudaMemcpyAsync(d_e0, e0.data(), sizeof(double) * nruns, cudaMemcpyHostToDevice, h->st));
      CU(cudaMemcpyAsync(h->d_czt_de, de.data(), sizeof(double) * nruns, cudaMemcpyHostToDevice,
                         h->st));
      CU(launch_czt_tables(nruns, h->ne, h->dt, d_e0, h->d_czt_de, h->d_czt_tw, h->d_czt_g,
                           h->d_czt_b, h->st));
      g_launches++;
      CU(cudaStreamSynchronize(h->st));       // e0, de: host vectors of this scope
    }
  }
  const char *path = getenv("QD_COLUMN_PATH");   // "simt" forces the SIMT column pass
  if (!f64 && !(path && std::string(path) == "simt")) {
    std::vector<const double *> lp(h->nsets);
    for (int t = 0; t < h->nsets; t++) lp[t] = set_leg[t].data();
    int rc = tc_plan_create(h->tc, h->nth, h->nl, h->nsets, lp.data(), set_nl.data(),
                            d->theta.w, h->st);
    if (rc == QD_OK) h->use_tc = true;
    else if (rc != QD_ERR_UNSUPPORTED) return rc;
  }
  TRY(tune_column(h));
  TRY(tune_slice(h));
  TRY(tune_flux(h));
  CU(cudaStreamSynchronize(h->st));
  return QD_OK;
}

// theta-space psi of every run into d_psi_z (B psi_l and the absorber)
// (once per propagated state: qd_download reads every run from one staging)
int stage_psi(qd_handle *h)
{
  if (!h->started || h->psi_z_valid) return QD_OK;   // d_psi_z holds the input / the state
  if (h->prec == QD_PREC_FP64) TRY(issue_column<double>(h, COL_TAIL, false, nullptr, true));
  else TRY(issue_column<float>(h, COL_TAIL, false, nullptr, true));
  h->psi_z_valid = true;
  return QD_OK;
}

int get_psi(qd_handle *h, int run, double *psi_out)
{
  if (run < 0 || run >= h->nruns) return set_err(QD_ERR_INVALID, "run %d of %d", run, h->nruns);
  const long npt = h->n12 * h->nth;
  TRY(stage_psi(h));
  if (h->d_psi32) {             // complex64 form: every value is a complex64 one
    CU(launch_narrow_c(h->d_psi_z + (long)run * npt, h->d_psi32 + (long)run * npt, npt, h->st));
    g_launches++;
    Staging::Piece pc{psi_out, h->d_psi32 + (long)run * npt, sizeof(float2) * npt, true};
    CU(Staging::get().download(&pc, 1, h->st));
    return QD_OK;
  }
  CU(Staging::get().download(psi_out, h->d_psi_z + (long)run * npt, sizeof(double2) * npt,
                             h->st));
  return QD_OK;
}

int get_crp(qd_handle *h, int run, double *crp_out)
{
  if (!h->do_crp) return set_err(QD_ERR_INVALID, "CRP.calculate_CRP is 0");
  if (run < 0 || run >= h->nruns) return set_err(QD_ERR_INVALID, "run %d of %d", run, h->nruns);
  if (!h->started) {
    for (int e = 0; e < h->ne; e++) crp_out[e] = 0.0;
    return QD_OK;
  }
  TRY(compute_crp(h));
  CU(cudaMemcpyAsync(crp_out, h->d_crp + (long)run * h->ne, sizeof(double) * h->ne,
                     cudaMemcpyDeviceToHost, h->st));
  CU(cudaStreamSynchronize(h->st));
  return QD_OK;
}

// Energies of the current theta-space state of one run (timeEvol.C:256-360):
// kinetic from the 2-D DFT of each l-slice, rotational and potential by
// direct sums; all reductions in FP64.
int energies(qd_handle *h, int run, double out4[4])
{
  if (run < 0 || run >= h->nruns) return set_err(QD_ERR_INVALID, "run %d of %d", run, h->nruns);
  TRY(stage_psi(h));
  EnergyParams e{};
  e.n1 = h->n1; e.n2 = h->n2; e.nth = h->nth; e.nl = h->nl; e.n12 = h->n12;
  e.psi_z = h->d_psi_z + (long)run * h->n12 * h->nth;
  e.pot = h->d_pot + (long)run * h->vrun;
  const long soff = (long)h->run_set[run] * h->nth * h->nl;
  e.w = h->d_w; e.P = h->d_P + soff; e.WP = h->d_WP + soff; e.K = h->run_k[run];
  e.T1 = h->d_T1; e.T2 = h->d_T2; e.I1 = h->d_I1; e.I2 = h->d_I2;
  e.tw1 = h->d_tw1_64; e.tw2 = h->d_tw2_64; e.pl1 = h->pl1; e.pl2 = h->pl2;
  // the DFT scratch and the sums stay with the handle (its memory pool)
  // after the first call
  if (!h->d_escratch) {
    TRY(h->alloc(h->d_escratch, (size_t)h->n12 * h->nth));
    TRY(h->alloc(h->d_esums3, 3));
  }
  e.sums = h->d_esums3;
  e.scratch = h->d_escratch;
  CU(cudaMemsetAsync(e.sums, 0, 3 * sizeof(double), h->st));
  CU(launch_energies(e, h->st));
  double s[3] = {0, 0, 0};
  CU(cudaMemcpyAsync(s, e.sums, sizeof s, cudaMemcpyDeviceToHost, h->st));
  CU(cudaStreamSynchronize(h->st));
  g_launches += energies_launches();
  const double dd = h->data->r1.dr * h->data->r2.dr;
  out4[0] = s[0] * dd / ((double)h->n1 * h->n2);   // kinetic (unnormalised DFT)
  out4[1] = s[1] * dd;                              // rotational
  out4[2] = s[2] * dd;                              // potential
  out4[3] = out4[0] + out4[1] + out4[2];
  return QD_OK;
}

// ---- checkpoint / restore ----------------------------------------------------
constexpr uint64_t CKPT_MAGIC = 0x33544b5044514251ull;   // file tag, layout version 3

struct CkptHeader {
  uint64_t magic;
  int32_t prec, nruns, n1, n2, nth, nl, ne, npts;
  int32_t steps, started, last_finalized, ring_fill, flux_pending;
  int32_t basis;               // l-space representation: 0 psi_l, 1 psi_l / sqrt(l+1/2)
  int64_t acc_done;
  int32_t ring;                // steps held by the flux history ring (QD_RING)
  int32_t reserved;
};

// The complex64 tensor-core column pass keeps psi_l in the orthonormal basis.
int lspace_basis(const qd_handle *h) { return h->prec == QD_PREC_FP32 && h->use_tc ? 1 : 0; }

int checkpoint(qd_handle *h, const char *path)
{
  CU(cudaStreamSynchronize(h->st));
  CkptHeader hd{};
  hd.magic = CKPT_MAGIC; hd.prec = h->prec; hd.nruns = h->nruns; hd.n1 = h->n1; hd.n2 = h->n2;
  hd.nth = h->nth; hd.nl = h->nl; hd.ne = h->do_crp ? h->ne : 0; hd.npts = h->npts;
  hd.steps = h->steps; hd.started = h->started; hd.last_finalized = h->last_finalized;
  hd.ring_fill = h->ring_fill; hd.flux_pending = h->flux_pending; hd.acc_done = h->acc_done;
  hd.basis = lspace_basis(h);
  hd.ring = QD_RING;
  const size_t csz = h->prec == QD_PREC_FP64 ? sizeof(double2) : sizeof(float2);
  std::vector<std::pair<const void *, size_t>> blocks;
  const size_t nq = (size_t)h->nth * h->n1;
  blocks.push_back({h->d_lpsi, csz * h->n12 * h->nl * h->nruns});
  blocks.push_back({h->d_psi_z, sizeof(double2) * h->n12 * h->nth * h->nruns});
  if (h->do_crp) {
    blocks.push_back({h->d_surf, csz * nq * (2 * h->h + 1) * h->nruns});
    blocks.push_back({h->d_ring_psi, sizeof(double2) * nq * QD_RING * h->nruns});
    blocks.push_back({h->d_ring_g, sizeof(double2) * nq * QD_RING * h->nruns});
    blocks.push_back({h->d_fai, sizeof(double2) * nq * h->ne * h->nruns});
    blocks.push_back({h->d_dfai, sizeof(double2) * nq * h->ne * h->nruns});
  }
  FILE *f = fopen(path, "wb");
  if (!f) return set_err(QD_ERR_IO, "cannot write \"%s\"", path);
  bool ok = fwrite(&hd, sizeof hd, 1, f) == 1;
  const uint64_t nnorm = h->norms_host.size();
  ok = ok && fwrite(&nnorm, sizeof nnorm, 1, f) == 1;
  ok = ok && (nnorm == 0 || fwrite(h->norms_host.data(), sizeof(double), nnorm, f) == nnorm);
  std::vector<unsigned char> buf;
  for (auto &b : blocks) {
    if (!ok) break;
    buf.resize(b.second);
    if (cudaMemcpy(buf.data(), b.first, b.second, cudaMemcpyDeviceToHost) != cudaSuccess) {
      fclose(f);
      return set_err(QD_ERR_CUDA, "checkpoint: %s", cudaGetErrorString(cudaGetLastError()));
    }
    ok = fwrite(buf.data(), 1, b.second, f) == b.second;
  }
  if (fclose(f) != 0) ok = false;
  return ok ? QD_OK : set_err(QD_ERR_IO, "short write to \"%s\"", path);
}

int restore(qd_handle *h, const char *path)
{
  FILE *f = fopen(path, "rb");
  if (!f) return set_err(QD_ERR_IO, "cannot read \"%s\"", path);
  CkptHeader hd{};
  if (fread(&hd, sizeof hd, 1, f) != 1 || hd.magic != CKPT_MAGIC) {
    fclose(f);
    return set_err(QD_ERR_IO, "\"%s\" is not a propagator checkpoint of this layout version",
                   path);
  }
  if (hd.ring != QD_RING) {
    fclose(f);
    return set_err(QD_ERR_INVALID, "checkpoint \"%s\" holds a flux history ring of %d steps, "
                   "this library %d", path, hd.ring, QD_RING);
  }
  if (hd.prec != h->prec || hd.nruns != h->nruns || hd.n1 != h->n1 || hd.n2 != h->n2 ||
      hd.nth != h->nth || hd.nl != h->nl || hd.ne != (h->do_crp ? h->ne : 0) ||
      hd.npts != h->npts) {
    fclose(f);
    return set_err(QD_ERR_INVALID, "checkpoint \"%s\" was written for other sizes", path);
  }
  if (hd.basis != lspace_basis(h)) {
    fclose(f);
    return set_err(QD_ERR_INVALID, "checkpoint \"%s\" was written by another column-pass kernel "
                   "(l-space basis %d, this handle %d)", path, hd.basis, lspace_basis(h));
  }
  uint64_t nnorm = 0;
  bool ok = fread(&nnorm, sizeof nnorm, 1, f) == 1 && nnorm < (1ull << 40);
  std::vector<double> norms(ok ? nnorm : 0);
  ok = ok && (nnorm == 0 || fread(norms.data(), sizeof(double), nnorm, f) == nnorm);
  const size_t csz = h->prec == QD_PREC_FP64 ? sizeof(double2) : sizeof(float2);
  const size_t nq = (size_t)h->nth * h->n1;
  std::vector<std::pair<void *, size_t>> blocks;
  blocks.push_back({h->d_lpsi, csz * h->n12 * h->nl * h->nruns});
  blocks.push_back({h->d_psi_z, sizeof(double2) * h->n12 * h->nth * h->nruns});
  if (h->do_crp) {
    blocks.push_back({h->d_surf, csz * nq * (2 * h->h + 1) * h->nruns});
    blocks.push_back({h->d_ring_psi, sizeof(double2) * nq * QD_RING * h->nruns});
    blocks.push_back({h->d_ring_g, sizeof(double2) * nq * QD_RING * h->nruns});
    blocks.push_back({h->d_fai, sizeof(double2) * nq * h->ne * h->nruns});
    blocks.push_back({h->d_dfai, sizeof(double2) * nq * h->ne * h->nruns});
  }
  std::vector<unsigned char> buf;
  for (auto &b : blocks) {
    if (!ok) break;
    buf.resize(b.second);
    ok = fread(buf.data(), 1, b.second, f) == b.second;
    if (ok && cudaMemcpy(b.first, buf.data(), b.second, cudaMemcpyHostToDevice) != cudaSuccess) {
      fclose(f);
      return set_err(QD_ERR_CUDA, "restore: %s", cudaGetErrorString(cudaGetLastError()));
    }
  }
  fclose(f);
  if (!ok) return set_err(QD_ERR_IO, "\"%s\" is truncated", path);
  h->steps = hd.steps; h->started = hd.started; h->last_finalized = hd.last_finalized;
  h->psi_z_valid = false;
  h->crp_valid = false;
  h->ring_fill = hd.ring_fill; h->flux_pending = hd.flux_pending; h->acc_done = hd.acc_done;
  h->norms_host = norms;
  h->failed = false;
  return QD_OK;
}

int refuse_failed(const qd_handle *h)
{
  return set_err(QD_ERR_NONFINITE, "the handle's last propagation stopped on a corrupted "
                 "wavepacket (step %d); restore a checkpoint or create a new handle", h->steps);
}

}  // namespace

extern "C" {

int qd_abi_version(void) { return QD_ABI_VERSION; }
const char *qd_last_error(void) { return g_err.c_str(); }
int64_t qd_kernel_launch_count(void) { return g_launches.load(); }

int qd_set_device(int32_t device)
{
  CU(cudaSetDevice(device));
  return QD_OK;
}

int qd_create_batch(const qd_data *runs, int32_t n_runs, qd_handle **out)
{
  if (!out) return set_err(QD_ERR_INVALID, "out is NULL");
  *out = nullptr;
  qd_handle *h = nullptr;
  int rc = create(runs, n_runs, &h);
  if (rc != QD_OK) {
    delete h;
    return rc;
  }
  *out = h;
  return QD_OK;
}

int qd_create(const qd_data *data, qd_handle **out)
{
  return qd_create_batch(data, 1, out);
}

int qd_n_runs(qd_handle *h, int32_t *n_out)
{
  if (!h || !n_out) return set_err(QD_ERR_INVALID, "NULL argument");
  *n_out = h->nruns;
  return QD_OK;
}

int qd_destroy(qd_handle *h)
{
  if (!h) return QD_OK;
  DevGuard g(h->dev);
  delete h;
  return QD_OK;
}

int qd_propagate(qd_handle *h, int32_t n_steps)
{
  if (!h) return set_err(QD_ERR_INVALID, "handle is NULL");
  if (n_steps < 0) return set_err(QD_ERR_INVALID, "n_steps < 0");
  if (h->failed) return refuse_failed(h);
  DevGuard g(h->dev);
  if (h->prec == QD_PREC_FP64) return propagate<double>(h, n_steps);
  return propagate<float>(h, n_steps);
}

int qd_propagate_timed(qd_handle *h, int32_t n_steps, int64_t flush_bytes, double *device_ms)
{
  if (!h || !device_ms) return set_err(QD_ERR_INVALID, "NULL argument");
  if (n_steps < 0 || flush_bytes < 0) return set_err(QD_ERR_INVALID, "negative argument");
  if (h->failed) return refuse_failed(h);
  DevGuard g(h->dev);
  if (h->prec == QD_PREC_FP64) return propagate<double>(h, n_steps, (size_t)flush_bytes, device_ms);
  return propagate<float>(h, n_steps, (size_t)flush_bytes, device_ms);
}

int qd_get_psi_run(qd_handle *h, int32_t run, double *psi_out)
{
  if (!h || !psi_out) return set_err(QD_ERR_INVALID, "NULL argument");
  DevGuard g(h->dev);
  return get_psi(h, run, psi_out);
}

int qd_get_psi(qd_handle *h, double *psi_out) { return qd_get_psi_run(h, 0, psi_out); }

int qd_get_crp_run(qd_handle *h, int32_t run, double *crp_out)
{
  if (!h || !crp_out) return set_err(QD_ERR_INVALID, "NULL argument");
  DevGuard g(h->dev);
  return get_crp(h, run, crp_out);
}

int qd_get_crp(qd_handle *h, double *crp_out) { return qd_get_crp_run(h, 0, crp_out); }

int qd_download(qd_handle *h)
{
  if (!h) return set_err(QD_ERR_INVALID, "handle is NULL");
  DevGuard g(h->dev);
  // every run's psi and P(E) in one pipelined transfer
  TRY(stage_psi(h));
  const bool crp = h->do_crp && h->started;
  if (crp) TRY(compute_crp(h));
  const long npt = h->n12 * h->nth;
  std::vector<Staging::Piece> pcs;
  if (h->d_psi32) {             // complex64 form: every value is a complex64 one
    CU(launch_narrow_c(h->d_psi_z, h->d_psi32, (size_t)npt * h->nruns, h->st));
    g_launches++;
  }
  for (int r = 0; r < h->nruns; r++) {
    if (h->d_psi32)
      pcs.push_back({h->runs[r]->psi, h->d_psi32 + (long)r * npt, sizeof(float2) * npt, true});
    else
      pcs.push_back({h->runs[r]->psi, h->d_psi_z + (long)r * npt, sizeof(double2) * npt});
    if (crp)
      pcs.push_back({h->runs[r]->CRP.CRP, h->d_crp + (long)r * h->ne, sizeof(double) * h->ne});
  }
  CU(Staging::get().download(pcs.data(), (int)pcs.size(), h->st));
  if (h->do_crp && !h->started)
    for (int r = 0; r < h->nruns; r++)
      for (int e = 0; e < h->ne; e++) h->runs[r]->CRP.CRP[e] = 0.0;
  for (int r = 0; r < h->nruns; r++) h->runs[r]->time.steps = h->steps;
  return QD_OK;
}

int qd_get_norms_run(qd_handle *h, int32_t run, double *norms_out, int32_t n)
{
  if (!h || !norms_out || n < 0) return set_err(QD_ERR_INVALID, "bad argument");
  if (run < 0 || run >= h->nruns) return set_err(QD_ERR_INVALID, "run %d of %d", run, h->nruns);
  const size_t avail = h->norms_host.size() / h->nruns;
  if ((size_t)n > avail)
    return set_err(QD_ERR_INVALID, "%d norms requested, %zu available", n, avail);
  for (int32_t s = 0; s < n; s++)
    norms_out[s] = h->norms_host[(avail - n + s) * h->nruns + run];
  return QD_OK;
}

int qd_get_norms(qd_handle *h, double *norms_out, int32_t n)
{
  return qd_get_norms_run(h, 0, norms_out, n);
}

int qd_steps(qd_handle *h, int32_t *steps_out)
{
  if (!h || !steps_out) return set_err(QD_ERR_INVALID, "NULL argument");
  *steps_out = h->steps;
  return QD_OK;
}

int qd_set_profiling(qd_handle *h, int32_t on)
{
  if (!h) return set_err(QD_ERR_INVALID, "handle is NULL");
  h->profiling = on != 0;
  return QD_OK;
}

int qd_kernel_choice(qd_handle *h, int32_t out[4])
{
  if (!h || !out) return set_err(QD_ERR_INVALID, "NULL argument");
  out[0] = h->slice_cluster;
  out[1] = h->use_tc ? 1 : 0;
  out[2] = h->flux_variant;
  out[3] = h->d_czt_b ? 1 : 0;
  return QD_OK;
}

int qd_kernel_times(qd_handle *h, double *ms_out, int32_t n, int32_t *n_written)
{
  if (!h || !n_written) return set_err(QD_ERR_INVALID, "NULL argument");
  int32_t k = 0;
  for (; k < n && k < (int32_t)h->kernel_ms.size(); k++) ms_out[k] = h->kernel_ms[k];
  *n_written = k;
  return QD_OK;
}

int qd_energies_run(qd_handle *h, int32_t run, double out4[4])
{
  if (!h || !out4) return set_err(QD_ERR_INVALID, "NULL argument");
  DevGuard g(h->dev);
  return energies(h, run, out4);
}

int qd_energies(qd_handle *h, double out4[4]) { return qd_energies_run(h, 0, out4); }

int qd_set_energy_interval(qd_handle *h, int32_t every)
{
  if (!h) return set_err(QD_ERR_INVALID, "handle is NULL");
  if (every < 0) return set_err(QD_ERR_INVALID, "energy interval %d < 0", every);
  h->energy_every = every;
  return QD_OK;
}

int qd_get_energy_log_run(qd_handle *h, int32_t run, double *out, int32_t cap, int32_t *n_out)
{
  if (!h || !n_out || cap < 0 || (cap > 0 && !out)) return set_err(QD_ERR_INVALID, "bad argument");
  if (run < 0 || run >= h->nruns) return set_err(QD_ERR_INVALID, "run %d of %d", run, h->nruns);
  std::vector<const double *> mine;
  for (size_t i = 0; i + 5 <= h->energy_log.size(); i += 5)
    if ((int)h->energy_log[i + 1] == run) mine.push_back(&h->energy_log[i]);
  const size_t k = std::min(mine.size(), (size_t)cap), first = mine.size() - k;
  for (size_t i = 0; i < k; i++) {
    const double *r = mine[first + i];
    out[5 * i] = r[0];
    out[5 * i + 1] = r[2];
    out[5 * i + 2] = r[3];
    out[5 * i + 3] = r[4];
    out[5 * i + 4] = r[2] + r[3] + r[4];
  }
  *n_out = (int32_t)k;
  return QD_OK;
}

int qd_checkpoint(qd_handle *h, const char *path)
{
  if (!h || !path) return set_err(QD_ERR_INVALID, "NULL argument");
  DevGuard g(h->dev);
  return checkpoint(h, path);
}

int qd_restore(qd_handle *h, const char *path)
{
  if (!h || !path) return set_err(QD_ERR_INVALID, "NULL argument");
  DevGuard g(h->dev);
  return restore(h, path);
}

// The MEX drop-in.  With options.steps_to_copy_psi_from_device_to_host = N
// > 0 it does what the reference's GPU loop does every N steps
// (common-cuda/evolutionCUDA2.cu:540-546: P(E) on steps % N == 0, psi copied
// back to the host and the Matlab script run): whenever time.steps reaches a
// multiple of N it writes psi, time.steps and CRP.CRP of every run into the
// caller's arrays and calls options.progress of each run that has one.  A
// non-zero return stops the call with QD_ERR_STOPPED, the arrays holding
// that step's state.
int qd_time_evolution_batch(qd_data *runs, int32_t n_runs)
{
  if (!runs || n_runs < 1) return set_err(QD_ERR_INVALID, "need at least one run");
  const int every = runs[0].options.steps_to_copy_psi_from_device_to_host;
  if (every < 0)
    return set_err(QD_ERR_INVALID, "options.steps_to_copy_psi_from_device_to_host = %d", every);
  qd_handle *h = nullptr;
  TRY(qd_create_batch(runs, n_runs, &h));
  const int total = runs[0].time.total_steps;
  int rc = QD_OK;
  if (every == 0) {
    rc = qd_propagate(h, total);
    if (rc == QD_OK) rc = qd_download(h);
  } else {
    bool fresh = true;                  // the caller's arrays hold the current state
    for (int done = 0; done < total && rc == QD_OK;) {
      const int n = std::min(every - h->steps % every, total - done);
      rc = qd_propagate(h, n);
      if (rc != QD_OK) break;
      done += n;
      fresh = false;
      if (h->steps % every != 0) continue;
      rc = qd_download(h);
      if (rc != QD_OK) break;
      fresh = true;
      const size_t last = h->norms_host.size() - (size_t)n_runs;
      for (int r = 0; r < n_runs && rc == QD_OK; r++) {
        const qd_options &o = runs[r].options;
        if (o.progress && o.progress(h->steps, h->norms_host[last + r], runs[r].psi,
                                     o.progress_ctx) != 0)
          rc = set_err(QD_ERR_STOPPED, "the progress callback of run %d stopped the "
                       "propagation at step %d", r, h->steps);
      }
    }
    if (rc == QD_OK && !fresh) rc = qd_download(h);
  }
  qd_destroy(h);
  return rc;
}

int qd_time_evolution(qd_data *data) { return qd_time_evolution_batch(data, 1); }

int qd_read_grids(const char *dir, int32_t n, double *x, double *w)
{
  if (!dir || !x || !w) return set_err(QD_ERR_INVALID, "NULL argument");
  if (n < 1 || n > 599) return set_err(QD_ERR_INVALID, "argument should be 1 <= n <= 599");
  std::string path = std::string(dir) + "/" + std::to_string(n) + "-LegendreGauss.grids";
  FILE *f = fopen(path.c_str(), "r");
  if (!f) return set_err(QD_ERR_IO, "\"%s\" does not exist", path.c_str());
  std::vector<double> xs, ws;
  double a, b;
  while (fscanf(f, "%lf %lf", &a, &b) == 2) { xs.push_back(a); ws.push_back(b); }
  fclose(f);
  const int nh = (int)xs.size();
  if (n != 2 * nh - (n % 2))
    return set_err(QD_ERR_IO, "%s: %d lines do not describe n = %d", path.c_str(), nh, n);
  // mirror the non-negative half (GaussLegendre2.m:19-25)
  int o = 0;
  const int start = (n % 2) ? nh - 1 : nh - 1;
  for (int i = start; i >= ((n % 2) ? 1 : 0); i--) { x[o] = -xs[i]; w[o] = ws[i]; o++; }
  for (int i = 0; i < nh; i++) { x[o] = xs[i]; w[o] = ws[i]; o++; }
  return QD_OK;
}

// Both angular-basis entry points: one FP64 kernel launch on the device.
static int legendre_basis(const char *who, int32_t n, int32_t K, int32_t m, const double *x,
                          double *legendre)
{
  if (!x || !legendre || n < 1 || m < 0 || K < 0)
    return set_err(QD_ERR_INVALID, "%s: bad argument (n %d, K %d, m %d)", who, n, K, m);
  for (int k = 0; k < n; k++)
    if (!(std::fabs(x[k]) <= 1.0))
      return set_err(QD_ERR_INVALID, "%s: node %d (%g) is outside [-1, 1]", who, k, x[k]);
  double *dx = nullptr, *dl = nullptr;
  CU(cudaMalloc(&dx, sizeof(double) * n));
  cudaError_t e = cudaMalloc(&dl, sizeof(double) * (size_t)n * (m + 1));
  if (e != cudaSuccess) { cudaFree(dx); CU(e); }
  int rc = QD_OK;
  if (cudaMemcpy(dx, x, sizeof(double) * n, cudaMemcpyHostToDevice) != cudaSuccess ||
      launch_legendre_basis(n, K, m, dx, dl, 0) != cudaSuccess ||
      cudaMemcpy(legendre, dl, sizeof(double) * (size_t)n * (m + 1), cudaMemcpyDeviceToHost) !=
          cudaSuccess)
    rc = set_err(QD_ERR_CUDA, "%s: %s", who, cudaGetErrorString(cudaGetLastError()));
  g_launches++;
  cudaFree(dx);
  cudaFree(dl);
  return rc;
}

int qd_legendre_matrix(int32_t n, int32_t m, const double *x, double *legendre)
{
  return legendre_basis("qd_legendre_matrix", n, 0, m, x, legendre);
}

int qd_cs_legendre(int32_t n, int32_t K, int32_t m, const double *x, double *legendre)
{
  return legendre_basis("qd_cs_legendre", n, K, m, x, legendre);
}

}  // extern "C"

// ---- energies with static scratch (qd_energies_noalloc) ------------------------
// One file-scope device array holds everything qd_energies_noalloc needs on the
// device: its first 16 double2 (256 bytes) carry the three FP64 energy sums, the
// rest the 2-D DFT of up to QD_ENERGIES_NOALLOC_MAX_POINTS theta-space points.
static __device__ __align__(256) double2 g_energy_scratch[16 + QD_ENERGIES_NOALLOC_MAX_POINTS];

namespace {

constexpr int QD_MAX_DEVICES = 64;
std::atomic<double2 *> g_energy_scratch_at[QD_MAX_DEVICES];   // per device, set once

// Device address of g_energy_scratch on the current device (the handle's:
// the entry point makes it current), looked up on the first call for that
// device (cudaGetSymbolAddress; two threads racing here both store the same
// address).
int energy_scratch(double2 **out)
{
  int dev = 0;
  CU(cudaGetDevice(&dev));
  if (dev < 0 || dev >= QD_MAX_DEVICES)
    return set_err(QD_ERR_DEVICE, "qd_energies_noalloc: device %d out of range", dev);
  double2 *p = g_energy_scratch_at[dev].load();
  if (!p) {
    cudaError_t e = cudaGetSymbolAddress((void **)&p, g_energy_scratch);
    if (e != cudaSuccess || !p)
      return set_err(QD_ERR_CUDA, "qd_energies_noalloc: cudaGetSymbolAddress failed: %s",
                     cudaGetErrorString(e));
    g_energy_scratch_at[dev].store(p);
  }
  *out = p;
  return QD_OK;
}

// energies() with the scratch and the sums in g_energy_scratch: no device
// memory is allocated or freed.
int energies_noalloc(qd_handle *h, int run, double out4[4])
{
  if (run < 0 || run >= h->nruns) return set_err(QD_ERR_INVALID, "run %d of %d", run, h->nruns);
  const long need = h->n12 * h->nth;
  if (need > QD_ENERGIES_NOALLOC_MAX_POINTS)
    return set_err(QD_ERR_INVALID,
                   "qd_energies_noalloc: %ld grid points per run exceed the static scratch "
                   "of %d points (use qd_energies_run)", need, QD_ENERGIES_NOALLOC_MAX_POINTS);
  double2 *base = nullptr;
  TRY(energy_scratch(&base));
  TRY(stage_psi(h));
  EnergyParams e{};
  e.n1 = h->n1; e.n2 = h->n2; e.nth = h->nth; e.nl = h->nl; e.n12 = h->n12;
  e.psi_z = h->d_psi_z + (long)run * h->n12 * h->nth;
  e.pot = h->d_pot + (long)run * h->vrun;
  const long soff = (long)h->run_set[run] * h->nth * h->nl;
  e.w = h->d_w; e.P = h->d_P + soff; e.WP = h->d_WP + soff; e.K = h->run_k[run];
  e.T1 = h->d_T1; e.T2 = h->d_T2; e.I1 = h->d_I1; e.I2 = h->d_I2;
  e.tw1 = h->d_tw1_64; e.tw2 = h->d_tw2_64; e.pl1 = h->pl1; e.pl2 = h->pl2;
  e.sums = reinterpret_cast<double *>(base);
  e.scratch = base + 16;
  CU(cudaMemsetAsync(e.sums, 0, 3 * sizeof(double), h->st));
  CU(launch_energies(e, h->st));
  double s[3] = {0, 0, 0};
  CU(cudaMemcpyAsync(s, e.sums, sizeof s, cudaMemcpyDeviceToHost, h->st));
  CU(cudaStreamSynchronize(h->st));
  g_launches += energies_launches();
  const double dd = h->data->r1.dr * h->data->r2.dr;
  out4[0] = s[0] * dd / ((double)h->n1 * h->n2);
  out4[1] = s[1] * dd;
  out4[2] = s[2] * dd;
  out4[3] = out4[0] + out4[1] + out4[2];
  return QD_OK;
}

}  // namespace

extern "C" int qd_energies_noalloc(qd_handle *h, int32_t run, double out4[4])
{
  if (!h || !out4) return set_err(QD_ERR_INVALID, "NULL argument");
  DevGuard g(h->dev);
  return energies_noalloc(h, run, out4);
}
