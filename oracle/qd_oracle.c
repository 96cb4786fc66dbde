/*
 * qd_oracle.c -- TEST INFRASTRUCTURE ONLY.  CPU FP64 restatement of the
 * reference propagator (wangsl/quantum-dynamics, common/timeEvol.C and the
 * Fortran kernels it calls).  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py may load this library; the product never does.
 *
 * Each function cites the reference file:line whose arithmetic it restates.
 * Complex arithmetic is written out the way the reference's Complex class
 * (common/complex.h) performs it, so that results agree to rounding.
 *
 * FFT: FFTW 3.3.4 (the reference's dependency, not vendored) is replaced by
 * an unnormalised mixed-radix DFT with the same sign convention
 * (FFTW_FORWARD = exp(-2 pi i jk/n), FFTW_BACKWARD = exp(+...)).
 *
 * One extension beyond the reference: for a centrifugal-sudden block
 * (qd_data.cs, zero for the reference's J = 0 case) the rotational phase and
 * energy use j = K + l; the angular basis and the centrifugal potential come
 * in through theta.legendre and pot like any other input.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#include <stdint.h>
#include "qd.h"
#include "qd_oracle.h"

#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct { double re, im; } cplx;

static inline cplx cmul(cplx a, cplx b)
{ cplx c = { a.re*b.re - a.im*b.im, a.re*b.im + a.im*b.re }; return c; }

/* ------------------------------------------------------------------------
 * FFT (stand-in for FFTW's fftw_plan_dft_2d, common/fftwinterface.C:70-76)
 * ---------------------------------------------------------------------- */

static int smallest_factor(int n)
{
  if (n % 4 == 0) return 4;
  for (int f = 2; f * f <= n; f++) if (n % f == 0) return f;
  return n;
}

/* Recursive decimation-in-time mixed-radix DFT of x[0..n) (stride s) into
 * y[0..n) (contiguous).  tw[k] = exp(sign*2*pi*i*k/ntot), ntot = nroot. */
static void dft_rec(const cplx *x, int s, cplx *y, int n, const cplx *tw,
                    int nroot, cplx *tmp)
{
  if (n == 1) { y[0] = x[0]; return; }
  int p = smallest_factor(n);
  int m = n / p;
  /* sub-transforms of the p decimated sequences */
  for (int q = 0; q < p; q++)
    dft_rec(x + q * s, s * p, y + q * m, m, tw, nroot, tmp + n);
  /* combine: Y[k + m*r] = sum_q W_n^{q(k+m r)} Y_q[k] */
  int step = nroot / n;
  for (int k = 0; k < m; k++) {
    for (int r = 0; r < p; r++) {
      cplx acc = {0.0, 0.0};
      for (int q = 0; q < p; q++) {
        long e = ((long)q * (k + m * r)) % n;
        cplx w = tw[e * step];
        cplx v = cmul(y[q * m + k], w);
        acc.re += v.re; acc.im += v.im;
      }
      tmp[k + m * r] = acc;
    }
  }
  memcpy(y, tmp, sizeof(cplx) * n);
}

static cplx *make_twiddles(int n, int sign)
{
  cplx *tw = (cplx *)malloc(sizeof(cplx) * n);
  for (int k = 0; k < n; k++) {
    long double a = (long double)sign * 2.0L * 3.141592653589793238462643383279502884L
                    * (long double)k / (long double)n;
    tw[k].re = (double)cosl(a);
    tw[k].im = (double)sinl(a);
  }
  return tw;
}

/* In-place unnormalised 1-D DFT of n points with stride `stride`. */
static void fft1d_strided(cplx *a, int n, long stride, const cplx *tw,
                          cplx *buf /* 4n */)
{
  cplx *x = buf, *y = buf + n, *tmp = buf + 2 * n;
  for (int i = 0; i < n; i++) x[i] = a[i * stride];
  dft_rec(x, 1, y, n, tw, n, tmp);
  for (int i = 0; i < n; i++) a[i * stride] = y[i];
}

/* 2-D DFT of a column-major n1 x n2 array (i fastest), as FFTW's
 * fftw_plan_dft_2d(n2, n1, ...) over that memory (fftwinterface.C:71-76). */
void qdo_fft2d(double *data, int n1, int n2, int sign)
{
  cplx *a = (cplx *)data;
  cplx *tw1 = make_twiddles(n1, sign);
  cplx *tw2 = make_twiddles(n2, sign);
  int nmax = n1 > n2 ? n1 : n2;
  cplx *buf = (cplx *)malloc(sizeof(cplx) * 4 * nmax * 2);
  for (int j = 0; j < n2; j++) fft1d_strided(a + (long)j * n1, n1, 1, tw1, buf);
  for (int i = 0; i < n1; i++) fft1d_strided(a + i, n2, n1, tw2, buf);
  free(buf); free(tw1); free(tw2);
}

/* One 2-D DFT split over threads by lines, as FFTW's threaded plans
 * (fftw_plan_with_nthreads, fftwinterface.C:44) parallelise a single plan. */
void qdo_fft2d_threaded(double *data, int n1, int n2, int sign)
{
  cplx *a = (cplx *)data;
  cplx *tw1 = make_twiddles(n1, sign);
  cplx *tw2 = make_twiddles(n2, sign);
  int nmax = n1 > n2 ? n1 : n2;
#pragma omp parallel
  {
    cplx *buf = (cplx *)malloc(sizeof(cplx) * 4 * nmax * 2);
#pragma omp for schedule(static)
    for (int j = 0; j < n2; j++) fft1d_strided(a + (long)j * n1, n1, 1, tw1, buf);
#pragma omp for schedule(static)
    for (int i = 0; i < n1; i++) fft1d_strided(a + i, n2, n1, tw2, buf);
    free(buf);
  }
  free(tw1); free(tw2);
}

/* Batched version over nb consecutive n1 x n2 slices (OpenMP over slices). */
static void fft2d_batch(cplx *a, int n1, int n2, int nb, int sign)
{
  cplx *tw1 = make_twiddles(n1, sign);
  cplx *tw2 = make_twiddles(n2, sign);
  int nmax = n1 > n2 ? n1 : n2;
#pragma omp parallel
  {
    cplx *buf = (cplx *)malloc(sizeof(cplx) * 4 * nmax * 2);
#pragma omp for schedule(static)
    for (int b = 0; b < nb; b++) {
      cplx *s = a + (long)b * n1 * n2;
      for (int j = 0; j < n2; j++) fft1d_strided(s + (long)j * n1, n1, 1, tw1, buf);
      for (int i = 0; i < n1; i++) fft1d_strided(s + i, n2, n1, tw2, buf);
    }
    free(buf);
  }
  free(tw1); free(tw2);
}

/* ------------------------------------------------------------------------
 * Coordinate tables
 * ---------------------------------------------------------------------- */

/* Momentum grid of an FFT of nm points over length xl
 * (common/fftwinterface.C:110-125): {0..nm/2, -nm/2+1..-1} * 2 pi / xl. */
int qdo_momentum(double *p, int nm, double xl)
{
  if (nm / 2 * 2 != nm) return QD_ERR_INVALID;
  const double two_pi_xl = 2.0 * M_PI / xl;
  const int half = nm / 2;
  double p1 = 0;
  for (int i = 0; i <= half; i++) { p[i] = p1; p1 += two_pi_xl; }
  p1 = two_pi_xl * (-half + 1);
  for (int i = half + 1; i < nm; i++) { p[i] = p1; p1 += two_pi_xl; }
  return QD_OK;
}

/* p^2/(2 m) and 1/(2 m r^2) (common/MatlabStructures.C:17-36). */
int qdo_radial_tables(const qd_radial *c, double *psq2m, double *one2mr2)
{
  int rc = qdo_momentum(psq2m, c->n, c->n * c->dr);
  if (rc) return rc;
  for (int i = 0; i < c->n; i++) psq2m[i] = psq2m[i] * psq2m[i] / (2 * c->mass);
  const double m2 = c->mass + c->mass;
  for (int i = 0; i < c->n; i++) one2mr2[i] = 1.0 / (m2 * c->r[i] * c->r[i]);
  return QD_OK;
}

/* The reference's complex sqrt: pow(c, 0.5) with arg() from asin
 * (common/complex.h:60-68, 149-159). */
static double ref_arg(cplx c)
{
  double a = asin(c.im / sqrt(c.re * c.re + c.im * c.im));
  if (c.re < 0 && c.im > 0) return M_PI - a;
  if (c.re < 0 && c.im < 0) return -(M_PI + a);
  return a;
}
static cplx ref_sqrt(cplx c)
{
  double th = 0.5 * ref_arg(c);
  double r = pow(c.re * c.re + c.im * c.im, 0.25);
  cplx s = { r * cos(th), r * sin(th) };
  return s;
}
/* c1 / c2 = c1 / abs2(c2) * conj(c2) (common/complex.h:130-131). */
static cplx ref_div(cplx c1, cplx c2)
{
  double a2 = c2.re * c2.re + c2.im * c2.im;
  cplx t = { c1.re / a2, c1.im / a2 };
  cplx cc = { c2.re, -c2.im };
  return cmul(t, cc);
}
/* exp(Complex(0, -x)) as the reference evaluates it (complex.h:133-134). */
static cplx ref_expi(double x)
{
  cplx c = { cos(x), sin(x) };
  return c;
}

/* ------------------------------------------------------------------------
 * The propagator state
 * ---------------------------------------------------------------------- */

struct qdo_state {
  qd_data *d;
  int n1, n2, nth, nl;
  long n12;
  double *psq2m1, *psq2m2, *one2mr21, *one2mr22;
  cplx *psi;        /* aliases d->psi                          */
  cplx *lpsi;       /* n1*n2*nl                                */
  cplx *exp_ipot_dt, *exp_irot_dt_2, *exp_ikin_dt;
  double *weight_legendre;   /* n_theta x nl column-major        */
  double *dump;              /* n1 x n2                           */
  cplx *exp_ienergy_dt, *exp_ienergy_t;
  cplx *psi_surface, *d_psi_surface, *fai_surface, *d_fai_surface;
};

static void free_state(qdo_state *s)
{
  if (!s) return;
  free(s->psq2m1); free(s->psq2m2); free(s->one2mr21); free(s->one2mr22);
  free(s->lpsi); free(s->exp_ipot_dt); free(s->exp_irot_dt_2); free(s->exp_ikin_dt);
  free(s->weight_legendre); free(s->dump);
  free(s->exp_ienergy_dt); free(s->exp_ienergy_t);
  free(s->psi_surface); free(s->d_psi_surface); free(s->fai_surface); free(s->d_fai_surface);
  free(s);
}

qdo_state *qdo_create(qd_data *d)
{
  qdo_state *s = (qdo_state *)calloc(1, sizeof(qdo_state));
  s->d = d;
  s->n1 = d->r1.n; s->n2 = d->r2.n; s->nth = d->theta.n; s->nl = d->theta.m + 1;
  s->n12 = (long)s->n1 * s->n2;
  s->psq2m1 = malloc(sizeof(double) * s->n1); s->one2mr21 = malloc(sizeof(double) * s->n1);
  s->psq2m2 = malloc(sizeof(double) * s->n2); s->one2mr22 = malloc(sizeof(double) * s->n2);
  if (qdo_radial_tables(&d->r1, s->psq2m1, s->one2mr21) ||
      qdo_radial_tables(&d->r2, s->psq2m2, s->one2mr22)) { free_state(s); return NULL; }
  s->psi = (cplx *)d->psi;
  s->lpsi = (cplx *)calloc(s->n12 * s->nl, sizeof(cplx));
  return s;
}

void qdo_destroy(qdo_state *s) { free_state(s); }

/* setup_weight_legendre (timeEvol.C:737-760): wp(k,l) = (l+1/2) w_k P(l,k). */
static void setup_weight_legendre(qdo_state *s)
{
  if (s->weight_legendre) return;
  const int nth = s->nth, m = s->nl;
  s->weight_legendre = malloc(sizeof(double) * nth * m);
  const double *w = s->d->theta.w, *P = s->d->theta.legendre;
  for (int l = 0; l < m; l++) {
    const double f = l + 0.5;
    for (int k = 0; k < nth; k++) s->weight_legendre[k + (long)l * nth] = f * w[k] * P[l + (long)k * m];
  }
}

/* ForwardLegendreTransform (LegTransform.F:6-31):
 * LPsi(I,L) = sum_K CPsi(I,K) WLegP(K,L). */
void qdo_forward_legendre(const double *cpsi, double *lpsi, long NR, int NT, int NL,
                          const double *wlegp)
{
  const cplx *C = (const cplx *)cpsi; cplx *O = (cplx *)lpsi;
  memset(O, 0, sizeof(cplx) * NR * NL);
#pragma omp parallel for schedule(static, 1)
  for (int L = 0; L < NL; L++)
    for (int K = 0; K < NT; K++) {
      const double wlp = wlegp[K + (long)L * NT];
      const cplx *c = C + (long)K * NR;
      cplx *o = O + (long)L * NR;
      for (long I = 0; I < NR; I++) { o[I].re += c[I].re * wlp; o[I].im += c[I].im * wlp; }
    }
}

/* BackwardLegendreTransform (LegTransform.F:34-59):
 * CPsi(I,K) = sum_L LPsi(I,L) LegP(L,K). */
void qdo_backward_legendre(double *cpsi, const double *lpsi, long NR, int NT, int NL,
                           const double *legp)
{
  cplx *O = (cplx *)cpsi; const cplx *C = (const cplx *)lpsi;
  memset(O, 0, sizeof(cplx) * NR * NT);
#pragma omp parallel for schedule(static, 1)
  for (int K = 0; K < NT; K++)
    for (int L = 0; L < NL; L++) {
      const double p = legp[L + (long)K * NL];
      const cplx *c = C + (long)L * NR;
      cplx *o = O + (long)K * NR;
      for (long I = 0; I < NR; I++) { o[I].re += c[I].re * p; o[I].im += c[I].im * p; }
    }
}

static void forward_legendre(qdo_state *s)
{
  setup_weight_legendre(s);
  qdo_forward_legendre((const double *)s->psi, (double *)s->lpsi, s->n12, s->nth, s->nl,
                       s->weight_legendre);
}

static void backward_legendre(qdo_state *s)
{
  qdo_backward_legendre((double *)s->psi, (const double *)s->lpsi, s->n12, s->nth, s->nl,
                        s->d->theta.legendre);
}

/* setup_exp_ipot_dt (timeEvol.C:438-463). */
static void setup_exp_ipot_dt(qdo_state *s)
{
  if (s->exp_ipot_dt) return;
  const long n = s->n12 * s->nth;
  s->exp_ipot_dt = malloc(sizeof(cplx) * n);
  const double dt = s->d->time.time_step;
#pragma omp parallel for schedule(static)
  for (long q = 0; q < n; q++) s->exp_ipot_dt[q] = ref_expi(-dt * s->d->pot[q]);
}

/* setup_exp_irot_dt_2 (timeEvol.C:465-491). */
static void setup_exp_irot_dt_2(qdo_state *s)
{
  if (s->exp_irot_dt_2) return;
  const int n1 = s->n1, n2 = s->n2, m = s->nl;
  s->exp_irot_dt_2 = malloc(sizeof(cplx) * s->n12 * m);
  const double dt2 = s->d->time.time_step / 2;
#pragma omp parallel for schedule(static, 1)
  for (int l = 0; l < m; l++)
    for (int j = 0; j < n2; j++)
      for (int i = 0; i < n1; i++) {
        /* exp(l(l+1)(I1+I2) * Complex(0,-dt/2)): the real part of the product
           is l(l+1)(I1+I2)*0 = 0 and exp(0) = 1 */
        const double jr = (double)(s->d->cs.K + l);   /* j = K + l (centrifugal sudden) */
        const double x = jr * (jr + 1) * (s->one2mr21[i] + s->one2mr22[j]);
        s->exp_irot_dt_2[i + (long)n1 * (j + (long)n2 * l)] = ref_expi(x * -dt2);
      }
}

/* setup_exp_ikin_dt (timeEvol.C:493-517): exp(-i(T1+T2)dt)/n1/n2. */
static void setup_exp_ikin_dt(qdo_state *s)
{
  if (s->exp_ikin_dt) return;
  const int n1 = s->n1, n2 = s->n2;
  s->exp_ikin_dt = malloc(sizeof(cplx) * s->n12);
  const double dt = s->d->time.time_step;
  for (int j = 0; j < n2; j++)
    for (int i = 0; i < n1; i++) {
      cplx e = ref_expi((s->psq2m1[i] + s->psq2m2[j]) * -dt);
      e.re = e.re / n1 / n2; e.im = e.im / n1 / n2;
      s->exp_ikin_dt[i + (long)n1 * j] = e;
    }
}

/* pre_evolution_with_potential_dt_2 (timeEvol.C:519-538): psi /= sqrt(v). */
static void pre_evolution(qdo_state *s)
{
  setup_exp_ipot_dt(s);
  const long n = s->n12 * s->nth;
#pragma omp parallel for schedule(static)
  for (long q = 0; q < n; q++) s->psi[q] = ref_div(s->psi[q], ref_sqrt(s->exp_ipot_dt[q]));
}

static void mul_table(cplx *a, const cplx *t, long n)
{
#pragma omp parallel for schedule(static)
  for (long q = 0; q < n; q++) a[q] = cmul(a[q], t[q]);
}

/* evolution_with_potential_dt (timeEvol.C:540-559). */
static void evolution_with_potential(qdo_state *s)
{ setup_exp_ipot_dt(s); mul_table(s->psi, s->exp_ipot_dt, s->n12 * s->nth); }

/* evolution_with_rotational_dt_2 (timeEvol.C:561-582). */
static void evolution_with_rotational(qdo_state *s)
{ setup_exp_irot_dt_2(s); mul_table(s->lpsi, s->exp_irot_dt_2, s->n12 * s->nl); }

/* evolution_with_kinetic_dt (timeEvol.C:584-606). */
static void evolution_with_kinetic(qdo_state *s)
{
  setup_exp_ikin_dt(s);
#pragma omp parallel for schedule(static)
  for (int l = 0; l < s->nl; l++) {
    cplx *p = s->lpsi + (long)l * s->n12;
    for (long q = 0; q < s->n12; q++) p[q] = cmul(p[q], s->exp_ikin_dt[q]);
  }
}

/* kinetic_energy_for_legendre_psi(0) (timeEvol.C:390-436), momentum space. */
static double kinetic_energy_lpsi_kspace(qdo_state *s)
{
  const int n1 = s->n1, n2 = s->n2;
  double sum = 0.0;
#pragma omp parallel for schedule(static, 1) reduction(+:sum)
  for (int l = 0; l < s->nl; l++) {
    const cplx *p = s->lpsi + (long)l * s->n12;
    double sl = 0.0;
    for (int j = 0; j < n2; j++)
      for (int i = 0; i < n1; i++) {
        cplx c = p[i + (long)n1 * j];
        sl += (c.re * c.re + c.im * c.im) * (s->psq2m1[i] + s->psq2m2[j]);
      }
    sum += sl / (l + 0.5);
  }
  double e = sum * s->d->r1.dr * s->d->r2.dr;
  return e * (n1 * n2);
}

/* rotational_energy(0) (timeEvol.C:323-360). */
static double rotational_energy_lpsi(qdo_state *s)
{
  const int n1 = s->n1, n2 = s->n2;
  double sum = 0.0;
#pragma omp parallel for schedule(static, 1) reduction(+:sum)
  for (int l = 0; l < s->nl; l++) {
    const cplx *p = s->lpsi + (long)l * s->n12;
    double sl = 0.0;
    for (int j = 0; j < n2; j++)
      for (int i = 0; i < n1; i++) {
        cplx c = p[i + (long)n1 * j];
        sl += (c.re * c.re + c.im * c.im) * (s->one2mr21[i] + s->one2mr22[j]);
      }
    const double jr = (double)(s->d->cs.K + l);
    sum += sl * jr * (jr + 1) / (l + 0.5);
  }
  return sum * s->d->r1.dr * s->d->r2.dr;
}

/* potential_energy (timeEvol.C:256-283). */
static double potential_energy(qdo_state *s)
{
  double sum = 0.0;
  const double *w = s->d->theta.w;
#pragma omp parallel for schedule(static, 1) reduction(+:sum)
  for (int k = 0; k < s->nth; k++) {
    const cplx *p = s->psi + (long)k * s->n12;
    const double *v = s->d->pot + (long)k * s->n12;
    double sk = 0.0;
    for (long q = 0; q < s->n12; q++) sk += (p[q].re * p[q].re + p[q].im * p[q].im) * v[q];
    sum += w[k] * sk;
  }
  return sum * s->d->r1.dr * s->d->r2.dr;
}

/* module_for_psi (timeEvol.C:220-243). */
double qdo_module_for_psi(qdo_state *s)
{
  double sum = 0.0;
  const double *w = s->d->theta.w;
#pragma omp parallel for schedule(static, 1) reduction(+:sum)
  for (int k = 0; k < s->nth; k++) {
    const cplx *p = s->psi + (long)k * s->n12;
    double sk = 0.0;
    for (long q = 0; q < s->n12; q++) sk += p[q].re * p[q].re + p[q].im * p[q].im;
    sum += w[k] * sk;
  }
  return sum * s->d->r1.dr * s->d->r2.dr;
}

/* evolution_dt (timeEvol.C:619-647); energies[0..3] = kin, rot, pot, tot. */
static void evolution_dt(qdo_state *s, double *energies)
{
  evolution_with_potential(s);
  forward_legendre(s);
  evolution_with_rotational(s);
  fft2d_batch(s->lpsi, s->n1, s->n2, s->nl, -1);
  evolution_with_kinetic(s);
  double e_kin = energies ? kinetic_energy_lpsi_kspace(s) : 0.0;
  fft2d_batch(s->lpsi, s->n1, s->n2, s->nl, +1);
  evolution_with_rotational(s);
  double e_rot = energies ? rotational_energy_lpsi(s) : 0.0;
  backward_legendre(s);
  double e_pot = energies ? potential_energy(s) : 0.0;
  if (energies) {
    energies[0] = e_kin; energies[1] = e_rot; energies[2] = e_pot;
    energies[3] = e_kin + e_rot + e_pot;
  }
}

/* setup_dump + dump_psi (timeEvol.C:687-735). */
static void dump_psi(qdo_state *s)
{
  const qd_data *d = s->d;
  if (!(d->dump1.dump && d->dump2.dump)) return;
  const int n1 = s->n1, n2 = s->n2;
  if (!s->dump) {
    s->dump = malloc(sizeof(double) * s->n12);
    for (int j = 0; j < n2; j++)
      for (int i = 0; i < n1; i++) s->dump[i + (long)n1 * j] = d->dump1.dump[i] * d->dump2.dump[j];
  }
#pragma omp parallel for schedule(static, 1)
  for (int k = 0; k < s->nth; k++) {
    cplx *p = s->psi + (long)k * s->n12;
    for (long q = 0; q < s->n12; q++) { p[q].re *= s->dump[q]; p[q].im *= s->dump[q]; }
  }
}

/* setup_CRP_data (timeEvol.C:762-805). */
static void setup_crp(qdo_state *s)
{
  if (s->exp_ienergy_dt && s->exp_ienergy_t) return;
  const int n1 = s->n1, nth = s->nth, ne = s->d->CRP.n_energies;
  s->psi_surface = calloc((long)n1 * nth, sizeof(cplx));
  s->d_psi_surface = calloc((long)n1 * nth, sizeof(cplx));
  s->fai_surface = calloc((long)n1 * nth * ne, sizeof(cplx));
  s->d_fai_surface = calloc((long)n1 * nth * ne, sizeof(cplx));
  s->exp_ienergy_dt = malloc(sizeof(cplx) * ne);
  s->exp_ienergy_t = malloc(sizeof(cplx) * ne);
  const double dt = s->d->time.time_step;
  for (int i = 0; i < ne; i++) {
    /* exp(I*e*dt): I*e = Complex(0*e, e); exp(0)=1 */
    s->exp_ienergy_dt[i] = ref_expi(s->d->CRP.energies[i] * dt);
    s->exp_ienergy_t[i].re = dt; s->exp_ienergy_t[i].im = 0.0;
  }
}

/* Gradient3D (Gradient3.F:9-167): value and central difference of F along
 * the second index at the 1-based row N2P. */
int qdo_gradient3d(int N1, int N2, int N3, int N2P, double Dx, const double *Fd,
                   double *Vd, double *Gd, int NPoints)
{
  const cplx *F = (const cplx *)Fd; cplx *V = (cplx *)Vd, *G = (cplx *)Gd;
  int h = (NPoints - 1) / 2;
  if (NPoints != 3 && NPoints != 5 && NPoints != 7 && NPoints != 9 && NPoints != 11)
    return QD_ERR_INVALID;
  if (N2P - 1 - h < 0 || N2P - 1 + h > N2 - 1) return QD_ERR_INVALID;
#define FF(I, J, K) F[(I) + (long)N1 * ((J) - 1 + (long)N2 * (K))]
  for (int K = 0; K < N3; K++)
    for (int I = 0; I < N1; I++) {
      cplx g = {0, 0};
      double den = 0;
#define DIF(mm) cplx d##mm = { FF(I, N2P + mm, K).re - FF(I, N2P - mm, K).re, \
                               FF(I, N2P + mm, K).im - FF(I, N2P - mm, K).im }
      if (NPoints == 3) {
        DIF(1);
        g = d1; den = 2 * Dx;
      } else if (NPoints == 5) {
        DIF(1); DIF(2);
        g.re = -d2.re + 8 * d1.re; g.im = -d2.im + 8 * d1.im; den = 12 * Dx;
      } else if (NPoints == 7) {
        DIF(1); DIF(2); DIF(3);
        g.re = d3.re - 9 * d2.re + 45 * d1.re; g.im = d3.im - 9 * d2.im + 45 * d1.im; den = 60 * Dx;
      } else if (NPoints == 9) {
        DIF(1); DIF(2); DIF(3); DIF(4);
        g.re = -3 * d4.re + 32 * d3.re - 168 * d2.re + 672 * d1.re;
        g.im = -3 * d4.im + 32 * d3.im - 168 * d2.im + 672 * d1.im; den = 840 * Dx;
      } else {
        DIF(1); DIF(2); DIF(3); DIF(4); DIF(5);
        g.re = 2 * d5.re - 25 * d4.re + 150 * d3.re - 600 * d2.re + 2100 * d1.re;
        g.im = 2 * d5.im - 25 * d4.im + 150 * d3.im - 600 * d2.im + 2100 * d1.im; den = 2520 * Dx;
      }
#undef DIF
      V[I + (long)N1 * K] = FF(I, N2P, K);
      G[I + (long)N1 * K].re = g.re / den;
      G[I + (long)N1 * K].im = g.im / den;
    }
#undef FF
  return QD_OK;
}

/* PsiTimeToPsiEnergyOnSurface (CRPAux.F:4-31):
 * faiE(:,:,IE) += ExpIETDt(IE) * PsiT, DFaiE likewise. */
void qdo_psi_time_to_fai(int N1, int NTheta, int NE, const double *expiet,
                         const double *psit, const double *dpsit, double *faie,
                         double *dfaie)
{
  const long ns = (long)N1 * NTheta;
  const cplx *E = (const cplx *)expiet, *P = (const cplx *)psit, *DP = (const cplx *)dpsit;
#pragma omp parallel for schedule(static, 1)
  for (int e = 0; e < NE; e++) {
    const cplx c = E[e];
    cplx *f = (cplx *)faie + (long)e * ns, *df = (cplx *)dfaie + (long)e * ns;
    for (long q = 0; q < ns; q++) {
      cplx a = cmul(c, P[q]), b = cmul(c, DP[q]);
      f[q].re += a.re; f[q].im += a.im;
      df[q].re += b.re; df[q].im += b.im;
    }
  }
}

static void psi_time_to_fai_energy(qdo_state *s)
{
  qdo_psi_time_to_fai(s->n1, s->nth, s->d->CRP.n_energies, (const double *)s->exp_ienergy_t,
                      (const double *)s->psi_surface, (const double *)s->d_psi_surface,
                      (double *)s->fai_surface, (double *)s->d_fai_surface);
}

/* CalculateCRP (CRPAux.F:34-66). */
void qdo_calculate_crp(int N1, int NTheta, int NE, double Dr1, double mu2,
                       const double *W, const double *EtaSq, const double *Faid,
                       const double *DFaid, double *CRP)
{
  const cplx *Fai = (const cplx *)Faid, *DFai = (const cplx *)DFaid;
  const double dr1mu2 = Dr1 / mu2;
#pragma omp parallel for schedule(static, 1)
  for (int e = 0; e < NE; e++) {
    cplx ce = {0, 0};
    for (int k = 0; k < NTheta; k++) {
      cplx c3 = {0, 0};
      for (int i = 0; i < N1; i++) {
        long q = i + (long)N1 * (k + (long)NTheta * e);
        cplx a = { Fai[q].re, -Fai[q].im };
        cplx p = cmul(a, DFai[q]);
        c3.re += p.re; c3.im += p.im;
      }
      ce.re += W[k] * c3.re; ce.im += W[k] * c3.im;
    }
    CRP[e] = ce.im / EtaSq[e] * dr1mu2;
  }
}

/* calculate_reaction_probabilities (timeEvol.C:870-878). */
static int calculate_reaction_probabilities(qdo_state *s)
{
  qd_data *d = s->d;
  setup_crp(s);
  int rc = qdo_gradient3d(s->n1, s->n2, s->nth, d->CRP.n_dividing_surface, d->r2.dr,
                          (const double *)s->psi, (double *)s->psi_surface,
                          (double *)s->d_psi_surface, d->CRP.n_gradient_points);
  if (rc) return rc;
  for (int e = 0; e < d->CRP.n_energies; e++)          /* update_exp_ienergy_t, :807-817 */
    s->exp_ienergy_t[e] = cmul(s->exp_ienergy_t[e], s->exp_ienergy_dt[e]);
  psi_time_to_fai_energy(s);
  qdo_calculate_crp(s->n1, s->nth, d->CRP.n_energies, d->r1.dr, d->r2.mass, d->theta.w,
                    d->CRP.eta_sq, (const double *)s->fai_surface,
                    (const double *)s->d_fai_surface, d->CRP.CRP);
  return QD_OK;
}

/* time_evolution (timeEvol.C:649-685).  norms/energies: optional per-step
 * outputs (total_steps and 4*total_steps doubles). */
int qdo_run_steps(qdo_state *s, int nsteps, double *norms, double *energies)
{
  qd_data *d = s->d;
  for (int i_step = 0; i_step < nsteps; i_step++) {
    if (i_step == 0 && d->time.steps == 0) pre_evolution(s);
    evolution_dt(s, energies ? energies + 4 * i_step : NULL);
    dump_psi(s);
    if (norms) norms[i_step] = qdo_module_for_psi(s);
    if (d->CRP.calculate_CRP) {
      int rc = calculate_reaction_probabilities(s);
      if (rc) return rc;
    }
    d->time.steps++;
  }
  return QD_OK;
}

int qdo_time_evolution(qd_data *d, double *norms, double *energies)
{
  qdo_state *s = qdo_create(d);
  if (!s) return QD_ERR_INVALID;
  int rc = qdo_run_steps(s, d->time.total_steps, norms, energies);
  qdo_destroy(s);
  return rc;
}

/* Energies of the theta-space psi in d (no side effects on d->psi):
 * kinetic_energy_for_psi (timeEvol.C:285-321), rotational_energy(1)
 * (:323-360), potential_energy (:256-283); out = kin, rot, pot, total. */
int qdo_energies(qd_data *d, double *out)
{
  qdo_state *s = qdo_create(d);
  if (!s) return QD_ERR_INVALID;
  const int n1 = s->n1, n2 = s->n2, nth = s->nth;
  const long n12 = s->n12;
  cplx *work = malloc(sizeof(cplx) * n12 * nth);
  memcpy(work, s->psi, sizeof(cplx) * n12 * nth);
  fft2d_batch(work, n1, n2, nth, -1);
  double e = 0.0;
  for (int k = 0; k < nth; k++) {
    double ek = 0.0;
    for (int j = 0; j < n2; j++)
      for (int i = 0; i < n1; i++) {
        cplx c = work[i + (long)n1 * (j + (long)n2 * k)];
        ek += (c.re * c.re + c.im * c.im) * (s->psq2m1[i] + s->psq2m2[j]);
      }
    e += d->theta.w[k] * ek;
  }
  out[0] = e * d->r1.dr * d->r2.dr / (n1 * n2);
  forward_legendre(s);
  out[1] = rotational_energy_lpsi(s);
  out[2] = potential_energy(s);
  out[3] = out[0] + out[1] + out[2];
  free(work);
  qdo_destroy(s);
  return QD_OK;
}

int qdo_num_threads(void)
{
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
