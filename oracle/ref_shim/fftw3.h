/* fftw3.h -- TEST INFRASTRUCTURE ONLY.  The subset of the FFTW3 API that the
 * reference's common/fftwinterface.C calls (plans, execute, threads), backed
 * by the oracle's own unnormalised DFT.  FFTW itself is not installed. */
#ifndef QD_SHIM_FFTW3_H
#define QD_SHIM_FFTW3_H

typedef double fftw_complex[2];
typedef struct qd_shim_plan *fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign,
                           unsigned flags);
fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex *in, fftw_complex *out,
                           int sign, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
int fftw_init_threads(void);
void fftw_plan_with_nthreads(int n);

#endif
