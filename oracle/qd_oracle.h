/* qd_oracle.h -- TEST INFRASTRUCTURE ONLY: CPU FP64 oracle of the reference
 * propagator (see qd_oracle.c).  Never linked into the product. */
#ifndef QD_ORACLE_H
#define QD_ORACLE_H
#include "qd.h"
#ifdef __cplusplus
extern "C" {
#endif

typedef struct qdo_state qdo_state;

void qdo_fft2d(double *data, int n1, int n2, int sign);
int qdo_momentum(double *p, int nm, double xl);
int qdo_radial_tables(const qd_radial *c, double *psq2m, double *one2mr2);
int qdo_gradient3d(int N1, int N2, int N3, int N2P, double Dx, const double *F,
                   double *V, double *G, int NPoints);
void qdo_forward_legendre(const double *cpsi, double *lpsi, long NR, int NT, int NL,
                          const double *wlegp);
void qdo_backward_legendre(double *cpsi, const double *lpsi, long NR, int NT, int NL,
                           const double *legp);
void qdo_psi_time_to_fai(int N1, int NTheta, int NE, const double *expiet,
                         const double *psit, const double *dpsit, double *faie,
                         double *dfaie);
void qdo_fft2d_threaded(double *data, int n1, int n2, int sign);
void qdo_calculate_crp(int N1, int NTheta, int NE, double Dr1, double mu2,
                       const double *W, const double *EtaSq, const double *Fai,
                       const double *DFai, double *CRP);

qdo_state *qdo_create(qd_data *d);
void qdo_destroy(qdo_state *s);
int qdo_run_steps(qdo_state *s, int nsteps, double *norms, double *energies);
double qdo_module_for_psi(qdo_state *s);
int qdo_time_evolution(qd_data *d, double *norms, double *energies);
int qdo_num_threads(void);
int qdo_energies(qd_data *d, double *out4);

#ifdef __cplusplus
}
#endif
#endif
