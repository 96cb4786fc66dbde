/* shim.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * Lets the reference's own CPU propagator (common/timeEvol.C driven by
 * common/TimeEvolutionMex.C:18-78), compiled unmodified from the reference
 * sources, run without Matlab, FFTW or a Fortran compiler:
 *   - the mx* / mex* calls it makes are served from a tree of views built
 *     over a qd_data (no copies: psi, time.steps and CRP.CRP are written in
 *     place, as Matlab arrays would be);
 *   - the FFTW3 calls of common/fftwinterface.C run the oracle's DFT;
 *   - the Fortran kernels (LegTransform.F, CRPAux.F, Gradient3.F) are the
 *     oracle's C restatements under their Fortran symbol names.
 * Entry point: qdref_time_evolution(qd_data*).  mexErrMsgTxt unwinds with a
 * C++ exception that the entry point turns into a status code.
 */
#include <cstring>
#include <cstdlib>
#include <string>
#include <vector>
#include <map>
#include <memory>
#include <stdexcept>
#include <iostream>
#include <sstream>
#include "mex.h"
#include "fftw3.h"
#include "qd.h"
#include "qd_oracle.h"

struct mxArray {
  std::map<std::string, mxArray *> fields;
  void *data = nullptr;
  std::string str;
  bool is_string = false;
};

namespace {
struct MexError : std::runtime_error { using std::runtime_error::runtime_error; };

std::vector<std::unique_ptr<mxArray>> g_pool;

mxArray *view(const void *p)
{
  g_pool.emplace_back(new mxArray);
  g_pool.back()->data = const_cast<void *>(p);
  return g_pool.back().get();
}
mxArray *strct() { g_pool.emplace_back(new mxArray); return g_pool.back().get(); }
mxArray *string(const char *s)
{
  g_pool.emplace_back(new mxArray);
  g_pool.back()->is_string = true;
  g_pool.back()->str = s;
  return g_pool.back().get();
}

mxArray *radial(const qd_radial &c)
{
  mxArray *m = strct();
  m->fields["n"] = view(&c.n);
  m->fields["r"] = view(c.r);
  m->fields["dr"] = view(&c.dr);
  m->fields["mass"] = view(&c.mass);
  return m;
}
}  // namespace

mxArray *mxGetField(const mxArray *mx, int, const char *field)
{
  if (!mx) return nullptr;
  auto it = mx->fields.find(field);
  return it == mx->fields.end() ? nullptr : it->second;
}
void *mxGetData(const mxArray *mx) { return mx ? mx->data : nullptr; }
double *mxGetPr(const mxArray *mx) { return (double *)mxGetData(mx); }
char *mxArrayToString(const mxArray *mx)
{
  if (!mx || !mx->is_string) return nullptr;
  char *s = (char *)malloc(mx->str.size() + 1);
  memcpy(s, mx->str.c_str(), mx->str.size() + 1);
  return s;
}
void mxFree(void *p) { free(p); }
void mexErrMsgTxt(const char *msg) { throw MexError(msg); }
int mexCallMATLAB(int, mxArray **, int, mxArray **, const char *) { return 0; }

/* ---- FFTW3 subset ------------------------------------------------------ */
struct qd_shim_plan { int n0, n1; double *data; int sign; };

fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *, int sign, unsigned)
{ return new qd_shim_plan{1, n, (double *)in, sign}; }
/* Row-major n0 x n1 (last index fastest) = column-major n1 x n0. */
fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex *in, fftw_complex *, int sign, unsigned)
{ return new qd_shim_plan{n0, n1, (double *)in, sign}; }
void fftw_execute(const fftw_plan p) { qdo_fft2d_threaded(p->data, p->n1, p->n0, p->sign); }
void fftw_destroy_plan(fftw_plan p) { delete p; }
int fftw_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int) {}

/* ---- Fortran kernels under their Fortran names (fort.h: FORT(x) x##_) --- */
extern "C" {
void forwardlegendretransform_(const double *CPsi, double *LPsi, const int &NR,
                               const int &NTheta, const int &NLeg, const double *WLegP)
{ qdo_forward_legendre(CPsi, LPsi, NR, NTheta, NLeg, WLegP); }
void backwardlegendretransform_(double *CPsi, const double *LPsi, const int &NR,
                                const int &NTheta, const int &NLeg, const double *LegP)
{ qdo_backward_legendre(CPsi, LPsi, NR, NTheta, NLeg, LegP); }
void gradient3d_(const int &N1, const int &N2, const int &N3, const int &N2P,
                 const double &Dx, const double *F, double *V, double *G, const int &NPoints)
{
  if (qdo_gradient3d(N1, N2, N3, N2P, Dx, F, V, G, NPoints))
    mexErrMsgTxt("NPoints error");   /* Gradient3.F:25 MCrash */
}
void psitimetopsienergyonsurface_(const int &N1, const int &NTheta, const int &NE,
                                  const double *ExpIETDt, const double *PsiT,
                                  const double *DPsiT, double *faiE, double *DFaiE)
{ qdo_psi_time_to_fai(N1, NTheta, NE, ExpIETDt, PsiT, DPsiT, faiE, DFaiE); }
void calculatecrp_(const int &N1, const int &NTheta, const int &NE, const double &Dr1,
                   const double &mu2, const double *W, const double *EtaSq,
                   const double *Fai, const double *DFai, double *CRP)
{ qdo_calculate_crp(N1, NTheta, NE, Dr1, mu2, W, EtaSq, Fai, DFai, CRP); }
}

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]);

/* Run the reference MEX entry point on d.  Returns 0 or -1 (error text in
 * err, up to errlen bytes).  verbose=0 discards the reference's per-step
 * console output. */
extern "C" int qdref_time_evolution(qd_data *d, int verbose, char *err, int errlen)
{
  g_pool.clear();
  mxArray *top = strct();
  top->fields["r1"] = radial(d->r1);
  top->fields["r2"] = radial(d->r2);
  mxArray *th = strct();
  th->fields["n"] = view(&d->theta.n);
  th->fields["m"] = view(&d->theta.m);
  th->fields["x"] = view(d->theta.x);
  th->fields["w"] = view(d->theta.w);
  th->fields["legendre"] = view(d->theta.legendre);
  top->fields["theta"] = th;
  top->fields["pot"] = view(d->pot);
  top->fields["psi"] = view(d->psi);
  mxArray *tm = strct();
  tm->fields["total_steps"] = view(&d->time.total_steps);
  tm->fields["time_step"] = view(&d->time.time_step);
  tm->fields["steps"] = view(&d->time.steps);
  top->fields["time"] = tm;
  mxArray *op = strct();
  if (d->options.test_name) op->fields["test_name"] = string(d->options.test_name);
  top->fields["options"] = op;
  mxArray *d1 = strct(), *d2 = strct();
  if (d->dump1.dump) d1->fields["dump"] = view(d->dump1.dump);
  if (d->dump2.dump) d2->fields["dump"] = view(d->dump2.dump);
  top->fields["dump1"] = d1;
  top->fields["dump2"] = d2;
  mxArray *crp = strct();
  crp->fields["n_dividing_surface"] = view(&d->CRP.n_dividing_surface);
  crp->fields["n_gradient_points"] = view(&d->CRP.n_gradient_points);
  crp->fields["n_energies"] = view(&d->CRP.n_energies);
  crp->fields["calculate_CRP"] = view(&d->CRP.calculate_CRP);
  crp->fields["energies"] = view(d->CRP.energies);
  crp->fields["eta_sq"] = view(d->CRP.eta_sq);
  crp->fields["CRP"] = view(d->CRP.CRP);
  top->fields["CRP"] = crp;

  std::ostringstream sink;
  std::streambuf *saved = nullptr;
  if (!verbose) saved = std::cout.rdbuf(sink.rdbuf());
  int rc = 0;
  try {
    const mxArray *args[1] = {top};
    mexFunction(0, nullptr, 1, args);
  } catch (const std::exception &e) {
    rc = -1;
    if (err && errlen > 0) { strncpy(err, e.what(), errlen - 1); err[errlen - 1] = 0; }
  }
  if (saved) std::cout.rdbuf(saved);
  g_pool.clear();
  return rc;
}
