/* mex.h -- TEST INFRASTRUCTURE ONLY.  Minimal stand-in for Matlab's MEX/mx
 * API, just enough to compile the reference's CPU propagator
 * (common/TimeEvolutionMex.C, common/MatlabStructures.C, common/matutils.*,
 * common/wave2matlab.C) without Matlab.  An mxArray is either a struct
 * (named fields) or a non-owning view of caller memory. */
#ifndef QD_SHIM_MEX_H
#define QD_SHIM_MEX_H
#include <cstddef>
#include <cstdio>   /* Matlab's mex.h pulls in stdio.h */
#include <unistd.h>

struct mxArray;

mxArray *mxGetField(const mxArray *mx, int index, const char *field);
void *mxGetData(const mxArray *mx);
double *mxGetPr(const mxArray *mx);
char *mxArrayToString(const mxArray *mx);
void mxFree(void *p);
void mexErrMsgTxt(const char *msg);
int mexCallMATLAB(int nlhs, mxArray *plhs[], int nrhs, mxArray *prhs[], const char *name);

#endif
