// qd_tc.h -- tensor-core (tcgen05) column pass for the complex64 propagation.
#pragma once
#include <cuda_runtime.h>
#include "qd_kernels.h"

struct TcPlan {
  int nth = 0, nl = 0;          // true sizes
  int S = 0;                    // max(n_l, n_theta) padded to 16 (MMA N and K)
  int renorm = 0;               // per-column isometry rescaling (n_l <= n_theta, Gauss nodes)
  void *mats = nullptr;         // device: B1, B2 hi|mid|lo images, then an int status word
  size_t mats_bytes = 0;
  int smem_bytes = 0;
  int grid = 0;
};

// Build the operand images of the two Legendre matrices from the host
// theta.legendre ((m+1) x n column-major), weights and nodes; returns
// QD_ERR_UNSUPPORTED when the sizes are outside what the kernel handles.
int tc_plan_create(TcPlan &plan, int nth, int nl, const double *legendre, const double *w,
                   const double *x, cudaStream_t s);
void tc_plan_destroy(TcPlan &plan);
// Device status word: 0 = ok, non-zero = a bounded wait in the kernel expired.
int *tc_status_ptr(const TcPlan &plan);
cudaError_t launch_column_tc(const TcPlan &plan, const ColumnParams &p, int mode,
                             cudaStream_t s);
