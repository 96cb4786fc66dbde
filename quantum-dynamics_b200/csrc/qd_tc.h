// qd_tc.h -- tensor-core (tcgen05) column pass for the complex64 propagation.
#pragma once
#include <cuda_runtime.h>
#include "qd_kernels.h"

struct TcPlan {
  int nth = 0, nl = 0;          // n_theta; n_l of the state layout (max over the sets)
  int S = 0;                    // max(n_l, n_theta) padded to 16 (MMA N and K)
  int renorm = 0;               // per-column isometry rescaling (orthonormal Q columns)
  int nsets = 0;                // angular bases (one operand image set each)
  size_t set_bytes = 0;         // bytes of one image set: Q hi|lo (FP16, times 2^12)
  void *mats = nullptr;         // device: the image sets, then an int status word
  size_t mats_bytes = 0;
  int smem_bytes = 0;
  int grid = 0;
};

// Build the operand images of the Legendre transform pair of each angular
// basis from the host theta.legendre matrices (leg[t]: nl_set[t] x n_theta,
// column-major, the reference's layout) and the weights; returns
// QD_ERR_UNSUPPORTED when the sizes are outside what the kernel handles.
int tc_plan_create(TcPlan &plan, int nth, int nl, int nsets, const double *const *leg,
                   const int *nl_set, const double *w, cudaStream_t s);
void tc_plan_destroy(TcPlan &plan, cudaStream_t s);   // stream-ordered free
// Device status word: 0 = ok, non-zero = a bounded wait in the kernel expired.
int *tc_status_ptr(const TcPlan &plan);
cudaError_t launch_column_tc(const TcPlan &plan, const ColumnParams &p, int mode,
                             cudaStream_t s);
