// qd_tc.h -- tensor-core (tcgen05) column pass for the complex64 propagation.
#pragma once
#include <cuda_runtime.h>
#include "qd_kernels.h"

struct TcPlan {
  int nth = 0, nl = 0;          // true sizes
  int mth = 0, ml = 0;          // padded sizes (MMA M and K multiples)
  void *mats = nullptr;         // device: split (hi, lo) tf32 operand images
  size_t mats_bytes = 0;
  int smem_bytes = 0;
  int grid = 0;
};

// Build the operand images of the two Legendre matrices; returns
// QD_ERR_UNSUPPORTED when the sizes are outside what the kernel handles.
int tc_plan_create(TcPlan &plan, int nth, int nl, const double *dP, const double *dWP,
                   cudaStream_t s);
void tc_plan_destroy(TcPlan &plan);
cudaError_t launch_column_tc(const TcPlan &plan, const ColumnParams &p, int mode,
                             cudaStream_t s);
