// k_column_tc.cu -- tensor-core column pass (placeholder until the tcgen05
// kernel lands: reports the sizes as unsupported so the SIMT pass runs).
#include "qd.h"
#include "qd_tc.h"

int tc_plan_create(TcPlan &, int, int, const double *, const double *, cudaStream_t)
{
  return QD_ERR_UNSUPPORTED;
}

void tc_plan_destroy(TcPlan &) {}

cudaError_t launch_column_tc(const TcPlan &, const ColumnParams &, int, cudaStream_t)
{
  return cudaErrorNotSupported;
}
