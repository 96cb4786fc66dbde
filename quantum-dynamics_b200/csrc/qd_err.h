// qd_err.h -- error reporting shared by the library's translation units.
#pragma once
#include <cstdarg>
#include <cstdio>
#include <cuda_runtime.h>
#include "qd.h"

int qd_set_error(int code, const char *msg);     // sets qd_last_error(), returns code
void qd_count_launches(int n);                    // qd_kernel_launch_count bookkeeping

inline int qd_errf(int code, const char *fmt, ...)
{
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  return qd_set_error(code, buf);
}

#define QD_CU(x)                                                                        \
  do {                                                                                  \
    cudaError_t e_ = (x);                                                               \
    if (e_ != cudaSuccess)                                                              \
      return qd_errf(QD_ERR_CUDA, "%s failed: %s (%s:%d)", #x, cudaGetErrorString(e_),   \
                     __FILE__, __LINE__);                                               \
  } while (0)
