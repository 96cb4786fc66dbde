// qd_cs.cu -- angular basis of a centrifugal-sudden block (J, K): the
// associated Legendre functions of order K normalised to one on [-1, 1],
// in the layout and scaling of the reference's theta.legendre
// (H3/main.m:98-101, common/LegendreP2.m:9-21 for K = 0).
#include <cmath>
#include <vector>
#include "qd_err.h"

extern "C" int qd_cs_legendre(int32_t n, int32_t K, int32_t m, const double *x, double *leg)
{
  if (!x || !leg || n < 1 || m < 0 || K < 0)
    return qd_errf(QD_ERR_INVALID, "qd_cs_legendre: bad argument (n %d, K %d, m %d)", n, K, m);
  const long ld = m + 1;                         // leg[l + k*(m+1)]
  for (int k = 0; k < n; k++) {
    double *col = leg + (long)k * ld;
    const double xk = x[k];
    if (K == 0) {                                // P_l by the recurrence of LegendreP2.m
      double p0 = 1.0, p1 = xk;
      col[0] = 1.0;
      if (m >= 1) col[1] = xk;
      for (int l = 2; l <= m; l++) {
        const double p2 = (2.0 - 1.0 / l) * xk * p1 - (1.0 - 1.0 / l) * p0;
        col[l] = p2;
        p0 = p1;
        p1 = p2;
      }
      continue;
    }
    const double s = std::sqrt(1.0 - xk * xk);
    double p0 = std::sqrt(0.5);                  // Pbar_0^0
    for (int mm = 1; mm <= K; mm++) p0 *= std::sqrt((2.0 * mm + 1.0) / (2.0 * mm)) * s;
    col[0] = p0;                                 // Pbar_K^K
    double p1 = 0.0;
    if (m >= 1) {
      p1 = std::sqrt(2.0 * K + 3.0) * xk * p0;   // Pbar_{K+1}^K
      col[1] = p1;
    }
    for (int l = 2; l <= m; l++) {
      const double j = K + l;
      const double a = std::sqrt((4.0 * j * j - 1.0) / (j * j - (double)K * K));
      const double b = std::sqrt(((j - 1) * (j - 1) - (double)K * K) / (4.0 * (j - 1) * (j - 1) - 1.0));
      const double p2 = a * (xk * p1 - b * p0);
      col[l] = p2;
      p0 = p1;
      p1 = p2;
    }
    for (int l = 0; l <= m; l++) col[l] /= std::sqrt(l + 0.5);
  }
  return QD_OK;
}
