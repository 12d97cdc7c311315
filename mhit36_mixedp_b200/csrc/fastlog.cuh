// Table-driven natural logarithm in float64 for the ACDI distance function.
//
// Method: P. T. P. Tang, "Table-driven implementation of the logarithm function in IEEE
// floating-point arithmetic", ACM TOMS 16(4), 1990.  x = 2^e m with m reduced to
// [sqrt(1/2), sqrt(2)); c = j/128 is the nearest table point (|m - c| <= 1/256, so f = m - c is
// exact by Sterbenz' lemma); r = f / c is formed as f * (1/c) with |r| < 0.0056, and
//   log x = e ln2 + log c + log1p(r),  log1p(r) = r - r^2/2 + r^3/3 - ... (through r^9/9).
// ln2 and log c are split in a high part and a low correction (ln2_hi has 42 significant bits,
// so e * ln2_hi is exact).  The table of log c and 1/c is computed on the host in 80-bit
// arithmetic.  For m near 1 the table point is c = 1 exactly, so log x = r + (series) without
// cancellation.  Non-positive, NaN, infinite and subnormal arguments fall back to CUDA's log,
// which keeps log(0) = -inf and log(x < 0) = NaN.
//
// Accuracy (tests/test_gpu_fastlog.py): within 2 ulp of numpy.log over 1e-300 .. 1e300.
#pragma once
#include <cuda_runtime.h>

namespace mhit {

constexpr int FASTLOG_J0 = 90;              // smallest table index: 90/128 < sqrt(1/2)
constexpr int FASTLOG_J1 = 182;             // one past the largest: 181/128 > sqrt(2)
constexpr int FASTLOG_N = FASTLOG_J1 - FASTLOG_J0;
// table layout (doubles): [0,N) log c hi | [N,2N) log c lo | [2N,3N) 1/c | ln2_hi | ln2_lo
constexpr int FASTLOG_TABLE_LEN = 3 * FASTLOG_N + 2;

__device__ __forceinline__ double fast_log(double x, const double* __restrict__ tab) {
  const int hi = __double2hiint(x);
  const int lo = __double2loint(x);
  const int bexp = (hi >> 20) & 0x7ff;
  if (!(x > 0.0) || bexp == 0 || bexp == 0x7ff) return log(x);  // 0, < 0, NaN, subnormal, inf
  int e = bexp - 1023;
  double m = __hiloint2double((hi & 0x000fffff) | 0x3ff00000, lo);  // [1, 2)
  if (m > 1.4142135623730951) {
    m = m * 0.5;
    e += 1;
  }
  const int j = __double2int_rz(fma(m, 128.0, 0.5));  // nearest j/128, in [90, 181]
  const double c = (double)j * 0.0078125;
  const double f = m - c;
  const double r = f * __ldg(tab + 2 * FASTLOG_N + (j - FASTLOG_J0));
  // log1p(r) - r, Horner in r
  double q = 1.0 / 9.0;
  q = fma(q, r, -1.0 / 8.0);
  q = fma(q, r, 1.0 / 7.0);
  q = fma(q, r, -1.0 / 6.0);
  q = fma(q, r, 1.0 / 5.0);
  q = fma(q, r, -0.25);
  q = fma(q, r, 1.0 / 3.0);
  q = fma(q, r, -0.5);
  q = q * (r * r);
  const double de = (double)e;
  const double big = fma(de, __ldg(tab + 3 * FASTLOG_N), __ldg(tab + (j - FASTLOG_J0)));
  const double small = fma(de, __ldg(tab + 3 * FASTLOG_N + 1), __ldg(tab + FASTLOG_N + (j - FASTLOG_J0)));
  return big + (r + (q + small));
}

}  // namespace mhit
