// Host table of the table-driven logarithm (fastlog.cuh) and its test hook.
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/mhit_b200.h"
#include "fastlog.cuh"
#include "kernels.h"

namespace mhit {

int set_error(int code, const std::string& msg);

// log c (split hi + lo) and 1/c for c = j/128, j in [90, 182), plus ln2 split so that
// e * ln2_hi is exact (ln2_hi has 42 significant bits).  80-bit arithmetic on the host.
std::vector<double> fastlog_table() {
  std::vector<double> t(FASTLOG_TABLE_LEN);
  for (int j = FASTLOG_J0; j < FASTLOG_J1; ++j) {
    const long double c = (long double)j / 128.0L;
    const long double lc = logl(c);
    const double h = (double)lc;
    t[j - FASTLOG_J0] = h;
    t[FASTLOG_N + j - FASTLOG_J0] = (double)(lc - (long double)h);
    t[2 * FASTLOG_N + j - FASTLOG_J0] = (double)(1.0L / c);
  }
  const long double ln2 = logl(2.0L);
  const double ln2_hi = (double)(floorl(ln2 * 4398046511104.0L) / 4398046511104.0L);  // 2^42
  t[3 * FASTLOG_N] = ln2_hi;
  t[3 * FASTLOG_N + 1] = (double)(ln2 - (long double)ln2_hi);
  return t;
}

__global__ void k_fastlog_probe(const double* __restrict__ x, double* __restrict__ y, int n,
                                const double* __restrict__ tab) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = fast_log(x[i], tab);
}

}  // namespace mhit

// Test hook: y = fast_log(x) for n host values (allocates; tests only).
extern "C" int mhit_debug_fastlog(const double* x, double* y, int n) {
  using namespace mhit;
  if (!x || !y || n < 0) return set_error(MHIT_ERR_ARG, "bad argument");
  if (n == 0) return MHIT_OK;
  std::vector<double> t = fastlog_table();
  double *dx = nullptr, *dy = nullptr, *dt = nullptr;
  const size_t b = (size_t)n * sizeof(double);
  int rc = MHIT_OK;
  cudaError_t e;
  if ((e = cudaMalloc(&dx, b)) != cudaSuccess || (e = cudaMalloc(&dy, b)) != cudaSuccess ||
      (e = cudaMalloc(&dt, t.size() * sizeof(double))) != cudaSuccess ||
      (e = cudaMemcpy(dx, x, b, cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemcpy(dt, t.data(), t.size() * sizeof(double), cudaMemcpyHostToDevice)) != cudaSuccess) {
    rc = set_cuda_error(e, "fastlog probe setup", __FILE__, __LINE__);
  } else {
    k_fastlog_probe<<<256, 256>>>(dx, dy, n, dt);
    if ((e = cudaGetLastError()) != cudaSuccess || (e = cudaMemcpy(y, dy, b, cudaMemcpyDeviceToHost)) != cudaSuccess)
      rc = set_cuda_error(e, "fastlog probe", __FILE__, __LINE__);
  }
  cudaFree(dx);
  cudaFree(dy);
  cudaFree(dt);
  return rc;
}
