// Pressure of the mixed-precision Poisson modes built from two FP32 arrays.
//
// MHIT_POISSON_FP32_REFINED: the reference's FP32 branch solves lap p = rho/dt div u* once in
// FP32 (multi/main.f90:833-912).  With the discrete (modified-wavenumber) Laplacian the operator
// is the 7-point stencil L_h, so the FP32 pressure p32 is corrected once in FP64:
//   r = rho/dt div u* - L_h p32      (FP64, rounded to FP32: k_div_fftx's residual source)
//   L_h delta = r                    (a second FP32 solve, same kernels)
//   p = p32 + delta                  (in FP64 inside k_correct)
// which brings the projected divergence back to FP64 round-off.
// k_combine materialises that pressure in FP64 for a download.
#include "common.cuh"
#include "kernels.h"

namespace mhit {

__global__ void k_combine(const float* __restrict__ p32, const float* __restrict__ d32, double* __restrict__ p64,
                          size_t n) {
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x)
    p64[c] = (double)p32[c] + (double)d32[c];
}

cudaError_t launch_combine(const float* p32, const float* d32, double* p64, size_t n, cudaStream_t st) {
  k_combine<<<148 * 8, 256, 0, st>>>(p32, d32, p64, n);
  return cudaGetLastError();
}

}  // namespace mhit
