// FP64 residual sweep of the mixed-precision Poisson solve (MHIT_POISSON_FP32_REFINED).
//
// The reference's FP32 branch solves lap p = rho/dt div u* once in FP32 (multi/main.f90:833-912).
// With the discrete (modified-wavenumber) Laplacian the operator is the 7-point stencil L_h, so
// the FP32 pressure p32 can be corrected once in FP64:
//   r = rho/dt div u* - L_h p32      (this kernel, FP64, stored as FP32)
//   L_h delta = r                    (a second FP32 solve, same kernels)
//   p = p32 + delta                  (in FP64 inside k_correct)
// which brings the projected divergence back to FP64 round-off.  The right-hand side is
// recomputed from u* in the same operation order as k_div_fftx (:841-843).
#include "common.cuh"
#include "kernels.h"

namespace mhit {

__global__ void __launch_bounds__(256) k_residual(ResidArgs a) {
  const Geo& g = a.g;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int i = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 8 + threadIdx.y, k = blockIdx.z;
  if (i >= nx || j >= ny) return;
  const int ip = wrapp(i, nx), im = wrapm(i, nx), jp = wrapp(j, ny), jm = wrapm(j, ny);
  const int kp = wrapp(k, nz), km = wrapm(k, nz);
  const size_t c = lin(i, j, k, nx, ny);
  const double cd = a.cdiv, ddxi = g.ddxi;
  double rhs = cd * (__ldg(a.u + lin(ip, j, k, nx, ny)) - __ldg(a.u + c));
  rhs = rhs + cd * (__ldg(a.v + lin(i, jp, k, nx, ny)) - __ldg(a.v + c));
  rhs = rhs + cd * (__ldg(a.w + lin(i, j, kp, nx, ny)) - __ldg(a.w + c));
  const double p0 = (double)__ldg(a.p + c);
  const double lap = ((double)__ldg(a.p + lin(ip, j, k, nx, ny)) - 2.0 * p0 + (double)__ldg(a.p + lin(im, j, k, nx, ny))) * ddxi +
                     ((double)__ldg(a.p + lin(i, jp, k, nx, ny)) - 2.0 * p0 + (double)__ldg(a.p + lin(i, jm, k, nx, ny))) * ddxi +
                     ((double)__ldg(a.p + lin(i, j, kp, nx, ny)) - 2.0 * p0 + (double)__ldg(a.p + lin(i, j, km, nx, ny))) * ddxi;
  a.r[c] = (float)(rhs - lap);
}

__global__ void k_combine(const float* __restrict__ p32, const float* __restrict__ d32, double* __restrict__ p64,
                          size_t n) {
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x)
    p64[c] = (double)p32[c] + (double)d32[c];
}

cudaError_t launch_combine(const float* p32, const float* d32, double* p64, size_t n, cudaStream_t st) {
  k_combine<<<148 * 8, 256, 0, st>>>(p32, d32, p64, n);
  return cudaGetLastError();
}

cudaError_t launch_residual(const ResidArgs& a, cudaStream_t st) {
  dim3 blk(32, 8);
  dim3 grd((a.g.nx + 31) / 32, (a.g.ny + 7) / 8, a.g.nz);
  k_residual<<<grd, blk, 0, st>>>(a);
  return cudaGetLastError();
}

}  // namespace mhit
