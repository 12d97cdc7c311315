// Field statistics of caller-owned device arrays without any device allocation.
//
// mhit_diagnostics computes max|div u|, the kinetic energy and the dissipation with a partials
// buffer that mhit_init allocates.  Some callers cannot let a library allocate: a Fortran host
// whose device arrays belong to its compiler runtime (OpenACC / CUDA Fortran) and that only
// wants statistics of fields it already holds, or a run that has committed almost all of the
// GPU's memory (a 1024^3 box) where one more cudaMalloc can fail and a cudaFree would
// synchronise the whole device in the middle of the timestep loop.  mhit_field_stats_noalloc
// serves them: the caller passes the three velocity arrays and a 3-double output on the device,
// and the only scratch is the file-scope array below, one partial-result slot per z plane.
//
// The array lives in every GPU that loads the library until the process exits (32 KB).  Its
// host-side symbol is not a device address: the address is looked up with cudaGetSymbolAddress
// by the first call made on a device, and again whenever the CUDA context current on that
// device has changed since (after a cudaDeviceReset the old address belongs to a destroyed
// context).  All calls share the array: two calls whose kernels overlap on the GPU (different
// streams, or different host threads on the same device) race on it and must be serialised by
// the caller.  Each call writes the slots of planes 0..nz-1 before it reads them, so nothing has
// to start at zero.
//
// The kinetic energy is that of the arrays as passed: no mean is removed (mhit_diagnostics
// subtracts its context's lazily removed mean first; on fields downloaded from a context, or
// with zero mean, the two agree).  A NaN anywhere in u, v or w makes stats[0] (and stats[1])
// NaN: the maxima propagate NaN instead of dropping it.
#include <cmath>
#include <cstdio>
#include <mutex>
#include <string>

#include "../../include/mhit_b200.h"
#include "common.cuh"
#include "kernels.h"

namespace mhit {

int set_error(int code, const std::string& msg);

namespace {

constexpr int STATS_NT = 256;
constexpr int STATS_SLOT = 4;  // maxdiv, sum u.u, sum S:S, unused

static __device__ __align__(256) double g_stats_scratch[MHIT_STATS_NOALLOC_MAX_PLANES * STATS_SLOT];

// one block per z plane: max |div|, sum of u.u and of S_ij S_ij over the plane
__global__ void __launch_bounds__(STATS_NT) k_stats_planes(int nx, int ny, int nz, double dxi, double h,
                                                           const double* __restrict__ U,
                                                           const double* __restrict__ V,
                                                           const double* __restrict__ W, double* __restrict__ slots) {
  const int k = blockIdx.x;
  const int kp = wrapp(k, nz), km = wrapm(k, nz);
  const int nplane = nx * ny;
  double mdiv = 0.0, ke = 0.0, ss = 0.0;
  for (int e = threadIdx.x; e < nplane; e += STATS_NT) {
    const int j = e / nx, i = e - j * nx;
    const int ip = wrapp(i, nx), im = wrapm(i, nx), jp = wrapp(j, ny), jm = wrapm(j, ny);
#define F(A, ii, jj, kk) __ldg(A + lin(ii, jj, kk, nx, ny))
    const double u0 = F(U, i, j, k), v0 = F(V, i, j, k), w0 = F(W, i, j, k);
    const double div = (F(U, ip, j, k) - u0) * dxi + (F(V, i, jp, k) - v0) * dxi + (F(W, i, j, kp) - w0) * dxi;
    mdiv = nanmax(mdiv, fabs(div));
    ke += u0 * u0 + v0 * v0 + w0 * w0;
    const double dudx = (F(U, ip, j, k) - F(U, im, j, k)) * h;
    const double dudy = (F(U, i, jp, k) - F(U, i, jm, k)) * h;
    const double dudz = (F(U, i, j, kp) - F(U, i, j, km)) * h;
    const double dvdx = (F(V, ip, j, k) - F(V, im, j, k)) * h;
    const double dvdy = (F(V, i, jp, k) - F(V, i, jm, k)) * h;
    const double dvdz = (F(V, i, j, kp) - F(V, i, j, km)) * h;
    const double dwdx = (F(W, ip, j, k) - F(W, im, j, k)) * h;
    const double dwdy = (F(W, i, jp, k) - F(W, i, jm, k)) * h;
    const double dwdz = (F(W, i, j, kp) - F(W, i, j, km)) * h;
#undef F
    const double s12 = 0.5 * (dudy + dvdx), s13 = 0.5 * (dudz + dwdx), s23 = 0.5 * (dvdz + dwdy);
    ss += dudx * dudx + dvdy * dvdy + dwdz * dwdz + 2.0 * (s12 * s12 + s13 * s13 + s23 * s23);
  }
  __shared__ double red[3][STATS_NT / 32];
  double vals[3] = {mdiv, ke, ss};
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    double x = vals[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double y = __shfl_down_sync(0xffffffffu, x, o);
      x = q == 0 ? nanmax(x, y) : x + y;
    }
    if ((threadIdx.x & 31) == 0) red[q][threadIdx.x >> 5] = x;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    const int q = threadIdx.x;
    double x = red[q][0];
    for (int wv = 1; wv < STATS_NT / 32; ++wv) x = q == 0 ? nanmax(x, red[q][wv]) : x + red[q][wv];
    slots[(size_t)k * STATS_SLOT + q] = x;
  }
}

// reduce the nz plane slots in a fixed order and write maxdiv, KE, dissipation
__global__ void __launch_bounds__(1024) k_stats_reduce(const double* __restrict__ slots, int nx, int ny, int nz,
                                                       double nu, double* __restrict__ out) {
  __shared__ double red[3][32];
  double vals[3] = {0.0, 0.0, 0.0};
  for (int k = threadIdx.x; k < nz; k += blockDim.x) {
    vals[0] = nanmax(vals[0], slots[(size_t)k * STATS_SLOT + 0]);
    vals[1] += slots[(size_t)k * STATS_SLOT + 1];
    vals[2] += slots[(size_t)k * STATS_SLOT + 2];
  }
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    double x = vals[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double y = __shfl_down_sync(0xffffffffu, x, o);
      x = q == 0 ? nanmax(x, y) : x + y;
    }
    if ((threadIdx.x & 31) == 0) red[q][threadIdx.x >> 5] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int nw = (blockDim.x + 31) / 32;
    double r[3];
    for (int q = 0; q < 3; ++q) {
      double x = red[q][0];
      for (int wv = 1; wv < nw; ++wv) x = q == 0 ? nanmax(x, red[q][wv]) : x + red[q][wv];
      r[q] = x;
    }
    const double n = (double)nx * ny * nz;
    out[0] = r[0];
    out[1] = 0.5 * r[1] / n;
    out[2] = 2.0 * nu * r[2] / n;
  }
}

std::mutex g_scratch_mutex;
struct ScratchSlot {
  void* ctx = nullptr;   // CUDA context the address belongs to
  void* addr = nullptr;  // device address of g_stats_scratch in that context
};
ScratchSlot g_scratch[64];

// The driver's cuCtxGetCurrent, reached through the runtime (the library links only cudart).
using CtxGetCurrentFn = int (*)(void**);
CtxGetCurrentFn ctx_get_current() {
  static CtxGetCurrentFn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<CtxGetCurrentFn>(p);
  }
  return fn;
}

void* current_context() {
  void* ctx = nullptr;
  CtxGetCurrentFn fn = ctx_get_current();
  if (fn && fn(&ctx) != 0) ctx = nullptr;
  return ctx;
}

// Device address of g_stats_scratch on the current device, looked up on the first call and
// again whenever the current context differs from the one the cached address belongs to.
int scratch_address(int dev, void** out) {
  if (dev < 0 || dev >= 64) return set_error(MHIT_ERR_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  ScratchSlot& slot = g_scratch[dev];
  void* ctx = current_context();
  if (!slot.addr || !ctx || ctx != slot.ctx) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_stats_scratch);
    if (e != cudaSuccess) return set_cuda_error(e, "cudaGetSymbolAddress(g_stats_scratch)", __FILE__, __LINE__);
    slot.addr = p;
    slot.ctx = current_context();  // the lookup made the device's primary context current if none was
  }
  *out = slot.addr;
  return MHIT_OK;
}

}  // namespace
}  // namespace mhit

extern "C" int mhit_field_stats_noalloc(int nx, int ny, int nz, double nu, const double* u, const double* v,
                                        const double* w, double* stats, void* stream) {
  using namespace mhit;
  if (!u || !v || !w || !stats) return set_error(MHIT_ERR_ARG, "null device pointer");
  if (nx < 2 || ny < 2 || nz < 2) return set_error(MHIT_ERR_ARG, "nx, ny and nz must be at least 2");
  if (nz > MHIT_STATS_NOALLOC_MAX_PLANES) {
    char b[160];
    snprintf(b, sizeof(b), "nz = %d exceeds the %d z planes of the no-allocation scratch", nz,
             MHIT_STATS_NOALLOC_MAX_PLANES);
    return set_error(MHIT_ERR_ARG, b);
  }
  if ((long long)nx * ny > (1LL << 30)) return set_error(MHIT_ERR_ARG, "nx*ny too large");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return set_cuda_error(e, "cudaGetDevice", __FILE__, __LINE__);
  void* scratch = nullptr;
  int rc = scratch_address(dev, &scratch);
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const double dx = 8.0 * atan(1.0) / nx;  // lx/nx as multi/readinput.f90:115-117
  const double dxi = 1.0 / dx, h = 0.5 / dx;
  k_stats_planes<<<nz, STATS_NT, 0, st>>>(nx, ny, nz, dxi, h, u, v, w, static_cast<double*>(scratch));
  e = cudaGetLastError();
  if (e != cudaSuccess) return set_cuda_error(e, "k_stats_planes launch", __FILE__, __LINE__);
  k_stats_reduce<<<1, 1024, 0, st>>>(static_cast<const double*>(scratch), nx, ny, nz, nu, stats);
  e = cudaGetLastError();
  if (e != cudaSuccess) return set_cuda_error(e, "k_stats_reduce launch", __FILE__, __LINE__);
  return MHIT_OK;
}
