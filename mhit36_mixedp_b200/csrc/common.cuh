// Shared definitions for the MHIT36 B200 timestep kernels (sm_100a).
//
// Field layout in HBM: every 3-D field is an x-fastest (nx, ny, nz) array without halo
// planes -- the layout of the reference's field files (multi/readwrite.f90:28-46).  The
// reference's y/z halo planes (multi/main.f90:93, refreshed by cudecompUpdateHalosX at 28
// call sites) are replaced by periodic index arithmetic inside the kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace mhit {

template <typename T> struct Cx { T x, y; };
template <> struct __align__(16) Cx<double> { double x, y; };
template <> struct __align__(8) Cx<float> { float x, y; };

template <typename T> __device__ __forceinline__ Cx<T> cx(T a, T b) { Cx<T> r; r.x = a; r.y = b; return r; }
template <typename T> __device__ __forceinline__ Cx<T> operator+(Cx<T> a, Cx<T> b) { return cx<T>(a.x + b.x, a.y + b.y); }
template <typename T> __device__ __forceinline__ Cx<T> operator-(Cx<T> a, Cx<T> b) { return cx<T>(a.x - b.x, a.y - b.y); }
template <typename T> __device__ __forceinline__ Cx<T> cmul(Cx<T> a, Cx<T> b) {
  return cx<T>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename T> __device__ __forceinline__ Cx<T> conj(Cx<T> a) { return cx<T>(a.x, -a.y); }
template <typename T> __device__ __forceinline__ Cx<T> scale(Cx<T> a, T s) { return cx<T>(a.x * s, a.y * s); }
// multiply by -i (forward) or +i (inverse)
template <typename T, bool INV> __device__ __forceinline__ Cx<T> mul_mi(Cx<T> a) {
  return INV ? cx<T>(-a.y, a.x) : cx<T>(a.y, -a.x);
}

// Per-context device-resident scalars, written by the reduction kernels and read by the
// next step's kernels (no host round trip inside a step).
struct DevScalars {
  double mean[3];      // mean of u,v,w removed lazily (multi/main.f90:967-981)
  double gumax;        // signed max over u,v,w after mean removal (multi/main.f90:998-1002)
  double cfl;          // gumax*dt*dxi (multi/main.f90:1003)
  int flag;            // bit0: NaN seen, bit1: CFL > 7 (multi/main.f90:1006)
  int pad;
  double diag[8];      // on-demand diagnostics: maxdiv, ke, eps, ...
};

// Geometry and physical constants passed by value to every kernel.
struct Geo {
  int nx, ny, nz;
  int nkx;      // nx/2+1
  int pitch;    // padded row pitch of the spectrum, in complex elements
  double dt, dx, dxi, ddxi, rhoi, mu, rho, eps, epsi, sigma;
  double f1, f2, f3;
};

// max that propagates NaN (fmax returns the other operand): a NaN anywhere in a reduced field
// shows up in the reduced maximum
__device__ __forceinline__ double nanmax(double a, double b) { return (a != a) ? a : ((b != b) ? b : fmax(a, b)); }

__device__ __forceinline__ int wrapp(int i, int n) { return (i + 1 == n) ? 0 : i + 1; }
__device__ __forceinline__ int wrapm(int i, int n) { return (i == 0) ? n - 1 : i - 1; }
__device__ __forceinline__ size_t lin(int i, int j, int k, int nx, int ny) {
  return ((size_t)k * ny + j) * nx + i;
}

}  // namespace mhit

#define MHIT_CUDA_TRY(expr)                                                      \
  do {                                                                           \
    cudaError_t _e = (expr);                                                     \
    if (_e != cudaSuccess) return ::mhit::set_cuda_error(_e, #expr, __FILE__, __LINE__); \
  } while (0)
