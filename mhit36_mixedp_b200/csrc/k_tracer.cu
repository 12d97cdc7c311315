// Lagrangian tracers: multi/main.f90:477-508 on one GPU (no sort, count or migration).
//
// Per tracer: velocity at the position (1-D linear per component as the reference,
// multi/particles.f90:96-117, or trilinear at the staggered face positions), AB2 position
// update with the flow's alpha/beta (:480-486), periodic wrap x - lx floor(x/lx)
// (multi/particles.f90:372-376), history shift u1 = u (:503-508).
//
// Table layout: structure of arrays, 12 columns of npmax doubles in the reference's column
// order (multi/particles.f90:17-22): tag, x, y, z, u, v, w, phi, u1, v1, w1, phi1.
// Reference y/z labelling: local index 1+floor(y/dx) is global plane floor(y/dx) - yz_shift.
#include "common.cuh"
#include "kernels.h"

namespace mhit {

__device__ __forceinline__ int pmod(long long i, int n) {
  long long r = i % n;
  return (int)(r < 0 ? r + n : r);
}

__device__ __forceinline__ double tri(const double* __restrict__ f, double m, const Geo& g, double x, double y,
                                      double z) {
  const double ix = floor(x), iy = floor(y), iz = floor(z);
  const double tx = x - ix, ty = y - iy, tz = z - iz;
  const int a0 = pmod((long long)ix, g.nx), a1 = pmod((long long)ix + 1, g.nx);
  const int b0 = pmod((long long)iy, g.ny), b1 = pmod((long long)iy + 1, g.ny);
  const int c0 = pmod((long long)iz, g.nz), c1 = pmod((long long)iz + 1, g.nz);
  const int nx = g.nx, ny = g.ny;
#define L(a, b, c) (__ldg(f + lin(a, b, c, nx, ny)) - m)
  const double c00 = (1.0 - tx) * L(a0, b0, c0) + tx * L(a1, b0, c0);
  const double c10 = (1.0 - tx) * L(a0, b1, c0) + tx * L(a1, b1, c0);
  const double c01 = (1.0 - tx) * L(a0, b0, c1) + tx * L(a1, b0, c1);
  const double c11 = (1.0 - tx) * L(a0, b1, c1) + tx * L(a1, b1, c1);
#undef L
  const double d0 = (1.0 - ty) * c00 + ty * c10;
  const double d1 = (1.0 - ty) * c01 + ty * c11;
  return (1.0 - tz) * d0 + tz * d1;
}

__global__ void __launch_bounds__(256) k_tracer(TracerArgs a) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= a.np) return;
  const Geo& g = a.g;
  const size_t S = (size_t)a.npmax;
  double* P = a.part;
  const double dx = g.dx;
  const double mu_ = a.sc->mean[0], mv_ = a.sc->mean[1], mw_ = a.sc->mean[2];
  double x = P[1 * S + q], y = P[2 * S + q], z = P[3 * S + q];
  double up, vp, wp;
  const int s = a.yz_shift;
  if (a.interp == 0) {
    // multi/particles.f90:96-117
    const double fx = floor(x / dx), fy = floor(y / dx), fz = floor(z / dx);
    const double tx = x / dx - fx, ty = y / dx - fy, tz = z / dx - fz;
    const int i0 = pmod((long long)fx, g.nx), i1 = pmod((long long)fx + 1, g.nx);
    const int j0 = pmod((long long)fy - s, g.ny), j1 = pmod((long long)fy - s + 1, g.ny);
    const int k0 = pmod((long long)fz - s, g.nz), k1 = pmod((long long)fz - s + 1, g.nz);
    const int nx = g.nx, ny = g.ny;
    up = (1.0 - tx) * (__ldg(a.u + lin(i0, j0, k0, nx, ny)) - mu_) + tx * (__ldg(a.u + lin(i1, j0, k0, nx, ny)) - mu_);
    vp = (1.0 - ty) * (__ldg(a.v + lin(i0, j0, k0, nx, ny)) - mv_) + ty * (__ldg(a.v + lin(i0, j1, k0, nx, ny)) - mv_);
    wp = (1.0 - tz) * (__ldg(a.w + lin(i0, j0, k0, nx, ny)) - mw_) + tz * (__ldg(a.w + lin(i0, j0, k1, nx, ny)) - mw_);
  } else {
    const double xs = x / dx, ys = y / dx, zs = z / dx;
    up = tri(a.u, mu_, g, xs + 0.5, ys - s, zs - s);
    vp = tri(a.v, mv_, g, xs, ys - (s - 0.5), zs - s);
    wp = tri(a.w, mw_, g, xs, ys - s, zs - (s - 0.5));
  }
  P[4 * S + q] = up;
  P[5 * S + q] = vp;
  P[6 * S + q] = wp;
  const double dt = g.dt, al = a.alpha, be = a.beta, lx = a.lx;
  // multi/main.f90:483-484
  x = x + dt * (al * up - be * P[8 * S + q]);
  y = y + dt * (al * vp - be * P[9 * S + q]);
  z = z + dt * (al * wp - be * P[10 * S + q]);
  // multi/particles.f90:372-376
  x = x - lx * floor(x / lx);
  y = y - lx * floor(y / lx);
  z = z - lx * floor(z / lx);
  P[1 * S + q] = x;
  P[2 * S + q] = y;
  P[3 * S + q] = z;
  // multi/main.f90:506
  P[8 * S + q] = up;
  P[9 * S + q] = vp;
  P[10 * S + q] = wp;
}

cudaError_t launch_tracer(const TracerArgs& a, cudaStream_t st) {
  if (a.np <= 0) return cudaSuccess;
  k_tracer<<<(a.np + 255) / 256, 256, 0, st>>>(a);
  return cudaGetLastError();
}

}  // namespace mhit
