// ACDI phase-field transport: multi/main.f90:522-636 in one kernel.
//
// The reference makes five passes with three stored intermediates (psidi, tanh_psi and the
// three normal components) and six halo exchanges.  Here a block owns a PTX x PTY column of
// cells and marches up a chunk of z planes keeping two rings of three planes in shared
// memory:
//   psi   = eps log((min(phi,1)+1e-16)/(1-min(phi,1)+1e-16))           (:527-528), halo 2
//   F     = 1/4 (1 - tanh(psi/(2 eps))^2) n/(|n|+1e-16), n = central psi differences
//           (:530, :559-561, :586-589, :609-614), halo 1
// and writes only phi^{n+1} and rhsphi_o.  psi and F are recomputed for the halo of the tile
// (x-y recompute factor (PTX+4)(PTY+4)/(PTX PTY)).  gamma = 1.0*gumax is read from the
// device scalars written by the previous projection (:536, :998-1002).
#include "common.cuh"
#include "kernels.h"

namespace mhit {

constexpr int PTX = 32, PTY = 8;
constexpr int PHX = PTX + 4, PHY = PTY + 4;  // psi tile (halo 2)
constexpr int PFX = PTX + 2, PFY = PTY + 2;  // F tile (halo 1)
constexpr int PNT = PTX * PTY;
constexpr int PZCHUNK = 32;
constexpr double ENUM = 1.0e-16;

__device__ __forceinline__ int wrapn(int i, int n) {
  i %= n;
  return i < 0 ? i + n : i;
}

__global__ void __launch_bounds__(PNT) k_phase(PhaseArgs a) {
  __shared__ double spsi[3][PHY][PHX];
  __shared__ double sF[3][3][PFY][PFX];
  const Geo& g = a.g;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int i0 = blockIdx.x * PTX, j0 = blockIdx.y * PTY;
  const int k0 = blockIdx.z * PZCHUNK;
  const int k1 = min(k0 + PZCHUNK, nz);
  const int tid = threadIdx.x;
  const double eps = g.eps, epsi = g.epsi;
  const double* __restrict__ phi = a.phi;

  auto slot = [&](int m) { return (m - k0 + 6) % 3; };
  auto psi_plane = [&](int m) {
    const int kw = wrapn(m, nz);
    const int s = slot(m);
    for (int e = tid; e < PHX * PHY; e += PNT) {
      const int y = e / PHX, x = e - y * PHX;
      const int gi = wrapn(i0 - 2 + x, nx), gj = wrapn(j0 - 2 + y, ny);
      const double val = fmin(__ldg(phi + lin(gi, gj, kw, nx, ny)), 1.0);
      spsi[s][y][x] = eps * log((val + ENUM) / (1.0 - val + ENUM));
    }
  };
  auto F_plane = [&](int m) {
    const int sm = slot(m - 1), s0 = slot(m), sp = slot(m + 1);
    const int sf = slot(m);
    for (int e = tid; e < PFX * PFY; e += PNT) {
      const int y = e / PFX, x = e - y * PFX;
      const int px = x + 1, py = y + 1;
      const double ps = spsi[s0][py][px];
      double nxr = spsi[s0][py][px + 1] - spsi[s0][py][px - 1];
      double nyr = spsi[s0][py + 1][px] - spsi[s0][py - 1][px];
      double nzr = spsi[sp][py][px] - spsi[sm][py][px];
      const double normag = 1.0 / (sqrt(nxr * nxr + nyr * nyr + nzr * nzr) + ENUM);
      nxr = nxr * normag;
      nyr = nyr * normag;
      nzr = nzr * normag;
      const double t = tanh(0.5 * ps * epsi);
      const double fac = 0.25 * (1.0 - t * t);
      sF[sf][0][y][x] = fac * nxr;
      sF[sf][1][y][x] = fac * nyr;
      sF[sf][2][y][x] = fac * nzr;
    }
  };

  // prologue: psi k0-2..k0+1, F k0-1, k0
  psi_plane(k0 - 2);
  psi_plane(k0 - 1);
  psi_plane(k0);
  __syncthreads();
  F_plane(k0 - 1);
  __syncthreads();
  psi_plane(k0 + 1);
  __syncthreads();
  F_plane(k0);
  __syncthreads();

  const double gamma = 1.0 * a.sc->gumax;
  const double mu_ = a.sc->mean[0], mv_ = a.sc->mean[1], mw_ = a.sc->mean[2];
  const double dxi = g.dxi, ddxi = g.ddxi, dt = g.dt;
  const int tx = tid % PTX, ty = tid / PTX;
  const int i = i0 + tx, j = j0 + ty;
  const bool own = (i < nx) && (j < ny);
  const int ip = wrapp(i % nx, nx), im = wrapm(i % nx, nx);
  const int jp = wrapp(j % ny, ny), jm = wrapm(j % ny, ny);

  for (int k = k0; k < k1; ++k) {
    psi_plane(k + 2);
    __syncthreads();
    F_plane(k + 1);
    __syncthreads();
    if (own) {
      const int kp = wrapp(k, nz), km = wrapm(k, nz);
      const size_t c = lin(i, j, k, nx, ny);
      const double p0 = __ldg(phi + c);
      const double pxp = __ldg(phi + lin(ip, j, k, nx, ny)), pxm = __ldg(phi + lin(im, j, k, nx, ny));
      const double pyp = __ldg(phi + lin(i, jp, k, nx, ny)), pym = __ldg(phi + lin(i, jm, k, nx, ny));
      const double pzp = __ldg(phi + lin(i, j, kp, nx, ny)), pzm = __ldg(phi + lin(i, j, km, nx, ny));
      const double u0 = __ldg(a.u + c) - mu_, uxp = __ldg(a.u + lin(ip, j, k, nx, ny)) - mu_;
      const double v0 = __ldg(a.v + c) - mv_, vyp = __ldg(a.v + lin(i, jp, k, nx, ny)) - mv_;
      const double w0 = __ldg(a.w + c) - mw_, wzp = __ldg(a.w + lin(i, j, kp, nx, ny)) - mw_;
      // :551-557
      double rhs = -((uxp * 0.5 * (pxp + p0) - u0 * 0.5 * (p0 + pxm)) * dxi) -
                   (vyp * 0.5 * (pyp + p0) - v0 * 0.5 * (p0 + pym)) * dxi -
                   (wzp * 0.5 * (pzp + p0) - w0 * 0.5 * (p0 + pzm)) * dxi +
                   gamma * (eps * (pxp - 2.0 * p0 + pxm) * ddxi + eps * (pyp - 2.0 * p0 + pym) * ddxi +
                            eps * (pzp - 2.0 * p0 + pzm) * ddxi);
      // :609-614
      const int fx = tx + 1, fy = ty + 1;
      const int s0 = slot(k), sm = slot(k - 1), sp = slot(k + 1);
      rhs = rhs - gamma * ((sF[s0][0][fy][fx + 1] - sF[s0][0][fy][fx - 1]) * 0.5 * dxi +
                           (sF[s0][1][fy + 1][fx] - sF[s0][1][fy - 1][fx]) * 0.5 * dxi +
                           (sF[sp][2][fy][fx] - sF[sm][2][fy][fx]) * 0.5 * dxi);
      // :625-626
      const double ro = a.rphio[c];
      a.phin[c] = p0 + dt * (a.alpha * rhs - a.beta * ro);
      a.rphio[c] = rhs;
    }
    __syncthreads();
  }
}

cudaError_t launch_phase(const PhaseArgs& a, cudaStream_t st) {
  dim3 grd((a.g.nx + PTX - 1) / PTX, (a.g.ny + PTY - 1) / PTY, (a.g.nz + PZCHUNK - 1) / PZCHUNK);
  k_phase<<<grd, PNT, 0, st>>>(a);
  return cudaGetLastError();
}

}  // namespace mhit
