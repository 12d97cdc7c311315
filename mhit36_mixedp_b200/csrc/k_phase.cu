// ACDI phase-field transport: multi/main.f90:522-636 in one kernel.
//
// The reference makes five passes with three stored intermediates (psidi, tanh_psi and the
// three normal components) and six halo exchanges.  Here a block owns a PTX x PTY column of
// cells and marches up a chunk of z planes, keeping three rings of planes in shared memory:
//   phi  planes k-2..k+5 (two planes in flight via cp.async), x/y halo 2
//   psi  = eps log((min(phi,1)+1e-16)/(1-min(phi,1)+1e-16))          (:527-528), halo 2
//   F    = 1/4 (1 - t^2) n/(|n|+1e-16), n = central psi differences (:559-561, :586-589,
//          :609-614), halo 1, with t = tanh(psi/(2 eps)) (:530)
// and writes only phi^{n+1} and rhsphi_o.  psi and F are recomputed on the x-y halo of the
// tile (factors (PTX+4)(PTY+4)/(PTX PTY) and (PTX+2)(PTY+2)/(PTX PTY)).
//
// t is evaluated in closed form: tanh(log(r)/2) = (r-1)/(r+1) with r = (val+1e-16)/(1-val+1e-16)
// gives t = (2 val - 1)/(1 + 2e-16) exactly in real arithmetic; in float64 it agrees with the
// reference's tanh(0.5*psi/eps) to 2.2e-16 over the whole range of phi (a NaN psi, from
// phi < -1e-16, still gives a NaN t as in the reference).
//
// With PhaseArgs::clamp (opt-in, off by default) phi is also clamped below at 0 before the
// log, so a cell undershooting to phi < -1e-16 no longer turns psi into NaN.
//
// gamma = 1.0*gumax is read from the device scalars written by the previous projection
// (:536, :998-1002); u, v, w are the stored fields minus the lazily removed mean.
#include <cuda_pipeline.h>

#include "common.cuh"
#include "kernels.h"

namespace mhit {

constexpr int PTX = 32, PTY = 16, PNT = PTX * PTY;
constexpr int PZC = 64;                      // default z planes per block
constexpr int PHX = PTX + 4, PHY = PTY + 4;  // phi / psi plane (halo 2)
constexpr int PHL = PHX * PHY;
constexpr int PFX = PTX + 2, PFY = PTY + 2;  // F plane (halo 1)
constexpr int PFL = PFX * PFY;
constexpr int PCPY = (PHL + PNT - 1) / PNT;
constexpr double ENUM = 1.0e-16;
constexpr double TNORM = 1.0 / (1.0 + 2.0 * ENUM);

struct PhaseSmem {
  double phi[7][PHL];   // planes k-2..k+4 (k+4, k+5 in flight while iteration k runs)
  double psi[4][PHL];   // planes k..k+3
  double F[3][3][PFL];  // planes k-1..k+1
};

__device__ __forceinline__ int pmodi(int x, int n) {
  x %= n;
  return x < 0 ? x + n : x;
}

// Software pipeline, two barriers per output plane k, phi prefetched two planes ahead:
//   wait phi(k+3); B1; cp.async phi(k+5); { psi(k+3), F(k+1) } as one task list; B2; out(k)
__global__ void __launch_bounds__(PNT, 2) k_phase(PhaseArgs a) {
  extern __shared__ __align__(16) unsigned char smraw[];
  PhaseSmem& S = *reinterpret_cast<PhaseSmem*>(smraw);
  const Geo& g = a.g;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const size_t plane = (size_t)nx * ny;
  const int i0 = blockIdx.x * PTX, j0 = blockIdx.y * PTY;
  const int zc = a.zchunk > 0 ? a.zchunk : PZC;
  const int k0 = blockIdx.z * zc;
  const int k1 = min(k0 + zc, nz);
  const int tid = threadIdx.x;
  const double eps = g.eps;
  const int clamp = a.clamp;
  const double* __restrict__ phig = a.phi;

  int poff[PCPY];
#pragma unroll
  for (int c = 0; c < PCPY; ++c) {
    const int e = tid + c * PNT;
    poff[c] = -1;
    if (e < PHL) {
      const int y = e / PHX, x = e - y * PHX;
      poff[c] = pmodi(j0 - 2 + y, ny) * nx + pmodi(i0 - 2 + x, nx);
    }
  }
  auto slot7 = [&](int m) { return (m - k0 + 9) % 7; };
  auto slot4 = [&](int m) { return (m - k0 + 8) & 3; };
  auto slot3 = [&](int m) { return (m - k0 + 6) % 3; };
  auto issue_phi = [&](int m) {
    const size_t base = (size_t)pmodi(m, nz) * plane;
    double* dst = S.phi[slot7(m)];
#pragma unroll
    for (int c = 0; c < PCPY; ++c)
      if (poff[c] >= 0) __pipeline_memcpy_async(dst + tid + c * PNT, phig + base + poff[c], 8);
  };
  // psi of element e of a plane (multi/main.f90:527-528)
  auto psi_at = [&](const double* __restrict__ P, double* __restrict__ Q, int e) {
    double val = fmin(P[e], 1.0);
    if (clamp) val = fmax(val, 0.0);
    Q[e] = eps * log((val + ENUM) / (1.0 - val + ENUM));
  };
  // F of one element (multi/main.f90:530, 559-561, 586-589, 609-614); q: psi-plane index,
  // f: F-plane index
  auto F_at = [&](const double* __restrict__ Qm, const double* __restrict__ Q0, const double* __restrict__ Qp,
                  const double* __restrict__ P, double* __restrict__ Fd, int q, int f) {
    double nxr = Q0[q + 1] - Q0[q - 1];
    double nyr = Q0[q + PHX] - Q0[q - PHX];
    double nzr = Qp[q] - Qm[q];
    const double normag = 1.0 / (sqrt(nxr * nxr + nyr * nyr + nzr * nzr) + ENUM);
    nxr = nxr * normag;
    nyr = nyr * normag;
    nzr = nzr * normag;
    const double ps = Q0[q];
    double val = fmin(P[q], 1.0);
    if (clamp) val = fmax(val, 0.0);
    const double t = (ps == ps) ? (2.0 * val - 1.0) * TNORM : ps;
    const double fac = 0.25 * (1.0 - t * t);
    Fd[f] = fac * nxr;
    Fd[PFL + f] = fac * nyr;
    Fd[2 * PFL + f] = fac * nzr;
  };
  auto F_plane_all = [&](int m) {
    const double* Qm = S.psi[slot4(m - 1)];
    const double* Q0 = S.psi[slot4(m)];
    const double* Qp = S.psi[slot4(m + 1)];
    const double* P = S.phi[slot7(m)];
    double* Fd = S.F[slot3(m)][0];
    for (int e = tid; e < PFL; e += PNT) {
      const int y = e / PFX, x = e - y * PFX;
      F_at(Qm, Q0, Qp, P, Fd, (y + 1) * PHX + (x + 1), e);
    }
  };

  // prologue: phi k0-2..k0+3; psi k0-2..k0+2 (ring of 4); F k0-1, k0
  for (int m = k0 - 2; m <= k0 + 3; ++m) issue_phi(m);
  __pipeline_commit();
  issue_phi(k0 + 4);
  __pipeline_commit();
  __pipeline_wait_prior(1);
  __syncthreads();
  for (int e = tid; e < 3 * PHL; e += PNT) {
    const int m = k0 - 2 + e / PHL;
    psi_at(S.phi[slot7(m)], S.psi[slot4(m)], e % PHL);
  }
  __syncthreads();
  F_plane_all(k0 - 1);
  __syncthreads();
  for (int e = tid; e < 2 * PHL; e += PNT) {
    const int m = k0 + 1 + e / PHL;
    psi_at(S.phi[slot7(m)], S.psi[slot4(m)], e % PHL);
  }
  __syncthreads();
  F_plane_all(k0);

  // this thread's share of the per-plane task list {psi(k+3) elements, F(k+1) elements}
  constexpr int NTASK = (PHL + PFL + PNT - 1) / PNT;
  int tq[NTASK], tf[NTASK];  // psi task: tq = e, tf = -1; F task: tq = psi index, tf = F index
#pragma unroll
  for (int r = 0; r < NTASK; ++r) {
    const int t = tid + r * PNT;
    if (t < PHL) {
      tq[r] = t;
      tf[r] = -1;
    } else if (t < PHL + PFL) {
      const int e = t - PHL, y = e / PFX, x = e - y * PFX;
      tq[r] = (y + 1) * PHX + (x + 1);
      tf[r] = e;
    } else {
      tq[r] = -1;
      tf[r] = -1;
    }
  }

  const double gamma = 1.0 * a.sc->gumax;
  const double mu_ = a.sc->mean[0], mv_ = a.sc->mean[1], mw_ = a.sc->mean[2];
  const double dxi = g.dxi, ddxi = g.ddxi, dt = g.dt;
  const double hdxi = 0.5 * dxi;  // (x*0.5)*dxi == x*(0.5*dxi) exactly
  const int tx = tid % PTX, ty = tid / PTX;
  const int i = i0 + tx, j = j0 + ty;
  const bool own = (i < nx) && (j < ny);
  const int ip = own ? wrapp(i, nx) : 0, jp = own ? wrapp(j, ny) : 0;
  const int hq = (ty + 2) * PHX + (tx + 2);  // own cell in the phi/psi plane
  const int fq = (ty + 1) * PFX + (tx + 1);  // own cell in the F plane
  // running pointers to the own cell of plane k (and its +x, +y, +z neighbours)
  const size_t c0 = (size_t)k0 * plane + (size_t)(own ? j : 0) * nx + (own ? i : 0);
  const double* pu = a.u + c0;
  const double* pv = a.v + c0;
  const double* pw = a.w + c0;
  const ptrdiff_t dux = (ptrdiff_t)ip - (own ? i : 0);
  const ptrdiff_t dvy = ((ptrdiff_t)jp - (own ? j : 0)) * nx;
  double* pphin = a.phin + c0;
  double* prphi = a.rphio + c0;

  for (int k = k0; k < k1; ++k) {
    // operands from HBM for this plane, issued before the barriers
    const ptrdiff_t dwz = (k + 1 == nz) ? -(ptrdiff_t)(nz - 1) * (ptrdiff_t)plane : (ptrdiff_t)plane;
    double u0 = 0, uxp = 0, v0 = 0, vyp = 0, w0 = 0, wzp = 0, ro = 0;
    if (own) {
      u0 = __ldg(pu);
      uxp = __ldg(pu + dux);
      v0 = __ldg(pv);
      vyp = __ldg(pv + dvy);
      w0 = __ldg(pw);
      wzp = __ldg(pw + dwz);
      ro = *prphi;
    }
    __pipeline_wait_prior(1);  // phi(k+3) landed; phi(k+4) may still be in flight
    __syncthreads();
    issue_phi(k + 5);
    __pipeline_commit();
    {
      const double* P3 = S.phi[slot7(k + 3)];
      double* Q3 = S.psi[slot4(k + 3)];
      const double* Qm = S.psi[slot4(k)];
      const double* Q0 = S.psi[slot4(k + 1)];
      const double* Qp = S.psi[slot4(k + 2)];
      const double* P1 = S.phi[slot7(k + 1)];
      double* Fd = S.F[slot3(k + 1)][0];
#pragma unroll
      for (int r = 0; r < NTASK; ++r) {
        if (tf[r] >= 0) F_at(Qm, Q0, Qp, P1, Fd, tq[r], tf[r]);
        else if (tq[r] >= 0) psi_at(P3, Q3, tq[r]);
      }
    }
    __syncthreads();
    if (own) {
      u0 -= mu_;
      uxp -= mu_;
      v0 -= mv_;
      vyp -= mv_;
      w0 -= mw_;
      wzp -= mw_;
      const double* P0 = S.phi[slot7(k)];
      const double p0 = P0[hq];
      const double pxp = P0[hq + 1], pxm = P0[hq - 1], pyp = P0[hq + PHX], pym = P0[hq - PHX];
      const double pzp = S.phi[slot7(k + 1)][hq], pzm = S.phi[slot7(k - 1)][hq];
      // multi/main.f90:551-557
      double rhs = -((uxp * 0.5 * (pxp + p0) - u0 * 0.5 * (p0 + pxm)) * dxi) -
                   (vyp * 0.5 * (pyp + p0) - v0 * 0.5 * (p0 + pym)) * dxi -
                   (wzp * 0.5 * (pzp + p0) - w0 * 0.5 * (p0 + pzm)) * dxi +
                   gamma * (eps * (pxp - 2.0 * p0 + pxm) * ddxi + eps * (pyp - 2.0 * p0 + pym) * ddxi +
                            eps * (pzp - 2.0 * p0 + pzm) * ddxi);
      // :609-614
      const double* F0x = S.F[slot3(k)][0];
      const double* F0y = S.F[slot3(k)][1];
      rhs = rhs - gamma * ((F0x[fq + 1] - F0x[fq - 1]) * hdxi + (F0y[fq + PFX] - F0y[fq - PFX]) * hdxi +
                           (S.F[slot3(k + 1)][2][fq] - S.F[slot3(k - 1)][2][fq]) * hdxi);
      // :625-626
      *pphin = p0 + dt * (a.alpha * rhs - a.beta * ro);
      *prphi = rhs;
    }
    pu += plane;
    pv += plane;
    pw += plane;
    pphin += plane;
    prphi += plane;
  }
  __pipeline_wait_prior(0);
}

cudaError_t launch_phase(const PhaseArgs& a, cudaStream_t st) {
  const size_t smem = sizeof(PhaseSmem);
  static int attr_set[64] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && !attr_set[dev]) {
    cudaError_t e = cudaFuncSetAttribute(k_phase, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr_set[dev] = 1;
  }
  const int zc = a.zchunk > 0 ? a.zchunk : PZC;
  dim3 grd((a.g.nx + PTX - 1) / PTX, (a.g.ny + PTY - 1) / PTY, (a.g.nz + zc - 1) / zc);
  k_phase<<<grd, PNT, smem, st>>>(a);
  return cudaGetLastError();
}

}  // namespace mhit
