// Momentum predictor: multi/main.f90:658-802 in one pass over the grid.
//
// Per cell: conservative advection (h11..h33, :672-694), viscous Laplacian (:696-707), ABC
// forcing from the per-axis sin/cos tables (:712-714), and with the phase field the
// chemical-potential surface-tension force recomputed on chip at the cell and at its -x,-y,-z
// neighbours (:734-739) and averaged to the faces (:768-770) -- the reference's fxst/fyst/fzst
// arrays and their 6 halo exchanges (:746-757) are never stored.  Then the AB2 update
// u* = u + dt (alpha rhs - beta rhs_o), rhs_o = rhs (:771-776 / :787-792).
//
// The velocity read here is the stored one minus the running mean of the previous
// projection (DevScalars::mean); subtracting on read is exactly the reference's
// u = u - gumean (:977-981) done lazily.
#include "common.cuh"
#include "kernels.h"

namespace mhit {

__device__ __forceinline__ double chempot_at(const double* __restrict__ phi, int i, int j, int k, const Geo& g) {
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int ip = wrapp(i, nx), im = wrapm(i, nx), jp = wrapp(j, ny), jm = wrapm(j, ny);
  const int kp = wrapp(k, nz), km = wrapm(k, nz);
  const double c = __ldg(phi + lin(i, j, k, nx, ny));
  const double s = __ldg(phi + lin(ip, j, k, nx, ny)) + __ldg(phi + lin(im, j, k, nx, ny)) +
                   __ldg(phi + lin(i, jp, k, nx, ny)) + __ldg(phi + lin(i, jm, k, nx, ny)) +
                   __ldg(phi + lin(i, j, kp, nx, ny)) + __ldg(phi + lin(i, j, km, nx, ny));
  // multi/main.f90:735
  return c * (1.0 - c) * (1.0 - 2.0 * c) * g.epsi - g.eps * (s - 6.0 * c) * g.ddxi;
}

template <bool PHI>
__global__ void __launch_bounds__(256) k_mom(MomArgs a) {
  const Geo& g = a.g;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  if (i >= nx || j >= ny || k >= nz) return;
  const int ip = wrapp(i, nx), im = wrapm(i, nx), jp = wrapp(j, ny), jm = wrapm(j, ny);
  const int kp = wrapp(k, nz), km = wrapm(k, nz);
  const double mu_ = a.sc->mean[0], mv_ = a.sc->mean[1], mw_ = a.sc->mean[2];
  const double* __restrict__ U = a.u;
  const double* __restrict__ V = a.v;
  const double* __restrict__ W = a.w;
#define LU(ii, jj, kk) (__ldg(U + lin(ii, jj, kk, nx, ny)) - mu_)
#define LV(ii, jj, kk) (__ldg(V + lin(ii, jj, kk, nx, ny)) - mv_)
#define LW(ii, jj, kk) (__ldg(W + lin(ii, jj, kk, nx, ny)) - mw_)
  const double u0 = LU(i, j, k), v0 = LV(i, j, k), w0 = LW(i, j, k);
  const double uxp = LU(ip, j, k), uxm = LU(im, j, k), uyp = LU(i, jp, k), uym = LU(i, jm, k);
  const double uzp = LU(i, j, kp), uzm = LU(i, j, km);
  const double vxp = LV(ip, j, k), vxm = LV(im, j, k), vyp = LV(i, jp, k), vym = LV(i, jm, k);
  const double vzp = LV(i, j, kp), vzm = LV(i, j, km);
  const double wxp = LW(ip, j, k), wxm = LW(im, j, k), wyp = LW(i, jp, k), wym = LW(i, jm, k);
  const double wzp = LW(i, j, kp), wzm = LW(i, j, km);
  const double v_imjp = LV(im, jp, k), w_imkp = LW(im, j, kp), u_ipjm = LU(ip, jm, k);
  const double w_jmkp = LW(i, jm, kp), u_ipkm = LU(ip, j, km), v_jpkm = LV(i, jp, km);
#undef LU
#undef LV
#undef LW
  const double dxi = g.dxi, ddxi = g.ddxi, rhoi = g.rhoi, mu = g.mu;
  // multi/main.f90:672-680
  double h11 = (uxp + u0) * (uxp + u0) - (u0 + uxm) * (u0 + uxm);
  double h12 = (uyp + u0) * (vyp + v_imjp) - (u0 + uym) * (v0 + vxm);
  double h13 = (uzp + u0) * (wzp + w_imkp) - (u0 + uzm) * (w0 + wxm);
  double h21 = (uxp + u_ipjm) * (vxp + v0) - (u0 + uym) * (v0 + vxm);
  double h22 = (vyp + v0) * (vyp + v0) - (v0 + vym) * (v0 + vym);
  double h23 = (wzp + w_jmkp) * (vzp + v0) - (w0 + wym) * (v0 + vzm);
  double h31 = (wxp + w0) * (uxp + u_ipkm) - (w0 + wxm) * (u0 + uzm);
  double h32 = (vyp + v_jpkm) * (wyp + w0) - (v0 + vzm) * (w0 + wym);
  double h33 = (wzp + w0) * (wzp + w0) - (w0 + wzm) * (w0 + wzm);
  // :682-694
  double ru = -(h11 * 0.25 * dxi + h12 * 0.25 * dxi + h13 * 0.25 * dxi);
  double rv = -(h21 * 0.25 * dxi + h22 * 0.25 * dxi + h23 * 0.25 * dxi);
  double rw = -(h31 * 0.25 * dxi + h32 * 0.25 * dxi + h33 * 0.25 * dxi);
  // :696-707
  h11 = mu * (uxp - 2.0 * u0 + uxm) * ddxi;
  h12 = mu * (uyp - 2.0 * u0 + uym) * ddxi;
  h13 = mu * (uzp - 2.0 * u0 + uzm) * ddxi;
  h21 = mu * (vxp - 2.0 * v0 + vxm) * ddxi;
  h22 = mu * (vyp - 2.0 * v0 + vym) * ddxi;
  h23 = mu * (vzp - 2.0 * v0 + vzm) * ddxi;
  h31 = mu * (wxp - 2.0 * w0 + wxm) * ddxi;
  h32 = mu * (wyp - 2.0 * w0 + wym) * ddxi;
  h33 = mu * (wzp - 2.0 * w0 + wzm) * ddxi;
  ru = ru + (h11 + h12 + h13) * rhoi;
  rv = rv + (h21 + h22 + h23) * rhoi;
  rw = rw + (h31 + h32 + h33) * rhoi;
  // :712-714, tables: sx cx | sy cy | sz cz
  const double* t = a.tabs;
  const double sxi = __ldg(t + i), cxi = __ldg(t + nx + i);
  const double syj = __ldg(t + 2 * nx + j), cyj = __ldg(t + 2 * nx + ny + j);
  const double szk = __ldg(t + 2 * nx + 2 * ny + k), czk = __ldg(t + 2 * nx + 2 * ny + nz + k);
  ru = ru + g.f3 * szk + g.f2 * cyj;
  rv = rv + g.f1 * sxi + g.f3 * czk;
  rw = rw + g.f2 * syj + g.f1 * cxi;
  if constexpr (PHI) {
    // :734-739 at the cell and its -x/-y/-z neighbours, :768-770 face average
    const double* __restrict__ P = a.phi;
    const double s6 = 6.0 * g.sigma;
    const double c0 = chempot_at(P, i, j, k, g);
    const double p_xp = __ldg(P + lin(ip, j, k, nx, ny)), p_xm = __ldg(P + lin(im, j, k, nx, ny));
    const double p_yp = __ldg(P + lin(i, jp, k, nx, ny)), p_ym = __ldg(P + lin(i, jm, k, nx, ny));
    const double p_zp = __ldg(P + lin(i, j, kp, nx, ny)), p_zm = __ldg(P + lin(i, j, km, nx, ny));
    const double p_c = __ldg(P + lin(i, j, k, nx, ny));
    const int imm = wrapm(im, nx), jmm = wrapm(jm, ny), kmm = wrapm(km, nz);
    const double fx0 = s6 * c0 * 0.5 * (p_xp - p_xm) * dxi;
    const double fy0 = s6 * c0 * 0.5 * (p_yp - p_ym) * dxi;
    const double fz0 = s6 * c0 * 0.5 * (p_zp - p_zm) * dxi;
    const double cxm = chempot_at(P, im, j, k, g);
    const double cym = chempot_at(P, i, jm, k, g);
    const double czm = chempot_at(P, i, j, km, g);
    const double fxm = s6 * cxm * 0.5 * (p_c - __ldg(P + lin(imm, j, k, nx, ny))) * dxi;
    const double fym = s6 * cym * 0.5 * (p_c - __ldg(P + lin(i, jmm, k, nx, ny))) * dxi;
    const double fzm = s6 * czm * 0.5 * (p_c - __ldg(P + lin(i, j, kmm, nx, ny))) * dxi;
    ru = ru + 0.5 * (fxm + fx0) * rhoi;
    rv = rv + 0.5 * (fym + fy0) * rhoi;
    rw = rw + 0.5 * (fzm + fz0) * rhoi;
  }
  const size_t c = lin(i, j, k, nx, ny);
  const double dt = g.dt, al = a.alpha, be = a.beta;
  const double ruo = a.ru[c], rvo = a.rv[c], rwo = a.rw[c];
  a.un[c] = u0 + dt * (al * ru - be * ruo);
  a.vn[c] = v0 + dt * (al * rv - be * rvo);
  a.wn[c] = w0 + dt * (al * rw - be * rwo);
  a.ru[c] = ru;
  a.rv[c] = rv;
  a.rw[c] = rw;
}

cudaError_t launch_mom(const MomArgs& a, cudaStream_t st) {
  dim3 blk(32, 4, 2);
  dim3 grd((a.g.nx + 31) / 32, (a.g.ny + 3) / 4, (a.g.nz + 1) / 2);
  if (a.phi) k_mom<true><<<grd, blk, 0, st>>>(a);
  else k_mom<false><<<grd, blk, 0, st>>>(a);
  return cudaGetLastError();
}

}  // namespace mhit
