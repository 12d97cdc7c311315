// Projection and the per-step reductions: multi/main.f90:942-1007.
//
// k_correct     u** = u* - dt/rho (p(i) - p(i-1)) dxi (and v, w along y, z; :953-955) in place,
//               with per-block partial sums (mean, :956-958) and maxima (:998-1000).
// k_finalize    one block reduces the partials in a fixed order (run-to-run deterministic),
//               writes mean = sum/nx/ny/nz (:967-969), gumax = max over components of
//               (max - mean) -- equal to maxval(u - mean) because rounding is monotonic --,
//               cfl = gumax dt dxi (:1003) and the NaN / CFL>7 flags (:1006).
// The mean is not subtracted here: the next step's kernels and the download subtract it on
// read, which saves a full read+write pass of u, v, w.
#include "common.cuh"
#include "kernels.h"

namespace mhit {

constexpr int CNT = 256;

constexpr int CTX = 32, CTY = 16, CZC = 16;  // x-y tile and default z chunk of k_correct

// Pressure sources of the projection: a pair of x-adjacent values and a single value, widened
// to FP64.  PSum is the refinement's p = p32 + delta, formed on the fly exactly as a stored
// (double)p32 + (double)delta would be.
struct PDouble {
  const double* p;
  __device__ __forceinline__ double2 pair(size_t o) const { return *reinterpret_cast<const double2*>(p + o); }
  __device__ __forceinline__ double one(size_t o) const { return p[o]; }
};
struct PFloat {
  const float* p;
  __device__ __forceinline__ double2 pair(size_t o) const {
    const float2 v = *reinterpret_cast<const float2*>(p + o);
    return make_double2((double)v.x, (double)v.y);
  }
  __device__ __forceinline__ double one(size_t o) const { return (double)p[o]; }
};
struct PSum {
  const float* p;
  const float* d;
  __device__ __forceinline__ double2 pair(size_t o) const {
    const float2 a = *reinterpret_cast<const float2*>(p + o), b = *reinterpret_cast<const float2*>(d + o);
    return make_double2((double)a.x + (double)b.x, (double)a.y + (double)b.y);
  }
  __device__ __forceinline__ double one(size_t o) const { return (double)p[o] + (double)d[o]; }
};

// Each thread owns two adjacent x cells (16-byte loads of u, v, w) of one tile row and marches
// up zc planes two at a time: p(k-1) is carried in registers from the previous plane,
// p(i-1) comes from the neighbouring lane of the 16-lane row, p(j-1) from L1.
template <typename S>
__global__ void __launch_bounds__(CNT) k_correct(CorrectArgs a, S ps, int zc) {
  const Geo& g = a.g;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const size_t plane = (size_t)nx * ny;
  double* __restrict__ U = a.u;
  double* __restrict__ V = a.v;
  double* __restrict__ W = a.w;
  const double cc = g.dt / g.rho, dxi = g.dxi;
  const int lx = threadIdx.x & 15, ty = threadIdx.x >> 4;  // 16 lanes x 16 rows
  const int i = blockIdx.x * CTX + 2 * lx, j = blockIdx.y * CTY + ty;
  const int k0 = blockIdx.z * zc, k1 = min(k0 + zc, nz);
  const bool own = i < nx && j < ny;
  const int ic = own ? i : 0, jc = own ? j : 0;
  const int im = wrapm(ic, nx), jm = wrapm(jc, ny);
  const bool edge = (lx == 0) || (nx < CTX);
  double su = 0.0, sv = 0.0, sw = 0.0;
  double mu = -INFINITY, mv = -INFINITY, mw = -INFINITY;
  const size_t r0 = (size_t)jc * nx + ic;
  const ptrdiff_t dym = ((ptrdiff_t)jm - jc) * nx;
  const double2 pk = ps.pair((size_t)wrapm(k0, nz) * plane + r0);
  double pkm0 = pk.x, pkm1 = pk.y;
  auto plane_step = [&](size_t c, const double2 pc2, const double2 py2, const double pxm_edge, const double2 uo,
                        const double2 vo, const double2 wo) {
    const double pc0 = pc2.x, pc1 = pc2.y;
    double pxm0 = __shfl_up_sync(0xffffffffu, pc1, 1, 16);
    if (edge) pxm0 = pxm_edge;
    // multi/main.f90:953-955
    const double u0 = uo.x - cc * (pc0 - pxm0) * dxi, u1 = uo.y - cc * (pc1 - pc0) * dxi;
    const double v0 = vo.x - cc * (pc0 - py2.x) * dxi, v1 = vo.y - cc * (pc1 - py2.y) * dxi;
    const double w0 = wo.x - cc * (pc0 - pkm0) * dxi, w1 = wo.y - cc * (pc1 - pkm1) * dxi;
    pkm0 = pc0;
    pkm1 = pc1;
    if (own) {
      *reinterpret_cast<double2*>(U + c) = make_double2(u0, u1);
      *reinterpret_cast<double2*>(V + c) = make_double2(v0, v1);
      *reinterpret_cast<double2*>(W + c) = make_double2(w0, w1);
      su += u0 + u1;
      sv += v0 + v1;
      sw += w0 + w1;
      mu = fmax(mu, fmax(u0, u1));
      mv = fmax(mv, fmax(v0, v1));
      mw = fmax(mw, fmax(w0, w1));
    }
  };
  int k = k0;
  for (; k + 1 < k1; k += 2) {
    const size_t ca = (size_t)k * plane + r0, cb = ca + plane;
    const double2 pa = ps.pair(ca), pb = ps.pair(cb);
    const double2 ya = ps.pair(ca + dym), yb = ps.pair(cb + dym);
    const double xa = edge ? ps.one(ca - ic + im) : 0.0, xb = edge ? ps.one(cb - ic + im) : 0.0;
    const double2 ua = *reinterpret_cast<const double2*>(U + ca), ub = *reinterpret_cast<const double2*>(U + cb);
    const double2 va = *reinterpret_cast<const double2*>(V + ca), vb = *reinterpret_cast<const double2*>(V + cb);
    const double2 wa = *reinterpret_cast<const double2*>(W + ca), wb = *reinterpret_cast<const double2*>(W + cb);
    plane_step(ca, pa, ya, xa, ua, va, wa);
    plane_step(cb, pb, yb, xb, ub, vb, wb);
  }
  if (k < k1) {
    const size_t ca = (size_t)k * plane + r0;
    const double2 pa = ps.pair(ca);
    const double2 ya = ps.pair(ca + dym);
    const double xa = edge ? ps.one(ca - ic + im) : 0.0;
    plane_step(ca, pa, ya, xa, *reinterpret_cast<const double2*>(U + ca), *reinterpret_cast<const double2*>(V + ca),
               *reinterpret_cast<const double2*>(W + ca));
  }
  // block reduction (fixed tree)
  __shared__ double red[6][CNT / 32];
  double vals[6] = {su, sv, sw, mu, mv, mw};
  const int t = threadIdx.x, lane = t & 31;
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    double x = vals[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double y = __shfl_down_sync(0xffffffffu, x, o);
      x = q < 3 ? x + y : fmax(x, y);
    }
    if (lane == 0) red[q][t >> 5] = x;
  }
  __syncthreads();
  if (t < 6) {
    double x = red[t][0];
    for (int wv = 1; wv < CNT / 32; ++wv) x = t < 3 ? x + red[t][wv] : fmax(x, red[t][wv]);
    const size_t bid = ((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
    a.partials[bid * 6 + t] = x;
  }
}

__global__ void __launch_bounds__(1024) k_finalize(const double* __restrict__ partials, int nblocks, Geo g,
                                                   DevScalars* sc) {
  __shared__ double red[6][32];
  double vals[6] = {0.0, 0.0, 0.0, -INFINITY, -INFINITY, -INFINITY};
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      const double x = partials[(size_t)b * 6 + q];
      vals[q] = q < 3 ? vals[q] + x : fmax(vals[q], x);
    }
  }
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    double x = vals[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double y = __shfl_down_sync(0xffffffffu, x, o);
      x = q < 3 ? x + y : fmax(x, y);
    }
    if ((threadIdx.x & 31) == 0) red[q][threadIdx.x >> 5] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double r[6];
    const int nw = (blockDim.x + 31) / 32;
    for (int q = 0; q < 6; ++q) {
      double x = red[q][0];
      for (int wv = 1; wv < nw; ++wv) x = q < 3 ? x + red[q][wv] : fmax(x, red[q][wv]);
      r[q] = x;
    }
    const double nxd = g.nx, nyd = g.ny, nzd = g.nz;
    int flag = 0;
    for (int q = 0; q < 3; ++q) {
      const double m = r[q] / nxd / nyd / nzd;  // multi/main.f90:967-969
      sc->mean[q] = m;
      r[3 + q] = r[3 + q] - m;
      if (!(r[q] == r[q])) flag |= 1;
    }
    const double gumax = fmax(r[5], fmax(r[3], r[4]));  // :1001
    sc->gumax = gumax;
    sc->cfl = gumax * g.dt * g.dxi;
    if (!(gumax == gumax)) flag |= 1;
    if (sc->cfl > 7.0) flag |= 2;  // :1006
    sc->flag |= flag;
  }
}

// z planes per block: 64 where that still leaves eight waves of two blocks on each of the 148
// SMs (each chunk re-reads the p plane below it: 1.106 against 1.135 ms FP32, 1.209 against
// 1.250 ms FP64 at 512^3), otherwise CZC
static int correct_chunk(const Geo& g) {
  const long long cols = (long long)((g.nx + CTX - 1) / CTX) * ((g.ny + CTY - 1) / CTY);
  return cols * ((g.nz + 63) / 64) >= 8 * 148 * 2 ? 64 : CZC;
}

static dim3 correct_grid(const Geo& g) {
  const int zc = correct_chunk(g);
  return dim3((g.nx + CTX - 1) / CTX, (g.ny + CTY - 1) / CTY, (g.nz + zc - 1) / zc);
}

int correct_blocks(const Geo& g) {
  const dim3 d = correct_grid(g);
  return (int)(d.x * d.y * d.z);
}

cudaError_t launch_correct(const CorrectArgs& a, cudaStream_t st) {
  const dim3 grd = correct_grid(a.g), blk(CNT);
  const int zc = correct_chunk(a.g);
  if (a.pd) k_correct<<<grd, blk, 0, st>>>(a, PSum{static_cast<const float*>(a.p), a.pd}, zc);
  else if (a.fp32) k_correct<<<grd, blk, 0, st>>>(a, PFloat{static_cast<const float*>(a.p)}, zc);
  else k_correct<<<grd, blk, 0, st>>>(a, PDouble{static_cast<const double*>(a.p)}, zc);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return launch_finalize(a.partials, a.nblocks, a.g, a.sc, st);
}

cudaError_t launch_finalize(const double* partials, int nblocks, const Geo& g, DevScalars* sc, cudaStream_t st) {
  k_finalize<<<1, 1024, 0, st>>>(partials, nblocks, g, sc);
  return cudaGetLastError();
}

// ------------------------------------------------------------------ diagnostics
// max |div u| (the operator of :841-843 without rho/dt), kinetic energy, and the dissipation
// 2 nu <S_ij S_ij> with central differences (post/compute_diss/main.f90:72-117).  The maximum
// propagates NaN, so a NaN velocity gives a NaN max|div| as well as a NaN KE.
__global__ void __launch_bounds__(CNT) k_diag(DiagArgs a) {
  const Geo& g = a.g;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const size_t ntot = (size_t)nx * ny * nz;
  const double mu_ = a.sc->mean[0], mv_ = a.sc->mean[1], mw_ = a.sc->mean[2];
  const double* __restrict__ U = a.u;
  const double* __restrict__ V = a.v;
  const double* __restrict__ W = a.w;
  const double dxi = g.dxi, h = 0.5 / a.dxd;
  double mdiv = 0.0, ke = 0.0, ss = 0.0;
  const size_t stride = (size_t)gridDim.x * CNT;
  for (size_t c = (size_t)blockIdx.x * CNT + threadIdx.x; c < ntot; c += stride) {
    const int i = (int)(c % nx);
    const size_t r = c / nx;
    const int j = (int)(r % ny), k = (int)(r / ny);
    const int ip = wrapp(i, nx), im = wrapm(i, nx), jp = wrapp(j, ny), jm = wrapm(j, ny);
    const int kp = wrapp(k, nz), km = wrapm(k, nz);
#define F(A, m, ii, jj, kk) (__ldg(A + lin(ii, jj, kk, nx, ny)) - m)
    const double u0 = F(U, mu_, i, j, k), v0 = F(V, mv_, i, j, k), w0 = F(W, mw_, i, j, k);
    const double div = (F(U, mu_, ip, j, k) - u0) * dxi + (F(V, mv_, i, jp, k) - v0) * dxi +
                       (F(W, mw_, i, j, kp) - w0) * dxi;
    mdiv = nanmax(mdiv, fabs(div));
    ke += u0 * u0 + v0 * v0 + w0 * w0;
    const double dudx = (F(U, mu_, ip, j, k) - F(U, mu_, im, j, k)) * h;
    const double dudy = (F(U, mu_, i, jp, k) - F(U, mu_, i, jm, k)) * h;
    const double dudz = (F(U, mu_, i, j, kp) - F(U, mu_, i, j, km)) * h;
    const double dvdx = (F(V, mv_, ip, j, k) - F(V, mv_, im, j, k)) * h;
    const double dvdy = (F(V, mv_, i, jp, k) - F(V, mv_, i, jm, k)) * h;
    const double dvdz = (F(V, mv_, i, j, kp) - F(V, mv_, i, j, km)) * h;
    const double dwdx = (F(W, mw_, ip, j, k) - F(W, mw_, im, j, k)) * h;
    const double dwdy = (F(W, mw_, i, jp, k) - F(W, mw_, i, jm, k)) * h;
    const double dwdz = (F(W, mw_, i, j, kp) - F(W, mw_, i, j, km)) * h;
#undef F
    const double s12 = 0.5 * (dudy + dvdx), s13 = 0.5 * (dudz + dwdx), s23 = 0.5 * (dvdz + dwdy);
    ss += dudx * dudx + dvdy * dvdy + dwdz * dwdz + 2.0 * (s12 * s12 + s13 * s13 + s23 * s23);
  }
  __shared__ double red[3][CNT / 32];
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
    for (int wv = 1; wv < CNT / 32; ++wv) x = q == 0 ? nanmax(x, red[q][wv]) : x + red[q][wv];
    a.partials[(size_t)blockIdx.x * 4 + q] = x;
  }
}

__global__ void __launch_bounds__(1024) k_diag_finalize(const double* __restrict__ partials, int nblocks, Geo g,
                                                        double nu, DevScalars* sc) {
  __shared__ double red[3][32];
  double vals[3] = {0.0, 0.0, 0.0};
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
    vals[0] = nanmax(vals[0], partials[(size_t)b * 4 + 0]);
    vals[1] += partials[(size_t)b * 4 + 1];
    vals[2] += partials[(size_t)b * 4 + 2];
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
    const double n = (double)g.nx * g.ny * g.nz;
    sc->diag[0] = r[0];
    sc->diag[1] = 0.5 * r[1] / n;
    sc->diag[2] = 2.0 * nu * r[2] / n;
  }
}

cudaError_t launch_diag(const DiagArgs& a, cudaStream_t st) {
  k_diag<<<a.nblocks, CNT, 0, st>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_diag_finalize<<<1, 1024, 0, st>>>(a.partials, a.nblocks, a.g, a.nu, a.sc);
  return cudaGetLastError();
}

__global__ void k_fill(double* p, size_t n, double v) {
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) p[c] = v;
}

cudaError_t launch_fill(double* p, size_t n, double v, cudaStream_t st) {
  k_fill<<<148 * 4, 256, 0, st>>>(p, n, v);
  return cudaGetLastError();
}

}  // namespace mhit
