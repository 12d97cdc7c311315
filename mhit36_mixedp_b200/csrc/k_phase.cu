// ACDI phase-field transport: multi/main.f90:522-636 in one kernel.
//
// The reference makes five passes with three stored intermediates (psidi, tanh_psi and the
// three normal components) and six halo exchanges.  Here a block owns a TX x TY column of
// cells and marches up a chunk of z planes.  It has one thread per position of the tile plus
// its x/y halo of 2 ((TX+4)(TY+4) threads), and each thread keeps its own z column in
// registers:
//   phi  planes k-1..k+3 (k+3 loaded one plane ahead)
//   psi  = eps log((min(phi,1)+1e-16)/(1-min(phi,1)+1e-16))            (:527-528), k..k+2
//   Fz   of F = 1/4 (1 - t^2) n/(|n|+1e-16), n = central psi differences (:559-561,
//        :586-589, :609-614), t = tanh(psi/(2 eps)) (:530),               planes k-1..k+1
//        (n/(|n|+1e-16) is evaluated as n rsqrt(|n|^2), see F_of)
// Only x/y neighbours go through shared memory: psi(k+1), phi(k) and Fx, Fy(k), each
// double-buffered.  Every shared read of plane k's iteration reads what the previous
// iteration wrote, so one barrier per plane suffices.  psi is evaluated on the halo of 2 and F
// on the halo of 1 (factors (TX+4)(TY+4)/(TX TY) and (TX+2)(TY+2)/(TX TY)); threads are
// numbered so that the TX x TY output cells fill whole warps, then the F ring, then the outer
// psi-only ring.  The kernel writes only phi^{n+1} and rhsphi_o.
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
#include <type_traits>

#include "common.cuh"
#include "kernels.h"

namespace mhit {

// 32 x 16 output cells per block, one block per SM (two blocks of 16 x 16 or 16 x 12 outputs,
// with more halo, were slower: 2.90 and 3.08 against 2.64 ms at 512^3)
constexpr int PTX = 32, PTY = 16;  // output cells per block in x, y
constexpr int PMINB = 1;           // resident blocks per SM
constexpr int PHX = PTX + 4, PHY = PTY + 4;  // positions with the halo of 2
constexpr int PNT = PHX * PHY;               // threads per block = positions
constexpr int PNI = PTX * PTY;               // output cells
constexpr int PNF = (PHX - 2) * (PHY - 2);   // F positions (halo 1)
constexpr int PZC = 64;                      // default z planes per block
constexpr double ENUM = 1.0e-16;
constexpr double TNORM = 1.0 / (1.0 + 2.0 * ENUM);

// a / b for b in [1e-16, 2] to within an ulp, in FMAs: the reciprocal from an FP32 seed (24
// bits) refined by two Newton-Raphson steps r <- r + r (1 - b r) (48, then 53 bits), the quotient
// q = a r corrected once with its residual, q <- q + r (a - b q) (Markstein's scheme).  Used for
// psi's quotient, whose error enters the normals only through psi differences.
__device__ __forceinline__ double div_nr(double a, double b) {
  double r = (double)__fdividef(1.0f, (float)b);
  double e = __fma_rn(-b, r, 1.0);
  r = __fma_rn(r, e, r);
  e = __fma_rn(-b, r, 1.0);
  r = __fma_rn(r, e, r);
  const double q = a * r;
  return __fma_rn(r, __fma_rn(-b, q, a), q);
}

__device__ __forceinline__ int pmodi(int x, int n) {
  x %= n;
  return x < 0 ? x + n : x;
}

// position of ring element r of the w x h rectangle perimeter starting at (x0, y0): top row,
// bottom row, left column, right column
__device__ __forceinline__ void ring_pos(int r, int x0, int y0, int w, int h, int& x, int& y) {
  if (r < w) { x = x0 + r; y = y0; return; }
  r -= w;
  if (r < w) { x = x0 + r; y = y0 + h - 1; return; }
  r -= w;
  if (r < h - 2) { x = x0; y = y0 + 1 + r; return; }
  r -= h - 2;
  x = x0 + w - 1;
  y = y0 + 1 + r;
}

// One z column of PTX x PTY cells, tile (bx, by), chunk bz, of the box a; dta, dtb = dt alpha,
// dt beta of the AB2 update.
template <bool CLAMP>
__device__ __forceinline__ void phase_tile(const PhaseArgs& a, double dta, double dtb, int bx, int by, int bz,
                                           unsigned char* smraw) {
  // thread -> position (hx, hy) in the (PHX x PHY) grid of the tile with its halo
  const int tid = threadIdx.x;
  int hx, hy;
  if (tid < PNI) {
    hx = 2 + tid % PTX;
    hy = 2 + tid / PTX;
  } else if (tid < PNF) {
    ring_pos(tid - PNI, 1, 1, PHX - 2, PHY - 2, hx, hy);
  } else {
    ring_pos(tid - PNF, 0, 0, PHX, PHY, hx, hy);
  }
  const int q = hy * PHX + hx;  // this position in a shared plane
  // shared planes at this position: psi[2], phi[2], Fx[2], Fy[2]
  double* sps = reinterpret_cast<double*>(smraw) + q;
  double* sph = sps + 2 * PNT;
  double* sfx = sph + 2 * PNT;
  double* sfy = sfx + 2 * PNT;

  const Geo& g = a.g;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int plane = nx * ny, ntot = plane * nz;
  const int i0 = bx * PTX, j0 = by * PTY;
  const int zc = a.zchunk > 0 ? a.zchunk : PZC;
  const int k0 = bz * zc, k1 = min(k0 + zc, nz);
  const int i = i0 - 2 + hx, j = j0 - 2 + hy;
  const int col = pmodi(j, ny) * nx + pmodi(i, nx);
  const bool frole = tid < PNF;
  const bool orole = tid < PNI && i < nx && j < ny;
  const double eps = g.eps;
  const double* __restrict__ phig = a.phi;

  auto clampv = [](double ph) {
    double val = fmin(ph, 1.0);
    if (CLAMP) val = fmax(val, 0.0);
    return val;
  };
  auto psi_of = [&](double ph) {  // multi/main.f90:527-528
    const double val = clampv(ph);
    return eps * log(div_nr(val + ENUM, 1.0 - val + ENUM));
  };
  // F of this position at one plane (multi/main.f90:530, 559-561, 586-589, 609-614): Q the
  // plane's shared psi at this position, dz the psi difference along z, ph/ps this position's
  // phi/psi.  The fused multiply-adds are written out, so the rounding does not depend on how
  // the compiler contracts each copy of the loop body.
  auto F_of = [&](const double* __restrict__ Q, double dz, double ph, double ps, double& fx, double& fy,
                  double& fz) {
    double nxr = Q[1] - Q[-1];
    double nyr = Q[PHX] - Q[-PHX];
    double nzr = dz;
    const double n2 = __fma_rn(nzr, nzr, __fma_rn(nyr, nyr, __dmul_rn(nxr, nxr)));
    // n/(|n| + 1e-16) as n rsqrt(|n|^2), 0 for n = 0: one reciprocal square root instead of a
    // square root and a division (k_phase 2.58 -> 2.38 ms at 512^3).  It differs from the
    // reference's quotient by 1e-16/|n| relative: far below rounding where the interface makes
    // |n| large, and where psi is flat (|n| tiny) 1/4 (1 - t^2) ~ phi (1 - phi) ~ 0 multiplies it.
    const double normag = n2 > 0.0 ? rsqrt(n2) : 0.0;
    nxr = nxr * normag;
    nyr = nyr * normag;
    nzr = nzr * normag;
    const double val = clampv(ph);
    const double tt = (ps == ps) ? (2.0 * val - 1.0) * TNORM : ps;
    const double fac = 0.25 * __fma_rn(-tt, tt, 1.0);
    fx = fac * nxr;
    fy = fac * nyr;
    fz = fac * nzr;
  };

  const double gamma = 1.0 * a.sc->gumax;
  const double mu_ = a.sc->mean[0], mv_ = a.sc->mean[1], mw_ = a.sc->mean[2];
  const double dxi = g.dxi, ddxi = g.ddxi;
  const double hdxi = 0.5 * dxi;  // (x*0.5)*dxi == x*(0.5*dxi) exactly
  // the right-hand side's constant factors, applied once per sum of terms (see the output block)
  const double c_lap = gamma * (eps * ddxi), c_shp = gamma * -hdxi;
  int c = k0 * plane + col;  // own cell (output role)
  const int dux = (i + 1 == nx) ? 1 - nx : 1;
  const int dvy = (j + 1 == ny) ? (1 - ny) * nx : nx;
  double w0 = orole ? __ldg(a.w + c) : 0.0;

  // Iteration k computes psi(k+2), F(k+1) and the output plane k.  The loop starts four planes
  // below the chunk: k0-4 and k0-3 only fill psi(k0-2), psi(k0-1), k0-2 and k0-1 add F(k0-1),
  // F(k0).  Every psi and F is thus evaluated by the loop body, so the values of a plane do
  // not depend on where a z chunk starts.  Register state entering iteration k: phi k-1..k+2,
  // psi k, k+1, Fz k-1, k.
  double f_m1 = 0.0, f_0 = 0.0, f_p1 = 0.0, f_p2 = phig[pmodi(k0 - 2, nz) * plane + col];
  double s_0 = 0.0, s_p1 = 0.0, z_m1 = 0.0, z_0 = 0.0;
  int o3 = pmodi(k0 - 1, nz) * plane + col;  // phi(k+3) of the first iteration

  // One plane of the loop; P is the parity of k, so the double-buffer slots are compile-time
  // offsets: slot(k) = slot(k + 2) = P PNT, slot(k + 1) = (1 - P) PNT.
  auto plane_iter = [&](auto par, int k) {
    constexpr int P = decltype(par)::value;
    constexpr int SK = P * PNT, SK1 = (1 - P) * PNT;
    const bool out = orole && k >= k0;
    const double f_p3 = (k + 1 < k1) ? phig[o3] : 0.0;
    o3 += plane;
    if (o3 >= ntot) o3 -= ntot;
    double u0 = 0, uxp = 0, v0 = 0, vyp = 0, wzp = 0, ro = 0;
    if (out) {
      const int cz = (k + 1 == nz) ? c - (nz - 1) * plane : c + plane;
      u0 = __ldg(a.u + c);
      uxp = __ldg(a.u + c + dux);
      v0 = __ldg(a.v + c);
      vyp = __ldg(a.v + c + dvy);
      wzp = __ldg(a.w + cz);
      ro = a.rphio[c];
    }
    // psi(k+2) of this position; phi(k+1) for the next plane's neighbours
    const double s_p2 = psi_of(f_p2);
    sps[SK] = s_p2;
    sph[SK1] = f_p1;
    // F(k+1) from the shared psi(k+1) (written last iteration) and the own psi(k+2) - psi(k)
    double z_p1 = 0.0;
    if (frole && k >= k0 - 2) {
      double fx, fy;
      F_of(sps + SK1, s_p2 - s_0, f_p1, s_p1, fx, fy, z_p1);
      sfx[SK1] = fx;
      sfy[SK1] = fy;
    }
    // output plane k from the shared phi(k), Fx/Fy(k) and the own column
    if (out) {
      const double u_0 = u0 - mu_, u_x = uxp - mu_, v_0 = v0 - mv_, v_y = vyp - mv_;
      const double w_0 = w0 - mw_, w_z = wzp - mw_;
      const double* P0 = sph + SK;
      const double p0 = f_0;
      const double pxp = P0[1], pxm = P0[-1], pyp = P0[PHX], pym = P0[-PHX];
      const double pzp = f_p1, pzm = f_m1;
      // multi/main.f90:551-557 and :609-614, with each group's constant factor taken out of its
      // sum (the same expression up to rounding: a few ulp of the terms, far inside the 1e-12
      // parity bound):
      //   rhs = -dxi/2 sum_d (u_d+ (phi+ + phi) - u_d (phi + phi-))                 advection
      //         + gamma eps ddxi (sum of the six neighbours - 6 phi)                diffusion
      //         - gamma dxi/2 sum_d (F_d+ - F_d-)                                   sharpening
      const double* Fx = sfx + SK;
      const double* Fy = sfy + SK;
      const double adv = (__fma_rn(u_x, pxp + p0, -u_0 * (p0 + pxm)) + __fma_rn(v_y, pyp + p0, -v_0 * (p0 + pym))) +
                         __fma_rn(w_z, pzp + p0, -w_0 * (p0 + pzm));
      const double lap = ((pxp + pxm) + (pyp + pym)) + __fma_rn(-6.0, p0, pzp + pzm);
      const double shp = ((Fx[1] - Fx[-1]) + (Fy[PHX] - Fy[-PHX])) + (z_p1 - z_m1);
      const double rhs = __fma_rn(-hdxi, adv, __fma_rn(c_lap, lap, c_shp * shp));
      // :625-626
      a.phin[c] = __fma_rn(dta, rhs, __fma_rn(-dtb, ro, p0));
      a.rphio[c] = rhs;
      w0 = wzp;
      c += plane;
    }
    __syncthreads();
    f_m1 = f_0;
    f_0 = f_p1;
    f_p1 = f_p2;
    f_p2 = f_p3;
    s_0 = s_p1;
    s_p1 = s_p2;
    z_m1 = z_0;
    z_0 = z_p1;
  };
  // k0 and the chunk are even (launch_phase), so k0 - 4 is even and the trip count too; two
  // planes per iteration, four per unrolled body (2.58 ms at 512^3 with runtime slots, against
  // 2.67 for two, 2.69 for one and 2.60 for eight planes, where it spills); the same bits for
  // every unroll factor
#pragma unroll 2
  for (int k = k0 - 4; k < k1; k += 2) {
    plane_iter(std::integral_constant<int, 0>{}, k);
    plane_iter(std::integral_constant<int, 1>{}, k + 1);
  }
}

template <bool CLAMP>
__global__ void __launch_bounds__(PNT, PMINB) k_phase(const __grid_constant__ PhaseArgs a) {
  extern __shared__ __align__(16) unsigned char smraw[];
  phase_tile<CLAMP>(a, a.dta, a.dtb, blockIdx.x, blockIdx.y, blockIdx.z, smraw);
}

// The phase step of many boxes in one launch: persistent blocks (one per SM) take work items
// (box, tile x, tile y, z chunk) from a device queue until it is empty.  A box's arguments
// (including its resolved z chunk) come from b.args; alpha, beta are the step's.  The boxes of
// one launch share the psi clamp (CLAMP).
template <bool CLAMP>
__global__ void __launch_bounds__(PNT, PMINB) k_phase_batch(const __grid_constant__ BatchArgs<PhaseArgs> b) {
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ int s_item;
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(b.counter, 1);
    __syncthreads();
    const int it = s_item;
    __syncthreads();  // every thread has the item before thread 0 takes the next one
    if (it >= b.nitems) break;
    const int4 w = b.items[it];
    const PhaseArgs& a = b.args[w.x];
    phase_tile<CLAMP>(a, a.g.dt * b.alpha, a.g.dt * b.beta, w.y, w.z, w.w, smraw);
  }
}

int phase_zchunk(const Geo& g, int requested) {
  // Default chunk: 256 planes where that still leaves six waves of one block on each of the 148
  // SMs (the four planes of warm-up below a chunk cost 1.6%: 2.27 against 2.31 ms at 512^3 with
  // 128 planes), else 128 planes where that leaves eight waves (3% instead of 6%: 2.667 against
  // 2.723 ms at 512^3 with 64), otherwise PZC.  Results do not depend on the chunk.
  if (requested > 0) return requested;
  const long long cols = (long long)((g.nx + PTX - 1) / PTX) * ((g.ny + PTY - 1) / PTY);
  if (cols * ((g.nz + 255) / 256) >= 6 * 148) return 256;
  return cols * ((g.nz + 127) / 128) >= 8 * 148 ? 128 : PZC;
}

dim3 phase_grid(const Geo& g, int zc) {
  return dim3((g.nx + PTX - 1) / PTX, (g.ny + PTY - 1) / PTY, (g.nz + zc - 1) / zc);
}

cudaError_t launch_phase_batch(const BatchArgs<PhaseArgs>& b, bool clamp, int nsm, cudaStream_t st) {
  constexpr size_t smem = 8 * sizeof(double) * PNT;
  auto kern = clamp ? k_phase_batch<true> : k_phase_batch<false>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(b.counter, 0, sizeof(int), st);
  if (e != cudaSuccess) return e;
  kern<<<b.nitems < nsm ? b.nitems : nsm, PNT, smem, st>>>(b);
  return cudaGetLastError();
}

cudaError_t launch_phase(const PhaseArgs& a, cudaStream_t st) {
  constexpr size_t smem = 8 * sizeof(double) * PNT;  // psi, phi, Fx, Fy: two planes each
  auto kern = a.clamp ? k_phase<true> : k_phase<false>;
  static int attr_set[64][2] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 64 || !attr_set[dev][a.clamp ? 1 : 0]) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    if (dev < 64) attr_set[dev][a.clamp ? 1 : 0] = 1;
  }
  PhaseArgs b = a;
  b.dta = a.g.dt * a.alpha;
  b.dtb = a.g.dt * a.beta;
  b.zchunk = phase_zchunk(a.g, a.zchunk);
  const int zc = b.zchunk;
  if (zc % 2 || a.g.nz % 2) return cudaErrorInvalidValue;  // the plane loop runs two planes at a time
  kern<<<phase_grid(a.g, zc), PNT, smem, st>>>(b);
  return cudaGetLastError();
}

}  // namespace mhit
