// Momentum predictor: multi/main.f90:658-802 in one pass over the grid.
//
// Per cell: conservative advection (h11..h33, :672-694), viscous Laplacian (:696-707), ABC
// forcing from the per-axis sin/cos tables (:712-714), and with the phase field the
// chemical-potential surface-tension force (:734-739) averaged to the faces (:768-770) -- the
// reference's fxst/fyst/fzst arrays and their 6 halo exchanges (:746-757) are never stored.
// Then the AB2 update u* = u + dt (alpha rhs - beta rhs_o), rhs_o = rhs (:771-776 / :787-792).
//
// Blocking: a block owns a MTX x MTY column of cells and marches up a chunk of z planes.
// Rings of z planes live in shared memory, filled with cp.async one plane ahead of use:
//   u, v, w   planes k-1..k+1 read, k+2 in flight (4 slots), y halo 1, x rows [-2, MTX+2)
//   phi^{n+1} planes k-2..k+2 read, k+3 in flight (8 slots), y halo [-2,+1], x rows [-2, MTX+2)
//   chempot   planes k-1, k read, k+1 written (4 slots) over x [-1, MTX-1], y [-1, MTY-1]
// so every input byte crosses HBM once (plus the x/y halo re-read from L2) and the chemical
// potential is evaluated once per cell.  Iteration k computes the chemical potential of plane
// k+1 and the output of plane k after a single barrier: every shared read of the iteration
// reads what earlier iterations wrote or copied.  The rows start at x = -2, an even column because the
// tile origin and nx are even, so they are copied as 16-byte pairs with cp.async.cg, which
// bypasses L1: with 8-byte copies (which allocate in L1) the kernel was 3.06 ms at 512^3 and
// 4.24 ms when the shared-memory carveout left L1 small; with 16-byte L2-only copies it is
// 2.96 ms whatever the carveout.
//
// The velocity read here is the stored one minus the running mean of the previous
// projection (DevScalars::mean); subtracting on read is exactly the reference's
// u = u - gumean (:977-981) done lazily.
#include <cuda_pipeline.h>

#include "common.cuh"
#include "kernels.h"

namespace mhit {

constexpr int MTX = 32, MTY = 8, MNT = MTX * MTY;
constexpr int MZC = 32;                       // default z planes per block
constexpr int UPX = MTX + 4, UPY = MTY + 2;   // u/v/w plane: x in [-2, T+2), y in [-1, T+1)
constexpr int UPL = UPX * UPY;
constexpr int PPX = MTX + 4, PPY = MTY + 3;   // phi plane: x in [-2, T+2), y in [-2, T+1)
constexpr int PPL = PPX * PPY;
constexpr int CPX = MTX + 1, CPY = MTY + 1;   // chempot plane: x,y in [-1, T)
constexpr int CPL = CPX * CPY;
constexpr int UPAIRS = UPY * (UPX / 2), PPAIRS = PPY * (PPX / 2);  // 16-byte copies per plane
static_assert(UPAIRS <= MNT && PPAIRS <= MNT, "one pair per thread and plane");
// ring slots padded to whole 128-byte lines, the alignment a TMA box destination needs
constexpr int UPS = (UPL * 8 + 127) / 128 * 16, PPS = (PPL * 8 + 127) / 128 * 16;  // doubles
constexpr unsigned UBYTES = UPL * 8, PBYTES = PPL * 8;  // bytes of one box

template <bool PHI> struct MomSmem;
template <> struct MomSmem<false> {
  double u[4][UPS], v[4][UPS], w[4][UPS];
  unsigned long long bar[2];  // TMA completion, one per alternating group of boxes
};
template <> struct MomSmem<true> {
  double u[4][UPS], v[4][UPS], w[4][UPS];
  double phi[8][PPS];
  double cp[4][CPL];
  unsigned long long bar[2];
};

constexpr long long MOM_WAIT_LIMIT = 1ll << 26;  // polls of an mbarrier before giving up (seconds)

__device__ __forceinline__ uint32_t sm_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void tma_box(const void* dst, const CUtensorMap* map, int x, int y, int z, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
      ::"r"(sm_addr(dst)), "l"(map), "r"(x), "r"(y), "r"(z), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void expect_tx(uint32_t bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t parity) {
  for (long long it = 0; it < MOM_WAIT_LIMIT; ++it) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if (it > 64) __nanosleep(32);
  }
  return false;
}

// 16-byte global -> shared copy through L2 only (cp.async.cg)
__device__ __forceinline__ void cp16(void* dst, const void* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}

__device__ __forceinline__ int pmod_int(int x, int n) {
  x %= n;
  return x < 0 ? x + n : x;
}

// One z column of MTX x MTY cells, tile (bx, by), chunk bz, of the box a, with the step's
// alpha, beta (AB2 weights).
template <bool PHI>
__device__ __forceinline__ void mom_tile(const MomArgs& a, double alpha, double beta, int bx, int by, int bz,
                                         unsigned char* smraw) {
  MomSmem<PHI>& S = *reinterpret_cast<MomSmem<PHI>*>(smraw);
  const Geo& g = a.g;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const size_t plane = (size_t)nx * ny;
  const int i0 = bx * MTX, j0 = by * MTY;
  const int zc = a.zchunk > 0 ? a.zchunk : MZC;
  const int k0 = bz * zc;
  const int k1 = min(k0 + zc, nz);
  const int tid = threadIdx.x;

  // this thread's 16-byte pair of a u/v/w plane and of a phi plane: source offset in the
  // plane, destination index in the ring plane (-1: no pair)
  int up_src = -1, up_dst = 0, pp_src = -1, pp_dst = 0;
  if (tid < UPAIRS) {
    const int y = tid / (UPX / 2), xp = tid - y * (UPX / 2);
    up_src = pmod_int(j0 - 1 + y, ny) * nx + pmod_int(i0 - 2 + 2 * xp, nx);
    up_dst = y * UPX + 2 * xp;
  }
  if (PHI && tid < PPAIRS) {
    const int y = tid / (PPX / 2), xp = tid - y * (PPX / 2);
    pp_src = pmod_int(j0 - 2 + y, ny) * nx + pmod_int(i0 - 2 + 2 * xp, nx);
    pp_dst = y * PPX + 2 * xp;
  }
  auto copy_phi = [&](int m, size_t base) {
    if constexpr (PHI) {
      if (pp_src >= 0)
        cp16(&reinterpret_cast<MomSmem<true>&>(S).phi[(m - k0 + 16) & 7][pp_dst], a.phi + base + pp_src);
    }
  };
  auto issue_uvw = [&](int m) {
    const size_t base = (size_t)pmod_int(m, nz) * plane;
    const int su = (m - k0 + 16) & 3;
    if (up_src >= 0) {
      cp16(&S.u[su][up_dst], a.u + base + up_src);
      cp16(&S.v[su][up_dst], a.v + base + up_src);
      cp16(&S.w[su][up_dst], a.w + base + up_src);
    }
  };
  auto issue_phi = [&](int m) { copy_phi(m, (size_t)pmod_int(m, nz) * plane); };

  // A block whose rings need no periodic wrap in x and y has every ring plane in one TMA box per
  // field (x from i0-2, y from j0-1 for u, v, w and from j0-2 for phi; z wraps by the plane
  // index): one thread issues the boxes of a plane group and an mbarrier tracks their bytes.
  // The other blocks copy 16-byte pairs per thread (cp.async).  Groups alternate between the two
  // barriers: group g (0: the loop's prologue, then one per iteration) completes phase g/2 of
  // bar[g % 2].
  const bool tma = a.tma && i0 >= 2 && i0 + MTX + 2 <= nx && j0 >= 2 && j0 + MTY + 1 <= ny;
  const uint32_t bar0 = sm_addr(&S.bar[0]);
  if (tma && tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar0) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar0 + 8) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (tma) __syncthreads();
  auto tma_uvw = [&](int m, uint32_t bar) {
    const int su = (m - k0 + 16) & 3, z = pmod_int(m, nz);
    tma_box(&S.u[su][0], &a.tmu, i0 - 2, j0 - 1, z, bar);
    tma_box(&S.v[su][0], &a.tmv, i0 - 2, j0 - 1, z, bar);
    tma_box(&S.w[su][0], &a.tmw, i0 - 2, j0 - 1, z, bar);
  };
  auto tma_phi = [&](int m, uint32_t bar) {
    if constexpr (PHI)
      tma_box(&reinterpret_cast<MomSmem<true>&>(S).phi[(m - k0 + 16) & 7][0], &a.tmphi, i0 - 2, j0 - 2,
              pmod_int(m, nz), bar);
  };
  bool waits_ok = true;

  const double eps = g.eps, epsi = g.epsi, ddxi = g.ddxi, dxi = g.dxi;
  // chemical potential (multi/main.f90:735) of plane m over the CPX x CPY region
  auto chempot_plane = [&](int m) {
    if constexpr (PHI) {
      auto& P = reinterpret_cast<MomSmem<true>&>(S).phi;
      const int pm = (m - k0 + 15) & 7, p0 = (m - k0 + 16) & 7, pp = (m - k0 + 17) & 7;
      const int sc = (m - k0 + 16) & 3;
      for (int e = tid; e < CPL; e += MNT) {
        const int y = e / CPX, x = e - y * CPX;
        const int q = (y + 1) * PPX + (x + 1);  // phi index of (i0-1+x, j0-1+y)
        const double c = P[p0][q];
        const double s = P[p0][q + 1] + P[p0][q - 1] + P[p0][q + PPX] + P[p0][q - PPX] + P[pp][q] + P[pm][q];
        reinterpret_cast<MomSmem<true>&>(S).cp[sc][e] = c * (1.0 - c) * (1.0 - 2.0 * c) * epsi - eps * (s - 6.0 * c) * ddxi;
      }
    }
  };

  const double mu_ = a.sc->mean[0], mv_ = a.sc->mean[1], mw_ = a.sc->mean[2];

  // Iteration k computes the chemical potential of plane k+1 and the output of plane k after
  // one barrier; the copies it waits for (u, v, w(k+1), phi(k+2)) were issued one iteration
  // earlier.  With the phase field the loop starts at k0-2 (k0-2, k0-1 only fill the chemical
  // potential of k0-1 and k0), so every chemical potential comes from the loop body.
  const int ks = PHI ? k0 - 2 : k0;
  if (tma) {
    if (tid == 0) {
      if constexpr (PHI) {
        expect_tx(bar0, 3 * UBYTES + 3 * PBYTES);
        tma_phi(k0 - 2, bar0);
        tma_phi(k0 - 1, bar0);
        tma_phi(k0, bar0);
        tma_uvw(k0 - 1, bar0);
      } else {
        expect_tx(bar0, 9 * UBYTES);
        tma_uvw(k0 - 1, bar0);
        tma_uvw(k0, bar0);
        tma_uvw(k0 + 1, bar0);
      }
    }
  } else {
    if constexpr (PHI) {
      issue_phi(k0 - 2);
      issue_phi(k0 - 1);
      issue_phi(k0);
      issue_uvw(k0 - 1);
    } else {
      issue_uvw(k0 - 1);
      issue_uvw(k0);
      issue_uvw(k0 + 1);
    }
    __pipeline_commit();
  }

  const int tx = tid % MTX, ty = tid / MTX;
  const int i = i0 + tx, j = j0 + ty;
  const bool own = i < nx && j < ny;
  const double* t = a.tabs;
  const double sxi = own ? __ldg(t + i) : 0.0, cxi = own ? __ldg(t + nx + i) : 0.0;
  const double syj = own ? __ldg(t + 2 * nx + j) : 0.0, cyj = own ? __ldg(t + 2 * nx + ny + j) : 0.0;
  // constant factors of the right-hand side, applied once per sum of terms (the reference's
  // expression up to rounding: a few ulp of the terms, far inside the 1e-12 parity bound)
  const double c_adv = -0.25 * dxi;                    // -(h11 + h12 + h13) / 4 dxi
  const double c_vis = g.mu * ddxi * g.rhoi;           // mu lap(u) / rho
  const double c_st = 6.0 * g.sigma * 0.25 * dxi * g.rhoi;  // face average of the force / rho
  const double dta = g.dt * alpha, dtb = g.dt * beta;
  const int uq = (ty + 1) * UPX + (tx + 2);   // own cell in the u/v/w plane
  const int pq = (ty + 2) * PPX + (tx + 2);   // own cell in the phi plane
  const int cq = (ty + 1) * CPX + (tx + 1);   // own cell in the chempot plane

  // four planes per unrolled body: 2.86 ms at 512^3 against 2.91 not unrolled and 2.93 unrolled
  // twice; the same bits
#pragma unroll 4
  for (int k = ks; k < k1; ++k) {
    const bool out = own && k >= k0;
    const size_t c = (size_t)(k >= k0 ? k : k0) * plane + (size_t)(own ? j : 0) * nx + (own ? i : 0);
    double ruo = 0.0, rvo = 0.0, rwo = 0.0;
    if (out) {
      ruo = a.ru[c];
      rvo = a.rv[c];
      rwo = a.rw[c];
    }
    // the copies issued one iteration earlier have landed (this thread's, or the block's TMA
    // group); after the barrier everyone's have, and everyone is done with iteration k-1
    if (tma) {
      const int gi = k - ks;
      if (!bar_wait(bar0 + 8 * (gi & 1), (gi >> 1) & 1)) waits_ok = false;
    } else {
      __pipeline_wait_prior(0);
    }
    __syncthreads();
    if (k + 1 < k1) {
      if (tma) {
        if (tid == 0) {
          const uint32_t b = bar0 + 8 * ((k - ks + 1) & 1);
          expect_tx(b, PHI ? 3 * UBYTES + PBYTES : 3 * UBYTES);
          tma_uvw(k + 2, b);
          tma_phi(k + 3, b);
        }
      } else {
        issue_uvw(k + 2);
        issue_phi(k + 3);
      }
    }
    if (!tma) __pipeline_commit();
    if (k + 1 < k1) chempot_plane(k + 1);
    if (out) {
      const int sm = (k - k0 + 15) & 3, s0 = (k - k0 + 16) & 3, sp = (k - k0 + 17) & 3;
      const double* U0 = S.u[s0];
      const double* V0 = S.v[s0];
      const double* W0 = S.w[s0];
      const double u0 = U0[uq] - mu_, v0 = V0[uq] - mv_, w0 = W0[uq] - mw_;
      const double uxp = U0[uq + 1] - mu_, uxm = U0[uq - 1] - mu_, uyp = U0[uq + UPX] - mu_, uym = U0[uq - UPX] - mu_;
      const double uzp = S.u[sp][uq] - mu_, uzm = S.u[sm][uq] - mu_;
      const double vxp = V0[uq + 1] - mv_, vxm = V0[uq - 1] - mv_, vyp = V0[uq + UPX] - mv_, vym = V0[uq - UPX] - mv_;
      const double vzp = S.v[sp][uq] - mv_, vzm = S.v[sm][uq] - mv_;
      const double wxp = W0[uq + 1] - mw_, wxm = W0[uq - 1] - mw_, wyp = W0[uq + UPX] - mw_, wym = W0[uq - UPX] - mw_;
      const double wzp = S.w[sp][uq] - mw_, wzm = S.w[sm][uq] - mw_;
      const double v_imjp = V0[uq + UPX - 1] - mv_, w_imkp = S.w[sp][uq - 1] - mw_, u_ipjm = U0[uq - UPX + 1] - mu_;
      const double w_jmkp = S.w[sp][uq - UPX] - mw_, u_ipkm = S.u[sm][uq + 1] - mu_, v_jpkm = S.v[sm][uq + UPX] - mv_;
      // multi/main.f90:672-694: the fluxes h = a^2 - b^2 and h = a c - b d as one product and
      // one fused multiply-add each
      auto dsq = [](double a1, double b1) { return __fma_rn(a1, a1, -(b1 * b1)); };
      auto dpr = [](double a1, double c1, double b1, double d1) { return __fma_rn(a1, c1, -(b1 * d1)); };
      const double h11 = dsq(uxp + u0, u0 + uxm);
      const double h12 = dpr(uyp + u0, vyp + v_imjp, u0 + uym, v0 + vxm);
      const double h13 = dpr(uzp + u0, wzp + w_imkp, u0 + uzm, w0 + wxm);
      const double h21 = dpr(uxp + u_ipjm, vxp + v0, u0 + uym, v0 + vxm);
      const double h22 = dsq(vyp + v0, v0 + vym);
      const double h23 = dpr(wzp + w_jmkp, vzp + v0, w0 + wym, v0 + vzm);
      const double h31 = dpr(wxp + w0, uxp + u_ipkm, w0 + wxm, u0 + uzm);
      const double h32 = dpr(vyp + v_jpkm, wyp + w0, v0 + vzm, w0 + wym);
      const double h33 = dsq(wzp + w0, w0 + wzm);
      // :696-707: mu (sum of the six neighbours - 6 u) ddxi / rho
      const double lu = ((uxp + uxm) + (uyp + uym)) + __fma_rn(-6.0, u0, uzp + uzm);
      const double lv = ((vxp + vxm) + (vyp + vym)) + __fma_rn(-6.0, v0, vzp + vzm);
      const double lw = ((wxp + wxm) + (wyp + wym)) + __fma_rn(-6.0, w0, wzp + wzm);
      double ru = __fma_rn(c_adv, (h11 + h12) + h13, c_vis * lu);
      double rv = __fma_rn(c_adv, (h21 + h22) + h23, c_vis * lv);
      double rw = __fma_rn(c_adv, (h31 + h32) + h33, c_vis * lw);
      // :712-714
      const double szk = __ldg(t + 2 * nx + 2 * ny + k), czk = __ldg(t + 2 * nx + 2 * ny + nz + k);
      ru = __fma_rn(g.f3, szk, __fma_rn(g.f2, cyj, ru));
      rv = __fma_rn(g.f1, sxi, __fma_rn(g.f3, czk, rv));
      rw = __fma_rn(g.f2, syj, __fma_rn(g.f1, cxi, rw));
      if constexpr (PHI) {
        // :737-739 at the cell and at its -x/-y/-z neighbours, :768-770 face average:
        // 6 sigma mu_c grad(phi) / rho averaged to the face, the central differences taken as
        // (phi+ - phi-) dxi / 2
        auto& SP = reinterpret_cast<MomSmem<true>&>(S);
        const int pmm = (k - k0 + 14) & 7, pm = (k - k0 + 15) & 7, p0 = (k - k0 + 16) & 7, pp = (k - k0 + 17) & 7;
        const int c0s = (k - k0 + 16) & 3, cms = (k - k0 + 15) & 3;
        const double* P0 = SP.phi[p0];
        const double pc = P0[pq];
        const double c0 = SP.cp[c0s][cq];
        const double fx = __fma_rn(c0, P0[pq + 1] - P0[pq - 1], SP.cp[c0s][cq - 1] * (pc - P0[pq - 2]));
        const double fy = __fma_rn(c0, P0[pq + PPX] - P0[pq - PPX], SP.cp[c0s][cq - CPX] * (pc - P0[pq - 2 * PPX]));
        const double fz = __fma_rn(c0, SP.phi[pp][pq] - SP.phi[pm][pq], SP.cp[cms][cq] * (pc - SP.phi[pmm][pq]));
        ru = __fma_rn(c_st, fx, ru);
        rv = __fma_rn(c_st, fy, rv);
        rw = __fma_rn(c_st, fz, rw);
      }
      // :771-776 / :787-792
      a.un[c] = __fma_rn(dta, ru, __fma_rn(-dtb, ruo, u0));
      a.vn[c] = __fma_rn(dta, rv, __fma_rn(-dtb, rvo, v0));
      a.wn[c] = __fma_rn(dta, rw, __fma_rn(-dtb, rwo, w0));
      a.ru[c] = ru;
      a.rv[c] = rv;
      a.rw[c] = rw;
    }
  }
  __pipeline_wait_prior(0);
  // a TMA wait that ran out (the boxes never arrived) is reported through the flag word; the
  // step then fails with MHIT_ERR_TIMEOUT
  if (!waits_ok) atomicOr(&const_cast<DevScalars*>(a.sc)->flag, 4);
}

template <bool PHI>
__global__ void __launch_bounds__(MNT, 3) k_mom(const __grid_constant__ MomArgs a) {
  extern __shared__ __align__(128) unsigned char smraw[];
  mom_tile<PHI>(a, a.alpha, a.beta, blockIdx.x, blockIdx.y, blockIdx.z, smraw);
}

// The momentum step of many boxes in one launch: persistent blocks (three per SM) take work items
// (box, tile x, tile y, z chunk) from a device queue until it is empty.  The boxes' arguments live
// in device memory, so their rings are filled by per-thread copies (no TMA).
template <bool PHI>
__global__ void __launch_bounds__(MNT, 3) k_mom_batch(const __grid_constant__ BatchArgs<MomArgs> b) {
  extern __shared__ __align__(128) unsigned char smraw[];
  __shared__ int s_item;
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(b.counter, 1);
    __syncthreads();
    const int it = s_item;
    __syncthreads();  // every thread has the item before thread 0 takes the next one
    if (it >= b.nitems) break;
    const int4 w = b.items[it];
    mom_tile<PHI>(b.args[w.x], b.alpha, b.beta, w.y, w.z, w.w, smraw);
    __syncthreads();  // the rings are reused by the next item
  }
}

int mom_zchunk(const Geo& g, int requested) {
  // Default chunk: 64 planes where that still leaves eight waves of three blocks on each of the
  // 148 SMs (2.896 against 2.928 ms at 512^3), otherwise MZC.  Results do not depend on it.
  if (requested > 0) return requested;
  const long long cols = (long long)((g.nx + MTX - 1) / MTX) * ((g.ny + MTY - 1) / MTY);
  return cols * ((g.nz + 63) / 64) >= 8 * 148 * 3 ? 64 : MZC;
}

dim3 mom_grid(const Geo& g, int zc) {
  return dim3((g.nx + MTX - 1) / MTX, (g.ny + MTY - 1) / MTY, (g.nz + zc - 1) / zc);
}

cudaError_t launch_mom_batch(const BatchArgs<MomArgs>& b, bool phi, int nsm, cudaStream_t st) {
  const size_t smem = phi ? sizeof(MomSmem<true>) : sizeof(MomSmem<false>);
  auto kern = phi ? k_mom_batch<true> : k_mom_batch<false>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(b.counter, 0, sizeof(int), st);
  if (e != cudaSuccess) return e;
  const int grid = b.nitems < 3 * nsm ? b.nitems : 3 * nsm;
  kern<<<grid, MNT, smem, st>>>(b);
  return cudaGetLastError();
}

template <bool PHI>
static cudaError_t launch_mom_t(const MomArgs& a, cudaStream_t st) {
  const size_t smem = sizeof(MomSmem<PHI>);
  static int attr_set[64] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && !attr_set[dev]) {
    cudaError_t e = cudaFuncSetAttribute(k_mom<PHI>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr_set[dev] = 1;
  }
  MomArgs b = a;
  b.zchunk = mom_zchunk(a.g, a.zchunk);
  k_mom<PHI><<<mom_grid(a.g, b.zchunk), MNT, smem, st>>>(b);
  return cudaGetLastError();
}

cudaError_t launch_mom(const MomArgs& a, cudaStream_t st) {
  return a.phi ? launch_mom_t<true>(a, st) : launch_mom_t<false>(a, st);
}

int mom_field_map(CUtensorMap* map, const double* field, int nx, int ny, int nz, bool phi) {
  EncodeTiledFn enc = tensor_map_encoder();
  if (!enc) return set_error(MHIT_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
  // x-fastest float64 field; box UPX x UPY (PPX x PPY for phi) x 1 plane.  The row stride nx * 8
  // bytes is a multiple of 16 (nx is even) and the box rows are 288 bytes.
  const cuuint64_t dims[3] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz};
  const cuuint64_t strides[2] = {(cuuint64_t)nx * 8, (cuuint64_t)nx * ny * 8};
  const cuuint32_t box[3] = {(cuuint32_t)UPX, (cuuint32_t)(phi ? PPY : UPY), 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<double*>(field), dims, strides, box, estr,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return set_error(MHIT_ERR_CUDA, "cuTensorMapEncodeTiled failed for a momentum ring map");
  return MHIT_OK;
}

}  // namespace mhit
