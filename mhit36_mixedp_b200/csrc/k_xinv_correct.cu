// The inverse x transform fused with the projection: multi/main.f90:909-912 and :942-1003 in one
// pass over HBM.
//
// Apart, k_fftx_inv writes the pressure and k_correct reads it back beside u*, v*, w* (the
// pressure's -x, -y and -z neighbours of each cell).  Here a block owns XO = 7 consecutive y
// lines of a chunk of z planes and marches up z.  Per plane the block
//   1. fetches the plane's 8 half-spectrum rows (its 7 lines and the line below them, j0 - 1,
//      the -y neighbour of its first line) with cp.async, two planes ahead, into a ring of three
//      tile buffers in shared memory;
//   2. C2R-transforms the 8 rows in place (the untangle and the Stockham stages of k_fftx_inv, so
//      the on-demand transform of the same spectrum gives the same doubles);
//   3. projects its 7 lines (u -= dt/rho (p - p(i-1)) dxi, and v, w along y, z: :953-955) with
//      p(i-1) and p(j-1) from the tile and p(k-1) carried by each thread for its own x pairs from
//      the plane below (the loop starts one plane below the chunk for them), and accumulates the
//      per-block sums and maxima of k_correct.
// The warps are specialised so the two kinds of work overlap: the transform warps (steps 1-2,
// synchronising among themselves on named barrier 1) transform plane i while the stream warps
// (step 3: the u, v, w traffic) project plane i - 1.  At nx = 512 each stream thread stages its
// u, v, w pairs of the next plane in shared memory by cp.async as it finishes each pair of the
// current one, so a whole plane's loads are in flight without holding registers.  A tile buffer
// passes between them by named barriers: "ready" (2 + buffer: transform warps arrive, stream
// warps wait) and "free" (5 + buffer: stream warps arrive, transform warps wait before fetching
// plane i + 2 into the buffer of plane i - 1).  Hardware barriers, no spin loops; every arrival
// has its matching wait, and a barrier's next phase starts only after its last one completed.
//
// The pressure never goes to HBM: the library transforms it from the spectrum, which stays intact
// until the next step's x pass, when something reads it.  Per cell this moves the spectrum once
// (8/7 of it, the halo line) and u, v, w in and out: 48 + 8 (FP64) or 48 + 4 (FP32) bytes of the
// 72 / 60 of the two passes.
//
// INC (incremental FP32 solve): the transform is the correction delta; the pressure is
// qold + delta formed in FP64 (qold, the FP32 predictor, read at the cell and its -x and -y
// neighbours), and fl32 of it goes to qnew, the next step's predictor (a second buffer, so no
// block overwrites a predictor another block still reads).
#include <cuda_pipeline.h>

#include <algorithm>

#include "common.cuh"
#include "fft_core.cuh"
#include "kernels.h"

namespace mhit {

constexpr int XL = 8;       // lines transformed per plane (a power of two: the tile swizzle)
constexpr int XO = XL - 1;  // lines projected per plane: tile line 0 is the -y halo
constexpr int XZC_MIN = 8;  // fewest z planes per block of the default chunking
constexpr int XNB = 3;      // tile buffers: loading, transforming, being projected

// transform threads: one butterfly of the schedule's largest radix each (at most 256: larger tiles
// loop), at least 64
template <int M> __host__ __device__ constexpr int xc_maxr() {
  int m = 0;
  for (int s = 0; s < Radix<M>::ns; ++s) m = Radix<M>::r[s] > m ? Radix<M>::r[s] : m;
  return m;
}
template <int M> __host__ __device__ constexpr int xc_nf() {
  return M / xc_maxr<M>() * XL > 256 ? 256 : (M / xc_maxr<M>() * XL < 64 ? 64 : M / xc_maxr<M>() * XL);
}
// stream threads: 7 x pairs of the 7 lines each at nx = 512, 14 at nx = 1024
template <int M> __host__ __device__ constexpr int xc_ns() { return M >= 256 ? 256 : 128; }
template <int M> __host__ __device__ constexpr int xc_ppt() { return (XO * M + xc_ns<M>() - 1) / xc_ns<M>(); }
template <typename T, int M> __host__ __device__ constexpr size_t xc_spec_bytes() {
  return (size_t)XNB * (M + 1) * XL * sizeof(Cx<T>);
}
// incremental solve: beside each spectrum tile, the 8 lines of the FP32 predictor (row-major)
template <typename T, int M, bool INC> __host__ __device__ constexpr size_t xc_tile_bytes() {
  return xc_spec_bytes<T, M>() + (INC ? (size_t)XNB * XL * 2 * M * sizeof(float) : 0);
}
// The pressure each stream thread carries to the next plane (the -z neighbour) lives in shared
// memory where it fits beside the tiles (in registers it would crowd out the loads), else in
// registers (FP64 at nx = 1024).
template <typename T, int M, bool INC> __host__ __device__ constexpr bool xc_pz_shared() {
  return xc_tile_bytes<T, M, INC>() + (size_t)xc_ns<M>() * xc_ppt<M>() * 16 <= 227 * 1024;
}
template <typename T, int M, bool INC> __host__ __device__ constexpr size_t xc_smem() {
  return xc_tile_bytes<T, M, INC>() + (xc_pz_shared<T, M, INC>() ? (size_t)xc_ns<M>() * xc_ppt<M>() * 16 : 0);
}
// where the loads go through registers: x pairs a stream thread loads before computing any of them
template <typename T, int M, bool INC> __host__ __device__ constexpr int xc_pb() {
  return xc_pz_shared<T, M, INC>() ? 7 : 2;
}
// Where it fits as well (nx = 512), each stream thread stages its u, v, w pairs of the NEXT plane
// in shared memory with cp.async, pair by pair as it finishes the current plane's pair (one
// commit group per pair), so a whole plane's loads (~86 KB per SM) are in flight while the
// current plane is projected and no registers hold them.
template <typename T, int M, bool INC> __host__ __device__ constexpr size_t xc_uvw_bytes() {
  return (size_t)3 * xc_ns<M>() * xc_ppt<M>() * 16;
}
template <typename T, int M, bool INC> __host__ __device__ constexpr bool xc_uvw_shared() {
  return xc_pz_shared<T, M, INC>() && xc_smem<T, M, INC>() + xc_uvw_bytes<T, M, INC>() <= 227 * 1024;
}
template <typename T, int M, bool INC> __host__ __device__ constexpr size_t xc_smem_all() {
  return xc_smem<T, M, INC>() + (xc_uvw_shared<T, M, INC>() ? xc_uvw_bytes<T, M, INC>() : 0);
}

__device__ __forceinline__ void bar_sync(int id, int count) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}
__device__ __forceinline__ void bar_arrive(int id, int count) {
  asm volatile("bar.arrive %0, %1;" ::"r"(id), "r"(count) : "memory");
}

template <typename T, int M, bool INC>
__global__ void __launch_bounds__(xc_nf<M>() + xc_ns<M>(), 1) k_xinv_correct(const XcArgs a) {
  constexpr int NF = xc_nf<M>(), NS = xc_ns<M>(), NT = NF + NS;
  constexpr int TL = (M + 1) * XL;         // elements of one tile buffer
  constexpr int NP = XO * M;               // x pairs projected per plane
  constexpr int PPT = xc_ppt<M>();         // ... per stream thread
  constexpr int XPB = xc_pb<T, M, INC>();
  constexpr bool PZS = xc_pz_shared<T, M, INC>();
  constexpr bool UVS = xc_uvw_shared<T, M, INC>();
  constexpr int nx = 2 * M;
  constexpr int QL = XL * nx;              // floats of one predictor tile
  extern __shared__ __align__(16) unsigned char smraw[];
  Cx<T>* tiles = reinterpret_cast<Cx<T>*>(smraw);
  float* qtiles = reinterpret_cast<float*>(smraw + xc_spec_bytes<T, M>());
  const Geo& g = a.g;
  const int ny = g.ny, nz = g.nz;
  const int j0 = blockIdx.x * XO;
  const int k0 = blockIdx.y * a.zc, k1 = min(k0 + a.zc, nz);
  const int nplanes = k1 - k0 + 1;  // with the plane below the chunk
  const int tid = threadIdx.x;
  double su = 0.0, sv = 0.0, sw_ = 0.0;
  double mu = -INFINITY, mv = -INFINITY, mw = -INFINITY;

  if (tid < NF) {
    // ---------------------------------------------------------- transform warps
    const Cx<T>* __restrict__ spec = static_cast<const Cx<T>*>(a.spec);
    const Cx<T>* __restrict__ twx = static_cast<const Cx<T>*>(a.twx);
    const int pitch = g.pitch;
    // rows j0-1 .. j0+6 of plane index i (plane k0 - 1 + i, periodic in y and z; rows past ny in
    // a tail tile wrap and are transformed but not projected)
    auto fetch = [&](int i) {
      int kk = k0 - 1 + i;
      kk = kk < 0 ? kk + nz : kk;
      const Cx<T>* src = spec + (size_t)kk * ny * pitch;
      Cx<T>* s = tiles + (i % XNB) * TL;
      for (int e = tid; e < TL; e += NF) {
        const int b = e / (M + 1), kx = e - b * (M + 1);
        int j = j0 - 1 + b;
        j = j < 0 ? j + ny : (j >= ny ? j - ny : j);
        __pipeline_memcpy_async(&s[sw<XL>(kx, b)], &src[(size_t)j * pitch + kx], sizeof(Cx<T>));
      }
      if constexpr (INC) {
        // the same 8 lines of the predictor, 16-byte chunks (a line is nx floats, nx % 4 == 0)
        const float* qsrc = a.qold + (size_t)kk * ny * nx;
        float* qs = qtiles + (i % XNB) * QL;
        for (int e = tid; e < QL / 4; e += NF) {
          const int b = e / (nx / 4), c4 = e - b * (nx / 4);
          int j = j0 - 1 + b;
          j = j < 0 ? j + ny : (j >= ny ? j - ny : j);
          __pipeline_memcpy_async(&qs[b * nx + 4 * c4], &qsrc[(size_t)j * nx + 4 * c4], 16);
        }
      }
      __pipeline_commit();
    };
    fetch(0);
    if (nplanes > 1) fetch(1);
    for (int i = 0; i < nplanes; ++i) {
      Cx<T>* s = tiles + (i % XNB) * TL;
      if (i + 1 < nplanes) __pipeline_wait_prior(1);  // plane i's rows (plane i+1's may still fly)
      else __pipeline_wait_prior(0);
      bar_sync(1, NF);
      c2r_untangle<T, M, XL, NF>(s, twx);
      bar_sync(1, NF);
      fft_tile<T, M, XL, NF, true, Radix<M>, SyncNamed<1, NF>>(s, twx, 2);
      bar_arrive(2 + i % XNB, NT);  // plane i's pressure is in its buffer
      if (i + 2 < nplanes) {
        // the buffer of plane i + 2 held plane i - 1: wait until the stream warps are done with it
        if (i >= 1) bar_sync(5 + (i - 1) % XNB, NT);
        fetch(i + 2);
      }
    }
  } else {
    // ---------------------------------------------------------- stream warps
    const int st = tid - NF;
    const size_t plane = (size_t)nx * ny;
    double* __restrict__ U = a.u;
    double* __restrict__ V = a.v;
    double* __restrict__ W = a.w;
    const double cc = g.dt / g.rho, dxi = g.dxi;
    // pressure of the thread's x pairs at the plane below: [pair][stream thread] in shared memory
    // after the tiles (each thread its own 16-byte slots: conflict-free), or in registers
    double2* pzs = reinterpret_cast<double2*>(smraw + xc_tile_bytes<T, M, INC>()) + st;
    double2 pzr[PZS ? 1 : PPT] = {};
    auto pz_get = [&](int m) -> double2 {
      if constexpr (PZS) return pzs[m * NS];
      else return pzr[m];
    };
    auto pz_set = [&](int m, double2 v) {
      if constexpr (PZS) pzs[m * NS] = v;
      else pzr[m] = v;
    };
    // staged u, v, w of pair m, field f: uvs[(f * PPT + m) * NS] (each thread its own slots)
    double2* uvs = reinterpret_cast<double2*>(smraw + xc_smem<T, M, INC>()) + st;
    // pair m of plane index ip into its slots, as one commit group (empty for pairs without a cell,
    // and past the last plane, so every thread commits PPT groups per plane)
    auto stage_pair = [&](int ip, int m) {
      if constexpr (UVS) {
        const int e = st + m * NS;
        if (ip < nplanes && (NP % NS == 0 || e < NP)) {
          const int l = e / M, n = e - l * M;
          const int j = j0 + l;
          if (j < ny) {
            const size_t o = (size_t)(k0 - 1 + ip) * plane + (size_t)j * nx + 2 * n;  // ip >= 1: no wrap
            __pipeline_memcpy_async(&uvs[(0 * PPT + m) * NS], U + o, 16);
            __pipeline_memcpy_async(&uvs[(1 * PPT + m) * NS], V + o, 16);
            __pipeline_memcpy_async(&uvs[(2 * PPT + m) * NS], W + o, 16);
          }
        }
        __pipeline_commit();
      }
    };
    for (int i = 0; i < nplanes; ++i) {
      const Cx<T>* s = tiles + (i % XNB) * TL;
      const float* qs = qtiles + (i % XNB) * QL;
      const int k = k0 - 1 + i;
      const int kk = k < 0 ? k + nz : k;
      bar_sync(2 + i % XNB, NT);  // plane i's pressure (and predictor rows) are ready
      if constexpr (UVS) {
#pragma unroll
        for (int m = 0; m < PPT; ++m) {
          const int e = st + m * NS;
          if (NP % NS == 0 || e < NP) {
            const int l = e / M, n = e - l * M;  // output line l = tile line l + 1
            const int j = j0 + l;
            const Cx<T> z = s[sw<XL>(n, l + 1)];
            const T zxm = s[sw<XL>(n == 0 ? M - 1 : n - 1, l + 1)].y;
            const Cx<T> zy = s[sw<XL>(n, l)];
            double p0, p1, pxm, py0, py1;
            if constexpr (INC) {
              const float2 qc = *reinterpret_cast<const float2*>(qs + (l + 1) * nx + 2 * n);
              // the -x neighbour as the odd half of the aligned pair below (8-byte loads at an
              // 8-byte stride: no bank conflict)
              const float qx = reinterpret_cast<const float2*>(qs + (l + 1) * nx)[n == 0 ? M - 1 : n - 1].y;
              const float2 qy = *reinterpret_cast<const float2*>(qs + l * nx + 2 * n);
              p0 = (double)qc.x + (double)z.x;
              p1 = (double)qc.y + (double)z.y;
              pxm = (double)qx + (double)zxm;
              py0 = (double)qy.x + (double)zy.x;
              py1 = (double)qy.y + (double)zy.y;
            } else {
              p0 = (double)z.x;
              p1 = (double)z.y;
              pxm = (double)zxm;
              py0 = (double)zy.x;
              py1 = (double)zy.y;
            }
            if (i > 0 && j < ny) {
              // this pair's staged plane: every group but the newest PPT - 1 (the plane's later
              // pairs, the next plane's earlier ones) is complete
              __pipeline_wait_prior(PPT - 1);
              const double2 uo = uvs[(0 * PPT + m) * NS], vo = uvs[(1 * PPT + m) * NS], wo = uvs[(2 * PPT + m) * NS];
              const size_t o = (size_t)kk * plane + (size_t)j * nx + 2 * n;
              // multi/main.f90:953-955, the expressions of k_correct
              const double u0 = uo.x - cc * (p0 - pxm) * dxi, u1 = uo.y - cc * (p1 - p0) * dxi;
              const double v0 = vo.x - cc * (p0 - py0) * dxi, v1 = vo.y - cc * (p1 - py1) * dxi;
              const double2 pk = pz_get(m);
              const double w0 = wo.x - cc * (p0 - pk.x) * dxi, w1 = wo.y - cc * (p1 - pk.y) * dxi;
              *reinterpret_cast<double2*>(U + o) = make_double2(u0, u1);
              *reinterpret_cast<double2*>(V + o) = make_double2(v0, v1);
              *reinterpret_cast<double2*>(W + o) = make_double2(w0, w1);
              if constexpr (INC) *reinterpret_cast<float2*>(a.qnew + o) = make_float2((float)p0, (float)p1);
              su += u0 + u1;
              sv += v0 + v1;
              sw_ += w0 + w1;
              mu = fmax(mu, fmax(u0, u1));
              mv = fmax(mv, fmax(v0, v1));
              mw = fmax(mw, fmax(w0, w1));
            }
            pz_set(m, make_double2(p0, p1));
          }
          // the slots are free (their values consumed above): the next plane's pair goes in
          stage_pair(i + 1, m);
        }
      } else {
#pragma unroll
        for (int m0 = 0; m0 < PPT; m0 += XPB) {
          // the batch's loads first (u, v, w of up to XPB pairs in flight per thread), then the math
          double2 uo[XPB], vo[XPB], wo[XPB];
#pragma unroll
          for (int mb = 0; mb < XPB && m0 + mb < PPT; ++mb) {
            const int e = st + (m0 + mb) * NS;
            if (NP % NS == 0 || e < NP) {
              const int l = e / M, n = e - l * M;
              const int j = j0 + l;
              if (i > 0 && j < ny) {
                const size_t o = (size_t)kk * plane + (size_t)j * nx + 2 * n;
                uo[mb] = *reinterpret_cast<const double2*>(U + o);
                vo[mb] = *reinterpret_cast<const double2*>(V + o);
                wo[mb] = *reinterpret_cast<const double2*>(W + o);
              }
            }
          }
#pragma unroll
          for (int mb = 0; mb < XPB && m0 + mb < PPT; ++mb) {
            const int m = m0 + mb;
            const int e = st + m * NS;
            if (NP % NS == 0 || e < NP) {
              const int l = e / M, n = e - l * M;  // output line l = tile line l + 1
              const int j = j0 + l;
              const Cx<T> z = s[sw<XL>(n, l + 1)];
              const T zxm = s[sw<XL>(n == 0 ? M - 1 : n - 1, l + 1)].y;
              const Cx<T> zy = s[sw<XL>(n, l)];
              double p0, p1, pxm, py0, py1;
              if constexpr (INC) {
                // the sums k_fftx_inv forms for the FP64 pressure (same doubles), the predictor at the
                // cell pair and its -x and -y neighbours from the tile's predictor rows
                const float2 qc = *reinterpret_cast<const float2*>(qs + (l + 1) * nx + 2 * n);
                // the -x neighbour as the odd half of the aligned pair below (8-byte loads at an
                // 8-byte stride: no bank conflict)
                const float qx = reinterpret_cast<const float2*>(qs + (l + 1) * nx)[n == 0 ? M - 1 : n - 1].y;
                const float2 qy = *reinterpret_cast<const float2*>(qs + l * nx + 2 * n);
                p0 = (double)qc.x + (double)z.x;
                p1 = (double)qc.y + (double)z.y;
                pxm = (double)qx + (double)zxm;
                py0 = (double)qy.x + (double)zy.x;
                py1 = (double)qy.y + (double)zy.y;
              } else {
                p0 = (double)z.x;
                p1 = (double)z.y;
                pxm = (double)zxm;
                py0 = (double)zy.x;
                py1 = (double)zy.y;
              }
              if (i > 0 && j < ny) {
                const size_t o = (size_t)kk * plane + (size_t)j * nx + 2 * n;
                // multi/main.f90:953-955, the expressions of k_correct
                const double u0 = uo[mb].x - cc * (p0 - pxm) * dxi, u1 = uo[mb].y - cc * (p1 - p0) * dxi;
                const double v0 = vo[mb].x - cc * (p0 - py0) * dxi, v1 = vo[mb].y - cc * (p1 - py1) * dxi;
                const double2 pk = pz_get(m);
                const double w0 = wo[mb].x - cc * (p0 - pk.x) * dxi, w1 = wo[mb].y - cc * (p1 - pk.y) * dxi;
                *reinterpret_cast<double2*>(U + o) = make_double2(u0, u1);
                *reinterpret_cast<double2*>(V + o) = make_double2(v0, v1);
                *reinterpret_cast<double2*>(W + o) = make_double2(w0, w1);
                if constexpr (INC) *reinterpret_cast<float2*>(a.qnew + o) = make_float2((float)p0, (float)p1);
                su += u0 + u1;
                sv += v0 + v1;
                sw_ += w0 + w1;
                mu = fmax(mu, fmax(u0, u1));
                mv = fmax(mv, fmax(v0, v1));
                mw = fmax(mw, fmax(w0, w1));
              }
              pz_set(m, make_double2(p0, p1));
            }
          }
        }
      }
      // the transform warps wait for this buffer only if they fetch plane i + 3 into it
      if (i + 3 < nplanes) bar_arrive(5 + i % XNB, NT);
    }
    if constexpr (UVS) __pipeline_wait_prior(0);  // no copy into the block's shared memory outlives it
  }
  // block reduction (fixed tree, as k_correct; the transform warps add the identities)
  __syncthreads();
  __shared__ double red[6][NT / 32];
  double vals[6] = {su, sv, sw_, mu, mv, mw};
  const int lane = tid & 31;
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    double x = vals[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double y = __shfl_down_sync(0xffffffffu, x, o);
      x = q < 3 ? x + y : fmax(x, y);
    }
    if (lane == 0) red[q][tid >> 5] = x;
  }
  __syncthreads();
  if (tid < 6) {
    double x = red[tid][0];
    for (int wv = 1; wv < NT / 32; ++wv) x = tid < 3 ? x + red[tid][wv] : fmax(x, red[tid][wv]);
    const size_t bid = (size_t)blockIdx.y * gridDim.x + blockIdx.x;
    a.partials[bid * 6 + tid] = x;
  }
}

// z planes per block: by default as many as make the grid one wave of one block per SM (148 on
// a B200; at 512^3 the 74 columns of 7 lines times 2 halves of z), so each block fills its
// transform-to-stream pipeline once for a long run of planes
static int xc_chunk(const Geo& g, int zc) {
  if (zc <= 0) {
    const int ncols = (g.ny + XO - 1) / XO;
    const int per = std::max(1, 148 / ncols);
    zc = std::max(XZC_MIN, (g.nz + per - 1) / per);
  }
  return zc < g.nz ? zc : g.nz;
}

static dim3 xc_grid(const Geo& g, int zc) {
  const int c = xc_chunk(g, zc);
  return dim3((g.ny + XO - 1) / XO, (g.nz + c - 1) / c);
}

int xc_blocks(const Geo& g, int zc) {
  const dim3 d = xc_grid(g, zc);
  return (int)(d.x * d.y);
}

template <typename T, int M>
static cudaError_t launch_xc_m(const XcArgs& a, cudaStream_t st) {
  constexpr int NT = xc_nf<M>() + xc_ns<M>();
  // the incremental solve is an FP32 mode: its variant exists for float tiles only
  constexpr bool HAS_INC = sizeof(T) == 4;
  static_assert(xc_smem_all<T, M, false>() <= 227 * 1024 && (!HAS_INC || xc_smem_all<T, M, HAS_INC>() <= 227 * 1024),
                "tiles exceed the shared memory of a block");
  const size_t smem = a.qold ? xc_smem_all<T, M, HAS_INC>() : xc_smem_all<T, M, false>();
  auto kern = a.qold ? k_xinv_correct<T, M, HAS_INC> : k_xinv_correct<T, M, false>;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  XcArgs b = a;
  b.zc = xc_chunk(a.g, a.zc);
  const dim3 grid = xc_grid(a.g, a.zc);
  kern<<<grid, NT, smem, st>>>(b);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return launch_finalize(a.partials, (int)(grid.x * grid.y), a.g, a.sc, st);
}

template <typename T>
static cudaError_t launch_xc_t(const XcArgs& a, cudaStream_t st) {
  switch (a.g.nx / 2) {
#define C(m) case m: return launch_xc_m<T, m>(a, st);
    C(8) C(16) C(32) C(64) C(96) C(128) C(256) C(512)
#undef C
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_xinv_correct(const XcArgs& a, cudaStream_t st) {
  if (a.qold && !a.fp32) return cudaErrorInvalidValue;  // the incremental solve is an FP32 mode
  return a.fp32 ? launch_xc_t<float>(a, st) : launch_xc_t<double>(a, st);
}

}  // namespace mhit
