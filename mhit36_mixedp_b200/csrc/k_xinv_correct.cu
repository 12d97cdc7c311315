// The inverse x transform fused with the projection: multi/main.f90:909-912 and :942-1003 in one
// pass over HBM.
//
// Apart, k_fftx_inv writes the pressure and k_correct reads it back beside u*, v*, w* (the
// pressure's -x, -y and -z neighbours of each cell).  Here a block owns XO = 7 consecutive y
// lines of a chunk of z planes and marches up z.  Per plane it
//   1. has the plane's 8 half-spectrum rows in shared memory (its 7 lines and the line below
//      them, j0 - 1, the -y neighbour of its first line), fetched by cp.async one plane ahead
//      into the other of two tile buffers;
//   2. C2R-transforms the 8 rows in place (the untangle and Stockham stages of k_fftx_inv, so
//      the pressure values are the same doubles);
//   3. projects its 7 lines (u -= dt/rho (p - p(i-1)) dxi, and v, w along y, z: :953-955) with
//      p(i-1) and p(j-1) from the tile and p(k-1) from the thread's registers, which hold the
//      pressure of its own x pairs at the plane below (the loop starts one plane below the
//      chunk for them), and accumulates the per-block sums and maxima of k_correct.
// The pressure never goes to HBM: the library materialises it from the spectrum, which stays
// intact until the next step's x pass, when something reads it.  Per cell this moves the spectrum
// once (8/7 of it: the halo line) and u, v, w in and out: 48 + 8 (FP64) or 48 + 4 (FP32) bytes
// of the 72 / 60 of the two passes.
//
// INC (incremental FP32 solve): the transform is the correction delta; the pressure is
// qold + delta formed in FP64 (qold, the FP32 predictor, read at the cell and its -x and -y
// neighbours), and fl32 of it goes to qnew, the next step's predictor (a second buffer, so no
// block overwrites a predictor another block still reads).
#include <cuda_pipeline.h>

#include "common.cuh"
#include "fft_core.cuh"
#include "kernels.h"

namespace mhit {

constexpr int XL = 8;       // lines transformed per plane (a power of two: the tile swizzle)
constexpr int XO = XL - 1;  // lines projected per plane: tile line 0 is the -y halo
constexpr int XZC = 16;     // default z planes per block

template <int M> __host__ __device__ constexpr int xc_max_radix() {
  int m = 0;
  for (int s = 0; s < XcRadix<M>::ns; ++s) m = XcRadix<M>::r[s] > m ? XcRadix<M>::r[s] : m;
  return m;
}

// threads: one per x pair of a line (coalesced 16-byte rows), at least one butterfly each
template <int M> __host__ __device__ constexpr int xc_threads() {
  return M / xc_max_radix<M>() * XL > M ? M / xc_max_radix<M>() * XL : (M < 64 ? 64 : M);
}

// resident blocks per SM the register budget is sized for (the tile buffers allow 3 of 256
// threads in FP64 at nx = 512)
#ifndef XC_MINB
#define XC_MINB 2
#endif
template <typename T, int M> __host__ __device__ constexpr int xc_minb() {
  return xc_threads<M>() >= 512 ? 1 : (xc_threads<M>() >= 256 ? XC_MINB : 4);
}

template <typename T, int M, bool INC>
__global__ void __launch_bounds__(xc_threads<M>(), (xc_minb<T, M>())) k_xinv_correct(const XcArgs a) {
  constexpr int NT = xc_threads<M>();
  constexpr int TL = (M + 1) * XL;         // elements of one tile buffer
  constexpr int NP = XO * M;               // x pairs projected per plane
  constexpr int PPT = (NP + NT - 1) / NT;  // ... per thread
  constexpr int nx = 2 * M;
  extern __shared__ __align__(16) unsigned char smraw[];
  Cx<T>* tiles = reinterpret_cast<Cx<T>*>(smraw);
  const Geo& g = a.g;
  const int ny = g.ny, nz = g.nz;
  const size_t plane = (size_t)nx * ny;
  const int pitch = g.pitch;
  const int j0 = blockIdx.x * XO;
  const int zc = a.zc;
  const int k0 = blockIdx.y * zc, k1 = min(k0 + zc, nz);
  const Cx<T>* __restrict__ spec = static_cast<const Cx<T>*>(a.spec);
  const Cx<T>* __restrict__ twx = static_cast<const Cx<T>*>(a.twx);
  double* __restrict__ U = a.u;
  double* __restrict__ V = a.v;
  double* __restrict__ W = a.w;
  const double cc = g.dt / g.rho, dxi = g.dxi;

  // rows j0-1 .. j0+6 of plane k (periodic in y and z; rows past ny in a tail tile wrap and
  // are transformed but not projected)
  auto fetch = [&](int k, Cx<T>* s) {
    const int kk = k < 0 ? k + nz : k;
    const Cx<T>* src = spec + (size_t)kk * ny * pitch;
    for (int e = threadIdx.x; e < TL; e += NT) {
      const int b = e / (M + 1), kx = e - b * (M + 1);
      int j = j0 - 1 + b;
      j = j < 0 ? j + ny : (j >= ny ? j - ny : j);
      __pipeline_memcpy_async(&s[sw<XL>(kx, b)], &src[(size_t)j * pitch + kx], sizeof(Cx<T>));
    }
    __pipeline_commit();
  };

  double pz[PPT][2];  // pressure of the thread's x pairs at the plane below
  double su = 0.0, sv = 0.0, sw_ = 0.0;
  double mu = -INFINITY, mv = -INFINITY, mw = -INFINITY;
  fetch(k0 - 1, tiles);
  int it = 0;
  for (int k = k0 - 1; k < k1; ++k, ++it) {
    Cx<T>* s = tiles + (it & 1) * TL;
    __pipeline_wait_prior(0);
    __syncthreads();  // plane k's tile is complete; no thread still reads the other buffer
    if (k + 1 < k1) fetch(k + 1, tiles + ((it + 1) & 1) * TL);
    c2r_untangle<T, M, XL, NT>(s, twx);
    __syncthreads();
    fft_tile<T, M, XL, NT, true, XcRadix<M>>(s, twx, 2);  // returns after a barrier
    const int kk = k < 0 ? k + nz : k;
    const bool out = k >= k0;
#pragma unroll
    for (int m = 0; m < PPT; ++m) {
      const int e = threadIdx.x + m * NT;
      if (NP % NT == 0 || e < NP) {
        const int l = e / M, n = e - l * M;  // output line l = tile line l + 1
        const int j = j0 + l;
        const Cx<T> z = s[sw<XL>(n, l + 1)];
        const T zxm = s[sw<XL>(n == 0 ? M - 1 : n - 1, l + 1)].y;
        const Cx<T> zy = s[sw<XL>(n, l)];
        double p0, p1, pxm, py0, py1;
        if constexpr (INC) {
          const int jj = j < ny ? j : j - ny;
          const int jm = jj == 0 ? ny - 1 : jj - 1;
          const float* q = a.qold + (size_t)kk * plane;
          const float2 qc = __ldg(reinterpret_cast<const float2*>(q + (size_t)jj * nx + 2 * n));
          const float qx = __ldg(q + (size_t)jj * nx + (n == 0 ? nx - 1 : 2 * n - 1));
          const float2 qy = __ldg(reinterpret_cast<const float2*>(q + (size_t)jm * nx + 2 * n));
          // the sums k_fftx_inv forms for the FP64 pressure (same doubles)
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
        if (out && j < ny) {
          const size_t o = (size_t)kk * plane + (size_t)j * nx + 2 * n;
          const double2 uo = *reinterpret_cast<const double2*>(U + o);
          const double2 vo = *reinterpret_cast<const double2*>(V + o);
          const double2 wo = *reinterpret_cast<const double2*>(W + o);
          // multi/main.f90:953-955, the expressions of k_correct
          const double u0 = uo.x - cc * (p0 - pxm) * dxi, u1 = uo.y - cc * (p1 - p0) * dxi;
          const double v0 = vo.x - cc * (p0 - py0) * dxi, v1 = vo.y - cc * (p1 - py1) * dxi;
          const double w0 = wo.x - cc * (p0 - pz[m][0]) * dxi, w1 = wo.y - cc * (p1 - pz[m][1]) * dxi;
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
        pz[m][0] = p0;
        pz[m][1] = p1;
      }
    }
  }
  // block reduction (fixed tree, as k_correct)
  __shared__ double red[6][NT / 32];
  double vals[6] = {su, sv, sw_, mu, mv, mw};
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
    for (int wv = 1; wv < NT / 32; ++wv) x = t < 3 ? x + red[t][wv] : fmax(x, red[t][wv]);
    const size_t bid = (size_t)blockIdx.y * gridDim.x + blockIdx.x;
    a.partials[bid * 6 + t] = x;
  }
}

static int xc_chunk(const Geo& g, int zc) {
  const int c = zc > 0 ? zc : XZC;
  return c < g.nz ? c : g.nz;
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
  constexpr int NT = xc_threads<M>();
  const size_t smem = 2 * (size_t)(M + 1) * XL * sizeof(Cx<T>);
  auto kern = a.qold ? k_xinv_correct<T, M, true> : k_xinv_correct<T, M, false>;
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
