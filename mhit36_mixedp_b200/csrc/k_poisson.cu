// Pressure Poisson solve on one GPU: multi/main.f90:833-923 without cuFFT or cuDecomp.
//
//   k_div_fftx   rho/dt * div(u*) in FP64 (:833-843), cast to the Poisson precision (:844),
//                and the x-direction R2C transform (:853) of a tile of B x-lines, fused.
//   k_fft_cols   C2C transform along y (:860, :906) or along z fused with the spectral divide
//                -rhs/k^2/(nx ny nz), zero mode := 0, and the inverse z transform
//                (:865, :883-896, :901).  The transposes of :858,863,904,909 disappear: a
//                tile is B adjacent kx columns of the x-fastest spectrum, read with stride.
//   k_fftx_inv   C2R along x (:912) into the pressure array (FP32 or FP64).
//
// Spectrum layout: [z][y][kx], kx fastest, row pitch padded to a multiple of 16 complex so
// every tile row starts on a 128-byte boundary.  Half-length real transforms: the x line of
// nx reals is packed as nx/2 complex (even + i*odd), transformed, and untangled with the
// exp(-2 pi i k/nx) twiddles (and the mirror image for C2R).
#include <cuda_pipeline.h>

#include <type_traits>

#include "common.cuh"
#include "fft_core.cuh"
#include "kernels.h"

namespace mhit {

template <typename T> struct Tile;
template <> struct Tile<double> { static constexpr int B = 8; };
template <> struct Tile<float> { static constexpr int B = 16; };

template <typename T> __device__ __forceinline__ void store2(T* p, T a, T b);
template <> __device__ __forceinline__ void store2<double>(double* p, double a, double b) {
  *reinterpret_cast<double2*>(p) = make_double2(a, b);
}
template <> __device__ __forceinline__ void store2<float>(float* p, float a, float b) {
  *reinterpret_cast<float2*>(p) = make_float2(a, b);
}

// x-pass threads: one butterfly of the largest radix per thread (as the column passes)
template <typename T, int M> __host__ __device__ constexpr int xpass_threads() { return fft_threads<M, Tile<T>::B>(); }
// Resident blocks the forward x pass is compiled for (0: no bound).  The FP32 256-point pass
// (nx = 512) asks for four blocks of 256 threads, the residency its 33 KB tiles allow anyway,
// which lets it use 64 registers instead of the 48 / 56 the compiler picks without the bound, at
// the same 32 warps per SM: the residual source (the
// incremental solve's right-hand side) 0.90 against 0.96 ms at 512^3, the same bits; the
// divergence source unchanged (0.71 ms).  Other lengths and FP64 keep the compiler's choice.
template <typename T, int M> __host__ __device__ constexpr int xpass_minblocks() {
  return (sizeof(T) == 4 && M == 256) ? 4 : 0;
}

// ------------------------------------------------------------------ forward x + divergence
// SRC 0: the divergence of u*; SRC 2: the real FP64 field `u` (the energy spectrum of a
// velocity component); SRC 3: the FP64 residual rho/dt div(u*) - L_h q of the FP32 pressure q in
// `rr` (L_h the 7-point Laplacian, the operator whose symbol the modified divide uses), rounded
// to FP32 -- the right-hand side of the refinement sweep and of the incremental solve.
template <typename T, int M, int SRC>
__global__ void __launch_bounds__(xpass_threads<T, M>(), xpass_minblocks<T, M>())
k_div_fftx(const double* __restrict__ u, const double* __restrict__ v, const double* __restrict__ w,
           const float* __restrict__ rr, Cx<T>* __restrict__ spec, const Cx<T>* __restrict__ twx, Geo g,
           double cdiv) {
  constexpr int B = Tile<T>::B;
  constexpr int NT = xpass_threads<T, M>();
  extern __shared__ __align__(16) unsigned char smraw[];
  Cx<T>* s = reinterpret_cast<Cx<T>*>(smraw);
  const int nx = 2 * M, ny = g.ny, nz = g.nz;
  const int nlines = ny * nz;
  const int line0 = blockIdx.x * B;

  // Element e of the tile: line e / M, complex point e % M.  The FP64 256-point tile (nx = 512)
  // loads in a loop of compile-time length unrolled twice (88 registers, twelve loads in flight
  // per thread): 0.85 ms at 512^3 against 1.00 ms for the strided loop; so does the FP32 tile
  // of the residual source (its 13 loads per pair); the FP32 divergence tile keeps the strided
  // loop (0.707 against 0.715 ms), and so do the other lengths (not measured).
  auto load = [&](int e) {
    const int b = e / M, n = e - b * M;
    const int line = min(line0 + b, nlines - 1);  // a tail tile repeats the last line
    Cx<T> z;
    if constexpr (SRC == 2) {
      const double2 r2 = __ldg(reinterpret_cast<const double2*>(u + (size_t)line * nx + 2 * n));
      z.x = (T)r2.x;
      z.y = (T)r2.y;
    } else {
      const int k = line / ny, j = line - k * ny;
      const int jp = wrapp(j, ny), kp = wrapp(k, nz);
      const int i = 2 * n;
      const size_t row = ((size_t)k * ny + j) * nx;
      const size_t rowy = ((size_t)k * ny + jp) * nx;
      const size_t rowz = ((size_t)kp * ny + j) * nx;
      // every operand is an independent load (taking the x neighbours from adjacent lanes by
      // shuffles serialised them: k_div_fftx 0.79 against 0.70 ms at 512^3 in FP32)
      const double2 uu = __ldg(reinterpret_cast<const double2*>(u + row + i));
      const double un = __ldg(u + row + (i + 2 == nx ? 0 : i + 2));
      const double2 vv = __ldg(reinterpret_cast<const double2*>(v + row + i));
      const double2 vp = __ldg(reinterpret_cast<const double2*>(v + rowy + i));
      const double2 ww = __ldg(reinterpret_cast<const double2*>(w + row + i));
      const double2 wp = __ldg(reinterpret_cast<const double2*>(w + rowz + i));
      // multi/main.f90:841-843, summed in the reference's order
      double r0 = cdiv * (uu.y - uu.x);
      r0 = r0 + cdiv * (vp.x - vv.x);
      r0 = r0 + cdiv * (wp.x - ww.x);
      double r1 = cdiv * (un - uu.y);
      r1 = r1 + cdiv * (vp.y - vv.y);
      r1 = r1 + cdiv * (wp.y - ww.y);
      if constexpr (SRC == 3) {
        // L_h q at cells i and i+1, summed per axis as (q+ - 2 q + q-) ddxi
        const int jm = wrapm(j, ny), km = wrapm(k, nz);
        const double ddxi = g.ddxi;
        const float2 qc = __ldg(reinterpret_cast<const float2*>(rr + row + i));
        const float qxm = __ldg(rr + row + (i == 0 ? nx - 1 : i - 1));
        const float qxp = __ldg(rr + row + (i + 2 == nx ? 0 : i + 2));
        const float2 qyp = __ldg(reinterpret_cast<const float2*>(rr + rowy + i));
        const float2 qym = __ldg(reinterpret_cast<const float2*>(rr + ((size_t)k * ny + jm) * nx + i));
        const float2 qzp = __ldg(reinterpret_cast<const float2*>(rr + rowz + i));
        const float2 qzm = __ldg(reinterpret_cast<const float2*>(rr + ((size_t)km * ny + j) * nx + i));
        const double q0 = (double)qc.x, q1 = (double)qc.y;
        const double l0 = ((double)qc.y - 2.0 * q0 + (double)qxm) * ddxi +
                          ((double)qyp.x - 2.0 * q0 + (double)qym.x) * ddxi +
                          ((double)qzp.x - 2.0 * q0 + (double)qzm.x) * ddxi;
        const double l1 = ((double)qxp - 2.0 * q1 + (double)qc.x) * ddxi +
                          ((double)qyp.y - 2.0 * q1 + (double)qym.y) * ddxi +
                          ((double)qzp.y - 2.0 * q1 + (double)qzm.y) * ddxi;
        r0 = r0 - l0;
        r1 = r1 - l1;
      }
      z.x = (T)r0;
      z.y = (T)r1;
    }
    s[sw<B>(n, b)] = z;
  };
  // The divergence sources marching down the tile's B lines (consecutive y at one z when
  // ny % B == 0): each thread keeps its x pairs' v(j+1), and for the residual q(j+1) and q(j), in
  // registers for the next line instead of loading them again (10 loads per pair and line instead
  // of 13 for the residual, 5 instead of 6 for the divergence: less L1/L2 traffic).  The same
  // expressions in the same order as `load`.
  constexpr int PP = M / NT > 0 ? M / NT : 1;  // x pairs per thread and line (march: M % NT == 0)
  auto march = [&]() {
    const int k = line0 / ny, jb = line0 - k * ny;
    const int kp = wrapp(k, nz), km = wrapm(k, nz);
    const size_t pk = (size_t)k * ny * nx, pkp = (size_t)kp * ny * nx, pkm = (size_t)km * ny * nx;
    double2 vcur[PP];
    float2 qcur[PP], qprev[PP];
#pragma unroll
    for (int p = 0; p < PP; ++p) {
      const int i = 2 * (threadIdx.x + p * NT);
      vcur[p] = __ldg(reinterpret_cast<const double2*>(v + pk + (size_t)jb * nx + i));
      if constexpr (SRC == 3) {
        qcur[p] = __ldg(reinterpret_cast<const float2*>(rr + pk + (size_t)jb * nx + i));
        qprev[p] = __ldg(reinterpret_cast<const float2*>(rr + pk + (size_t)wrapm(jb, ny) * nx + i));
      }
    }
#pragma unroll 2
    for (int b = 0; b < B; ++b) {
      const int j = jb + b, jp = wrapp(j, ny);
      const size_t row = pk + (size_t)j * nx, rowy = pk + (size_t)jp * nx;
      const size_t rowz = pkp + (size_t)j * nx, rowzm = pkm + (size_t)j * nx;
#pragma unroll
      for (int p = 0; p < PP; ++p) {
        const int n = threadIdx.x + p * NT, i = 2 * n;
        const double2 uu = __ldg(reinterpret_cast<const double2*>(u + row + i));
        const double un = __ldg(u + row + (i + 2 == nx ? 0 : i + 2));
        const double2 vv = vcur[p];
        const double2 vp = __ldg(reinterpret_cast<const double2*>(v + rowy + i));
        const double2 ww = __ldg(reinterpret_cast<const double2*>(w + row + i));
        const double2 wp = __ldg(reinterpret_cast<const double2*>(w + rowz + i));
        // multi/main.f90:841-843, summed in the reference's order
        double r0 = cdiv * (uu.y - uu.x);
        r0 = r0 + cdiv * (vp.x - vv.x);
        r0 = r0 + cdiv * (wp.x - ww.x);
        double r1 = cdiv * (un - uu.y);
        r1 = r1 + cdiv * (vp.y - vv.y);
        r1 = r1 + cdiv * (wp.y - ww.y);
        if constexpr (SRC == 3) {
          const double ddxi = g.ddxi;
          const float2 qc = qcur[p], qym = qprev[p];
          const float qxm = __ldg(rr + row + (i == 0 ? nx - 1 : i - 1));
          const float qxp = __ldg(rr + row + (i + 2 == nx ? 0 : i + 2));
          const float2 qyp = __ldg(reinterpret_cast<const float2*>(rr + rowy + i));
          const float2 qzp = __ldg(reinterpret_cast<const float2*>(rr + rowz + i));
          const float2 qzm = __ldg(reinterpret_cast<const float2*>(rr + rowzm + i));
          const double q0 = (double)qc.x, q1 = (double)qc.y;
          const double l0 = ((double)qc.y - 2.0 * q0 + (double)qxm) * ddxi +
                            ((double)qyp.x - 2.0 * q0 + (double)qym.x) * ddxi +
                            ((double)qzp.x - 2.0 * q0 + (double)qzm.x) * ddxi;
          const double l1 = ((double)qxp - 2.0 * q1 + (double)qc.x) * ddxi +
                            ((double)qyp.y - 2.0 * q1 + (double)qym.y) * ddxi +
                            ((double)qzp.y - 2.0 * q1 + (double)qzm.y) * ddxi;
          r0 = r0 - l0;
          r1 = r1 - l1;
          qprev[p] = qc;
          qcur[p] = qyp;
        }
        vcur[p] = vp;
        Cx<T> z;
        z.x = (T)r0;
        z.y = (T)r1;
        s[sw<B>(n, b)] = z;
      }
    }
  };
  if constexpr ((SRC == 0 || SRC == 3) && M % NT == 0) {
    if (ny % B == 0) march();
    else
      for (int e = threadIdx.x; e < M * B; e += NT) load(e);
  } else if constexpr ((sizeof(T) == 8 || SRC == 3) && M == 256 && (M * B) % NT == 0) {
#pragma unroll 2
    for (int it = 0; it < M * B / NT; ++it) load(threadIdx.x + it * NT);
  } else {
    for (int e = threadIdx.x; e < M * B; e += NT) load(e);
  }
  __syncthreads();
  fft_tile<T, M, B, NT, false>(s, twx, 2);

  // untangle: X[k] = (Z[k] + Z*[M-k])/2 - i/2 W^k (Z[k] - Z*[M-k]),  W = exp(-2 pi i/nx)
  for (int e = threadIdx.x; e < (M / 2 + 1) * B; e += NT) {
    const int kk = e / B, b = e - kk * B;
    if (kk == 0) {
      const Cx<T> z0 = s[sw<B>(0, b)];
      s[sw<B>(0, b)] = cx<T>(z0.x + z0.y, (T)0);
      s[sw<B>(M, b)] = cx<T>(z0.x - z0.y, (T)0);
    } else {
      const Cx<T> zk = s[sw<B>(kk, b)];
      const Cx<T> zm = s[sw<B>(M - kk, b)];
      const T h = (T)0.5;
      {
        const Cx<T> a = scale(zk + conj(zm), h);
        const Cx<T> d = zk - conj(zm);
        const Cx<T> t = cmul(twx[kk], d);  // W^k d
        s[sw<B>(kk, b)] = cx<T>(a.x + h * t.y, a.y - h * t.x);  // a - i/2 t
      }
      if (kk != M - kk) {
        const Cx<T> a = scale(zm + conj(zk), h);
        const Cx<T> d = zm - conj(zk);
        const Cx<T> t = cmul(twx[M - kk], d);
        s[sw<B>(M - kk, b)] = cx<T>(a.x + h * t.y, a.y - h * t.x);
      }
    }
  }
  __syncthreads();
  const int pitch = g.pitch;
  for (int e = threadIdx.x; e < (M + 1) * B; e += NT) {
    const int b = e / (M + 1), kx = e - b * (M + 1);
    const int line = line0 + b;
    if (line < nlines) spec[(size_t)line * pitch + kx] = s[sw<B>(kx, b)];
  }
}

// ------------------------------------------------------------------ inverse x -> pressure
// INC (incremental FP32 solve): the transform is the correction delta; with q the FP32 predictor
// in `qin`, the pressure s = q + delta is formed in FP64 and written to `p64` (what the
// projection reads), and fl32(s) to `qout` (the next step's predictor; skipped when null).
template <typename T, int M, bool INC>
__global__ void __launch_bounds__(xpass_threads<T, M>())
k_fftx_inv(const Cx<T>* __restrict__ spec, T* __restrict__ p, const Cx<T>* __restrict__ twx, Geo g,
           const float* __restrict__ qin, float* __restrict__ qout, double* __restrict__ p64) {
  constexpr int B = Tile<T>::B;
  constexpr int NT = xpass_threads<T, M>();
  extern __shared__ __align__(16) unsigned char smraw[];
  Cx<T>* s = reinterpret_cast<Cx<T>*>(smraw);
  const int nx = 2 * M;
  const int nlines = g.ny * g.nz;
  const int line0 = blockIdx.x * B;
  const int pitch = g.pitch;
  for (int e = threadIdx.x; e < (M + 1) * B; e += NT) {
    const int b = e / (M + 1), kx = e - b * (M + 1);
    const int line = min(line0 + b, nlines - 1);  // a tail tile repeats the last line
    __pipeline_memcpy_async(&s[sw<B>(kx, b)], &spec[(size_t)line * pitch + kx], sizeof(Cx<T>));
  }
  __pipeline_commit();
  __pipeline_wait_prior(0);
  __syncthreads();
  c2r_untangle<T, M, B, NT>(s, twx);
  __syncthreads();
  fft_tile<T, M, B, NT, true>(s, twx, 2);
  for (int e = threadIdx.x; e < M * B; e += NT) {
    const int b = e / M, n = e - b * M;
    const int line = line0 + b;
    if (line < nlines) {
      const Cx<T> z = s[sw<B>(n, b)];
      if constexpr (INC) {
        const size_t o = (size_t)line * nx + 2 * n;
        const float2 q2 = *reinterpret_cast<const float2*>(qin + o);
        const double s0 = (double)q2.x + (double)z.x, s1 = (double)q2.y + (double)z.y;
        if (qout) *reinterpret_cast<float2*>(qout + o) = make_float2((float)s0, (float)s1);
        *reinterpret_cast<double2*>(p64 + o) = make_double2(s0, s1);
      } else {
        store2<T>(p + (size_t)line * nx + 2 * n, z.x, z.y);
      }
    }
  }
}

// ------------------------------------------------------------------ y / z column passes
// MODE 0: forward, 1: inverse, 2: forward + spectral divide + inverse (z only)
// The first stage reads its operands straight from global memory and the last stage stores
// its results straight to global memory; in MODE 2 the forward transform's last stage, the
// divide and the inverse transform's first stage (radices in reversed order, so it works on the
// same strided element set) stay in registers: 4 shared-memory passes over the tile per
// transform of three stages instead of 8.
//
// Tiles are 8 columns wide (64-byte rows of float complex: whole DRAM sectors, one butterfly
// per thread and stage for the 512-point transforms), except for the FP64 512-point z solve.
// The z solve keeps two transforms' worth of butterflies in registers (128 per thread in FP64);
// the FP32 one runs two blocks per SM, the single transforms of up to 512 points fit two blocks
// per SM.  Measured at 512^3 FP32: 16-column tiles 0.603 ms for the z solve, 8 columns
// 0.551 ms, 4 columns 0.68 ms.  The FP64 512-point z solve runs 4-column tiles (64-byte rows)
// of 256 threads, two blocks per SM, so one block's loads overlap the other's butterflies:
// 0.865 ms against 0.97 ms for one 8-column block of 512 threads per SM (2 columns: 1.24 ms).
// Radix schedule of the FP32 512-point y passes: 16 x 32 with 128 threads (two radix-16 and one
// radix-32 butterfly per thread, four blocks per SM), one shared-memory round trip per transform
// instead of two for 8 x 8 x 8: y passes 0.222 / 0.231 against 0.269 / 0.271 ms at 512^3 (with
// 256 threads, half of them idle in the 32-point stage: 0.237 / 0.246).  The z solve keeps
// 8 x 8 x 8: 16 x 32 holds two transforms' registers across the divide and spills (0.63 against
// 0.57 ms with 128 threads; 0.81 ms with 256, half of them idle in the 32-point stages).  With
// 128 threads and fewer blocks per SM it spills less and loses warps: three blocks (168
// registers, 24 bytes spilled) 0.61 against 0.59 ms, two (201 registers, none spilled) 0.81 ms.
// The 8 x 8 x 8 solve spills 88 bytes per thread at its 64-register bound and is still faster:
// the pass needs the 32 warps per SM more than it loses to the spills.  The y passes at three
// blocks per SM instead of four: no change.
struct ColRadix512f { static constexpr int ns = 2; static constexpr int r[3] = {16, 32, 0}; };
template <typename T, int N, int MODE> struct ColSched {
  using S = Radix<N>;
  static constexpr int NT = fft_threads<N, 8>();
  static constexpr int MINB = N >= 1024 ? 1 : 2;
};
template <int MODE> struct ColSched<float, 512, MODE> {
  static constexpr bool Y = MODE != 2;
  using S = std::conditional_t<Y, ColRadix512f, Radix<512>>;
  static constexpr int NT = Y ? 128 : fft_threads<512, 8>();
  static constexpr int MINB = Y ? 4 : 2;
};
// The FP32 1024-point y passes (1024^3) in radix 32 x 32: two stages instead of three, one radix-32
// butterfly per thread and stage (256 threads per 8-column tile, two tiles per SM).
struct ColRadix1024f { static constexpr int ns = 2; static constexpr int r[3] = {32, 32, 0}; };
template <int MODE> struct ColSched<float, 1024, MODE> {
  static constexpr bool Y = MODE != 2;
  using S = std::conditional_t<Y, ColRadix1024f, Radix<1024>>;
  static constexpr int NT = Y ? 256 : fft_threads<1024, 8>();
  static constexpr int MINB = Y ? 2 : 1;
};

template <typename T, int N, int MODE> struct ColTile {
  static constexpr bool Z64 = MODE == 2 && N == 512 && sizeof(T) == 8;
  static constexpr int B = Z64 ? 4 : 8;
  static constexpr int NT = Z64 ? fft_threads<N, 4>() : ColSched<T, N, MODE>::NT;
  static constexpr int MINB = Z64 ? 2 : ((MODE == 2 && sizeof(T) == 8) ? 1 : ColSched<T, N, MODE>::MINB);
  using S = typename ColSched<T, N, MODE>::S;
};

template <typename T, int N, int MODE>
__global__ void __launch_bounds__(ColTile<T, N, MODE>::NT, ColTile<T, N, MODE>::MINB)
k_fft_cols(Cx<T>* __restrict__ spec, const Cx<T>* __restrict__ tw, Geo g, size_t stride_n,
           size_t stride_outer, const double* __restrict__ k2x, const double* __restrict__ k2y,
           const double* __restrict__ k2z, double ntot) {
  constexpr int B = ColTile<T, N, MODE>::B;
  constexpr int NT = ColTile<T, N, MODE>::NT;
  using S = typename ColTile<T, N, MODE>::S;
  constexpr int NS = S::ns;
  constexpr int RA = srad<S, false>(0), RL = srad<S, false>(NS - 1);
  constexpr int BA = StageShape<N, B, NT, RA>::BPT, BL = StageShape<N, B, NT, RL>::BPT;
  extern __shared__ __align__(16) unsigned char smraw[];
  Cx<T>* s = reinterpret_cast<Cx<T>*>(smraw);
  const int kx0 = blockIdx.x * B;
  const int outer = blockIdx.y;
  const int nkx = g.nkx;
  Cx<T>* base = spec + (size_t)outer * stride_outer + kx0;
  // The row pitch is a multiple of 16 complex and the padding columns stay zero, so every
  // B-wide tile is in bounds.
  Cx<T> a[BA][RA];
#pragma unroll
  for (int m = 0; m < BA; ++m) {
    if (st_valid<N, B, NT, RA>(m)) {
      const int q = threadIdx.x + m * NT, b = q % B, t = q / B;
#pragma unroll
      for (int r = 0; r < RA; ++r) a[m][r] = base[(size_t)(t + r * (N / RA)) * stride_n + b];
    }
  }
  Cx<T> z[BL][RL];
  fft_regs<T, N, B, NT, MODE == 1, false, S>(s, tw, 1, a, z);
  if constexpr (MODE == 2) {
    // multi/main.f90:889-895: phi3d = -phi3d/k2/(nx*ny*nz) in FP64, phi3d(1,1,1) = 0.
    // One reciprocal of k2*N per element (within 2 ulp of the reference's two divides).
    const double ky2 = k2y[outer];
#pragma unroll
    for (int m = 0; m < BL; ++m) {
      if (st_valid<N, B, NT, RL>(m)) {
        const int q = threadIdx.x + m * NT, b = q % B, t = q / B;
        const int kx = kx0 + b;
#pragma unroll
        for (int r = 0; r < RL; ++r) {
          const int n = t + r * (N / RL);
          double re = 0.0, im = 0.0;
          if (kx < nkx && !(kx == 0 && outer == 0 && n == 0)) {
            const double k2 = (k2x[kx] + ky2) + k2z[n];
            const double inv = 1.0 / (k2 * ntot);
            re = -(double)z[m][r].x * inv;
            im = -(double)z[m][r].y * inv;
          }
          z[m][r] = cx<T>((T)re, (T)im);
        }
      }
    }
    __syncthreads();  // every thread has read the forward transform's last stage
    fft_regs<T, N, B, NT, true, true, S>(s, tw, 1, z, a);
#pragma unroll
    for (int m = 0; m < BA; ++m) {
      if (st_valid<N, B, NT, RA>(m)) {
        const int q = threadIdx.x + m * NT, b = q % B, t = q / B;
        if (kx0 + b < nkx) {
#pragma unroll
          for (int r = 0; r < RA; ++r) base[(size_t)(t + r * (N / RA)) * stride_n + b] = a[m][r];
        }
      }
    }
  } else {
#pragma unroll
    for (int m = 0; m < BL; ++m) {
      if (st_valid<N, B, NT, RL>(m)) {
        const int q = threadIdx.x + m * NT, b = q % B, t = q / B;
        if (kx0 + b < nkx) {
#pragma unroll
          for (int r = 0; r < RL; ++r) base[(size_t)(t + r * (N / RL)) * stride_n + b] = z[m][r];
        }
      }
    }
  }
}
// The same passes with the whole tile staged in shared memory (cp.async in, every stage
// through shared memory, stores from shared memory): fewer registers per thread, which wins for
// the short transforms whose register-staged version needs 16-point butterflies.
template <typename T, int N, int MODE>
__global__ void __launch_bounds__(fft_threads<N, Tile<T>::B>())
k_fft_cols_smem(Cx<T>* __restrict__ spec, const Cx<T>* __restrict__ tw, Geo g, size_t stride_n,
           size_t stride_outer, const double* __restrict__ k2x, const double* __restrict__ k2y,
           const double* __restrict__ k2z, double ntot) {
  constexpr int B = Tile<T>::B;
  constexpr int NT = fft_threads<N, B>();
  extern __shared__ __align__(16) unsigned char smraw[];
  Cx<T>* s = reinterpret_cast<Cx<T>*>(smraw);
  const int kx0 = blockIdx.x * B;
  const int outer = blockIdx.y;
  const int nkx = g.nkx;
  Cx<T>* base = spec + (size_t)outer * stride_outer + kx0;
  // The row pitch is a multiple of 16 complex and the padding columns stay zero, so every
  // B-wide tile is in bounds: all loads of the tile go out back to back as async copies.
  for (int e = threadIdx.x; e < N * B; e += NT) {
    const int n = e / B, b = e - n * B;
    __pipeline_memcpy_async(&s[sw<B>(n, b)], &base[(size_t)n * stride_n + b], sizeof(Cx<T>));
  }
  __pipeline_commit();
  __pipeline_wait_prior(0);
  __syncthreads();
  fft_tile<T, N, B, NT, MODE == 1>(s, tw, 1);
  if constexpr (MODE == 2) {
    // multi/main.f90:889-895: phi3d = -phi3d/k2/(nx*ny*nz) in FP64, phi3d(1,1,1) = 0.
    // One reciprocal of k2*N per element (within 2 ulp of the reference's two divides).
    const double ky2 = k2y[outer];
    for (int e = threadIdx.x; e < N * B; e += NT) {
      const int n = e / B, b = e - n * B;
      const int kx = kx0 + b;
      if (kx < nkx) {
        const double k2 = (k2x[kx] + ky2) + k2z[n];
        const Cx<T> z = s[sw<B>(n, b)];
        const double inv = 1.0 / (k2 * ntot);
        double re = -(double)z.x * inv;
        double im = -(double)z.y * inv;
        if (kx == 0 && outer == 0 && n == 0) { re = 0.0; im = 0.0; }
        s[sw<B>(n, b)] = cx<T>((T)re, (T)im);
      }
    }
    __syncthreads();
    fft_tile<T, N, B, NT, true>(s, tw, 1);
  }
  for (int e = threadIdx.x; e < N * B; e += NT) {
    const int n = e / B, b = e - n * B;
    if (kx0 + b < nkx) base[(size_t)n * stride_n + b] = s[sw<B>(n, b)];
  }
}

// ------------------------------------------------------------------ host launchers
template <typename KernelT>
static cudaError_t prep_smem(KernelT kern, size_t smem) {
  if (smem > 48 * 1024) return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  return cudaSuccess;
}

template <typename T, int M>
static cudaError_t launch_xfwd_m(const PoissonArgs& a, cudaStream_t st) {
  constexpr int B = Tile<T>::B;
  const size_t smem = (size_t)(M + 1) * B * sizeof(Cx<T>);
  auto kern = a.presid ? k_div_fftx<T, M, 3> : (a.real64 ? k_div_fftx<T, M, 2> : k_div_fftx<T, M, 0>);
  cudaError_t e = prep_smem(kern, smem);
  if (e != cudaSuccess) return e;
  const int nlines = a.g.ny * a.g.nz;
  kern<<<(nlines + B - 1) / B, xpass_threads<T, M>(), smem, st>>>(a.u, a.v, a.w, a.presid, (Cx<T>*)a.spec,
                                                                  (const Cx<T>*)a.twx, a.g, a.cdiv);
  return cudaGetLastError();
}

template <typename T, int M>
static cudaError_t launch_xinv_m(const PoissonArgs& a, cudaStream_t st) {
  constexpr int B = Tile<T>::B;
  const size_t smem = (size_t)(M + 1) * B * sizeof(Cx<T>);
  auto kern = a.qin ? k_fftx_inv<T, M, true> : k_fftx_inv<T, M, false>;
  cudaError_t e = prep_smem(kern, smem);
  if (e != cudaSuccess) return e;
  const int nlines = a.g.ny * a.g.nz;
  kern<<<(nlines + B - 1) / B, xpass_threads<T, M>(), smem, st>>>((const Cx<T>*)a.spec, (T*)a.p, (const Cx<T>*)a.twx,
                                                                  a.g, a.qin, a.qout, a.p64);
  return cudaGetLastError();
}

template <typename T, int N, int MODE>
static cudaError_t launch_cols_n(const PoissonArgs& a, int axis, cudaStream_t st) {
  // the 256-point z solve runs faster staged in shared memory (measured at 256^3: 0.066 vs
  // 0.072 ms FP32, 0.105 vs 0.117 ms FP64); every other pass and size register-staged
  constexpr bool staged = MODE == 2 && N == 256;
  constexpr int B = staged ? Tile<T>::B : ColTile<T, N, MODE>::B;
  constexpr int NT = staged ? fft_threads<N, B>() : ColTile<T, N, MODE>::NT;
  const size_t smem = (size_t)N * B * sizeof(Cx<T>);
  auto kern = staged ? k_fft_cols_smem<T, N, MODE> : k_fft_cols<T, N, MODE>;
  cudaError_t e = prep_smem(kern, smem);
  if (e != cudaSuccess) return e;
  const Geo& g = a.g;
  const int ntile = (g.nkx + B - 1) / B;
  const size_t pitch = (size_t)g.pitch;
  const bool ya = axis == 1;  // along y: one tile per (kx tile, z); along z: per (kx tile, y)
  const size_t stride_n = ya ? pitch : (size_t)g.ny * pitch;
  const size_t stride_outer = ya ? (size_t)g.ny * pitch : pitch;
  dim3 grid(ntile, ya ? g.nz : g.ny);
  kern<<<grid, NT, smem, st>>>((Cx<T>*)a.spec, (const Cx<T>*)(ya ? a.twy : a.twz), g, stride_n, stride_outer, a.k2x,
                               a.k2y, a.k2z, a.ntot);
  return cudaGetLastError();
}

#define MHIT_XSIZES(X) X(8) X(16) X(32) X(64) X(96) X(128) X(256) X(512)
#define MHIT_NSIZES(X) X(16) X(32) X(64) X(128) X(192) X(256) X(512) X(1024)

template <typename T>
static cudaError_t launch_xfwd(const PoissonArgs& a, cudaStream_t st) {
  switch (a.g.nx / 2) {
#define C(m) case m: return launch_xfwd_m<T, m>(a, st);
    MHIT_XSIZES(C)
#undef C
  }
  return cudaErrorInvalidValue;
}
template <typename T>
static cudaError_t launch_xinv(const PoissonArgs& a, cudaStream_t st) {
  switch (a.g.nx / 2) {
#define C(m) case m: return launch_xinv_m<T, m>(a, st);
    MHIT_XSIZES(C)
#undef C
  }
  return cudaErrorInvalidValue;
}
template <typename T, int MODE>
static cudaError_t launch_cols(const PoissonArgs& a, int axis, cudaStream_t st) {
  const int n = axis == 1 ? a.g.ny : a.g.nz;
  switch (n) {
#define C(m) case m: return launch_cols_n<T, m, MODE>(a, axis, st);
    MHIT_NSIZES(C)
#undef C
  }
  return cudaErrorInvalidValue;
}

bool poisson_size_supported(int n, bool is_x) {
  if (is_x) {
    if (n % 2) return false;
    switch (n / 2) {
#define C(m) case m: return true;
      MHIT_XSIZES(C)
#undef C
    }
    return false;
  }
  switch (n) {
#define C(m) case m: return true;
    MHIT_NSIZES(C)
#undef C
  }
  return false;
}

template <typename T>
static cudaError_t poisson_stage_t(const PoissonArgs& a, int stage, cudaStream_t st) {
  switch (stage) {
    case PSTAGE_XFWD: return launch_xfwd<T>(a, st);
    case PSTAGE_YFWD: return launch_cols<T, 0>(a, 1, st);
    case PSTAGE_ZSOLVE:
      if (sizeof(T) == 4 && a.tcz) return launch_zsolve_tc(a.tcz, a, a.sc, st);
      return launch_cols<T, 2>(a, 2, st);
    case PSTAGE_YINV: return launch_cols<T, 1>(a, 1, st);
    case PSTAGE_XINV: return launch_xinv<T>(a, st);
    case PSTAGE_ZFWD: return launch_cols<T, 0>(a, 2, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t poisson_stage(const PoissonArgs& a, int stage, cudaStream_t st) {
  return a.fp32 ? poisson_stage_t<float>(a, stage, st) : poisson_stage_t<double>(a, stage, st);
}

}  // namespace mhit
