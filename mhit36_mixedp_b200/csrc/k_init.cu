// Initial conditions synthesised on the device: the O(N^3) part of the reference's start-up
// (multi/main.f90:322-415) and of the seeded benchmark fields.  The one-dimensional tables
// (coordinates, sines, complex exponentials) and the random mode amplitudes are O(N) host work
// done by the library's caller or its host code; the kernels here combine them over the grid.
//
//   k_tg        Taylor-Green, multi/main.f90:324-337: u = sin(x - dx/2) cos(y) cos(z),
//               v = -cos(x) sin(y - dx/2) cos(z), w = 0, from per-axis tables of the
//               accumulated coordinates (products formed left to right, as the reference).
//   k_modes_*   u(x) = Re sum_k c_k exp(i k.x) over a (2K+1)^3 cube of integer wavenumbers,
//               evaluated in three separable sums (over kx, then ky, then kz), then scaled to a
//               given rms: the random solenoidal field of the benchmark configurations.
//   k_drops     phi = 0.5 (1 - tanh((r - R)/(2 eps))) with r the periodic minimum-image distance
//               to the nearest of n centres: the centred drop of multi/main.f90:370-382
//               generalised to many drops.
//   k_particles the tracer table of multi/particles.f90:37-76 from a counter-based generator.
// Every product and sum is written with explicit IEEE operations (no contraction), so the
// device fields equal a host evaluation in the same order except where CUDA's tanh differs
// from the host's by an ulp.
#include "common.cuh"
#include "kernels.h"

namespace mhit {

constexpr int ITHREADS = 256;

__global__ void k_tg(double* __restrict__ u, double* __restrict__ v, double* __restrict__ w,
                     const double* __restrict__ tab, int nx, int ny, int nz) {
  // tab: sin(x_i - dx/2), cos(x_i) (nx each); sin(y_j - dx/2), cos(y_j) (ny each); cos(z_k) (nz)
  const double* sxh = tab;
  const double* cxs = sxh + nx;
  const double* syh = cxs + nx;
  const double* cys = syh + ny;
  const double* czs = cys + ny;
  const size_t n = (size_t)nx * ny * nz;
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(c % nx);
    const size_t r = c / nx;
    const int j = (int)(r % ny), k = (int)(r / ny);
    u[c] = __dmul_rn(__dmul_rn(sxh[i], cys[j]), czs[k]);
    v[c] = __dmul_rn(__dmul_rn(-cxs[i], syh[j]), czs[k]);
    w[c] = 0.0;
  }
}

// A[kz][ky][i] = sum_kx c[kz][ky][kx] ex[i][kx]   (K = 2 kmax + 1 wavenumbers per axis)
__global__ void k_modes_x(const Cx<double>* __restrict__ cm, const Cx<double>* __restrict__ ex, int K, int nx,
                          Cx<double>* __restrict__ A) {
  const int total = K * K * nx;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const int i = t % nx, kk = t / nx;  // kk = kz*K + ky
    double re = 0.0, im = 0.0;
    for (int q = 0; q < K; ++q) {
      const Cx<double> a = cm[(size_t)kk * K + q], b = ex[(size_t)i * K + q];
      re = __dadd_rn(re, __dsub_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)));
      im = __dadd_rn(im, __dadd_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x)));
    }
    A[t] = cx<double>(re, im);
  }
}

// B[kz][j][i] = sum_ky ey[j][ky] A[kz][ky][i]
__global__ void k_modes_y(const Cx<double>* __restrict__ A, const Cx<double>* __restrict__ ey, int K, int nx, int ny,
                          Cx<double>* __restrict__ Bt) {
  const size_t total = (size_t)K * ny * nx;
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(t % nx);
    const size_t r = t / nx;
    const int j = (int)(r % ny), kz = (int)(r / ny);
    double re = 0.0, im = 0.0;
    for (int q = 0; q < K; ++q) {
      const Cx<double> a = ey[(size_t)j * K + q], b = A[((size_t)kz * K + q) * nx + i];
      re = __dadd_rn(re, __dsub_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)));
      im = __dadd_rn(im, __dadd_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x)));
    }
    Bt[t] = cx<double>(re, im);
  }
}

// f[k][j][i] = sum_kz Re(ez[k][kz]) Re(B[kz][j][i]) - sum_kz Im(ez[k][kz]) Im(B[kz][j][i]); one
// thread per (j, i) column marching in k (its B column is read from L1 after the first plane),
// with per-block partial sums of f^2 for the rms scaling.
__global__ void __launch_bounds__(ITHREADS) k_modes_z(const Cx<double>* __restrict__ Bt,
                                                      const Cx<double>* __restrict__ ez, int K, int nx, int ny,
                                                      int nz, double* __restrict__ f, double* __restrict__ partials) {
  const size_t plane = (size_t)nx * ny;
  double ss = 0.0;
  for (size_t col = (size_t)blockIdx.x * ITHREADS + threadIdx.x; col < plane; col += (size_t)gridDim.x * ITHREADS) {
    for (int k = 0; k < nz; ++k) {
      double sr = 0.0, si = 0.0;
      for (int q = 0; q < K; ++q) {
        const Cx<double> e = ez[(size_t)k * K + q];
        const Cx<double> b = Bt[(size_t)q * plane + col];
        sr = __dadd_rn(sr, __dmul_rn(e.x, b.x));
        si = __dadd_rn(si, __dmul_rn(e.y, b.y));
      }
      const double val = __dsub_rn(sr, si);
      f[(size_t)k * plane + col] = val;
      ss = __fma_rn(val, val, ss);
    }
  }
  __shared__ double red[ITHREADS / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) ss += __shfl_down_sync(0xffffffffu, ss, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = ss;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = red[0];
    for (int q = 1; q < ITHREADS / 32; ++q) t += red[q];
    partials[blockIdx.x] = t;
  }
}

__global__ void k_scale(double* __restrict__ f, size_t n, double s) {
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x)
    f[c] = __dmul_rn(f[c], s);
}

// phi from the nearest of nd centres (cx, cy, cz), minimum image in a box lx x ly x lz; the
// coordinates are x = i dx, y = (j + s) dx, z = (k + s) dx (the reference labelling, s = yz_shift)
__global__ void k_drops(double* __restrict__ phi, const double* __restrict__ centres, int nd, int nx, int ny, int nz,
                        int s, double dx, double lx, double ly, double lz, double radius, double eps) {
  const size_t n = (size_t)nx * ny * nz;
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(c % nx);
    const size_t r = c / nx;
    const int j = (int)(r % ny), k = (int)(r / ny);
    const double x = __dmul_rn((double)i, dx), y = __dmul_rn((double)(j + s), dx), z = __dmul_rn((double)(k + s), dx);
    double rmin = INFINITY;
    for (int d = 0; d < nd; ++d) {
      double ddx = __dsub_rn(x, __ldg(centres + 3 * d));
      double ddy = __dsub_rn(y, __ldg(centres + 3 * d + 1));
      double ddz = __dsub_rn(z, __ldg(centres + 3 * d + 2));
      ddx = __dsub_rn(ddx, __dmul_rn(lx, rint(__ddiv_rn(ddx, lx))));
      ddy = __dsub_rn(ddy, __dmul_rn(ly, rint(__ddiv_rn(ddy, ly))));
      ddz = __dsub_rn(ddz, __dmul_rn(lz, rint(__ddiv_rn(ddz, lz))));
      const double d2 = __dadd_rn(__dadd_rn(__dmul_rn(ddz, ddz), __dmul_rn(ddy, ddy)), __dmul_rn(ddx, ddx));
      rmin = fmin(rmin, __dsqrt_rn(d2));
    }
    phi[c] = __dmul_rn(0.5, __dsub_rn(1.0, tanh(__ddiv_rn(__ddiv_rn(__dsub_rn(rmin, radius), 2.0), eps))));
  }
}

// Tracer table of multi/particles.f90:37-76 (particlegenerator with inflag = 1): tag i, position
// uniform in the box, everything else zero.  The reference draws from an unseeded
// RANDOM_NUMBER; here position a of tracer i is splitmix64(seed + (3 i + a + 1) G) (Steele, Lea
// and Flood, "Fast splittable pseudorandom number generators", OOPSLA 2014; G the golden-ratio
// increment 0x9E3779B97F4A7C15) mapped to [0, 1) by its top 53 bits, times the box length.
__device__ __forceinline__ unsigned long long splitmix64(unsigned long long z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__global__ void k_particles(double* __restrict__ part, int np, unsigned long long seed, double lx, double ly,
                            double lz) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x) {
    const double len[3] = {lx, ly, lz};
    part[i] = (double)(i + 1);  // Itag
    for (int a = 0; a < 3; ++a) {
      const unsigned long long r = splitmix64(seed + (3ull * (unsigned long long)i + a + 1) * 0x9E3779B97F4A7C15ull);
      const double u01 = (double)(r >> 11) * 0x1.0p-53;
      part[(size_t)(1 + a) * np + i] = __dmul_rn(u01, len[a]);
    }
    for (int c = 4; c < 12; ++c) part[(size_t)c * np + i] = 0.0;
  }
}

static int grid_for(size_t n) {
  const size_t b = (n + ITHREADS - 1) / ITHREADS;
  return (int)(b < 148 * 16 ? (b ? b : 1) : 148 * 16);
}

cudaError_t launch_init_tg(double* u, double* v, double* w, const double* tab, int nx, int ny, int nz,
                           cudaStream_t st) {
  k_tg<<<grid_for((size_t)nx * ny * nz), ITHREADS, 0, st>>>(u, v, w, tab, nx, ny, nz);
  return cudaGetLastError();
}

int modes_partials(int nx, int ny) { return grid_for((size_t)nx * ny); }

cudaError_t launch_init_modes(const ModeArgs& a, cudaStream_t st) {
  k_modes_x<<<grid_for((size_t)a.K * a.K * a.nx), ITHREADS, 0, st>>>(a.cm, a.ex, a.K, a.nx, a.A);
  k_modes_y<<<grid_for((size_t)a.K * a.ny * a.nx), ITHREADS, 0, st>>>(a.A, a.ey, a.K, a.nx, a.ny, a.Bt);
  k_modes_z<<<modes_partials(a.nx, a.ny), ITHREADS, 0, st>>>(a.Bt, a.ez, a.K, a.nx, a.ny, a.nz, a.f, a.partials);
  return cudaGetLastError();
}

cudaError_t launch_scale(double* f, size_t n, double s, cudaStream_t st) {
  k_scale<<<grid_for(n), ITHREADS, 0, st>>>(f, n, s);
  return cudaGetLastError();
}

cudaError_t launch_init_particles(double* part, int np, unsigned long long seed, double lx, double ly, double lz,
                                  cudaStream_t st) {
  k_particles<<<grid_for((size_t)np), ITHREADS, 0, st>>>(part, np, seed, lx, ly, lz);
  return cudaGetLastError();
}

cudaError_t launch_init_drops(const DropInitArgs& a, cudaStream_t st) {
  k_drops<<<grid_for((size_t)a.nx * a.ny * a.nz), ITHREADS, 0, st>>>(a.phi, a.centres, a.nd, a.nx, a.ny, a.nz, a.s,
                                                                       a.dx, a.lx, a.ly, a.lz, a.radius, a.eps);
  return cudaGetLastError();
}

}  // namespace mhit
