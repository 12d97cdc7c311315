// Shell-summed kinetic-energy spectrum of the velocity on the device.  The reference has no
// three-dimensional spectrum tool (its post-processing computes dissipation and drop statistics,
// post/compute_diss, post/unionfind_periodic); this is the textbook definition
//   E(k) = 1/2 sum over |kappa| in [k - 1/2, k + 1/2) of |u_kappa|^2 + |v_kappa|^2 + |w_kappa|^2,
//   u_kappa = (1/N) sum_x u(x) exp(-i kappa.x),   N = nx ny nz,
// so that sum_k E(k) = 1/2 <u.u> (Parseval), the kinetic energy of multi/main.f90's diagnostics.
// Wavenumbers are in units of 2 pi / Lx: kappa_x = m_x, kappa_y = m_y nx/ny, kappa_z = m_z nx/nz
// for a box of nx dx by ny dx by nz dx with Lx = 2 pi.
//
// Each component is transformed by the Poisson solver's own FP64 passes (x real-to-complex, then
// y and z forward) into the x-half spectrum [nz][ny][pitch]; k_spec_bin adds each element's
// energy (weight 2 for 0 < kx < nx/2, the conjugate half) to a block histogram in shared memory,
// and k_spec_reduce sums the block histograms in block order.  The shared-memory atomics make the
// last bits depend on scheduling.
#include "common.cuh"
#include "kernels.h"

namespace mhit {

constexpr int SPT = 256;

__global__ void __launch_bounds__(SPT) k_spec_bin(const Cx<double>* __restrict__ spec, Geo g,
                                                  const DevScalars* __restrict__ sc, int comp, int nbins,
                                                  double* __restrict__ partials) {
  extern __shared__ double hist[];
  for (int b = threadIdx.x; b < nbins; b += SPT) hist[b] = 0.0;
  __syncthreads();
  const int nx = g.nx, ny = g.ny, nz = g.nz, nkx = g.nkx, pitch = g.pitch;
  const double ntot = (double)nx * ny * nz, invn = 1.0 / ntot;
  const double sy = (double)nx / ny, sz = (double)nx / nz;
  const double mean = sc->mean[comp];  // the stored field still carries the lazily removed mean
  const int rows = ny * nz;
  for (int row = blockIdx.x; row < rows; row += gridDim.x) {
    const int j = row % ny, k = row / ny;
    const double my = (double)(2 * j <= ny ? j : j - ny) * sy;
    const double mz = (double)(2 * k <= nz ? k : k - nz) * sz;
    const double kyz = my * my + mz * mz;
    for (int kx = threadIdx.x; kx < nkx; kx += SPT) {
      Cx<double> c = spec[(size_t)row * pitch + kx];
      if (row == 0 && kx == 0) c.x -= mean * ntot;
      const double re = c.x * invn, im = c.y * invn;
      const double w = (kx == 0 || 2 * kx == nx) ? 0.5 : 1.0;
      const int shell = (int)rint(sqrt((double)kx * kx + kyz));
      if (shell < nbins) atomicAdd(&hist[shell], w * (re * re + im * im));
    }
  }
  __syncthreads();
  for (int b = threadIdx.x; b < nbins; b += SPT) partials[(size_t)blockIdx.x * nbins + b] = hist[b];
}

__global__ void k_spec_reduce(const double* __restrict__ partials, int nblocks, int nbins, double* __restrict__ E) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nbins; b += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int q = 0; q < nblocks; ++q) s += partials[(size_t)q * nbins + b];
    E[b] += s;
  }
}

int spectrum_blocks(const Geo& g) {
  const int rows = g.ny * g.nz;
  return rows < 148 * 2 ? rows : 148 * 2;
}

cudaError_t launch_spectrum_bin(const Cx<double>* spec, const Geo& g, const DevScalars* sc, int comp, int nbins,
                                double* partials, double* E, cudaStream_t st) {
  const int nb = spectrum_blocks(g);
  const size_t smem = (size_t)nbins * sizeof(double);
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k_spec_bin, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  k_spec_bin<<<nb, SPT, smem, st>>>(spec, g, sc, comp, nbins, partials);
  k_spec_reduce<<<(nbins + 255) / 256, 256, 0, st>>>(partials, nb, nbins, E);
  return cudaGetLastError();
}

}  // namespace mhit
