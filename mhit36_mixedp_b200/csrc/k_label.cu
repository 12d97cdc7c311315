// Droplet labelling: the connected components of phi >= thresh with periodic boundaries and
// their statistics, as post/unionfind_periodic/main.f90 computes them (mask :137-151, 6- or
// 26-neighbour connectivity :33-48, periodic halos :152-157/:251-258, per-drop volume, circular
// mean centre and mean velocity :276-336, volume = cells dx^3 :436).
//
// The reference iterates min-label propagation over 16^3 tiles until nothing changes.  Here the
// components come from a lock-free union-find over the cell indices (Playne and Hawick, "A New
// Algorithm for Parallel Connected-Component Labelling on GPUs", IEEE TPDS 2018): every masked
// cell starts as its own root; for each masked neighbour pair the two roots are joined by an
// atomicMin that hangs the larger root under the smaller, so the final root of a component is its
// smallest cell index (k, j, i order) whatever the scheduling; a flatten pass points every cell at
// its root.  Drops are numbered by that smallest index, so the order is deterministic.
//
// Every loop that follows parent pointers or retries a link is bounded (a chain or a retry
// sequence can never be longer than the number of cells); hitting the bound sets an error flag
// that the host turns into an error status instead of looping.
#include "common.cuh"
#include "kernels.h"

namespace mhit {

// forward half of the neighbourhood (dz, dy, dx): the other half is reached from the neighbour
__constant__ int8_t c_fwd[13][3] = {{0, 0, 1},  {0, 1, 0},  {1, 0, 0},  {0, 1, 1},  {0, 1, -1},
                                    {1, 0, 1},  {1, 0, -1}, {1, 1, 0},  {1, -1, 0}, {1, 1, 1},
                                    {1, 1, -1}, {1, -1, 1}, {1, -1, -1}};

// Root of x with path halving: each visited node is re-pointed at its grandparent.  A node's
// ancestors stay its ancestors (roots are only ever hung under smaller roots) and parents only
// decrease, so a plain store of the grandparent is safe under concurrent links and halvings.
__device__ __forceinline__ int find_root(int* lab, int x, long long bound, int* err) {
  volatile int* vl = lab;  // parents change under concurrent links: read them from L2
  for (long long it = 0; it < bound; ++it) {
    const int y = vl[x];
    if (y == x) return x;
    const int z = vl[y];
    if (z == y) return y;
    vl[x] = z;
    x = z;
  }
  atomicExch(err, 1);
  return x;
}

__device__ __forceinline__ void unite(int* lab, int a, int b, long long bound, int* err) {
  for (long long it = 0; it < bound; ++it) {
    a = find_root(lab, a, bound, err);
    b = find_root(lab, b, bound, err);
    if (a == b) return;
    if (a > b) {
      const int t = a;
      a = b;
      b = t;
    }
    const int old = atomicMin(&lab[b], a);
    if (old == b) return;  // b was still a root and now hangs under a
    b = old;               // b was linked meanwhile: continue from its new parent
  }
  atomicExch(err, 1);
}

__global__ void k_lab_init(const double* __restrict__ phi, double thresh, int* __restrict__ lab, int n) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
    lab[c] = phi[c] >= thresh ? c : -1;  // post/unionfind_periodic/main.f90:141
}

__global__ void k_lab_merge(int* lab, int nx, int ny, int nz, int nfwd, long long bound, int* err) {
  const int n = nx * ny * nz;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    if (lab[c] < 0) continue;
    const int i = c % nx, j = (c / nx) % ny, k = c / (nx * ny);
    for (int q = 0; q < nfwd; ++q) {
      int ii = i + c_fwd[q][2], jj = j + c_fwd[q][1], kk = k + c_fwd[q][0];
      ii = ii < 0 ? ii + nx : (ii >= nx ? ii - nx : ii);
      jj = jj < 0 ? jj + ny : (jj >= ny ? jj - ny : jj);
      kk = kk >= nz ? kk - nz : kk;
      const int d = (kk * ny + jj) * nx + ii;
      if (d != c && lab[d] >= 0) unite(lab, c, d, bound, err);
    }
  }
}

__global__ void k_lab_flatten(int* lab, int n, long long bound, int* err) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
    if (lab[c] >= 0) lab[c] = find_root(lab, c, bound, err);
}

// roots per chunk of LCHUNK consecutive cells (one block per chunk)
constexpr int LTHREADS = 256, LCHUNK = 8192;

__global__ void k_lab_count(const int* __restrict__ lab, int n, int* __restrict__ counts) {
  __shared__ int s;
  if (threadIdx.x == 0) s = 0;
  __syncthreads();
  const int c0 = blockIdx.x * LCHUNK, c1 = min(c0 + LCHUNK, n);
  int local = 0;
  for (int c = c0 + threadIdx.x; c < c1; c += LTHREADS) local += lab[c] == c;
  atomicAdd(&s, local);
  __syncthreads();
  if (threadIdx.x == 0) counts[blockIdx.x] = s;
}

// number the roots in index order: the root of drop d (0-based) gets -(d + 2), so that any cell
// finds its drop as -lab[lab[c]] - 2 (or -lab[c] - 2 at the root itself)
__global__ void k_lab_number(int* __restrict__ lab, int n, const int* __restrict__ offsets) {
  __shared__ int warp_tot[LTHREADS / 32];
  __shared__ int base;
  if (threadIdx.x == 0) base = offsets[blockIdx.x];
  __syncthreads();
  const int c0 = blockIdx.x * LCHUNK, c1 = min(c0 + LCHUNK, n);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int t0 = c0; t0 < c1; t0 += LTHREADS) {
    const int c = t0 + threadIdx.x;
    const int root = (c < c1 && lab[c] == c) ? 1 : 0;
    const unsigned bal = __ballot_sync(0xffffffffu, root);
    const int before = __popc(bal & ((1u << lane) - 1u));
    if (lane == 0) warp_tot[wid] = __popc(bal);
    __syncthreads();
    int wbase = 0;
    for (int q = 0; q < wid; ++q) wbase += warp_tot[q];
    if (root) lab[c] = -(base + wbase + before + 2);
    __syncthreads();
    if (threadIdx.x == 0) {
      int tot = 0;
      for (int q = 0; q < LTHREADS / 32; ++q) tot += warp_tot[q];
      base += tot;
    }
    __syncthreads();
  }
}

__device__ __forceinline__ int drop_of(const int* lab, int c) {
  const int r = lab[c];
  if (r == -1) return -1;
  return r < -1 ? -r - 2 : -lab[r] - 2;
}

// per drop: cells, sums of sin/cos of the cell centre per axis, sums of u, v, w
// (post/unionfind_periodic/main.f90:302-315); acc is [ndrops][9].  Cells of one drop are
// contiguous along x, so the 32 cells a warp visits mostly belong to one or two drops: the
// lanes of each drop are grouped (match_any), sum their values with shuffles, and one lane per
// group does the atomics -- a drop of 10^5 cells would otherwise serialise 10^6 atomics on nine
// addresses.
__global__ void k_lab_stats(const int* __restrict__ lab, int nx, int ny, int nz, const double* __restrict__ u,
                            const double* __restrict__ v, const double* __restrict__ w,
                            const double* __restrict__ trig, const DevScalars* __restrict__ sc,
                            double* __restrict__ acc, unsigned long long* __restrict__ cells) {
  const int n = nx * ny * nz;
  const double mu_ = sc->mean[0], mv_ = sc->mean[1], mw_ = sc->mean[2];
  // trig: sin x (nx), cos x (nx), sin y (ny), cos y (ny), sin z (nz), cos z (nz)
  const double* sx = trig;
  const double* cxs = sx + nx;
  const double* sy = cxs + nx;
  const double* cys = sy + ny;
  const double* sz = cys + ny;
  const double* czs = sz + nz;
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (blockDim.x >> 5);
  // warp-uniform loop: all 32 lanes take part in every match and shuffle
  for (int base = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 32; base < n; base += warps * 32) {
    const int c = base + lane;
    const int d = c < n ? drop_of(lab, c) : -1;
    if (__all_sync(0xffffffffu, d < 0)) continue;  // the whole warp is background (most warps)
    double val[9];
    if (d >= 0) {
      const int i = c % nx, j = (c / nx) % ny, k = c / (nx * ny);
      val[0] = sx[i];
      val[1] = cxs[i];
      val[2] = sy[j];
      val[3] = cys[j];
      val[4] = sz[k];
      val[5] = czs[k];
      val[6] = u[c] - mu_;
      val[7] = v[c] - mv_;
      val[8] = w[c] - mw_;
    } else {
#pragma unroll
      for (int q = 0; q < 9; ++q) val[q] = 0.0;
    }
    const unsigned grp = __match_any_sync(0xffffffffu, d);
    double sum[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) sum[q] = 0.0;
    // every lane of a group walks the same lanes in the same order: the sums are identical
    for (unsigned m = grp; m; m &= m - 1) {
      const int l = __ffs(m) - 1;
#pragma unroll
      for (int q = 0; q < 9; ++q) sum[q] += __shfl_sync(grp, val[q], l);
    }
    if (d >= 0 && lane == __ffs(grp) - 1) {
      double* a = acc + (size_t)d * 9;
      atomicAdd(&cells[d], (unsigned long long)__popc(grp));
#pragma unroll
      for (int q = 0; q < 9; ++q) atomicAdd(a + q, sum[q]);
    }
  }
}

// label field for the host: 0 background, 1.. drop number
__global__ void k_lab_final(const int* __restrict__ lab, int* __restrict__ out, int n) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) out[c] = drop_of(lab, c) + 1;
}

int label_chunks(int n) { return (n + LCHUNK - 1) / LCHUNK; }

cudaError_t launch_label_components(const LabelArgs& a, cudaStream_t st) {
  const int n = a.nx * a.ny * a.nz;
  const int grid = 148 * 8;
  k_lab_init<<<grid, 256, 0, st>>>(a.phi, a.thresh, a.lab, n);
  // the loops' bound: the cell count (no chain or retry sequence is longer), or a smaller test
  // bound that makes a legitimate chain run out and exercises the error path
  const long long bound = a.bound > 0 ? a.bound : n;
  k_lab_merge<<<grid, 256, 0, st>>>(a.lab, a.nx, a.ny, a.nz, a.connectivity == 26 ? 13 : 3, bound, a.err);
  k_lab_flatten<<<grid, 256, 0, st>>>(a.lab, n, bound, a.err);
  k_lab_count<<<label_chunks(n), LTHREADS, 0, st>>>(a.lab, n, a.counts);
  return cudaGetLastError();
}

cudaError_t launch_label_number(const LabelArgs& a, cudaStream_t st) {
  const int n = a.nx * a.ny * a.nz;
  k_lab_number<<<label_chunks(n), LTHREADS, 0, st>>>(a.lab, n, a.counts);
  return cudaGetLastError();
}

cudaError_t launch_label_stats(const LabelArgs& a, cudaStream_t st) {
  const int n = a.nx * a.ny * a.nz;
  k_lab_stats<<<148 * 8, 256, 0, st>>>(a.lab, a.nx, a.ny, a.nz, a.u, a.v, a.w, a.trig, a.sc, a.acc, a.cells);
  if (a.out) k_lab_final<<<148 * 8, 256, 0, st>>>(a.lab, a.out, n);
  return cudaGetLastError();
}

}  // namespace mhit
