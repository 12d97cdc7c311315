// Shared-memory mixed-radix Stockham FFT over a tile of B independent columns.
//
// Replaces the cuFFT 1-D plans of the reference (multi/main.f90:187-205, executed at
// :853,860,865,901,906,912).  Written from the DFT definition: a decimation-in-time
// Stockham autosort (one radix-R register butterfly per thread per stage, in-place in shared
// memory with a barrier between the read and the write half of each stage).
//
// Tile layout in shared memory: element (n, b) -- n along the transform, b the column --
// lives at n*B + (b ^ (n % B)).  A row of B elements is exactly 128 bytes (B = 8 double2 or
// 16 float2), so a warp touching whole rows is conflict-free, and the XOR swizzle keeps a
// warp walking down one column (the x-direction loads) conflict-free as well.
#pragma once
#include "common.cuh"

namespace mhit {

template <int N> struct Radix;  // radix schedule per transform length
template <> struct Radix<8>    { static constexpr int ns = 1; static constexpr int r[3] = {8, 0, 0}; };
template <> struct Radix<16>   { static constexpr int ns = 2; static constexpr int r[3] = {4, 4, 0}; };
template <> struct Radix<32>   { static constexpr int ns = 2; static constexpr int r[3] = {4, 8, 0}; };
template <> struct Radix<64>   { static constexpr int ns = 2; static constexpr int r[3] = {8, 8, 0}; };
template <> struct Radix<96>   { static constexpr int ns = 3; static constexpr int r[3] = {3, 4, 8}; };
template <> struct Radix<128>  { static constexpr int ns = 2; static constexpr int r[3] = {8, 16, 0}; };
template <> struct Radix<192>  { static constexpr int ns = 3; static constexpr int r[3] = {3, 8, 8}; };
template <> struct Radix<256>  { static constexpr int ns = 2; static constexpr int r[3] = {16, 16, 0}; };
template <> struct Radix<512>  { static constexpr int ns = 3; static constexpr int r[3] = {8, 8, 8}; };
template <> struct Radix<1024> { static constexpr int ns = 3; static constexpr int r[3] = {8, 8, 16}; };

template <int N> __host__ __device__ constexpr int max_radix() {
  int m = 0;
  for (int s = 0; s < Radix<N>::ns; ++s) m = Radix<N>::r[s] > m ? Radix<N>::r[s] : m;
  return m;
}

// threads per tile: one butterfly of the largest radix per thread, clamped to [64, 512]
template <int N, int B> __host__ __device__ constexpr int fft_threads() {
  int t = N / max_radix<N>() * B;
  return t < 64 ? 64 : (t > 512 ? 512 : t);
}

template <int B> __device__ __forceinline__ int sw(int n, int b) { return n * B + (b ^ (n & (B - 1))); }

// ---------------------------------------------------------------- register butterflies
template <typename T, bool INV> __device__ __forceinline__ void dft2(Cx<T>* a) {
  Cx<T> t = a[0];
  a[0] = t + a[1];
  a[1] = t - a[1];
}

template <typename T, bool INV> __device__ __forceinline__ void dft3(Cx<T>* a) {
  const T h = (T)0.5;
  const T s3 = (T)0.86602540378443864676372317075294;  // sqrt(3)/2
  Cx<T> s = a[1] + a[2];
  Cx<T> d = a[1] - a[2];
  Cx<T> m = a[0] - scale(s, h);
  // (-+ i sqrt(3)/2) * d
  Cx<T> r = INV ? cx<T>(-s3 * d.y, s3 * d.x) : cx<T>(s3 * d.y, -s3 * d.x);
  a[0] = a[0] + s;
  a[1] = m + r;
  a[2] = m - r;
}

template <typename T, bool INV> __device__ __forceinline__ void dft4(Cx<T>* a) {
  Cx<T> t0 = a[0] + a[2];
  Cx<T> t1 = a[0] - a[2];
  Cx<T> t2 = a[1] + a[3];
  Cx<T> t3 = mul_mi<T, INV>(a[1] - a[3]);
  a[0] = t0 + t2;
  a[2] = t0 - t2;
  a[1] = t1 + t3;
  a[3] = t1 - t3;
}

template <typename T, bool INV> __device__ __forceinline__ void dft8(Cx<T>* a) {
  const T r2 = (T)0.70710678118654752440084436210485;
  Cx<T> e[4] = {a[0], a[2], a[4], a[6]};
  Cx<T> o[4] = {a[1], a[3], a[5], a[7]};
  dft4<T, INV>(e);
  dft4<T, INV>(o);
  // o[k] *= w8^k, w8 = exp(-+ 2 pi i / 8)
  o[1] = INV ? cx<T>(r2 * (o[1].x - o[1].y), r2 * (o[1].x + o[1].y))
             : cx<T>(r2 * (o[1].x + o[1].y), r2 * (o[1].y - o[1].x));
  o[2] = mul_mi<T, INV>(o[2]);
  o[3] = INV ? cx<T>(-r2 * (o[3].x + o[3].y), r2 * (o[3].x - o[3].y))
             : cx<T>(r2 * (o[3].y - o[3].x), -r2 * (o[3].x + o[3].y));
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    a[k] = e[k] + o[k];
    a[k + 4] = e[k] - o[k];
  }
}

template <typename T, bool INV> __device__ __forceinline__ void dft16(Cx<T>* a) {
  // 16 = 4 x 4: columns n1, rows n2; y[k2 + 4 k1]
  const T c1 = (T)0.92387953251128675612818318939679;  // cos(pi/8)
  const T s1 = (T)0.38268343236508977172845998403040;  // sin(pi/8)
  const T r2 = (T)0.70710678118654752440084436210485;
  Cx<T> b[4][4];
#pragma unroll
  for (int n1 = 0; n1 < 4; ++n1) {
    Cx<T> t[4] = {a[n1], a[n1 + 4], a[n1 + 8], a[n1 + 12]};
    dft4<T, INV>(t);
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) b[n1][k2] = t[k2];
  }
  // twiddles w16^(n1*k2); for the inverse use the conjugate
  const T sg = INV ? (T)1 : (T)-1;
  auto tw = [&](Cx<T> v, T c, T s) { return cx<T>(v.x * c - v.y * (sg * s), v.x * (sg * s) + v.y * c); };
  b[1][1] = tw(b[1][1], c1, s1);
  b[1][2] = tw(b[1][2], r2, r2);
  b[1][3] = tw(b[1][3], s1, c1);
  b[2][1] = tw(b[2][1], r2, r2);
  b[2][2] = mul_mi<T, INV>(b[2][2]);
  b[2][3] = tw(b[2][3], -r2, r2);
  b[3][1] = tw(b[3][1], s1, c1);
  b[3][2] = tw(b[3][2], -r2, r2);
  b[3][3] = tw(b[3][3], -c1, -s1);
#pragma unroll
  for (int k2 = 0; k2 < 4; ++k2) {
    Cx<T> t[4] = {b[0][k2], b[1][k2], b[2][k2], b[3][k2]};
    dft4<T, INV>(t);
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) a[k2 + 4 * k1] = t[k1];
  }
}

template <typename T, bool INV> __device__ __forceinline__ void dft32(Cx<T>* a) {
  // 32 = 2 x 16: the 16-point DFTs of the even and odd elements, the odd half times
  // w32^k = exp(-+ 2 pi i k/32) = cos(pi k/16) -+ i sin(pi k/16), then one radix-2 step
  constexpr double C1 = 0.980785280403230449126182236134, C2 = 0.923879532511286756128183189397,
                   C3 = 0.831469612302545237078788377618, C4 = 0.707106781186547524400844362105,
                   C5 = 0.555570233019602224742830813949, C6 = 0.382683432365089771728459984030,
                   C7 = 0.195090322016128267848284868477;
  const T cs[16] = {(T)1.0, (T)C1, (T)C2, (T)C3, (T)C4, (T)C5, (T)C6, (T)C7,
                    (T)0.0, (T)-C7, (T)-C6, (T)-C5, (T)-C4, (T)-C3, (T)-C2, (T)-C1};
  const T sn[16] = {(T)0.0, (T)C7, (T)C6, (T)C5, (T)C4, (T)C3, (T)C2, (T)C1,
                    (T)1.0, (T)C1, (T)C2, (T)C3, (T)C4, (T)C5, (T)C6, (T)C7};
  Cx<T> e[16], o[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    e[k] = a[2 * k];
    o[k] = a[2 * k + 1];
  }
  dft16<T, INV>(e);
  dft16<T, INV>(o);
  const T sg = INV ? (T)1 : (T)-1;
#pragma unroll
  for (int k = 1; k < 16; ++k) {
    const T ck = cs[k], sk = sg * sn[k];
    o[k] = cx<T>(o[k].x * ck - o[k].y * sk, o[k].x * sk + o[k].y * ck);
  }
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    const Cx<T> t = o[k];
    a[k] = e[k] + t;
    a[k + 16] = e[k] - t;
  }
}

template <typename T, bool INV, int R> __device__ __forceinline__ void dftR(Cx<T>* a) {
  if constexpr (R == 2) dft2<T, INV>(a);
  else if constexpr (R == 3) dft3<T, INV>(a);
  else if constexpr (R == 4) dft4<T, INV>(a);
  else if constexpr (R == 8) dft8<T, INV>(a);
  else if constexpr (R == 16) dft16<T, INV>(a);
  else if constexpr (R == 32) dft32<T, INV>(a);
}

// Barrier of the threads that run a tile transform: the whole block by default; a named
// barrier (id, count) when only some warps of the block transform (warp-specialised kernels).
struct SyncBlock {
  __device__ __forceinline__ static void sync() { __syncthreads(); }
};
template <int ID, int COUNT> struct SyncNamed {
  __device__ __forceinline__ static void sync() { asm volatile("bar.sync %0, %1;" ::"n"(ID), "n"(COUNT) : "memory"); }
};

// ---------------------------------------------------------------- one Stockham stage
// tw: table of exp(-2 pi i m / L) for m in [0, L); twstride = L / N.  Threads 0..NT-1 take part.
template <typename T, int N, int B, int NT, int R, bool INV, typename SY = SyncBlock>
__device__ __forceinline__ void stockham_stage(Cx<T>* s, const Cx<T>* __restrict__ tw, int twstride, int p) {
  constexpr int NB = N / R * B;
  constexpr int BPT = (NB + NT - 1) / NT;
  Cx<T> a[BPT][R];
  const int tid = threadIdx.x;
#pragma unroll
  for (int m = 0; m < BPT; ++m) {
    const int q = tid + m * NT;
    if (NB % NT == 0 || q < NB) {
      const int b = q % B, t = q / B;
#pragma unroll
      for (int r = 0; r < R; ++r) a[m][r] = s[sw<B>(t + r * (N / R), b)];
    }
  }
  SY::sync();
#pragma unroll
  for (int m = 0; m < BPT; ++m) {
    const int q = tid + m * NT;
    if (NB % NT == 0 || q < NB) {
      const int b = q % B, t = q / B;
      const int k = t % p;
      if (p > 1) {
        // w^(r k) with w = exp(-+ 2 pi i / (p R)); table index r*k*(N/(pR))*twstride
        const int step = (N / (p * R)) * twstride;
#pragma unroll
        for (int r = 1; r < R; ++r) {
          Cx<T> w = tw[r * k * step];
          if (INV) w.y = -w.y;
          a[m][r] = cmul(a[m][r], w);
        }
      }
      dftR<T, INV, R>(a[m]);
      const int j = (t / p) * p * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) s[sw<B>(j + r * p, b)] = a[m][r];
    }
  }
  SY::sync();
}

// Full transform of the N x B tile in s (unnormalised in both directions, as cuFFT), in the
// radix schedule S (default Radix<N>), by threads 0..NT-1 synchronising with SY.  Caller
// synchronises before (tile loaded); returns after a barrier.
template <typename T, int N, int B, int NT, bool INV, typename S = Radix<N>, typename SY = SyncBlock>
__device__ __forceinline__ void fft_tile(Cx<T>* s, const Cx<T>* __restrict__ tw, int twstride) {
  constexpr int NS = S::ns;
  int p = 1;
  if constexpr (NS >= 1) {
    constexpr int R = S::r[0];
    stockham_stage<T, N, B, NT, R, INV, SY>(s, tw, twstride, p);
    p *= R;
  }
  if constexpr (NS >= 2) {
    constexpr int R = S::r[1];
    stockham_stage<T, N, B, NT, R, INV, SY>(s, tw, twstride, p);
    p *= R;
  }
  if constexpr (NS >= 3) {
    constexpr int R = S::r[2];
    stockham_stage<T, N, B, NT, R, INV, SY>(s, tw, twstride, p);
  }
}


// C2R preparation of B half spectra of length M+1 (kx = 0..M) in the tile s, in place: the
// packed half-length sequence Z[k] = (X[k] + X*[M-k]) + i W^-k (X[k] - X*[M-k]), W = exp(-2 pi
// i/(2M)), whose inverse transform gives the real line as (even + i odd) pairs; the imaginary
// parts of X[0] and X[M] are ignored.  Caller synchronises before (tile loaded) and after.
template <typename T, int M, int B, int NT>
__device__ __forceinline__ void c2r_untangle(Cx<T>* s, const Cx<T>* __restrict__ twx) {
  for (int e = threadIdx.x; e < (M / 2 + 1) * B; e += NT) {
    const int kk = e / B, b = e - kk * B;
    if (kk == 0) {
      const T a = s[sw<B>(0, b)].x, c = s[sw<B>(M, b)].x;
      s[sw<B>(0, b)] = cx<T>(a + c, a - c);
    } else {
      const Cx<T> xk = s[sw<B>(kk, b)];
      const Cx<T> xm = s[sw<B>(M - kk, b)];
      {
        const Cx<T> a = xk + conj(xm);
        const Cx<T> d = xk - conj(xm);
        const Cx<T> t = cmul(conj(twx[kk]), d);
        s[sw<B>(kk, b)] = cx<T>(a.x - t.y, a.y + t.x);
      }
      if (kk != M - kk) {
        const Cx<T> a = xm + conj(xk);
        const Cx<T> d = xm - conj(xk);
        const Cx<T> t = cmul(conj(twx[M - kk]), d);
        s[sw<B>(M - kk, b)] = cx<T>(a.x - t.y, a.y + t.x);
      }
    }
  }
}

// ---------------------------------------------------------------- stages with register I/O
// Stage s of the transform in radix order REV (false: Radix<N>::r[0..ns-1], true: reversed).
// Butterfly q = threadIdx.x + m NT works on column b = q % B, t = q / B: it reads elements
// t + r N/R and writes elements (t/p) p R + t%p + r p, p the product of the earlier radices.
// The first stage (p = 1) therefore reads, and the last stage (p = N/R) writes, the strided
// set t + r N/R: those two stages can take their operands from, and leave their results in,
// registers, so a tile loaded from (stored to) global memory skips a shared-memory pass.
// Radix of stage s, and the product of the earlier radices, of the schedule S (Radix<N>-like)
template <typename S, bool REV> __host__ __device__ constexpr int srad(int s) {
  return REV ? S::r[S::ns - 1 - s] : S::r[s];
}
template <typename S, bool REV> __host__ __device__ constexpr int spbefore(int s) {
  int p = 1;
  for (int i = 0; i < s; ++i) p *= srad<S, REV>(i);
  return p;
}
template <int N, bool REV> __host__ __device__ constexpr int rad(int s) { return srad<Radix<N>, REV>(s); }
template <int N, bool REV> __host__ __device__ constexpr int pbefore(int s) { return spbefore<Radix<N>, REV>(s); }
template <int N, int B, int NT, int R> struct StageShape {
  static constexpr int NB = N / R * B;
  static constexpr int BPT = (NB + NT - 1) / NT;
};
template <int N, int B, int NT, int R> __device__ __forceinline__ bool st_valid(int m) {
  constexpr int NB = StageShape<N, B, NT, R>::NB;
  return NB % NT == 0 || (int)threadIdx.x + m * NT < NB;
}

template <typename T, int N, int B, int NT, int R>
__device__ __forceinline__ void st_read(const Cx<T>* s, Cx<T> (&a)[StageShape<N, B, NT, R>::BPT][R]) {
#pragma unroll
  for (int m = 0; m < StageShape<N, B, NT, R>::BPT; ++m) {
    if (st_valid<N, B, NT, R>(m)) {
      const int q = threadIdx.x + m * NT, b = q % B, t = q / B;
#pragma unroll
      for (int r = 0; r < R; ++r) a[m][r] = s[sw<B>(t + r * (N / R), b)];
    }
  }
}

template <typename T, int N, int B, int NT, int R, bool INV>
__device__ __forceinline__ void st_compute(Cx<T> (&a)[StageShape<N, B, NT, R>::BPT][R], const Cx<T>* __restrict__ tw,
                                           int twstride, int p) {
#pragma unroll
  for (int m = 0; m < StageShape<N, B, NT, R>::BPT; ++m) {
    if (st_valid<N, B, NT, R>(m)) {
      const int q = threadIdx.x + m * NT, t = q / B, k = t % p;
      if (p > 1) {
        const int step = (N / (p * R)) * twstride;
#pragma unroll
        for (int r = 1; r < R; ++r) {
          Cx<T> w = tw[r * k * step];
          if (INV) w.y = -w.y;
          a[m][r] = cmul(a[m][r], w);
        }
      }
      dftR<T, INV, R>(a[m]);
    }
  }
}

template <typename T, int N, int B, int NT, int R>
__device__ __forceinline__ void st_write(Cx<T>* s, const Cx<T> (&a)[StageShape<N, B, NT, R>::BPT][R], int p) {
#pragma unroll
  for (int m = 0; m < StageShape<N, B, NT, R>::BPT; ++m) {
    if (st_valid<N, B, NT, R>(m)) {
      const int q = threadIdx.x + m * NT, b = q % B, t = q / B, k = t % p;
      const int j = (t / p) * p * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) s[sw<B>(j + r * p, b)] = a[m][r];
    }
  }
}

// Full transform in radix order REV: `in` holds the first stage's operands (elements
// t + r N/R0), `out` receives the last stage's results (elements t + r N/R_last).  s is used
// between stages; on entry no thread may still be reading s, and on return threads may still
// be reading it (the caller synchronises before writing s again).
template <typename T, int N, int B, int NT, bool INV, bool REV, typename S = Radix<N>>
__device__ __forceinline__ void fft_regs(
    Cx<T>* s, const Cx<T>* __restrict__ tw, int twstride,
    Cx<T> (&in)[StageShape<N, B, NT, srad<S, REV>(0)>::BPT][srad<S, REV>(0)],
    Cx<T> (&out)[StageShape<N, B, NT, srad<S, REV>(S::ns - 1)>::BPT][srad<S, REV>(S::ns - 1)]) {
  constexpr int NS = S::ns;
  constexpr int R0 = srad<S, REV>(0);
  st_compute<T, N, B, NT, R0, INV>(in, tw, twstride, 1);
  if constexpr (NS == 1) {
#pragma unroll
    for (int m = 0; m < StageShape<N, B, NT, R0>::BPT; ++m)
#pragma unroll
      for (int r = 0; r < R0; ++r) out[m][r] = in[m][r];
  } else {
    st_write<T, N, B, NT, R0>(s, in, 1);
    __syncthreads();
    if constexpr (NS == 3) {
      constexpr int R1 = srad<S, REV>(1);
      Cx<T> a1[StageShape<N, B, NT, R1>::BPT][R1];
      st_read<T, N, B, NT, R1>(s, a1);
      __syncthreads();
      st_compute<T, N, B, NT, R1, INV>(a1, tw, twstride, spbefore<S, REV>(1));
      st_write<T, N, B, NT, R1>(s, a1, spbefore<S, REV>(1));
      __syncthreads();
    }
    constexpr int RL = srad<S, REV>(NS - 1);
    st_read<T, N, B, NT, RL>(s, out);
    st_compute<T, N, B, NT, RL, INV>(out, tw, twstride, spbefore<S, REV>(NS - 1));
  }
}

}  // namespace mhit
