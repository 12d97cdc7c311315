// The 512-point z solve of the FP32 Poisson modes on the tensor cores (sm_100a tcgen05).
//
// Replaces, for nz = 512, the register/shared-memory Stockham z solve (k_fft_cols MODE 2): the
// forward z transform, the spectral divide -1/(k^2 N) with the zero mode cleared, and the
// inverse z transform (multi/main.f90:865, :883-896, :901).  Each 512-point DFT is factored
// 512 = 16 x 32 (Cooley-Tukey "four-step"): z index n = 32 n1 + n2, wavenumber k = k1 + 16 k2,
//   X[k1 + 16 k2] = sum_n2 W512^(n2 k1) W32^(n2 k2) sum_n1 x[32 n1 + n2] W16^(n1 k1),
// so a transform is a 16-point DFT-matrix GEMM, a twiddle multiply and a 32-point DFT-matrix
// GEMM.  The inverse uses conj(DFT(conj(.))) with the mirrored factorisation
// x[n2 + 32 n1] = sum_k1 W16^(-n1 k1) W512^(-n2 k1) sum_k2 X[k1 + 16 k2] W32^(-n2 k2).
//
// A complex GEMM is one real GEMM on interleaved (re, im) operands: the K index is 2 n + (0 re,
// 1 im) and the DFT matrix is the real block matrix [[Re W, -Im W], [Im W, Re W]].  Operands are
// BF16 split in three terms (x = x0 + x1 + x2, each the bf16 rounding of what the earlier terms
// left, 24 significant bits), and the six products x_i W_j with i + j <= 2 accumulate in FP32
// in tensor memory, which keeps FP32 accuracy (the dropped terms are below 2^-24 of the sum).
//
// A CTA owns a tile of 8 kx columns at one y: 512 x 8 complex FP32 values, brought into shared
// memory by two TMA boxes and written back the same way.  Its 128 threads (TMEM lanes 0-127)
// own one GEMM row each: stage 1 and 4 rows (c, n2) (256 rows, two M = 128 MMAs), stage 2 and 3
// rows (c, k1) (128 rows); two CTAs share an SM.  Between the GEMMs each thread reads its row of the accumulator
// (tcgen05.ld), applies the twiddles, the divide or the conjugations, splits the values into
// BF16 terms and writes the next GEMM's A operand (canonical K-major layout, no swizzle).  The
// DFT matrices (B operands) are staged once per CTA.  One elected thread issues the MMAs and
// commits them to an mbarrier.  Every wait is bounded: a wait that runs out sets bit 2 of the
// context's flag word, and the CTA stops, waits (bounded) for its MMAs, frees its tensor memory
// and returns.
#include <cuda.h>
#include <cuda_bf16.h>

#include <cmath>
#include <vector>

#include "common.cuh"
#include "kernels.h"

namespace mhit {

namespace {

constexpr int TC_NT = 128;          // threads per CTA (TMEM lanes 0-127)
constexpr int TC_C = 8;             // kx columns per tile
constexpr int TC_N = 512;           // transform length
constexpr int TC_TMEM_COLS = 64;    // accumulator columns (power of two >= 32)

// Canonical K-major layouts (no swizzle): a core matrix is 8 rows x 16 bytes; LBO is the byte
// distance between core matrices along K (dense: 128), SBO along M/N (all K chunks of a row
// group).  Row orders are chosen so that every shared-memory access of a warp is free of bank
// conflicts: stage 1 and 4 rows (c, n2) are m = 128 (n2 / 16) + 8 (n2 % 16) + c, stage 2 and 3 rows
// (c, k1) are m = 8 k1 + c, i.e. the tile column c runs fastest in both.
constexpr int A_LBO = 128;
constexpr int A1_SBO = 4 * A_LBO;           // K = 32: 4 chunks
constexpr int A2_SBO = 8 * A_LBO;           // K = 64: 8 chunks
constexpr int A_TERM = 32 * A1_SBO;         // 16384 bytes: 256 rows of K = 32 = 128 rows of K = 64
constexpr int B1_TERM = 4 * 512;            // N = 32, K = 32: 4 row groups x 4 chunks x 128 bytes
constexpr int B2_TERM = 8 * 1024;           // N = 64, K = 64
constexpr int B_IMAGE = 3 * (B1_TERM + B2_TERM);
static_assert(16 * A2_SBO <= A_TERM, "A region holds every stage's operand");

// shared memory plan (bytes from a 128-aligned base): 110 KB, two CTAs per SM
constexpr int SM_TILE = 0;                            // 512 x 8 complex float = 32768
constexpr int SM_A = SM_TILE + TC_N * TC_C * 8;       // 3 terms
constexpr int SM_B = SM_A + 3 * A_TERM;               // B1 terms then B2 terms
constexpr int SM_BAR = SM_B + B_IMAGE;                // two mbarriers + the TMEM address
constexpr int SM_TOTAL = SM_BAR + 64;
constexpr size_t SMEM_BYTES = SM_TOTAL + 128;         // slack for the 128-byte alignment

constexpr long long WAIT_LIMIT = 1ll << 26;  // polls of an mbarrier before giving up (seconds)

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  // start address, LBO and SBO in 16-byte units; version 1 (sm_100); no swizzle
  return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

// kind::f16 instruction descriptor: BF16 x BF16 -> F32, both operands K-major
__host__ __device__ constexpr uint32_t idesc_bf16(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (long long it = 0; it < WAIT_LIMIT; ++it) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if (it > 64) __nanosleep(64);
  }
  return false;
}

__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map, int x, int y, int z, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
      ::"r"(dst), "l"(map), "r"(x), "r"(y), "r"(z), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void tma_store_3d(const CUtensorMap* map, uint32_t src, int x, int y, int z) {
  asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%2, %3, %4}], [%1];"
               ::"l"(map), "r"(src), "r"(x), "r"(y), "r"(z)
               : "memory");
}

__device__ __forceinline__ void mma_bf16(uint32_t dtmem, uint64_t ad, uint64_t bd, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
      ::"r"(dtmem), "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// 32 consecutive accumulator columns of this thread's lane
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&r)[32]) {
  uint32_t u[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(u[0]), "=r"(u[1]), "=r"(u[2]), "=r"(u[3]), "=r"(u[4]), "=r"(u[5]), "=r"(u[6]), "=r"(u[7]), "=r"(u[8]),
        "=r"(u[9]), "=r"(u[10]), "=r"(u[11]), "=r"(u[12]), "=r"(u[13]), "=r"(u[14]), "=r"(u[15]), "=r"(u[16]),
        "=r"(u[17]), "=r"(u[18]), "=r"(u[19]), "=r"(u[20]), "=r"(u[21]), "=r"(u[22]), "=r"(u[23]), "=r"(u[24]),
        "=r"(u[25]), "=r"(u[26]), "=r"(u[27]), "=r"(u[28]), "=r"(u[29]), "=r"(u[30]), "=r"(u[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int q = 0; q < 32; ++q) r[q] = __uint_as_float(u[q]);
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// x = t0 + t1 + t2 in BF16 (each the rounding of what the earlier terms left)
__device__ __forceinline__ void split3(float x, __nv_bfloat16& t0, __nv_bfloat16& t1, __nv_bfloat16& t2) {
  t0 = __float2bfloat16_rn(x);
  const float r1 = x - __bfloat162float(t0);
  t1 = __float2bfloat16_rn(r1);
  t2 = __float2bfloat16_rn(r1 - __bfloat162float(t1));
}

__device__ __forceinline__ uint32_t pack2(__nv_bfloat16 a, __nv_bfloat16 b) {
  return (uint32_t)__bfloat16_as_ushort(a) | ((uint32_t)__bfloat16_as_ushort(b) << 16);
}

// byte offset of element (row m, K index k) in an A operand term with row-group stride sbo
__device__ __forceinline__ uint32_t a_off(int m, int k, int sbo) {
  return (uint32_t)((m >> 3) * sbo + (k >> 3) * A_LBO + (m & 7) * 16 + (k & 7) * 2);
}

// writes one complex value (re, im) at K = 2 kc, 2 kc + 1 of row m, in three BF16 terms
__device__ __forceinline__ void put_pair(unsigned char* A, int m, int kc, int sbo, float re, float im) {
  __nv_bfloat16 r0, r1, r2, i0, i1, i2;
  split3(re, r0, r1, r2);
  split3(im, i0, i1, i2);
  const uint32_t o = a_off(m, 2 * kc, sbo);
  *reinterpret_cast<uint32_t*>(A + o) = pack2(r0, i0);
  *reinterpret_cast<uint32_t*>(A + A_TERM + o) = pack2(r1, i1);
  *reinterpret_cast<uint32_t*>(A + 2 * A_TERM + o) = pack2(r2, i2);
}

// writes a whole row of 4 (nchunk 4) or 8 (nchunk 8) chunks from 16 or 32 complex values
template <int NC>
__device__ __forceinline__ void put_row(unsigned char* A, int m, int sbo, const float* v /* 2*4*NC floats */) {
#pragma unroll
  for (int q = 0; q < NC; ++q) {
    uint32_t w[3][4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      __nv_bfloat16 a0, a1, a2, b0, b1, b2;
      split3(v[8 * q + 2 * e], a0, a1, a2);
      split3(v[8 * q + 2 * e + 1], b0, b1, b2);
      w[0][e] = pack2(a0, b0);
      w[1][e] = pack2(a1, b1);
      w[2][e] = pack2(a2, b2);
    }
    const uint32_t o = (uint32_t)((m >> 3) * sbo + q * A_LBO + (m & 7) * 16);
#pragma unroll
    for (int t = 0; t < 3; ++t)
      *reinterpret_cast<uint4*>(A + t * A_TERM + o) = make_uint4(w[t][0], w[t][1], w[t][2], w[t][3]);
  }
}

// the six products x_i W_j (i + j <= 2) of one K-step into one accumulator
__device__ __forceinline__ void mma_products(uint32_t d, uint32_t a_base, uint32_t a_sbo, uint32_t b_base,
                                             uint32_t b_term, uint32_t b_sbo, uint32_t idesc, int kstep,
                                             bool first) {
  const int pi[6] = {0, 0, 1, 0, 1, 2}, pj[6] = {0, 1, 0, 2, 1, 0};
#pragma unroll
  for (int p = 0; p < 6; ++p) {
    const uint64_t ad = sdesc(a_base + pi[p] * A_TERM + kstep * 2 * A_LBO, A_LBO, a_sbo);
    const uint64_t bd = sdesc(b_base + pj[p] * b_term + kstep * 2 * 128, 128, b_sbo);
    mma_bf16(d, ad, bd, idesc, (first && p == 0) ? 0u : 1u);
  }
}

__device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__global__ void __launch_bounds__(TC_NT, 2)
k_zsolve_tc(const __grid_constant__ CUtensorMap tmap, const uint4* __restrict__ bimg,
            const float2* __restrict__ w512, Geo g, const double* __restrict__ k2x,
            const double* __restrict__ k2y, const double* __restrict__ k2z, double ntot, int ntx,
            DevScalars* __restrict__ sc) {
  extern __shared__ unsigned char smraw[];
  unsigned char* sm = reinterpret_cast<unsigned char*>(((uintptr_t)smraw + 127) & ~(uintptr_t)127);
  const int tid = threadIdx.x, warp = tid >> 5;
  float2* tile = reinterpret_cast<float2*>(sm + SM_TILE);
  unsigned char* A = sm + SM_A;
  const uint32_t a_base = smem_u32(A);
  const uint32_t b1_base = smem_u32(sm + SM_B), b2_base = b1_base + 3 * B1_TERM;
  uint64_t* bars = reinterpret_cast<uint64_t*>(sm + SM_BAR);
  const uint32_t tma_bar = smem_u32(&bars[0]), mma_bar = smem_u32(&bars[1]);
  uint32_t* tmem_holder = reinterpret_cast<uint32_t*>(sm + SM_BAR + 16);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_holder)),
                 "r"(TC_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    mbar_init(tma_bar, 1);
    mbar_init(mma_bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // the DFT matrices' B operand image (3 terms of the 16-point, then of the 32-point matrix)
  for (int q = tid; q < B_IMAGE / 16; q += TC_NT) reinterpret_cast<uint4*>(sm + SM_B)[q] = bimg[q];
  fence_async_smem();
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = *tmem_holder;
  const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);  // this warp's TMEM lane quarter

  constexpr uint32_t ID1 = idesc_bf16(128, 32), ID2 = idesc_bf16(128, 64);
  uint32_t tma_phase = 0, mma_phase = 0;
  bool ok = true, mma_pending = false;  // a committed MMA batch not yet waited for
  const int ntiles = ntx * g.ny;
  const int nkx = g.nkx;

  // waits for the committed MMAs; false (all threads agree) when the wait ran out
  auto wait_mma = [&]() {
    bool done = mbar_wait(mma_bar, mma_phase);
    done = __syncthreads_and(done);
    if (done) {
      mma_phase ^= 1;
      mma_pending = false;
    }
    fence_after_sync();
    return done;
  };
  // makes this thread's A writes visible to the tensor core, then thread 0 issues
  auto sync_for_mma = [&]() {
    fence_async_smem();
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
  };

  for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
    const int y = t / ntx, kx0 = (t - y * ntx) * TC_C;
    // ---- load the 512 x 8 tile (two boxes of 256 z rows)
    if (tid == 0) {
      asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");  // the previous tile's store
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tma_bar), "r"(TC_N * TC_C * 8)
                   : "memory");
      tma_load_3d(smem_u32(tile), &tmap, 2 * kx0, y, 0, tma_bar);
      tma_load_3d(smem_u32(tile) + 256 * TC_C * 8, &tmap, 2 * kx0, y, 256, tma_bar);
    }
    {
      bool done = mbar_wait(tma_bar, tma_phase);
      tma_phase ^= 1;
      if (!__syncthreads_and(done)) { ok = false; break; }
    }
    // ---- stage 1 operand: rows (c, n2) = 128 h + tid with c = tid % 8, n2 = 16 h + tid / 8;
    // K = (n1, re/im).  A warp reads 32 consecutive complex values of the tile per n1.
    const int cc = tid & 7, nq = tid >> 3;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int n2 = 16 * h + nq;
      float v[32];
#pragma unroll
      for (int n1 = 0; n1 < 16; ++n1) {
        const float2 z = tile[(32 * n1 + n2) * TC_C + cc];
        v[2 * n1] = z.x;
        v[2 * n1 + 1] = z.y;
      }
      put_row<4>(A, 128 * h + tid, A1_SBO, v);
    }
    sync_for_mma();
    if (tid == 0) {
#pragma unroll
      for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int s = 0; s < 2; ++s)
          mma_products(tmem + 32 * h, a_base + h * 16 * A1_SBO, A1_SBO, b1_base, B1_TERM, 512, ID1, s, s == 0);
      mma_commit(mma_bar);
    }
    mma_pending = true;
    if (!wait_mma()) { ok = false; break; }
    // ---- twiddle W512^(n2 k1), stage 2 operand: rows (c, k1) = 8 k1 + c, K = (n2, re/im)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      float r[32];
      tmem_ld32(lane_addr + 32 * h, r);
      const int n2 = 16 * h + nq;
#pragma unroll
      for (int k1 = 0; k1 < 16; ++k1) {
        const float2 z = cmulf(make_float2(r[2 * k1], r[2 * k1 + 1]), __ldg(&w512[(n2 * k1) & 511]));
        put_pair(A, 8 * k1 + cc, n2, A2_SBO, z.x, z.y);
      }
    }
    fence_before_sync();
    sync_for_mma();
    if (tid == 0) {
#pragma unroll
      for (int s = 0; s < 4; ++s) mma_products(tmem, a_base, A2_SBO, b2_base, B2_TERM, 1024, ID2, s, s == 0);
      mma_commit(mma_bar);
    }
    mma_pending = true;
    if (!wait_mma()) { ok = false; break; }
    // ---- divide (row (c, k1) = tid, columns k2), then the inverse's first operand: conj(X)
    {
      float r[64];
      tmem_ld32(lane_addr, *reinterpret_cast<float(*)[32]>(r));
      tmem_ld32(lane_addr + 32, *reinterpret_cast<float(*)[32]>(r + 32));
      const int c = cc, k1 = nq, kx = kx0 + c;  // row 8 k1 + c
      const bool col = kx < nkx;
      const double kxy = col ? k2x[kx] + k2y[y] : 0.0;
#pragma unroll
      for (int k2 = 0; k2 < 32; ++k2) {
        const int kz = k1 + 16 * k2;
        double re = 0.0, im = 0.0;
        // multi/main.f90:889-895 in FP64 (one reciprocal of k^2 N per element)
        if (col && !(kx == 0 && y == 0 && kz == 0)) {
          const double inv = 1.0 / ((kxy + k2z[kz]) * ntot);
          re = -(double)r[2 * k2] * inv;
          im = -(double)r[2 * k2 + 1] * inv;
        }
        r[2 * k2] = (float)re;
        r[2 * k2 + 1] = -(float)im;  // conjugate: the inverse runs as conj(DFT(conj(.)))
      }
      put_row<8>(A, tid, A2_SBO, r);
    }
    fence_before_sync();
    sync_for_mma();
    if (tid == 0) {
#pragma unroll
      for (int s = 0; s < 4; ++s) mma_products(tmem, a_base, A2_SBO, b2_base, B2_TERM, 1024, ID2, s, s == 0);
      mma_commit(mma_bar);
    }
    mma_pending = true;
    if (!wait_mma()) { ok = false; break; }
    // ---- twiddle W512^(n2 k1) of conj(Z), stage 4 operand: rows (c, n2) as in stage 1,
    // K = (k1, re/im)
    {
      float r[64];
      tmem_ld32(lane_addr, *reinterpret_cast<float(*)[32]>(r));
      tmem_ld32(lane_addr + 32, *reinterpret_cast<float(*)[32]>(r + 32));
      const int k1 = nq;
#pragma unroll
      for (int m2 = 0; m2 < 32; ++m2) {
        const float2 z = cmulf(make_float2(r[2 * m2], r[2 * m2 + 1]), __ldg(&w512[(m2 * k1) & 511]));
        put_pair(A, 128 * (m2 >> 4) + 8 * (m2 & 15) + cc, k1, A1_SBO, z.x, z.y);
      }
    }
    fence_before_sync();
    sync_for_mma();
    if (tid == 0) {
#pragma unroll
      for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int s = 0; s < 2; ++s)
          mma_products(tmem + 32 * h, a_base + h * 16 * A1_SBO, A1_SBO, b1_base, B1_TERM, 512, ID1, s, s == 0);
      mma_commit(mma_bar);
    }
    mma_pending = true;
    if (!wait_mma()) { ok = false; break; }
    // ---- x[32 n1 + n2] = conj(D4), back into the tile, then the TMA store
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      float r[32];
      tmem_ld32(lane_addr + 32 * h, r);
      const int n2 = 16 * h + nq;
#pragma unroll
      for (int n1 = 0; n1 < 16; ++n1) tile[(32 * n1 + n2) * TC_C + cc] = make_float2(r[2 * n1], -r[2 * n1 + 1]);
    }
    fence_async_smem();
    fence_before_sync();
    __syncthreads();
    if (tid == 0) {
      tma_store_3d(&tmap, smem_u32(tile), 2 * kx0, y, 0);
      tma_store_3d(&tmap, smem_u32(tile) + 256 * TC_C * 8, 2 * kx0, y, 256);
      asm volatile("cp.async.bulk.commit_group;" ::: "memory");
    }
  }
  if (tid == 0) {
    asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
    if (!ok) atomicOr(&sc->flag, 4);
  }
  if (mma_pending) {
    // an MMA batch may still be in flight after a wait ran out: wait for it (bounded) before
    // the tensor memory is freed
    mbar_wait(mma_bar, mma_phase);
  }
  fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    fence_after_sync();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_TMEM_COLS) : "memory");
  }
}

// ------------------------------------------------------------------ host side
// B operand image of one DFT matrix of length L (L = 16: rows 2 k + ro, K = 2 n + ri), three
// BF16 terms, canonical K-major layout with LBO = 128 and SBO = 128 * (2L / 8)
void dft_image(int L, unsigned char* out) {
  const int rows = 2 * L, kdim = 2 * L, nchunk = kdim / 8, sbo = 128 * nchunk, term = (rows / 8) * sbo;
  const long double pi = 3.141592653589793238462643383279502884L;
  for (int k = 0; k < L; ++k)
    for (int n = 0; n < L; ++n) {
      const long double ang = 2.0L * pi * (long double)((k * n) % L) / (long double)L;
      const double wr = (double)cosl(ang), wi = (double)(-sinl(ang));  // W_L^(nk) = exp(-2 pi i nk/L)
      for (int ro = 0; ro < 2; ++ro)
        for (int ri = 0; ri < 2; ++ri) {
          // [[Re W, -Im W], [Im W, Re W]]: (ro, ri)
          const double val = ro == 0 ? (ri == 0 ? wr : -wi) : (ri == 0 ? wi : wr);
          const int row = 2 * k + ro, kk = 2 * n + ri;
          const size_t off = (size_t)(row >> 3) * sbo + (size_t)(kk >> 3) * 128 + (row & 7) * 16 + (kk & 7) * 2;
          // three BF16 terms of the FP64 value
          double rem = val;
          for (int t = 0; t < 3; ++t) {
            const __nv_bfloat16 b = __float2bfloat16_rn((float)rem);
            rem -= (double)__bfloat162float(b);
            *reinterpret_cast<__nv_bfloat16*>(out + (size_t)t * term + off) = b;
          }
        }
    }
}

}  // namespace

EncodeTiledFn tensor_map_encoder() {
  static EncodeTiledFn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

struct ZsolveTc {
  CUtensorMap tmap;
  void* bimg = nullptr;
  void* w512 = nullptr;
};

bool zsolve_tc_supported(const Geo& g) { return g.nz == TC_N; }

int zsolve_tc_create(const Geo& g, void* spec, ZsolveTc** out) {
  *out = nullptr;
  if (!zsolve_tc_supported(g)) return set_error(MHIT_ERR_ARG, "the tensor-core z solve needs nz = 512");
  EncodeTiledFn enc = tensor_map_encoder();
  if (!enc) return set_error(MHIT_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
  ZsolveTc* z = new ZsolveTc();
  // the FP32 spectrum as a 3-D float tensor: x = 2 pitch floats, y, z; box 16 floats (8 complex,
  // 64 bytes) x 1 x 256.  The x coordinate of a box is 16 kx0 floats, a multiple of 16 floats.
  const cuuint64_t dims[3] = {(cuuint64_t)2 * g.pitch, (cuuint64_t)g.ny, (cuuint64_t)g.nz};
  const cuuint64_t strides[2] = {(cuuint64_t)g.pitch * 8, (cuuint64_t)g.pitch * 8 * g.ny};
  const cuuint32_t box[3] = {16, 1, 256};
  const cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = enc(&z->tmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, spec, dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    delete z;
    return set_error(MHIT_ERR_CUDA, "cuTensorMapEncodeTiled failed for the spectrum");
  }
  std::vector<unsigned char> img(B_IMAGE, 0);
  dft_image(16, img.data());
  dft_image(32, img.data() + 3 * B1_TERM);
  std::vector<float> w(2 * TC_N);
  const long double pi = 3.141592653589793238462643383279502884L;
  for (int m = 0; m < TC_N; ++m) {
    const long double ang = 2.0L * pi * (long double)m / (long double)TC_N;
    w[2 * m] = (float)(double)cosl(ang);
    w[2 * m + 1] = (float)(double)(-sinl(ang));
  }
  cudaError_t e = cudaMalloc(&z->bimg, B_IMAGE);
  if (e == cudaSuccess) e = cudaMemcpy(z->bimg, img.data(), B_IMAGE, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMalloc(&z->w512, w.size() * sizeof(float));
  if (e == cudaSuccess) e = cudaMemcpy(z->w512, w.data(), w.size() * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_zsolve_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_BYTES);
  if (e != cudaSuccess) {
    zsolve_tc_destroy(z);
    return set_cuda_error(e, "tensor-core z solve setup", __FILE__, __LINE__);
  }
  *out = z;
  return MHIT_OK;
}

void zsolve_tc_destroy(ZsolveTc* z) {
  if (!z) return;
  cudaFree(z->bimg);
  cudaFree(z->w512);
  delete z;
}

cudaError_t launch_zsolve_tc(const ZsolveTc* z, const PoissonArgs& a, DevScalars* sc, cudaStream_t st) {
  const Geo& g = a.g;
  const int ntx = (g.nkx + TC_C - 1) / TC_C;
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int ntiles = ntx * g.ny;
  const int grid = ntiles < 2 * nsm ? ntiles : 2 * nsm;  // two CTAs per SM
  k_zsolve_tc<<<grid, TC_NT, SMEM_BYTES, st>>>(z->tmap, static_cast<const uint4*>(z->bimg),
                                               static_cast<const float2*>(z->w512), g, a.k2x, a.k2y, a.k2z, a.ntot,
                                               ntx, sc);
  return cudaGetLastError();
}

}  // namespace mhit
