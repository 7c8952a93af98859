// The Greek coefficients of phase matrices tabulated at n_q Gauss-Legendre cosines, as dense
// contractions (engine.rs:2310-2355, fast.rs:210-271 with the projector of greek.rs:131-335):
// alpha1 = F11 D00, alpha4 = F33 D00, alpha2 +- alpha3 = (F11 +- F33) D22 / D2-2,
// beta1 = F12 D02, beta2 = F34 D02 with D = (2l+1)/2 w_k d_l(mu_k), one GEMM per combination,
// M = the tables (units), N = the orders, K = the cosines.
//
// Two forms:
//   * FP64 on the CUDA cores (greek_fp64_kernel): the parity form;
//   * 3xTF32 on the 5th-generation tensor cores (greek_tc_kernel): each operand split into a
//     TF32 head and a TF32 tail, A_h B_h + A_h B_t + A_t B_h accumulated in FP32 in tensor
//     memory (tcgen05.mma kind::tf32, M 128 x N 256 x K 8), operands staged by TMA
//     (cp.async.bulk.tensor, 128-byte swizzle) in a two-stage mbarrier pipeline.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cstdint>

#include "kernels.h"

namespace sb {

namespace {

constexpr int TC_M = 128, TC_N = 256, TC_KB = 32;  // tile and K block (128 bytes of TF32)
constexpr int A_BYTES = TC_M * TC_KB * 4;          // 16 KiB
constexpr int B_BYTES = TC_N * TC_KB * 4;          // 32 KiB
constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;
constexpr long long kSpinCycles = 4000000000LL;  // about 2 s at the B200's clocks

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(b)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(b)),
               "r"(bytes)
               : "memory");
}
// A bounded wait on phase `parity`: false (and the error flag set) if it did not complete.
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity, unsigned* err) {
  const long long t0 = clock64();
  for (;;) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_u32(b)), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > kSpinCycles) {
      atomicExch(err, 1u);
      return false;
    }
  }
}
__device__ __forceinline__ void tma_load(void* dst, const CUtensorMap* map, int x, int y,
                                         uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, "
      "{%2, %3}], [%4];\n" ::"r"(smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}
// A K-major operand tile in shared memory with the 128-byte swizzle: rows of 128 bytes, groups
// of 8 rows 1024 bytes apart (the canonical layout of the tcgen05 smem descriptor, version 1).
__device__ __forceinline__ uint64_t sdesc(const void* p) {
  uint64_t d = (smem_u32(p) >> 4) & 0x3FFF;
  d |= (uint64_t)1 << 16;            // leading byte offset (unused with the swizzle)
  d |= (uint64_t)(1024 >> 4) << 32;  // stride byte offset: 8 rows
  d |= (uint64_t)1 << 46;            // descriptor version
  d |= (uint64_t)2 << 61;            // 128-byte swizzle
  return d;
}
__device__ __forceinline__ void mma_tf32(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
          smem_u32(bar))
      : "memory");
}

// The TF32 head of x (round to nearest, ties away) and of its remainder.
__device__ __forceinline__ float to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

}  // namespace

// The six combinations of the tables as TF32 heads and tails: A[c][unit][k] for c = F11, F33,
// F11 + F33, F11 - F33, F12, F34, rows n_q_pad long (zero above n_q).
__global__ void greek_split_kernel(const double* __restrict__ phase, int64_t n_units, int n_q,
                                   int n_q_pad, float* __restrict__ hi, float* __restrict__ lo) {
  const int64_t total = 6 * n_units * (int64_t)n_q_pad;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int k = (int)(idx % n_q_pad);
    const int64_t row = idx / n_q_pad;
    const int c = (int)(row / n_units);
    const int64_t u = row % n_units;
    double v = 0.0;
    if (k < n_q) {
      // phase elements: F11 0, F12 1, F22 2, F33 3, F34 4, F44 5.
      const double f11 = phase[(0 * n_units + u) * n_q + k];
      const double f33 = phase[(3 * n_units + u) * n_q + k];
      switch (c) {
        case 0: v = f11; break;
        case 1: v = f33; break;
        case 2: v = f11 + f33; break;
        case 3: v = f11 - f33; break;
        case 4: v = phase[(1 * n_units + u) * n_q + k]; break;
        default: v = phase[(4 * n_units + u) * n_q + k]; break;
      }
    }
    const float h = to_tf32((float)v);
    hi[idx] = h;
    lo[idx] = to_tf32((float)(v - (double)h));
  }
}

// One 128 x 256 output tile of combination blockIdx.z: thread 0 streams K blocks of the four
// operands (A head, A tail, B head, B tail) by TMA into two stages and issues per block
// 3 products x 4 K steps of tcgen05.mma into the tile's FP32 accumulator in tensor memory;
// then every warp reads its 32 lanes (rows) back with tcgen05.ld. Every wait is bounded: on a
// timeout the kernel sets *err, skips the rest and frees its tensor memory.
__global__ void __launch_bounds__(128, 1)
    greek_tc_kernel(const __grid_constant__ CUtensorMap a_hi, const __grid_constant__ CUtensorMap a_lo,
                    const __grid_constant__ CUtensorMap b_hi, const __grid_constant__ CUtensorMap b_lo,
                    TcArgs a) {
  extern __shared__ __align__(1024) unsigned char tc_raw[];
  // 1024-byte alignment of the stages (the swizzle atom).
  unsigned char* base = (unsigned char*)(((uintptr_t)tc_raw + 1023) & ~(uintptr_t)1023);
  uint64_t* full = reinterpret_cast<uint64_t*>(base + 2 * STAGE_BYTES);
  uint64_t* empty = full + 2;
  uint64_t* done = full + 4;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(full + 5);
  const int t = threadIdx.x, w = t >> 5, lane = t & 31;
  const int c = blockIdx.z;
  const int mat = c < 2 ? 0 : c - 1 - (c == 5);  // combination -> projection matrix
  const int m0 = blockIdx.x * TC_M, n0 = blockIdx.y * TC_N;
  if (t == 0) {
    for (int i = 0; i < 2; ++i) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], 1);
    }
    mbar_init(done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (w == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(TC_N));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  const int nkb = (a.n_q_pad + TC_KB - 1) / TC_KB;
  const int arow = c * a.n_units + m0, brow = mat * a.len + n0;
  // Instruction descriptor: F32 accumulator, TF32 A and B, both K-major, N = 256, M = 128.
  const uint32_t idesc =
      (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TC_N >> 3) << 17) | ((uint32_t)(TC_M >> 4) << 24);
  bool ok = true;
  if (t == 0) {
    auto stage = [&](int s) { return base + s * STAGE_BYTES; };
    auto load = [&](int kb) {
      unsigned char* st = stage(kb & 1);
      mbar_expect_tx(&full[kb & 1], STAGE_BYTES);
      const int x = kb * TC_KB;
      tma_load(st, &a_hi, x, arow, &full[kb & 1]);
      tma_load(st + A_BYTES, &a_lo, x, arow, &full[kb & 1]);
      tma_load(st + 2 * A_BYTES, &b_hi, x, brow, &full[kb & 1]);
      tma_load(st + 2 * A_BYTES + B_BYTES, &b_lo, x, brow, &full[kb & 1]);
    };
    load(0);
    for (int kb = 0; kb < nkb && ok; ++kb) {
      if (kb + 1 < nkb) {
        // Stage (kb + 1) & 1 is free once the MMAs of block kb - 1 completed.
        if (kb >= 1) ok = mbar_wait(&empty[(kb + 1) & 1], ((kb - 1) >> 1) & 1, a.err);
        if (!ok) break;
        load(kb + 1);
      }
      ok = mbar_wait(&full[kb & 1], (kb >> 1) & 1, a.err);
      if (!ok) break;
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      unsigned char* st = stage(kb & 1);
      const uint64_t dah = sdesc(st), dal = sdesc(st + A_BYTES);
      const uint64_t dbh = sdesc(st + 2 * A_BYTES), dbl = sdesc(st + 2 * A_BYTES + B_BYTES);
#pragma unroll
      for (int k = 0; k < TC_KB / 8; ++k) {
        const uint64_t dk = (uint64_t)(k * 32 >> 4);  // 8 TF32 = 32 bytes along K
        const uint32_t acc = (kb > 0 || k > 0) ? 1u : 0u;
        mma_tf32(tmem, dah + dk, dbh + dk, idesc, acc);
        mma_tf32(tmem, dah + dk, dbl + dk, idesc, 1u);
        mma_tf32(tmem, dal + dk, dbh + dk, idesc, 1u);
      }
      mma_commit(&empty[kb & 1]);
    }
    mma_commit(done);
  }
  __syncthreads();
  ok = mbar_wait(done, 0, a.err);
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  // tcgen05.ld is warp-collective: the whole warp reads, or none of it.
  ok = __all_sync(0xffffffffu, ok && *(volatile unsigned*)a.err == 0);
  if (ok) {
    const int64_t row = m0 + 32 * w + lane;
    for (int c0 = 0; c0 < TC_N; c0 += 8) {
      uint32_t r[8];
      const uint32_t taddr = tmem + ((uint32_t)(32 * w) << 16) + (uint32_t)c0;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
            "=r"(r[7])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
      if (row < a.n_units) {
        float* out = a.out + ((int64_t)c * a.n_units + row) * a.len;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int l = n0 + c0 + j;
          if (l < a.len) out[l] = __uint_as_float(r[j]);
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (w == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TC_N));
}

// The coefficients from the six FP32 products: alpha1, alpha2 = (P + M) / 2, alpha3 =
// (P - M) / 2, alpha4, beta1, beta2, in FP64 ([6][n_units][len]).
__global__ void greek_assemble_kernel(const float* __restrict__ prod, int64_t n_units, int len,
                                      double* __restrict__ greek) {
  const int64_t total = n_units * (int64_t)len;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const double c0 = prod[idx], c1 = prod[total + idx], p = prod[2 * total + idx];
    const double m = prod[3 * total + idx], c4 = prod[4 * total + idx], c5 = prod[5 * total + idx];
    greek[idx] = c0;
    greek[total + idx] = (p + m) * 0.5;
    greek[2 * total + idx] = (p - m) * 0.5;
    greek[3 * total + idx] = c1;
    greek[4 * total + idx] = c4;
    greek[5 * total + idx] = c5;
  }
}

// The FP64 form: a tile of 32 tables x 32 orders per block of 256 threads; each thread owns
// 4 (table, order) pairs and all six combinations; K in steps of 16 cosines through shared
// memory. Sums in cosine order.
__global__ void __launch_bounds__(256) greek_fp64_kernel(const double* __restrict__ phase,
                                                        int64_t n_units, int n_q, int len,
                                                        const double* __restrict__ d,
                                                        double* __restrict__ greek) {
  __shared__ double fs[4][32][17];
  __shared__ double ds[4][16][33];
  const int t = threadIdx.x;
  const int64_t u0 = (int64_t)blockIdx.x * 32;
  const int l0 = blockIdx.y * 32;
  const int tl = t & 31, tu = t >> 5;  // order lane, unit group of 4
  double acc[4][6];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int e = 0; e < 6; ++e) acc[i][e] = 0.0;
  const int el[4] = {0, 1, 3, 4};  // F11, F12, F33, F34
  for (int k0 = 0; k0 < n_q; k0 += 16) {
    for (int idx = t; idx < 4 * 32 * 16; idx += 256) {
      const int kk = idx & 15, r = (idx >> 4) & 31, e = idx >> 9;
      const int64_t u = u0 + r;
      fs[e][r][kk] = (u < n_units && k0 + kk < n_q)
                         ? phase[((int64_t)el[e] * n_units + u) * n_q + k0 + kk]
                         : 0.0;
    }
    for (int idx = t; idx < 4 * 16 * 32; idx += 256) {
      const int r = idx & 31, kk = (idx >> 5) & 15, e = idx >> 9;
      const int l = l0 + r;
      ds[e][kk][r] = (l < len && k0 + kk < n_q) ? d[((int64_t)e * n_q + k0 + kk) * len + l] : 0.0;
    }
    __syncthreads();
    for (int kk = 0; kk < 16; ++kk) {
      const double d00 = ds[0][kk][tl], d22 = ds[1][kk][tl], d2m2 = ds[2][kk][tl],
                   d02 = ds[3][kk][tl];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int r = tu * 4 + i;
        const double f11 = fs[0][r][kk], f12 = fs[1][r][kk], f33 = fs[2][r][kk],
                     f34 = fs[3][r][kk];
        acc[i][0] = fma(f11, d00, acc[i][0]);
        acc[i][1] = fma(f33, d00, acc[i][1]);
        acc[i][2] = fma(f11 + f33, d22, acc[i][2]);
        acc[i][3] = fma(f11 - f33, d2m2, acc[i][3]);
        acc[i][4] = fma(f12, d02, acc[i][4]);
        acc[i][5] = fma(f34, d02, acc[i][5]);
      }
    }
    __syncthreads();
  }
  const int l = l0 + tl;
  if (l >= len) return;
  const int64_t total = n_units * (int64_t)len;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int64_t u = u0 + tu * 4 + i;
    if (u >= n_units) continue;
    const int64_t o = u * len + l;
    greek[o] = acc[i][0];
    greek[total + o] = (acc[i][2] + acc[i][3]) * 0.5;
    greek[2 * total + o] = (acc[i][2] - acc[i][3]) * 0.5;
    greek[3 * total + o] = acc[i][1];
    greek[4 * total + o] = acc[i][4];
    greek[5 * total + o] = acc[i][5];
  }
}

// B operands: the four matrices transposed ([4][len][n_q_pad], K-major) as TF32 heads and
// tails, from D [4][n_q][len].
__global__ void greek_split_d_kernel(const double* __restrict__ d, int n_q, int n_q_pad, int len,
                                     float* __restrict__ hi, float* __restrict__ lo) {
  const int64_t total = 4 * (int64_t)len * n_q_pad;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int k = (int)(idx % n_q_pad);
    const int64_t r = idx / n_q_pad;
    const int l = (int)(r % len), m = (int)(r / len);
    const double v = k < n_q ? d[((int64_t)m * n_q + k) * len + l] : 0.0;
    const float h = to_tf32((float)v);
    hi[idx] = h;
    lo[idx] = to_tf32((float)(v - (double)h));
  }
}

size_t greek_tc_smem() { return 2 * STAGE_BYTES + 1024 + 64; }

void launch_greek_split(const double* phase, int64_t n_units, int n_q, int n_q_pad, float* hi,
                        float* lo, cudaStream_t s) {
  const int64_t total = 6 * n_units * (int64_t)n_q_pad;
  const int grid = (int)std::min<int64_t>((total + 255) / 256, 148 * 32);
  if (grid > 0) greek_split_kernel<<<grid, 256, 0, s>>>(phase, n_units, n_q, n_q_pad, hi, lo);
}

void launch_greek_split_d(const double* d, int n_q, int n_q_pad, int len, float* hi, float* lo,
                          cudaStream_t s) {
  const int64_t total = 4 * (int64_t)len * n_q_pad;
  const int grid = (int)std::min<int64_t>((total + 255) / 256, 148 * 32);
  if (grid > 0) greek_split_d_kernel<<<grid, 256, 0, s>>>(d, n_q, n_q_pad, len, hi, lo);
}

cudaError_t launch_greek_tc(const CUtensorMap* maps, const TcArgs& a, cudaStream_t s) {
  static bool configured[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 64 && !configured[dev]) {
    cudaError_t e = cudaFuncSetAttribute(greek_tc_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)greek_tc_smem());
    if (e != cudaSuccess) return e;
    configured[dev] = true;
  }
  dim3 grid((unsigned)((a.n_units + TC_M - 1) / TC_M), (unsigned)((a.len + TC_N - 1) / TC_N), 6);
  greek_tc_kernel<<<grid, 128, greek_tc_smem(), s>>>(maps[0], maps[1], maps[2], maps[3], a);
  return cudaGetLastError();
}

void launch_greek_assemble(const float* prod, int64_t n_units, int len, double* greek,
                           cudaStream_t s) {
  const int64_t total = n_units * (int64_t)len;
  const int grid = (int)std::min<int64_t>((total + 255) / 256, 148 * 32);
  if (grid > 0) greek_assemble_kernel<<<grid, 256, 0, s>>>(prod, n_units, len, greek);
}

void launch_greek_fp64(const double* phase, int64_t n_units, int n_q, int len, const double* d,
                       double* greek, cudaStream_t s) {
  dim3 grid((unsigned)((n_units + 31) / 32), (unsigned)((len + 31) / 32));
  if (n_units > 0) greek_fp64_kernel<<<grid, 256, 0, s>>>(phase, n_units, n_q, len, d, greek);
}

}  // namespace sb
