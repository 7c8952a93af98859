// The mixed form of K-b and K-c (fixed grid, values): the angle GEMMs of the chunks with many
// terms as exact integer products on the 5th-generation tensor cores, the elements and their
// weighted sums over the chunk in FP64, into the same per-unit accumulators as unit_kernel.
//
// Per chunk the GEMMs C_E = G_E X and C_O = G_O X (scatrs/src/ensemble/fast.rs:141-145) run on
// digits: every table row and every coefficient column is a fixed-point integer of 40 bits
// (its own power-of-two scale) split into five balanced signed bytes (kernels.h).
// tcgen05.mma kind::i8 (M 128 x N 64 x K 32, operands in shared memory, INT32 accumulators in
// tensor memory) multiplies the digit pairs (i, j) with i + j < 5, each into the accumulator of
// its level i + j, where the sums are exact; the epilogue recombines the levels exactly in 64-bit
// integers, rounds once to FP64 and applies the row and column scales. Each product term keeps about 38 bits of the largest
// |G| |X| of its row and column, and the terms the truncation drops are centred on zero.
//
// A CTA (one per SM, persistent) takes work items (a unit and a share of its row tiles, the
// items of unit_kernel) in a static order. Its jobs are (chunk, M tile, 16-node half); an M tile
// is 64 angle pairs: 64 rows of G_E, then the same pairs' 64 rows of G_O. Warp 0 streams each
// job's K blocks (64 orders: the table's 5 digit slices of 128 rows and the chunk half's 5 slices
// of 64 columns, 60 KiB laid out in the 64-byte swizzle by the digit builders) with bulk copies
// into three stages; warp 1 issues the 15 products of every 32-order K step; warps 2-9 (two
// warpgroups, each half of the job's columns) read the level accumulators of their 32 lanes
// back, free the tensor memory for the next job's MMAs, and form the phase-matrix elements at
// +mu (E rows' threads) and -mu (O rows' threads), the pair's E and O rows being neighbouring
// lanes (an M tile's rows 2p, 2p + 1). Every output sum has one owner thread and runs over the
// chunks in order. Every wait is bounded: on a timeout the
// kernel sets *err, every role stops, and the tensor memory is freed.
#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.h"

namespace sb {

namespace {

constexpr double kPi = 3.14159265358979323846264338327950288;
constexpr int kThreads = 320;  // warp 0 copies, warp 1 MMAs, warps 2-9 the epilogue
constexpr int kStages = 3;
constexpr int kASlice = 128 * kI8KB;                                // 8 KiB
constexpr int kBSlice = 64 * kI8KB;                                 // 4 KiB
constexpr int kStageBytes = kI8Levels * (kASlice + kBSlice);        // 60 KiB
constexpr uint32_t kTmemCols = 512;
constexpr long long kSpinCycles = 4000000000LL;  // about 2 s at the B200's clocks

struct I8Smem {
  alignas(16) double side[2][kI8Side];  // two chunks' side records (column scales, node factors)
  double red[2][128][4];  // warpgroup 1's sums per row, handed to warpgroup 0
  unsigned long long full[kStages], empty[kStages], side_full[2], side_empty[2], tmem_full,
      tmem_empty, drained;
  uint32_t tmem_base;
  int abort;
  int stop;  // the epilogue warps' common decision to stop
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long* b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(b)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(b)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned long long* b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(b)) : "memory");
}
// One arrival for the calling warp, after all its lanes got here.
__device__ __forceinline__ void warp_arrive(unsigned long long* b) {
  __syncwarp();
  if ((threadIdx.x & 31) == 0) mbar_arrive(b);
}
// A bounded wait on phase `parity`: false if it gave up (then *err and sm.abort are set) or if
// another role gave up first.
__device__ __forceinline__ bool mbar_wait(unsigned long long* b, uint32_t parity, I8Smem& sm,
                                          unsigned* err) {
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
    if (*(volatile int*)&sm.abort) return false;
    if (clock64() - t0 > kSpinCycles) {
      atomicExch(err, 1u);
      *(volatile int*)&sm.abort = 1;
      return false;
    }
  }
}
// A bounded wait that ignores the abort flag: the drains of copies and MMAs in flight.
__device__ __forceinline__ void mbar_wait_drain(unsigned long long* b, uint32_t parity,
                                                unsigned* err) {
  const long long t0 = clock64();
  for (;;) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_u32(b)), "r"(parity)
        : "memory");
    if (done) return;
    if (clock64() - t0 > kSpinCycles) {
      atomicExch(err, 1u);
      return;
    }
  }
}
// Bulk copy of `bytes` (a multiple of 16) from global to shared memory, completing on `bar`.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes,
                                          unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
// A K-major operand in shared memory with the 64-byte swizzle: rows of 64 bytes, groups of 8
// rows 512 bytes apart (the canonical layout of the tcgen05 shared-memory descriptor).
__device__ __forceinline__ uint64_t sdesc64(uint32_t addr) {
  uint64_t d = (addr >> 4) & 0x3FFF;
  d |= (uint64_t)1 << 16;           // leading byte offset (unused with the swizzle)
  d |= (uint64_t)(512 >> 4) << 32;  // stride byte offset: 8 rows
  d |= (uint64_t)1 << 46;           // descriptor version
  d |= (uint64_t)4 << 61;           // 64-byte swizzle
  return d;
}
__device__ __forceinline__ void mma_i8(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                       uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}
__device__ __forceinline__ void mma_commit(unsigned long long* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
          smem_u32(bar))
      : "memory");
}
// Instruction descriptor: INT32 accumulator, A and B signed 8-bit, both K-major, N = 64,
// M = 128.
__device__ __forceinline__ uint32_t idesc_i8() {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(64 >> 3) << 17) |
         ((uint32_t)(128 >> 4) << 24);
}
// An INT32 accumulator value as a double, exactly: 2^52 + 2^31 + v read from its bits, less
// 2^52 + 2^31.
__device__ __forceinline__ double i32_to_f64(uint32_t bits) {
  return __hiloint2double(0x43300000, (int)(bits ^ 0x80000000u)) - 4503601774854144.0;
}
// F = d0 2^32 + d1 2^24 + d2 2^16 + d3 2^8 + d4 with every digit in [-128, 127] (each low digit
// the sign-extended low byte of what is left, so that the digits, and the products the five
// levels drop, are centred on zero); |F| < 127.5 2^32 keeps d0 in [-127, 127].
__device__ __forceinline__ void balanced_digits(long long f, int d[kI8Levels]) {
#pragma unroll
  for (int s = kI8Levels - 1; s > 0; --s) {
    d[s] = (int)(signed char)(f & 0xff);
    f = (f - d[s]) >> 8;
  }
  d[0] = (int)f;
}
__device__ __forceinline__ void epi_sync() { asm volatile("bar.sync 1, 256;\n" ::: "memory"); }

__device__ __forceinline__ void elements4(double s1r, double s1i, double s2r, double s2i,
                                          double e[4]) {
  // (|S1|^2+|S2|^2)/2, (|S2|^2-|S1|^2)/2, Re(S2 S1*), Im(S2 S1*) (scatrs/src/mie/phase.rs:54-59)
  double n1 = s1r * s1r + s1i * s1i, n2 = s2r * s2r + s2i * s2i;
  e[0] = 0.5 * (n1 + n2);
  e[1] = 0.5 * (n2 - n1);
  e[2] = s2r * s1r + s2i * s1i;
  e[3] = s2i * s1r - s2r * s1i;
}

// 16 consecutive columns of the warp's 32 lanes of tensor memory (one 32-bit value each).
__device__ __forceinline__ void tmem_ld16(uint32_t (&q)[16], uint32_t addr) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15}, [%16];\n"
      : "=r"(q[0]), "=r"(q[1]), "=r"(q[2]), "=r"(q[3]), "=r"(q[4]), "=r"(q[5]), "=r"(q[6]),
        "=r"(q[7]), "=r"(q[8]), "=r"(q[9]), "=r"(q[10]), "=r"(q[11]), "=r"(q[12]), "=r"(q[13]),
        "=r"(q[14]), "=r"(q[15])
      : "r"(addr));
}
// The level sums of 16 columns as values. With 5 levels: w = sum_s q[s] 2^(32 - 8 s) exactly
// in 64-bit integers (|q[s]| < 2^28.4, so |w| < 2^61), then w as a double, rounded once (the
// caller scales by 2^-32). With 6: sum_s q[s] 2^(-8 s) in FP64, rounding once per level.
template <int LEV>
__device__ __forceinline__ void recombine(const uint32_t (&q)[LEV][16], double* v) {
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    if constexpr (LEV == 5) {
      long long w = (long long)(int)q[0][k] * 4294967296LL;
      w += (long long)(int)q[1][k] * 16777216LL;
      w += (long long)(int)q[2][k] * 65536LL;
      w += (long long)(int)q[3][k] * 256LL;
      w += (long long)(int)q[4][k];
      const double hi = i32_to_f64((uint32_t)(w >> 32));
      const double lo = __hiloint2double(0x43300000, (int)(uint32_t)w) - 4503599627370496.0;
      v[k] = fma(hi, 4294967296.0, lo);
    } else {
      double acc = i32_to_f64(q[5][k]) * 0x1p-40;
      acc = fma(i32_to_f64(q[4][k]), 0x1p-32, acc);
      acc = fma(i32_to_f64(q[3][k]), 0x1p-24, acc);
      acc = fma(i32_to_f64(q[2][k]), 0x1p-16, acc);
      acc = fma(i32_to_f64(q[1][k]), 0x1p-8, acc);
      v[k] = i32_to_f64(q[0][k]) + acc;
    }
  }
}

__device__ __forceinline__ int band_of(int n) {
  int u = 1, idx = 0;
  while (u < n) {
    u = (int)ceil((double)u * 1.25);
    ++idx;
  }
  return idx;
}

// One job: chunk ci (nc terms, band b) of item unit ul, M tile `tile` (user tiles first), half.
struct Job {
  int ul;
  int64_t ci;
  int c;  // chunk within the unit
  int nc, b, tile, half;
};

// Calls f(job) for every job of this CTA, in the order every role sees them.
template <class F>
__device__ __forceinline__ void for_each_job(const UnitI8Args& a, F&& f) {
  const int t_user = (a.h_u + kI8Pairs - 1) / kI8Pairs;
  for (int item = blockIdx.x; item < a.n_items; item += gridDim.x) {
    const WorkItem it = a.items[item];
    for (int c = 0; c < a.cpu; ++c) {
      const int64_t ci = (int64_t)it.unit * a.cpu + c;
      if (a.chunk_xoff[ci] < 0) continue;
      const int nc = a.chunk_n[ci];
      const int b = a.greek_order >= 0 ? band_of(nc) : -1;
      const int t_band = b >= 0 ? (a.bands[b].h + kI8Pairs - 1) / kI8Pairs : 0;
      for (int tile = it.group; tile < t_user + t_band; tile += it.n_groups)
        for (int half = 0; half < 2; ++half)
          if (!f(Job{it.unit, ci, c, nc, b, tile, half})) return;
    }
  }
}

// The table of a job: its digits (tile's K block 0) and its rows' scales.
__device__ __forceinline__ const I8Table& job_table(const UnitI8Args& a, const Job& j,
                                                    int& tile_local) {
  const int t_user = (a.h_u + kI8Pairs - 1) / kI8Pairs;
  if (j.tile < t_user) {
    tile_local = j.tile;
    int v = 0;
    while ((kI8KB << v) < j.nc) ++v;  // the version covering the chunk's orders
    return a.user_tabs[v < a.n_user_tabs ? v : a.n_user_tabs - 1];
  }
  tile_local = j.tile - t_user;
  return a.band_tabs[j.b];
}

}  // namespace

template <int LEV>
__global__ void __launch_bounds__(kThreads, 1) unit_i8_kernel(UnitI8Args a) {
  extern __shared__ __align__(1024) unsigned char i8_raw[];
  unsigned char* stages =
      (unsigned char*)(((uintptr_t)i8_raw + 1023) & ~(uintptr_t)1023);  // swizzle atoms aligned
  I8Smem& sm = *reinterpret_cast<I8Smem*>(stages + kStages * kStageBytes);
  const int t = threadIdx.x, w = t >> 5, lane = t & 31;
  if (t == 0) {
    for (int i = 0; i < kStages; ++i) {
      mbar_init(&sm.full[i], 1);
      mbar_init(&sm.empty[i], 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(&sm.side_full[i], 1);
      mbar_init(&sm.side_empty[i], 8);  // one arrival per epilogue warp
    }
    mbar_init(&sm.tmem_full, 1);
    mbar_init(&sm.tmem_empty, 8);
    mbar_init(&sm.drained, 1);
    sm.abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (w == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(&sm.tmem_base)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = sm.tmem_base;

  if (w == 0) {
    // Copies: every chunk's side record into one of two slots, every job's K blocks into the
    // stages.
    if (lane == 0) {
      int it = 0, q = -1;
      int64_t cur = -1;
      for_each_job(a, [&](const Job& j) {
        if (j.ci != cur) {
          cur = j.ci;
          ++q;
          const int sl = q & 1;
          if (q >= 2 && !mbar_wait(&sm.side_empty[sl], ((q >> 1) - 1) & 1, sm, a.err))
            return false;
          mbar_expect_tx(&sm.side_full[sl], kI8Side * 8);
          bulk_load(sm.side[sl], a.xside + (int64_t)a.chunk_xidx[j.ci] * kI8Side, kI8Side * 8,
                    &sm.side_full[sl]);
        }
        int tl;
        const I8Table& tab = job_table(a, j, tl);
        const int n_kb = (j.nc + kI8KB - 1) / kI8KB;
        const unsigned char* A = a.tdig + tab.off + (int64_t)tl * tab.n_kb * kI8TileBytes;
        const unsigned char* B = a.xdig + a.chunk_xoff[j.ci] + (int64_t)j.half * n_kb * kI8HalfBytes;
        for (int kb = 0; kb < n_kb; ++kb, ++it) {
          const int st = it % kStages;
          if (it >= kStages && !mbar_wait(&sm.empty[st], ((it / kStages) - 1) & 1, sm, a.err))
            return false;
          unsigned char* dst = stages + st * kStageBytes;
          mbar_expect_tx(&sm.full[st], kStageBytes);
          bulk_load(dst, A + (int64_t)kb * kI8TileBytes, kI8TileBytes, &sm.full[st]);
          bulk_load(dst + kI8TileBytes, B + (int64_t)kb * kI8HalfBytes, kI8HalfBytes,
                    &sm.full[st]);
        }
        return true;
      });
      // The last copies have landed before the CTA can exit (they are the only ones that may
      // still be in flight when a role stopped early).
      for (int i = it > kStages ? it - kStages : 0; i < it; ++i)
        mbar_wait_drain(&sm.full[i % kStages], (i / kStages) & 1, a.err);
      for (int i = q > 1 ? q - 1 : 0; i <= q; ++i)
        mbar_wait_drain(&sm.side_full[i & 1], (i >> 1) & 1, a.err);
    }
  } else if (w == 1) {
    // MMAs: per job, per K block, per 32-order step the 15 digit products into their levels.
    if (lane == 0) {
      int it = 0, job = 0;
      const uint32_t idesc = idesc_i8();
      constexpr int n_lev = LEV;
      for_each_job(a, [&](const Job& j) {
        if (job > 0 && !mbar_wait(&sm.tmem_empty, (job - 1) & 1, sm, a.err)) return false;
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        const int n_kb = (j.nc + kI8KB - 1) / kI8KB;
        for (int kb = 0; kb < n_kb; ++kb, ++it) {
          const int st = it % kStages;
          if (!mbar_wait(&sm.full[st], (it / kStages) & 1, sm, a.err)) return false;
          asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
          const uint32_t sa = smem_u32(stages + st * kStageBytes);
          const uint32_t sb = sa + kI8TileBytes;
#pragma unroll
          for (int ks = 0; ks < kI8KB / 32; ++ks) {
#pragma unroll
            for (int i = 0; i < kI8Levels; ++i) {
              const uint64_t da = sdesc64(sa + i * kASlice + ks * 32);
#pragma unroll
              for (int k = 0; k < kI8Levels; ++k) {
                if (i + k >= n_lev) continue;
                const uint64_t db = sdesc64(sb + k * kBSlice + ks * 32);
                // The first product of each level at the job's first step starts its sum: (0, s)
                // for levels below kI8Levels, (s - 4, 4) for the levels above.
                const bool first = kb == 0 && ks == 0 && i == (i + k < kI8Levels ? 0 : i + k - 4);
                mma_i8(tmem + (uint32_t)((i + k) * 64), da, db, idesc, first ? 0u : 1u);
              }
            }
          }
          mma_commit(&sm.empty[st]);
        }
        mma_commit(&sm.tmem_full);
        ++job;
        return true;
      });
      // Everything issued has completed before the tensor memory is freed.
      mma_commit(&sm.drained);
      mbar_wait_drain(&sm.drained, 0, a.err);
    }
  } else {
    // Epilogue: warps 2-9, two warpgroups; warp w reads lane quarter (w & 3) of the
    // accumulators (row r) and the columns of its warpgroup e: nodes 8 e .. 8 e + 7 of the job's
    // 16-node half. Row r is pair r >> 1's E row (r even) or O row (r odd), so that a pair's two
    // rows are neighbouring lanes.
    const int r = 32 * (w & 3) + lane;
    const int e = (w - 2) >> 2;
    const int side = r & 1;            // 0: E row, elements at +mu; 1: O row, at -mu
    const int p = r >> 1;              // the angle pair within the tile
    const int e_thread = t - 64;       // 0 .. 255
    const int t_user = (a.h_u + kI8Pairs - 1) / kI8Pairs;
    int job = 0, q = -1;
    int64_t cur = -1;
    double out[4] = {0.0, 0.0, 0.0, 0.0};
    for_each_job(a, [&](const Job& j) {
      // The row's scale, read before the waits so that its latency hides behind them.
      int tl;
      const I8Table& tab = job_table(a, j, tl);
      // (times 2^-32 with 5 levels: the recombined values are in units of the lowest level)
      const double rs = a.tscale[tab.scale_off + (int64_t)tl * 128 + r] * (LEV == 5 ? 0x1p-32 : 1.0);
      if (j.ci != cur) {
        // The previous chunk's side record is free; this chunk's has landed.
        if (q >= 0) warp_arrive(&sm.side_empty[q & 1]);
        ++q;
        cur = j.ci;
        mbar_wait(&sm.side_full[q & 1], (q >> 1) & 1, sm, a.err);
      }
      // Every epilogue thread takes the same decision: one reads the abort flag between two
      // barriers that all of them reach.
      mbar_wait(&sm.tmem_full, job & 1, sm, a.err);
      epi_sync();
      if (e_thread == 0) sm.stop = *(volatile int*)&sm.abort;
      epi_sync();
      if (sm.stop) return false;
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      // The kept levels of this row's 32 columns: read back, the tensor memory freed for the
      // next job's MMAs, then recombined in FP64. With 5 levels all 160 sums are read before
      // the release; with 6, the first group is recombined before the second group's are read.
      double v[32];
      const uint32_t lane_base = tmem + ((uint32_t)(32 * (w & 3)) << 16) + (uint32_t)(32 * e);
      constexpr int kHeld = LEV == 5 ? 2 : 1;  // column groups held as sums across the release
      uint32_t sums[kHeld][LEV][16];
      if constexpr (LEV != 5) {
#pragma unroll
        for (int s = 0; s < LEV; ++s) tmem_ld16(sums[0][s], lane_base + (uint32_t)(s * 64));
        asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
        recombine<LEV>(sums[0], v);
      }
#pragma unroll
      for (int g = 2 - kHeld; g < 2; ++g)
#pragma unroll
        for (int s = 0; s < LEV; ++s)
          tmem_ld16(sums[g - (2 - kHeld)][s], lane_base + (uint32_t)(s * 64 + g * 16));
      asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
      warp_arrive(&sm.tmem_empty);
#pragma unroll
      for (int g = 2 - kHeld; g < 2; ++g) recombine<LEV>(sums[g - (2 - kHeld)], v + 16 * g);
      const bool user = j.tile < t_user;
      const double* cs = sm.side[q & 1];
      const double* nf = sm.side[q & 1] + 128;
      const double sg = side ? -1.0 : 1.0;
#pragma unroll
      for (int nd = 0; nd < 8; ++nd) {
        // Columns u.re, u.im, v.re, v.im of node 8 e + nd of the half; the pair's other row from
        // the neighbouring lane. S1 = E_u +- O_v, S2 = E_v +- O_u (fast.rs:151-204).
        double mine[4], other[4], E[4], O[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          mine[k] = v[4 * nd + k] * (rs * cs[j.half * 64 + 32 * e + 4 * nd + k]);
          other[k] = __shfl_xor_sync(0xffffffffu, mine[k], 1);
          E[k] = side ? other[k] : mine[k];
          O[k] = side ? mine[k] : other[k];
        }
        double el[4];
        elements4(E[0] + sg * O[2], E[1] + sg * O[3], E[2] + sg * O[0], E[3] + sg * O[1], el);
        const double f = nf[j.half * 16 + 8 * e + nd];
#pragma unroll
        for (int k = 0; k < 4; ++k) out[k] = fma(f, el[k], out[k]);
      }
      if (j.half == 1) {
        // The job pair's sums into this row's (pair, side) accumulators: warpgroup 1 hands its
        // sums to warpgroup 0 through shared memory (two buffers, one per parity of the pair).
        const int buf = (job >> 1) & 1;
        if (e == 1) {
#pragma unroll
          for (int k = 0; k < 4; ++k) sm.red[buf][r][k] = out[k];
        }
        epi_sync();
        if (e == 0) {
#pragma unroll
          for (int k = 0; k < 4; ++k) out[k] += sm.red[buf][r][k];
          int jo = -1;
          int64_t len;
          double* base;
          if (user) {
            const int row = j.tile * kI8Pairs + p;
            if (row < a.h_u) {
              const int2 mp = a.user_map[row];
              jo = side ? mp.y : mp.x;
            }
            len = a.n_mu;
            base = a.acc + a.unit_acc[j.ul];
          } else {
            const BandDesc B = a.bands[j.b];
            const int row = (j.tile - t_user) * kI8Pairs + p;
            if (row < B.h) {
              const int qn = B.n_q, jn = qn / 2 + row, mirror = qn - 1 - jn;
              if (side == 0 || mirror != jn) jo = side ? mirror : jn;
            }
            len = B.n_q;
            base = a.acc + a.chunk_acc[j.ci];
          }
          // Reductions without a reply: this thread's adds to one sum stay in its program order,
          // and no other thread adds to it while the kernel runs.
          if (jo >= 0)
#pragma unroll
            for (int k = 0; k < 4; ++k) atomicAdd(base + k * len + jo, out[k]);
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) out[k] = 0.0;
      }
      ++job;
      return true;
    });
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (w == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem),
                 "r"(kTmemCols));
}

// The digits of one int8 chunk's coefficient rows: thread c owns column c (node c / 4,
// component c % 4); its scale 2^-e puts the column's largest |X| (recorded by K-a) below
// 127 2^-e (in [63.5, 127) 2^-e), and each value's F = rint(X 2^(e + 32)) is written as its 5
// balanced digits, 16 orders at a time, into the (half, K block, digit) slices in the 64-byte
// swizzle (16-byte chunk q of row r at chunk q ^ ((r >> 1) & 3)).
__global__ void __launch_bounds__(128) x_split_kernel(XSplitArgs a) {
  const int ci = a.list[blockIdx.x];
  const int nc = a.chunk_n[ci];
  const double* X = a.X + a.chunk_row[ci] * 128;
  const int c = threadIdx.x;
  const double m = a.colmax[(int64_t)ci * 128 + c];
  int ex = 0;
  frexp(m, &ex);
  int e = 7 - ex;  // m 2^e in [64, 128)
  if (ldexp(m, e) >= 127.0) --e;
  double* side = a.xside + (int64_t)a.chunk_xidx[ci] * kI8Side;
  side[c] = m > 0.0 ? ldexp(1.0, -e) : 0.0;
  if (c < 32) {
    // The node factor w 4 pi r^2 / x^2 (the phase-matrix normalisation times the area); padding
    // nodes and nodes of zero radius weigh nothing.
    const int64_t unit = a.units[ci / a.cpu];
    const int64_t d = unit / a.n_wl, i = unit % a.n_wl;
    const int jn = (ci % a.cpu) * 32 + c;
    double f = 0.0;
    if (jn < a.n_nodes && a.radius[d * a.n_nodes + jn] > 0.0) {
      const double rad = a.radius[d * a.n_nodes + jn];
      const double x = 2.0 * kPi * rad / a.wl[i];
      f = a.weight[d * a.n_nodes + jn] * (4.0 / (x * x) * (kPi * rad * rad));
    }
    side[128 + c] = f;
  }
  const int half = c >> 6, row = c & 63;
  const int n_kb = (nc + kI8KB - 1) / kI8KB;
  unsigned char* base = a.xdig + a.chunk_xoff[ci];
  for (int kb = 0; kb < n_kb; ++kb) {
    for (int q2 = 0; q2 < kI8KB / 32; ++q2) {
      // 32 orders' values loaded before any is split, so that their loads are in flight together.
      double xv[32];
#pragma unroll
      for (int b = 0; b < 32; ++b) {
        const int k = kb * kI8KB + q2 * 32 + b;
        xv[b] = (k < nc && m > 0.0) ? X[(int64_t)k * 128 + c] : 0.0;
      }
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int q = 2 * q2 + h;
        uint32_t dg[kI8Levels][4];
#pragma unroll
        for (int s = 0; s < kI8Levels; ++s)
#pragma unroll
          for (int u = 0; u < 4; ++u) dg[s][u] = 0;
#pragma unroll
        for (int b = 0; b < 16; ++b) {
          long long f = __double2ll_rn(ldexp(xv[16 * h + b], e + 32));
          const int sh = 8 * (b & 3);
          int d[kI8Levels];
          balanced_digits(f, d);
#pragma unroll
          for (int s = 0; s < kI8Levels; ++s) dg[s][b >> 2] |= (uint32_t)(d[s] & 0xff) << sh;
        }
        const int qs = q ^ ((row >> 1) & 3);
#pragma unroll
        for (int s = 0; s < kI8Levels; ++s) {
          uint4* dst = reinterpret_cast<uint4*>(
              base + ((int64_t)(half * n_kb + kb) * kI8Levels + s) * (64 * kI8KB) + row * kI8KB +
              qs * 16);
          *dst = make_uint4(dg[s][0], dg[s][1], dg[s][2], dg[s][3]);
        }
      }
    }
  }
}

size_t units_i8_smem() { return kStages * kStageBytes + sizeof(I8Smem) + 1024; }

void launch_x_split(const XSplitArgs& a, cudaStream_t s) {
  if (a.n > 0) x_split_kernel<<<a.n, 128, 0, s>>>(a);
}

cudaError_t launch_units_i8(const UnitI8Args& a, int grid, cudaStream_t s) {
  static bool configured[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 64 && !configured[dev]) {
    for (auto f : {unit_i8_kernel<5>, unit_i8_kernel<6>}) {
      cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)units_i8_smem());
      if (e != cudaSuccess) return e;
    }
    configured[dev] = true;
  }
  if (grid > 0) {
    if (a.levels == 6)
      unit_i8_kernel<6><<<grid, kThreads, units_i8_smem(), s>>>(a);
    else
      unit_i8_kernel<5><<<grid, kThreads, units_i8_smem(), s>>>(a);
  }
  return cudaGetLastError();
}

}  // namespace sb
