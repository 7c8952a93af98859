// K-b, K-c and K-d for the fixed-grid ensemble: one persistent CTA works through whole
// (distribution, wavelength) units, each in a fixed order, so the sums are deterministic and
// need no atomics.
//
// Per unit, per chunk of 32 nodes (ascending radius):
//   * K-b: S1, S2 of the chunk's 32 spheres at the table cosines as real FP64 GEMMs,
//     C_E = G_E X and C_O = G_O X (scatrs/src/ensemble/fast.rs:141-145), against the shared
//     pi/tau tables of the requested cosines and of the chunk's projector band;
//   * K-c: the phase-matrix elements at mu and at -mu (fast.rs:151-204), scaled per sphere and
//     weighted by w_j u(r_j) r_j, summed over the chunk into the unit's accumulators;
//   * K-d: when the band changes, the band's averaged tables projected onto the Greek
//     coefficients with (2l+1)/2 w_k d_l(mu_k) (fast.rs:238-253, engine.rs:2310-2355).
// Then the averages and the outputs of engine.rs:2396-2497.
#include "kernels.h"

namespace sb {

namespace {

constexpr double kPi = 3.14159265358979323846264338327950288;
constexpr int KB = 8;     // orders per GEMM stage
constexpr int TR = 32;    // table rows per tile
constexpr int NT = 128;   // threads: 8 row groups of 4 rows x 16 node groups of 2 nodes
// The stage rows' strides in shared memory: 4 doubles past 32 and 128, so that the FP64 MMA's
// operand loads (lane = 4 g + q reads order k4 + q, row or column g) of a half-warp fall in 16
// distinct 8-byte banks.
constexpr int TRP = TR + 4;
constexpr int XP = 128 + 4;

__device__ __forceinline__ void elements4(double s1r, double s1i, double s2r, double s2i,
                                          double e[4]) {
  // (|S1|^2+|S2|^2)/2, (|S2|^2-|S1|^2)/2, Re(S2 S1*), Im(S2 S1*) (scatrs/src/mie/phase.rs:54-59)
  double n1 = s1r * s1r + s1i * s1i, n2 = s2r * s2r + s2i * s2i;
  e[0] = 0.5 * (n1 + n2);
  e[1] = 0.5 * (n2 - n1);
  e[2] = s2r * s1r + s2i * s1i;
  e[3] = s2i * s1r - s2r * s1i;
}

// element_derivatives (scatrs/src/mie/phase.rs:62-73): the elements' derivatives for amplitude
// derivatives (D1, D2).
__device__ __forceinline__ void element_derivs4(double s1r, double s1i, double s2r, double s2i,
                                                double d1r, double d1i, double d2r, double d2i,
                                                double e[4]) {
  const double r1 = s1r * d1r + s1i * d1i;
  const double r2 = s2r * d2r + s2i * d2i;
  e[0] = r1 + r2;
  e[1] = r2 - r1;
  e[2] = (d2r * s1r + d2i * s1i) + (s2r * d1r + s2i * d1i);
  e[3] = (d2i * s1r - d2r * s1i) + (s2i * d1r - s2r * d1i);
}

// The band of a chunk with n terms: the index of bucket(n) in 1, 2, 3, 4, 5, 7, ... (each the
// ceiling of 1.25 times the last; engine.rs:951-957).
__device__ __forceinline__ int band_of(int n) {
  int u = 1, idx = 0;
  while (u < n) {
    u = (int)ceil((double)u * 1.25);
    ++idx;
  }
  return idx;
}

struct Smem {
  double a[2][2][KB][TRP];  // [stage][G_E, G_O][order][row] (rows 32 .. 35 unused)
  double xs[2][KB][XP];    // [stage][order][4 columns x 32 nodes] (128 .. 131 unused)
  double w[32], cu[32], area[32], sc[32];
  double wth[3][32];  // the distribution parameters' weights (derivatives only)
  double wd[32], wthd[3][32];  // adaptive derivatives: the error weights (w_K - w_G) ...
  int nn[32];  // each node's number of terms plus one (an upper bound of K-a's), 0 for padding
  double S[8];
  int slot;
};

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::); }

// One stage: orders k0 .. k0+KB-1 (those below nc) of the 32 table rows and of the chunk's
// coefficient rows, copied asynchronously into stage buffer st. The tables are stored
// transposed (order-major, ldr doubles per order) so that each order's 32 rows are contiguous.
__device__ __forceinline__ void load_stage(Smem& sm, int st, const double* __restrict__ ge,
                                           const double* __restrict__ go, int ldr, int r0,
                                           int k0, int nc, const double* __restrict__ xc) {
  const int t = threadIdx.x;
#pragma unroll
  for (int i = t; i < KB * 16; i += NT) {
    const int kk = i >> 4, c = i & 15;
    if (k0 + kk < nc) {
      const int64_t off = (int64_t)(k0 + kk) * ldr + r0 + 2 * c;
      cp_async16(&sm.a[st][0][kk][2 * c], ge + off);
      cp_async16(&sm.a[st][1][kk][2 * c], go + off);
    }
  }
#pragma unroll
  for (int i = t; i < KB * 64; i += NT) {
    const int kk = i >> 6, c = i & 63;
    if (k0 + kk < nc) cp_async16(&sm.xs[st][kk][2 * c], xc + (int64_t)(k0 + kk) * 128 + 2 * c);
  }
  cp_commit();
}

// As load_stage, with the rows at or above nc zero-filled (cp.async with a zero source size), so
// that whole 4-order steps of the FP64 MMA can run past the chunk's last order.
__device__ __forceinline__ void cp_async16_zfill(void* dst, const void* src, bool valid) {
  unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  const int n = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(n));
}
__device__ __forceinline__ void load_stage_z(Smem& sm, int st, const double* __restrict__ ge,
                                             const double* __restrict__ go, int ldr, int r0,
                                             int k0, int nc, const double* __restrict__ xc) {
  const int t = threadIdx.x;
#pragma unroll
  for (int i = t; i < KB * 16; i += NT) {
    const int kk = i >> 4, c = i & 15;
    const bool valid = k0 + kk < nc;
    const int64_t off = valid ? (int64_t)(k0 + kk) * ldr + r0 + 2 * c : 0;
    cp_async16_zfill(&sm.a[st][0][kk][2 * c], ge + off, valid);
    cp_async16_zfill(&sm.a[st][1][kk][2 * c], go + off, valid);
  }
#pragma unroll
  for (int i = t; i < KB * 64; i += NT) {
    const int kk = i >> 6, c = i & 63;
    const bool valid = k0 + kk < nc;
    cp_async16_zfill(&sm.xs[st][kk][2 * c], xc + (valid ? (int64_t)(k0 + kk) * 128 + 2 * c : 0),
                     valid);
  }
  cp_commit();
}

// D (8x8) += A (8x4, row) B (4x8, col) in FP64 on the tensor cores (PTX mma.sync m8n8k4):
// lane l holds A[l/4][l%4], B[l%4][l/4] and D[l/4][2 (l%4) + {0, 1}].
__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// A row tile's table source: G_E, G_O (order-major, ldr doubles per order) from row r0.
struct TileSrc {
  const double* ge;
  const double* go;
  int ldr, r0;
};

// The tile C_E = G_E X, C_O = G_O X (32 rows x 128 columns) on the FP64 tensor path: warp w
// computes rows 8w .. 8w + 7 of all 128 columns as 16 MMA tiles of 8 columns (2 nodes) each for E
// and O; cE[nt] is D of columns 8 nt ... Every warp does the same work, the MMAs of a group of 4
// tiles (8 nodes) stopping above the group's largest number of terms (K-a writes zero rows up to
// the chunk's), so that no warp, and no SM sub-partition, carries the chunk's largest spheres
// alone.
// The tile's first stage is already in flight in buffer st0; with nx, the next tile's first stage
// (same chunk, same coefficient rows) is issued during this tile's last stage, so that the
// pipeline does not drain between tiles, and st0 returns the buffer it went to.
__device__ __forceinline__ void gemm_tile_mma(Smem& sm, const TileSrc& src, int nc,
                                              const double* __restrict__ xc, double cE[16][2],
                                              double cO[16][2], int& st0, const TileSrc* nx) {
  const double* __restrict__ ge = src.ge;
  const double* __restrict__ go = src.go;
  const int ldr = src.ldr, r0 = src.r0;
  const int t = threadIdx.x, w = t >> 5, lane = t & 31, q = lane & 3, g = lane >> 2;
#pragma unroll
  for (int nt = 0; nt < 16; ++nt) {
    cE[nt][0] = cE[nt][1] = 0.0;
    cO[nt][0] = cO[nt][1] = 0.0;
  }
  int gmax[4] = {0, 0, 0, 0};
#pragma unroll
  for (int i = 0; i < 32; ++i) gmax[i >> 3] = max(gmax[i >> 3], sm.nn[i]);
  int st = st0;
  for (int k0 = 0; k0 < nc; k0 += KB, st ^= 1) {
    cp_wait_all();
    __syncthreads();
    if (k0 + KB < nc)
      load_stage_z(sm, st ^ 1, ge, go, ldr, r0, k0 + KB, nc, xc);
    else if (nx)
      load_stage_z(sm, st ^ 1, nx->ge, nx->go, nx->ldr, nx->r0, 0, nc, xc);
    const int kend = nc - k0 < KB ? nc - k0 : KB;
#pragma unroll
    for (int k4 = 0; k4 < KB; k4 += 4) {
      if (k4 < kend) {
        const int kk = k4 + q;
        const double aE = sm.a[st][0][kk][8 * w + g];
        const double aO = sm.a[st][1][kk][8 * w + g];
#pragma unroll
        for (int gr = 0; gr < 4; ++gr) {
          if (k0 + k4 < gmax[gr]) {
            double b[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = sm.xs[st][kk][32 * gr + 8 * j + g];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              dmma(cE[4 * gr + j][0], cE[4 * gr + j][1], aE, b[j]);
              dmma(cO[4 * gr + j][0], cO[4 * gr + j][1], aO, b[j]);
            }
          }
        }
      }
    }
  }
  // The next tile's first stage went to buffer st; the next tile's second stage reuses this
  // tile's last buffer only after the next tile's first barrier, which every warp reaches after
  // its MMAs here.
  st0 = st;
}

// The elements of an MMA tile, scaled, weighted and summed over the chunk's 32 spheres. Lane
// pairs (q, q ^ 1) hold a node's (u) and (v) columns; after exchanging them the even lane forms
// the elements at +mu and the odd lane those at -mu of its row (8 w + g) for its node of each
// tile (2 nt + q / 2); the 16 nodes add in the thread, then node pairs across lanes q, q ^ 2.
// Thread t ends with v[0], v[1]: row t / 4, side t & 1, elements 2 ((t / 2) & 1) + {0, 1}.
template <bool kUser>
__device__ __forceinline__ void chunk_elements_mma(Smem& sm, const double cE[16][2],
                                                   const double cO[16][2], double v[2]) {
  const int lane = threadIdx.x & 31, q = lane & 3;
  const int side = q & 1;
  const double sg = side ? -1.0 : 1.0;
  double p[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
  for (int nt = 0; nt < 16; ++nt) {
    const int node = 2 * nt + (q >> 1);
    const double wt = sm.w[node], cu = sm.cu[node], ar = sm.area[node], sc = sm.sc[node];
    const double e0 = cE[nt][0], e1 = cE[nt][1];
    const double o0 = cO[nt][0], o1 = cO[nt][1];
    const double pe0 = __shfl_xor_sync(0xffffffffu, e0, 1);
    const double pe1 = __shfl_xor_sync(0xffffffffu, e1, 1);
    const double po0 = __shfl_xor_sync(0xffffffffu, o0, 1);
    const double po1 = __shfl_xor_sync(0xffffffffu, o1, 1);
    // The even lane of a pair holds u (re, im), the odd one v.
    const double eur = side ? pe0 : e0, eui = side ? pe1 : e1;
    const double evr = side ? e0 : pe0, evi = side ? e1 : pe1;
    const double our = side ? po0 : o0, oui = side ? po1 : o1;
    const double ovr = side ? o0 : po0, ovi = side ? o1 : po1;
    double e[4];
    elements4(eur + sg * ovr, eui + sg * ovi, evr + sg * our, evi + sg * oui, e);
#pragma unroll
    for (int k = 0; k < 4; ++k) p[k] += kUser ? wt * ((cu * e[k]) * ar) : wt * (sc * e[k]);
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) p[k] += __shfl_xor_sync(0xffffffffu, p[k], 2);
  const int e2 = 2 * (q >> 1);
  v[0] = e2 ? p[2] : p[0];
  v[1] = e2 ? p[3] : p[1];
}
// accE/accO[r][c] = sum_k G[r0 + 4 rg + r][k] X[k][4 ng + c (+ 64 for c >= 4)] for k < nc.
__device__ __forceinline__ void gemm_tile(Smem& sm, const double* __restrict__ ge,
                                          const double* __restrict__ go, int ldr, int r0, int nc,
                                          const double* __restrict__ xc, double accE[4][8],
                                          double accO[4][8]) {
  const int t = threadIdx.x, rg = t >> 4, ng = t & 15;
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      accE[r][c] = 0.0;
      accO[r][c] = 0.0;
    }
  load_stage(sm, 0, ge, go, ldr, r0, 0, nc, xc);
  int st = 0;
  for (int k0 = 0; k0 < nc; k0 += KB, st ^= 1) {
    cp_wait_all();
    __syncthreads();
    if (k0 + KB < nc) load_stage(sm, st ^ 1, ge, go, ldr, r0, k0 + KB, nc, xc);
    const int kend = nc - k0 < KB ? nc - k0 : KB;
#pragma unroll 8
    for (int kk = 0; kk < KB; ++kk) {
      if (kk < kend) {
        const double2 e01 = *reinterpret_cast<const double2*>(&sm.a[st][0][kk][rg * 4]);
        const double2 e23 = *reinterpret_cast<const double2*>(&sm.a[st][0][kk][rg * 4 + 2]);
        const double2 o01 = *reinterpret_cast<const double2*>(&sm.a[st][1][kk][rg * 4]);
        const double2 o23 = *reinterpret_cast<const double2*>(&sm.a[st][1][kk][rg * 4 + 2]);
        const double2 x0 = *reinterpret_cast<const double2*>(&sm.xs[st][kk][ng * 4]);
        const double2 x1 = *reinterpret_cast<const double2*>(&sm.xs[st][kk][ng * 4 + 2]);
        const double2 y0 = *reinterpret_cast<const double2*>(&sm.xs[st][kk][(ng + 16) * 4]);
        const double2 y1 = *reinterpret_cast<const double2*>(&sm.xs[st][kk][(ng + 16) * 4 + 2]);
        const double ae[4] = {e01.x, e01.y, e23.x, e23.y};
        const double ao[4] = {o01.x, o01.y, o23.x, o23.y};
        const double xv[8] = {x0.x, x0.y, x1.x, x1.y, y0.x, y0.y, y1.x, y1.y};
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
          for (int c = 0; c < 8; ++c) {
            accE[r][c] = fma(ae[r], xv[c], accE[r][c]);
            accO[r][c] = fma(ao[r], xv[c], accO[r][c]);
          }
      }
    }
  }
  __syncthreads();  // the stage buffers are free for the next tile
}

// Sums of p[32] over the 16 threads sharing a row group, scattered: thread ng ends with the
// sums of entries 2 ng and 2 ng + 1 in v. At offset o a lane keeps the lower half of its values
// if (ng & o) == 0.
__device__ __forceinline__ void reduce_scatter16(double p[32], double v[2]) {
  const int ng = threadIdx.x & 15;
#pragma unroll
  for (int lvl = 0, o = 8, h = 16; lvl < 4; ++lvl, o >>= 1, h >>= 1) {
    const bool lower = (ng & o) == 0;
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      if (i < h) {
        const double mine = lower ? p[i] : p[i + h];
        const double other = lower ? p[i + h] : p[i];
        p[i] = mine + __shfl_xor_sync(0xffffffffu, other, o);
      }
    }
  }
  v[0] = p[0];
  v[1] = p[1];
}

// The elements at +mu and -mu of this thread's 4 rows for its 2 spheres, scaled and weighted,
// summed over the chunk's 32 spheres by a reduce-scatter over the 16 threads sharing the rows:
// thread ng ends with v[0], v[1] of side ng >> 3 (0: +mu, 1: -mu), row (ng >> 1) & 3 and
// elements 2 (ng & 1) and 2 (ng & 1) + 1.
template <bool kUser>
__device__ __forceinline__ void chunk_elements(const Smem& sm, const double accE[4][8],
                                               const double accO[4][8], double v[2]) {
  const int ng = threadIdx.x & 15;
  double p[32];
#pragma unroll
  for (int i = 0; i < 32; ++i) p[i] = 0.0;
#pragma unroll
  for (int nd = 0; nd < 2; ++nd) {
    const int node = ng + 16 * nd;
    const double w = sm.w[node], cu = sm.cu[node], ar = sm.area[node], sc = sm.sc[node];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const double eur = accE[r][4 * nd], eui = accE[r][4 * nd + 1];
      const double evr = accE[r][4 * nd + 2], evi = accE[r][4 * nd + 3];
      const double our = accO[r][4 * nd], oui = accO[r][4 * nd + 1];
      const double ovr = accO[r][4 * nd + 2], ovi = accO[r][4 * nd + 3];
      double ep[4], em[4];
      elements4(eur + ovr, eui + ovi, evr + our, evi + oui, ep);
      elements4(eur - ovr, eui - ovi, evr - our, evi - oui, em);
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        // Requested cosines: W (4/x^2 F) pi r^2 (phase.rs:204-219, engine.rs:1075); band
        // tables: W (4/x^2 pi r^2) F (engine.rs:1655-1660).
        if (kUser) {
          p[r * 4 + e] += w * ((cu * ep[e]) * ar);
          p[16 + r * 4 + e] += w * ((cu * em[e]) * ar);
        } else {
          p[r * 4 + e] += w * (sc * ep[e]);
          p[16 + r * 4 + e] += w * (sc * em[e]);
        }
      }
    }
  }
  reduce_scatter16(p, v);
}

// The derivative blocks' elements of this thread's 4 rows for its one sphere (node
// 16 half + ng; accumulator columns 0-3 its (u, v) sums, 4-7 those of (du/dm, dv/dm)), for
// block blk: values (weight w), the distribution's parameters (their weights), Re m and Im m
// (weight w, the element derivatives along dS/dm and i dS/dm; phase.rs:322-335), reduced over
// the 16 spheres as chunk_elements does.
// kDiff: with the error weights (w_K - w_G) ... instead.
template <bool kUser, bool kDiff = false>
__device__ __forceinline__ void chunk_elements_d(const Smem& sm, const double accE[4][8],
                                                 const double accO[4][8], int half, int blk,
                                                 int n_theta, double v[2]) {
  const int ng = threadIdx.x & 15;
  const int node = 16 * half + ng;
  const int kind = blk == 0 ? 0 : (blk <= n_theta ? 0 : blk - n_theta);  // 0 f, 1 Re m, 2 Im m
  const double wt = kDiff ? ((blk >= 1 && blk <= n_theta) ? sm.wthd[blk - 1][node] : sm.wd[node])
                          : ((blk >= 1 && blk <= n_theta) ? sm.wth[blk - 1][node] : sm.w[node]);
  const double cu = sm.cu[node], ar = sm.area[node], sc = sm.sc[node];
  double p[32];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
#pragma unroll
    for (int sd = 0; sd < 2; ++sd) {
      const double sg = sd == 0 ? 1.0 : -1.0;
      const double s1r = accE[r][0] + sg * accO[r][2], s1i = accE[r][1] + sg * accO[r][3];
      const double s2r = accE[r][2] + sg * accO[r][0], s2i = accE[r][3] + sg * accO[r][1];
      double e[4];
      if (kind == 0) {
        elements4(s1r, s1i, s2r, s2i, e);
      } else {
        double d1r = accE[r][4] + sg * accO[r][6], d1i = accE[r][5] + sg * accO[r][7];
        double d2r = accE[r][6] + sg * accO[r][4], d2i = accE[r][7] + sg * accO[r][5];
        if (kind == 2) {
          const double t1 = d1r, t2 = d2r;
          d1r = -d1i;
          d1i = t1;
          d2r = -d2i;
          d2i = t2;
        }
        element_derivs4(s1r, s1i, s2r, s2i, d1r, d1i, d2r, d2i, e);
      }
#pragma unroll
      for (int k = 0; k < 4; ++k)
        p[sd * 16 + r * 4 + k] = kUser ? wt * ((cu * e[k]) * ar) : wt * (sc * e[k]);
    }
  }
  reduce_scatter16(p, v);
}

}  // namespace

// The error block of an adaptive call: |sum over panel A| + |sum over panel B| of the elements
// weighted by w_K - w_G (sm.wth[0]), the chunk's panels being nodes 0-15 (this thread's node
// ng) and 16-31 (node ng + 16); each panel reduced over its 16 nodes like chunk_elements.
template <bool kUser>
__device__ __forceinline__ void chunk_errors(const Smem& sm, const double accE[4][8],
                                             const double accO[4][8], double v[2]) {
  const int ng = threadIdx.x & 15;
  double out[2] = {0.0, 0.0};
#pragma unroll 1
  for (int nd = 0; nd < 2; ++nd) {
    const int node = ng + 16 * nd;
    const double w = sm.wth[0][node], cu = sm.cu[node], ar = sm.area[node], sc = sm.sc[node];
    double p[32];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      double eu_r = nd ? accE[r][4] : accE[r][0], eu_i = nd ? accE[r][5] : accE[r][1];
      double ev_r = nd ? accE[r][6] : accE[r][2], ev_i = nd ? accE[r][7] : accE[r][3];
      double ou_r = nd ? accO[r][4] : accO[r][0], ou_i = nd ? accO[r][5] : accO[r][1];
      double ov_r = nd ? accO[r][6] : accO[r][2], ov_i = nd ? accO[r][7] : accO[r][3];
      double ep[4], em[4];
      elements4(eu_r + ov_r, eu_i + ov_i, ev_r + ou_r, ev_i + ou_i, ep);
      elements4(eu_r - ov_r, eu_i - ov_i, ev_r - ou_r, ev_i - ou_i, em);
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        p[r * 4 + e] = kUser ? w * ((cu * ep[e]) * ar) : w * (sc * ep[e]);
        p[16 + r * 4 + e] = kUser ? w * ((cu * em[e]) * ar) : w * (sc * em[e]);
      }
    }
    double vv[2];
    reduce_scatter16(p, vv);
    out[0] += fabs(vv[0]);
    out[1] += fabs(vv[1]);
  }
  v[0] = out[0];
  v[1] = out[1];
}

// kMode 0: values; 1: with the derivative blocks; 2: adaptive panels (values and errors);
// 3: adaptive panels with the derivative blocks (each block's sums, then its error sums: every
// 16-node half of a chunk is one panel).
template <int kMode>
__device__ __forceinline__ void unit_body(const UnitArgs& a) {
  constexpr bool kDeriv = kMode == 1 || kMode == 3;
  constexpr bool kAdD = kMode == 3;
  extern __shared__ __align__(16) unsigned char unit_raw[];
  Smem& sm = *reinterpret_cast<Smem*>(unit_raw);
  const int t = threadIdx.x, rg = t >> 4, ng = t & 15;
  // This thread's share of a reduced tile: side (+mu, -mu), row, two elements.
  const int side = ng >> 3, rr = (ng >> 1) & 3, e0 = 2 * (ng & 1);
  const int t_user = (a.h_u + TR - 1) / TR;
  // Blocks of sums: the values, then (with derivatives) each distribution parameter, Re m and
  // Im m; halves: a chunk's coefficient rows are one 32-node tile, or two of 16 nodes with
  // their derivative columns.
  const int n_blk = kDeriv ? 3 + a.n_theta : (kMode == 2 ? 2 : 1);  // blocks of sums computed
  constexpr int kHalves = kDeriv ? 2 : 1;
  for (;;) {
    if (t == 0) sm.slot = atomicAdd(a.work_counter, 1);
    __syncthreads();
    const int slot = sm.slot;
    __syncthreads();
    if (slot >= a.n_items) break;
    const WorkItem it = a.items[slot];
    const int ul = it.unit;
    const int64_t unit = a.units[ul];
    const int64_t d = unit / a.n_wl, i = unit % a.n_wl;
    const double lam = a.wl[i];
    double* acc_user = a.acc + a.unit_acc[ul];
    for (int c = 0; c < a.cpu; ++c) {
      const int64_t ci = (int64_t)ul * a.cpu + c;
      const int nc = a.chunk_n[ci];
      if (nc == 0) continue;
      if (a.i8_above > 0 && nc > a.i8_above && nc <= kI8MaxTerms) continue;  // the int8 path's
      const int b = a.greek_order >= 0 ? band_of(nc) : -1;
      const int t_band = b >= 0 ? (a.bands[b].h + TR - 1) / TR : 0;
      if (it.group >= t_user + t_band) continue;
      if (t < 32) {
        const int j = c * 32 + t;
        double w = 0.0, cu = 0.0, ar = 0.0, sc = 0.0, wd = 0.0;
        int nn = 0;
        double wth[3] = {0.0, 0.0, 0.0}, wthd[3] = {0.0, 0.0, 0.0};
        const int64_t node = (a.per_unit ? unit : d) * a.n_nodes + j;
        if (j < a.n_nodes && a.radius[node] > 0.0) {
          const double r = a.radius[node];
          const double x = 2.0 * kPi * r / lam;
          // ceil(x + 6 x^(1/3) + 3), the truncation, plus one for a contraction's rounding.
          nn = (int)ceil(x + 6.0 * cbrt(x) + 3.0) + 1;
          w = a.weight[node];  // w_j u(r_j) r_j
          cu = 4.0 / (x * x);
          ar = kPi * r * r;
          sc = 4.0 / (x * x) * (kPi * r * r);
          if (kDeriv)
            for (int p = 0; p < a.n_theta; ++p) wth[p] = a.wtheta[node * 3 + p];
          if (kMode == 2) wth[0] = a.wdiff[node];
          if (kAdD) {
            wd = a.wdiff[node];
            for (int p = 0; p < a.n_theta; ++p) wthd[p] = a.wthdiff[node * 3 + p];
          }
        }
        sm.w[t] = w;
        sm.cu[t] = cu;
        sm.area[t] = ar;
        sm.sc[t] = sc;
        sm.nn[t] = nn;
        if (kDeriv || kMode == 2)
          for (int p = 0; p < 3; ++p) sm.wth[p][t] = wth[p];
        if (kAdD) {
          sm.wd[t] = wd;
          for (int p = 0; p < 3; ++p) sm.wthd[p][t] = wthd[p];
        }
      }
      __syncthreads();
      for (int half = 0; half < kHalves; ++half) {
        const double* xc = a.X + (a.chunk_row[ci] + (int64_t)half * nc) * 128;
        double v[2];
        // This thread's output of a reduced tile (kMode 0, the MMA tile, owns row t / 4).
        const int o_row = kMode == 0 ? (t >> 2) : rg * 4 + rr;
        const int o_side = kMode == 0 ? (t & 1) : side;
        const int o_e0 = kMode == 0 ? 2 * ((t >> 1) & 1) : e0;
        // A tile's table rows: the user cosines', then the band's.
        auto source = [&](int tl) {
          const bool u = tl < t_user;
          const BandDesc Bd = u ? BandDesc{} : a.bands[b];
          return TileSrc{u ? a.ge_u : a.band_ge + Bd.g_off, u ? a.go_u : a.band_go + Bd.g_off,
                         u ? a.h_u_pad : Bd.h_pad, (u ? tl : tl - t_user) * TR};
        };
        int st0 = 0;  // the stage buffer of the next MMA tile's first stage (kMode 0)
        if constexpr (kMode == 0) {
          const TileSrc s0 = source(it.group);
          load_stage_z(sm, 0, s0.ge, s0.go, s0.ldr, s0.r0, 0, nc, xc);
        }
        for (int tile = it.group; tile < t_user + t_band; tile += it.n_groups) {
          const bool user = tile < t_user;
          const BandDesc B = user ? BandDesc{} : a.bands[b];
          const int r0 = (user ? tile : tile - t_user) * TR;
          const double* ge = user ? a.ge_u : a.band_ge + B.g_off;
          const double* go = user ? a.go_u : a.band_go + B.g_off;
          const int ldr = user ? a.h_u_pad : B.h_pad;
          // The output index of this thread's sums, or -1.
          const int row = r0 + o_row;
          int j = -1;
          if (user) {
            if (row < a.h_u) {
              const int2 mp = a.user_map[row];
              j = o_side ? mp.y : mp.x;
            }
          } else if (row < B.h) {
            const int q = B.n_q, jn = q / 2 + row, mirror = q - 1 - jn;
            if (o_side == 0 || mirror != jn) j = o_side ? mirror : jn;
          }
          const int64_t len = user ? a.n_mu : B.n_q;
          double* base = user ? acc_user : a.acc + a.chunk_acc[ci];
          if constexpr (kMode == 0) {
            double cE[16][2], cO[16][2];
            const int tn = tile + it.n_groups;
            const TileSrc nx = source(tn < t_user + t_band ? tn : tile);
            gemm_tile_mma(sm, TileSrc{ge, go, ldr, r0}, nc, xc, cE, cO, st0,
                          tn < t_user + t_band ? &nx : nullptr);
            if (user)
              chunk_elements_mma<true>(sm, cE, cO, v);
            else
              chunk_elements_mma<false>(sm, cE, cO, v);
            if (j >= 0) {
              base[o_e0 * len + j] += v[0];
              base[(o_e0 + 1) * len + j] += v[1];
            }
          } else {
            double accE[4][8], accO[4][8];
            gemm_tile(sm, ge, go, ldr, r0, nc, xc, accE, accO);
            for (int blk = 0; blk < n_blk; ++blk) {
              if (user) {
                if (kDeriv)
                  chunk_elements_d<true>(sm, accE, accO, half, blk, a.n_theta, v);
                else if (kMode == 2 && blk == 1)
                  chunk_errors<true>(sm, accE, accO, v);
                else
                  chunk_elements<true>(sm, accE, accO, v);
              } else {
                if (kDeriv)
                  chunk_elements_d<false>(sm, accE, accO, half, blk, a.n_theta, v);
                else if (kMode == 2 && blk == 1)
                  chunk_errors<false>(sm, accE, accO, v);
                else
                  chunk_elements<false>(sm, accE, accO, v);
              }
              if (j >= 0) {
                double* ab = base + (int64_t)blk * 4 * len;
                ab[o_e0 * len + j] += v[0];
                ab[(o_e0 + 1) * len + j] += v[1];
              }
              if constexpr (kAdD) {
                // The panel's |Kronrod - Gauss| into the block's error sums.
                double ve[2];
                if (user)
                  chunk_elements_d<true, true>(sm, accE, accO, half, blk, a.n_theta, ve);
                else
                  chunk_elements_d<false, true>(sm, accE, accO, half, blk, a.n_theta, ve);
                if (j >= 0) {
                  double* ab = base + (int64_t)(n_blk + blk) * 4 * len;
                  ab[o_e0 * len + j] += fabs(ve[0]);
                  ab[(o_e0 + 1) * len + j] += fabs(ve[1]);
                }
              }
            }
          }
        }
      }
      __syncthreads();
    }
  }
}

// K-b and K-c: each work item runs its row tiles of every chunk of its unit and adds the
// reduced tiles into the unit's accumulators. Every output sum is owned by one thread of one
// work item and runs over the chunks in order, so the results do not depend on how a unit's
// tiles are split into work items.
__global__ void __launch_bounds__(NT, 3) unit_kernel(UnitArgs a) { unit_body<0>(a); }

// The same with the derivative blocks: per chunk, its two 16-node halves in order; per tile,
// every block's sums (values, distribution parameters, Re m, Im m), each into its own
// accumulator (4 n_mu or 4 n_q doubles apart).
__global__ void __launch_bounds__(NT) unit_deriv_kernel(UnitArgs a) { unit_body<1>(a); }

// Adaptive panels: per tile the values' sums and the sums of |Kronrod - Gauss| per panel.
__global__ void __launch_bounds__(NT) unit_adaptive_kernel(UnitArgs a) { unit_body<2>(a); }

// Adaptive panels with the derivative blocks: per tile every block's sums and error sums.
__global__ void __launch_bounds__(NT) unit_adaptive_deriv_kernel(UnitArgs a) { unit_body<3>(a); }

// K-d: the Greek coefficients of each band slot, (2l+1)/2 sum_k w_k F(mu_k) d_l(mu_k) with F
// the slot's averaged tables (fast.rs:238-253): a contraction over the band's n_q nodes shared
// by a tile of up to 32 slots. Lane s of each warp holds slot s; warp w the orders
// l0 + 9w + j (j < 9) of each block of 72 orders. The sums over k run in node order.
namespace {
constexpr int PQ = 32;   // nodes per stage
constexpr int PT = 256;  // threads
constexpr int PL = 72;   // orders per pass: 8 warps x 9
struct ProjSmem {
  double fs[4][PQ][33];  // F11, F12, F33, F34 per node and slot (padded against conflicts)
  double ds[4][PQ][PL];  // d00, d22, d2-2, d02 (scaled) per node and order
  double rz[32];         // 1/Z per slot
  double z[32], ez[32], tr[32];  // adaptive: Z, its error, the truncation term
  double dz[32], edz[32];        // adaptive derivatives: the slot's Z_p and its error
  int blk[32];                   // adaptive derivatives: the slot's block
  int64_t offs[32];
};
}  // namespace

// An adaptive call's table element o of slot s along its block b (engine.rs:1782-1836): the
// part's average (values) or its first-order error estimate (bounds), from the block's sums
// and error sums and the values' (a unit's slots per band: B value slots, then B error slots,
// 4 n_q doubles each). v = S_0/Z, e = (E_0 + |v| e_Z)/Z + t |v|; a parameter p:
// dv = (S_p - v Z_p)/Z, (E_p + |v| e_Zp + |dv| e_Z + e |Z_p|)/Z + t |dv|; along m: dv = S_m/Z,
// (E_m + |dv| e_Z)/Z + t |dv|.
__device__ __forceinline__ double ad_table(const ProjArgs& a, const ProjSmem& sm, int s,
                                           int64_t o, int q, bool bounds) {
  const int b = sm.blk[s], B = a.ad_blocks;
  const int64_t q4 = 4 * (int64_t)q;
  const double z = sm.z[s], ez = sm.ez[s], tr = sm.tr[s], dz = sm.dz[s], edz = sm.edz[s];
  if (!bounds) {
    const double v0 = a.acc[o - b * q4] / z;
    if (b == 0) return v0;
    if (b <= a.n_theta) return (a.acc[o] - v0 * dz) / z;
    return a.acc[o] / z;
  }
  const double v0 = a.acc[o - (B + b) * q4] / z, av0 = fabs(v0);
  const double e0 = (a.acc[o - b * q4] + av0 * ez) / z + tr * av0;
  if (b == 0) return e0;
  const double sb = a.acc[o - B * q4], eb = a.acc[o];
  if (b <= a.n_theta) {
    const double dv = (sb - v0 * dz) / z;
    return (eb + av0 * edz + fabs(dv) * ez + e0 * fabs(dz)) / z + tr * fabs(dv);
  }
  const double dv = sb / z;
  return (eb + fabs(dv) * ez) / z + tr * fabs(dv);
}

__global__ void __launch_bounds__(PT) proj_kernel(ProjArgs a) {
  extern __shared__ __align__(16) unsigned char proj_raw[];
  ProjSmem& sm = *reinterpret_cast<ProjSmem*>(proj_raw);
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  const int glen = a.greek_order + 1;
  for (int item = blockIdx.x; item < a.n_items; item += gridDim.x) {
    const ProjItem it = a.items[item];
    const BandDesc B = a.bands[it.band];
    const int q = B.n_q, len = B.order + 1;
    const bool bounds = it.kind == 1;
    if (t < 32) {
      double rz = 0.0;
      int64_t off = -1;
      if (t < it.count) {
        const BandSlot bs = a.slots[a.slot_index[it.first + t]];
        if (a.unit_norm) {
          const int stride = a.ad_blocks > 0 ? kNormStrideD : 8;
          const double* un = a.unit_norm + stride * (int64_t)a.units[bs.unit];
          sm.z[t] = un[0];
          sm.ez[t] = un[1];
          sm.tr[t] = un[2];
          if (a.ad_blocks > 0) {
            const int b = bs.pad, p = b - 1;
            sm.blk[t] = b;
            sm.dz[t] = (b >= 1 && b <= a.n_theta) ? un[8 + p] : 0.0;
            sm.edz[t] = (b >= 1 && b <= a.n_theta) ? un[11 + p] : 0.0;
          }
        } else if (a.raw) {
          rz = 1.0;
        } else {
          double z = 0.0;
          for (int c = 0; c < a.cpu; ++c) z += a.chunk_sums[((int64_t)bs.unit * a.cpu + c) * 8];
          rz = 1.0 / z;
        }
        off = bs.off;
      }
      sm.rz[t] = rz;
      sm.offs[t] = off;
    }
    __syncthreads();
    const double* D = a.band_d + B.d_off;
    for (int l0 = 0; l0 < len; l0 += PL) {
      double acc[9][6];
#pragma unroll
      for (int j = 0; j < 9; ++j)
#pragma unroll
        for (int e = 0; e < 6; ++e) acc[j][e] = 0.0;
      for (int k0 = 0; k0 < q; k0 += PQ) {
        const int kn = q - k0 < PQ ? q - k0 : PQ;
        // The averaged tables (S/Z) of the 32 slots at nodes k0..k0+kn-1; node fastest, so
        // each slot's run is one coalesced read.
        for (int idx = t; idx < 4 * 32 * PQ; idx += PT) {
          const int kk = idx % PQ, s = (idx / PQ) & 31, e = idx / (32 * PQ);
          double v = 0.0;
          const int64_t off = sm.offs[s];
          if (kk < kn && off >= 0) {
            const int64_t o = off + (int64_t)e * q + k0 + kk;
            if (a.ad_blocks > 0) {
              v = ad_table(a, sm, s, o, q, bounds);
            } else if (!a.unit_norm) {
              v = a.acc[o] * sm.rz[s];
            } else if (!bounds) {
              v = a.acc[o] / sm.z[s];
            } else {
              // The error sums of the slot after the values' (engine.rs:1782-1800).
              const double av = fabs(a.acc[o - 4 * (int64_t)q] / sm.z[s]);
              v = (a.acc[o] + av * sm.ez[s]) / sm.z[s] + sm.tr[s] * av;
            }
          }
          sm.fs[e][kk][s] = v;
        }
        for (int idx = t; idx < 4 * PQ * PL; idx += PT) {
          const int l = idx % PL, kk = (idx / PL) % PQ, m = idx / (PL * PQ);
          double v = 0.0;
          if (kk < kn && l0 + l < len) v = D[((int64_t)m * q + k0 + kk) * len + l0 + l];
          sm.ds[m][kk][l] = bounds ? fabs(v) : v;
        }
        __syncthreads();
        for (int kk = 0; kk < kn; ++kk) {
          const double f11 = sm.fs[0][kk][lane], f12 = sm.fs[1][kk][lane];
          const double f33 = sm.fs[2][kk][lane], f34 = sm.fs[3][kk][lane];
          // Bounds: alpha2 and alpha3 share the half sum of the bounds of alpha2 +- alpha3
          // (fast.rs:256-271).
          const double fp = f11 + f33, fm = bounds ? fp : f11 - f33;
#pragma unroll
          for (int j = 0; j < 9; ++j) {
            const int l = 9 * w + j;
            const double d00 = sm.ds[0][kk][l], d22 = sm.ds[1][kk][l];
            const double d2m2 = sm.ds[2][kk][l], d02 = sm.ds[3][kk][l];
            acc[j][0] = fma(f11, d00, acc[j][0]);
            acc[j][1] = fma(f33, d00, acc[j][1]);
            acc[j][2] = fma(fp, d22, acc[j][2]);
            acc[j][3] = fma(fm, d2m2, acc[j][3]);
            acc[j][4] = fma(f12, d02, acc[j][4]);
            acc[j][5] = fma(f34, d02, acc[j][5]);
          }
        }
        __syncthreads();
      }
      if (lane < it.count) {
        double* out = a.slot_greek + (int64_t)a.slot_index[it.first + lane] * 6 * glen;
#pragma unroll
        for (int j = 0; j < 9; ++j) {
          const int l = l0 + 9 * w + j;
          if (l < len) {
            const double p = acc[j][2], mi = acc[j][3];
            out[l] = acc[j][0];
            out[glen + l] = (p + mi) * 0.5;
            out[2 * glen + l] = bounds ? (p + mi) * 0.5 : (p - mi) * 0.5;
            out[3 * glen + l] = acc[j][1];
            out[4 * glen + l] = acc[j][4];
            out[5 * glen + l] = acc[j][5];
          }
        }
      }
    }
    __syncthreads();
  }
}

// The outputs per unit: the averages S/Z (engine.rs:1782-1836), the Greek coefficients summed
// over the unit's band slots in increasing band order (engine.rs:2310-2355), and the assembly
// of engine.rs:2396-2497.
__global__ void __launch_bounds__(NT) final_kernel(FinalArgs a) {
  __shared__ double S[8];
  __shared__ double a0s;
  const int t = threadIdx.x;
  const int L = a.greek_order;
  const int glen = L >= 0 ? L + 1 : 0;
  const int64_t nu = a.n_units_total;
  for (int ul = blockIdx.x; ul < a.n_units; ul += gridDim.x) {
    const int64_t unit = a.units[ul];
    const int64_t d = unit / a.n_wl, i = unit % a.n_wl;
    if (t < 8) {
      double s = 0.0;
      for (int c = 0; c < a.cpu; ++c) s += a.chunk_sums[((int64_t)ul * a.cpu + c) * 8 + t];
      S[t] = s;
    }
    __syncthreads();
    const double z = S[0];
    const double* acc_user = a.acc + a.unit_acc[ul];
    double v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = S[k] / z;
    const double ext = v[1], sca = v[2], scag = v[3], ab = v[4], back = v[5], r2 = v[6],
                 r3 = v[7];
    if (t == 0) {
      const bool bext = !(isfinite(ext) && ext != 0.0), bsca = !(isfinite(sca) && sca != 0.0);
      const bool bback = !(isfinite(back) && back != 0.0);
      if (bext || bsca || bback) {
        unsigned long long key = ((unsigned long long)(i * a.n_dist + d) << 2) |
                                 (unsigned long long)(bext ? 1 : (bsca ? 2 : 3));
        atomicMin(a.err + 1, key);
      }
      const double out[11] = {ext,         sca,        ab,  back,    sca / ext,
                              scag / sca, (4.0 * kPi) * (ext / back), 0.0, r3 / r2,
                              kPi * r2,   (4.0 * kPi / 3.0) * r3};
#pragma unroll
      for (int k = 0; k < 11; ++k) a.values[k * nu + unit] = out[k];
    }
    if (a.phase) {
      for (int j = t; j < a.n_mu; j += NT) {
        double f[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          f[e] = acc_user[e * a.n_mu + j] / z;
          if (a.normalized) f[e] = f[e] / sca;
        }
        const double o6[6] = {f[0], f[1], f[0], f[2], f[3], f[2]};
#pragma unroll
        for (int e = 0; e < 6; ++e) a.phase[((int64_t)e * nu + unit) * a.n_mu + j] = o6[e];
      }
    }
    if (glen > 0 && a.greek) {
      const int2 sl = a.unit_slots[ul];
      auto sum = [&](int idx) {
        const int e = idx / glen, l = idx % glen;
        double g = 0.0;
        for (int k = 0; k < sl.y; ++k) {
          const BandSlot bs = a.slots[sl.x + k];
          if (l <= a.bands[bs.band].order)
            g += a.slot_greek[(int64_t)(sl.x + k) * 6 * glen + (int64_t)e * glen + l];
        }
        return g;
      };
      if (t == 0) a0s = sum(0);
      __syncthreads();
      const double a0 = a0s;
      for (int idx = t; idx < 6 * glen; idx += NT) {
        const int e = idx / glen, l = idx % glen;
        double g = sum(idx);
        if (a.normalized) g = idx == 0 ? 1.0 : g / a0;
        a.greek[((int64_t)e * nu + unit) * glen + l] = g;
      }
    }
    __syncthreads();
  }
}

// The outputs and their derivatives per unit. Blocks b of the sums S_b (b = 0 the values,
// 1..P_theta the distribution's parameters, then Re m and Im m): the averages v = S_0/Z, along a
// parameter (S_p - v Z_p)/Z, along m S_m/Z (engine.rs:1782-1836); the ratios and the
// normalizations with the quotient rule of ensemble/lin.rs; the Greek coefficients from each
// block's projected raw sums, averaged the same way (the projection is linear).
__global__ void __launch_bounds__(NT) final_deriv_kernel(FinalArgs a) {
  __shared__ double S[6][8];
  __shared__ double a0s[6];
  const int t = threadIdx.x;
  const int L = a.greek_order;
  const int glen = L >= 0 ? L + 1 : 0;
  const int64_t nu = a.n_units_total;
  const int P = a.n_theta + 2, B = 1 + P, nth = a.n_theta;
  for (int ul = blockIdx.x; ul < a.n_units; ul += gridDim.x) {
    const int64_t unit = a.units[ul];
    const int64_t d = unit / a.n_wl, i = unit % a.n_wl;
    if (t < 8 * B) {
      const int b = t / 8, k = t % 8;
      double s = 0.0;
      for (int c = 0; c < a.cpu; ++c)
        s += a.chunk_sums[(((int64_t)ul * a.cpu + c) * B + b) * 8 + k];
      S[b][k] = s;
    }
    __syncthreads();
    const double z = S[0][0];
    // An average and its derivatives from the raw sums s_b of one quantity.
    auto avg = [&](const double* sb, int stride, double* out) {
      const double v = sb[0] / z;
      out[0] = v;
      for (int p = 0; p < P; ++p) {
        const double sp = sb[(1 + p) * stride];
        out[1 + p] = p < nth ? (sp - v * S[1 + p][0]) / z : sp / z;
      }
    };
    // x / y with derivatives (lin.rs Lin::div).
    auto ldiv = [&](const double* x, const double* y, double* out) {
      const double v = x[0] / y[0];
      out[0] = v;
      for (int p = 0; p < P; ++p) out[1 + p] = (x[1 + p] - v * y[1 + p]) / y[0];
    };
    const double* acc_user = a.acc + a.unit_acc[ul];
    if (t == 0) {
      double v[8][6];
      for (int k = 0; k < 8; ++k) avg(&S[0][k], 8, v[k]);
      const double ext = v[1][0], sca = v[2][0], back = v[5][0];
      const bool bext = !(isfinite(ext) && ext != 0.0), bsca = !(isfinite(sca) && sca != 0.0);
      const bool bback = !(isfinite(back) && back != 0.0);
      if (bext || bsca || bback) {
        unsigned long long key = ((unsigned long long)(i * a.n_dist + d) << 2) |
                                 (unsigned long long)(bext ? 1 : (bsca ? 2 : 3));
        atomicMin(a.err + 1, key);
      }
      double out[11][6];
      for (int p = 0; p <= P; ++p) {
        out[0][p] = v[1][p];
        out[1][p] = v[2][p];
        out[2][p] = v[4][p];
        out[3][p] = v[5][p];
        out[7][p] = 0.0;
        out[9][p] = kPi * v[6][p];
        out[10][p] = (4.0 * kPi / 3.0) * v[7][p];
      }
      ldiv(v[2], v[1], out[4]);
      ldiv(v[3], v[2], out[5]);
      ldiv(v[1], v[5], out[6]);
      for (int p = 0; p <= P; ++p) out[6][p] *= 4.0 * kPi;
      ldiv(v[7], v[6], out[8]);
      for (int k = 0; k < 11; ++k) {
        a.values[k * nu + unit] = out[k][0];
        for (int p = 0; p < P; ++p) a.d_values[((int64_t)p * 11 + k) * nu + unit] = out[k][1 + p];
      }
    }
    double sca[6];
    {
      double v[6];
      avg(&S[0][2], 8, v);
      for (int p = 0; p <= P; ++p) sca[p] = v[p];
    }
    if (a.phase) {
      const int64_t blk = 4 * (int64_t)a.n_mu;
      for (int j = t; j < a.n_mu; j += NT) {
        double f[4][6];
        for (int e = 0; e < 4; ++e) {
          avg(acc_user + e * a.n_mu + j, (int)blk, f[e]);
          if (a.normalized) {
            double o[6];
            ldiv(f[e], sca, o);
            for (int p = 0; p <= P; ++p) f[e][p] = o[p];
          }
        }
        const int src[6] = {0, 1, 0, 2, 3, 2};
        for (int e = 0; e < 6; ++e) {
          a.phase[((int64_t)e * nu + unit) * a.n_mu + j] = f[src[e]][0];
          for (int p = 0; p < P; ++p)
            a.d_phase[(((int64_t)p * 6 + e) * nu + unit) * a.n_mu + j] = f[src[e]][1 + p];
        }
      }
    }
    if (glen > 0 && a.greek) {
      // The unit's slots are B consecutive entries (one per block) per band, bands ascending.
      const int2 sl = a.unit_slots[ul];
      auto sum = [&](int b, int idx) {
        const int e = idx / glen, l = idx % glen;
        double g = 0.0;
        for (int k = b; k < sl.y; k += B) {
          const BandSlot bs = a.slots[sl.x + k];
          if (l <= a.bands[bs.band].order)
            g += a.slot_greek[(int64_t)(sl.x + k) * 6 * glen + (int64_t)e * glen + l];
        }
        return g;
      };
      auto coeff = [&](int idx, double* out) {
        double raw[6];
        for (int b = 0; b < B; ++b) raw[b] = sum(b, idx);
        avg(raw, 1, out);
      };
      if (t == 0) coeff(0, a0s);
      __syncthreads();
      for (int idx = t; idx < 6 * glen; idx += NT) {
        const int e = idx / glen, l = idx % glen;
        double c[6];
        coeff(idx, c);
        if (a.normalized) {
          if (idx == 0) {
            c[0] = 1.0;
            for (int p = 0; p < P; ++p) c[1 + p] = 0.0;
          } else {
            double o[6];
            ldiv(c, a0s, o);
            for (int p = 0; p <= P; ++p) c[p] = o[p];
          }
        }
        a.greek[((int64_t)e * nu + unit) * glen + l] = c[0];
        for (int p = 0; p < P; ++p)
          a.d_greek[(((int64_t)p * 6 + e) * nu + unit) * glen + l] = c[1 + p];
      }
    }
    __syncthreads();
  }
}

// The outputs of adaptive panels per unit with their error estimates: averages from the
// Kronrod sums and the moments' Z, errors (e + |v| e_Z)/Z + truncation |v| (engine.rs:
// 1782-1836), <r^2>, <r^3> from the moments (a single radius keeps its own), the ratios and
// normalizations with the first-order bounds of ensemble/lin.rs (Lin::div, Lin::scale), and the
// Greek coefficients summed over the bands, values and bounds (engine.rs:2310-2355).
namespace {
struct LinE {
  double v, e;
};
__device__ __forceinline__ LinE ldiv(LinE a, LinE b) {
  const double v = a.v / b.v;
  return {v, (a.e + fabs(v) * b.e) / fabs(b.v)};
}
__device__ __forceinline__ LinE lscale(LinE a, double c) { return {c * a.v, fabs(c) * a.e}; }
}  // namespace

// Stage 1 of the adaptive outputs: each (part, wavelength) unit's averages with their error
// estimates into `avg` (per unit: the 8 scalars, the 4 n_mu cosine tables, the 6 (L + 1) Greek
// sums, each as values then errors). The Greek sums are projected per part and mixed after
// (the projection is linear and its bounds are linear in the errors).
__global__ void __launch_bounds__(NT) final_adaptive_kernel(FinalArgs a) {
  __shared__ double S[2][8];
  const int t = threadIdx.x;
  const int L = a.greek_order;
  const int glen = L >= 0 ? L + 1 : 0;
  const int64_t stride = 16 + 8 * (int64_t)a.n_mu + 12 * (int64_t)glen;
  for (int ul = blockIdx.x; ul < a.n_units; ul += gridDim.x) {
    const int64_t unit = a.units[ul];
    if (t < 16) {
      double s = 0.0;
      for (int c = 0; c < a.cpu; ++c) s += a.chunk_sums[((int64_t)ul * a.cpu + c) * 16 + t];
      S[t / 8][t % 8] = s;
    }
    __syncthreads();
    const double* un = a.unit_norm + 8 * unit;
    const double z = un[0], ez = un[1], tr = un[2];
    const bool point = un[3] != 0.0;
    auto avg = [&](double s, double e) {
      const double v = s / z;
      return LinE{v, (e + fabs(v) * ez) / z + tr * fabs(v)};
    };
    double* out = a.avg + stride * unit;
    if (t < 8) {
      LinE v = avg(S[0][t], S[1][t]);
      // <r^2>, <r^3> from the moment integration (a single radius keeps its own).
      if (!point && t >= 6) v = LinE{un[4 + 2 * (t - 6)], un[5 + 2 * (t - 6)]};
      out[t] = v.v;
      out[8 + t] = v.e;
    }
    const double* acc_user = a.acc + a.unit_acc[ul];
    for (int j = t; j < 4 * a.n_mu; j += NT) {
      const LinE f = avg(acc_user[j], acc_user[4 * a.n_mu + j]);
      out[16 + j] = f.v;
      out[16 + 4 * a.n_mu + j] = f.e;
    }
    if (glen > 0) {
      // The unit's slots: per band a values slot, then its bounds slot.
      const int2 sl = a.unit_slots[ul];
      double* og = out + 16 + 8 * (int64_t)a.n_mu;
      for (int idx = t; idx < 6 * glen; idx += NT) {
        const int e = idx / glen, l = idx % glen;
        double gv = 0.0, ge = 0.0;
        for (int k = 0; k + 1 < sl.y; k += 2) {
          const BandSlot bs = a.slots[sl.x + k];
          if (l <= a.bands[bs.band].order) {
            gv += a.slot_greek[(int64_t)(sl.x + k) * 6 * glen + (int64_t)e * glen + l];
            ge += a.slot_greek[(int64_t)(sl.x + k + 1) * 6 * glen + (int64_t)e * glen + l];
          }
        }
        og[idx] = gv;
        og[6 * glen + idx] = ge;
      }
    }
    __syncthreads();
  }
}

// Stage 1 of an adaptive call with derivatives: each (part, wavelength) unit's averages along
// every block b < B (values, each distribution parameter, Re m, Im m) with their error
// estimates into `avg`, block after block: 8 scalars, 4 n_mu cosine values, 6 (L + 1) Greek
// coefficients, then the same for the errors (engine.rs:1782-1836 with the quotient rule of
// the parameter blocks). <r^2> and <r^3> and their parameter derivatives come from the moments
// (a single radius keeps its own; 0 along m). The Greek sums are already averaged per slot.
__global__ void __launch_bounds__(NT) final_adaptive_d_kernel(FinalArgs a) {
  __shared__ double S[12][8];
  const int t = threadIdx.x;
  const int L = a.greek_order;
  const int glen = L >= 0 ? L + 1 : 0;
  const int B = a.ad_blocks, nth = a.n_theta;
  const int64_t row = 8 + 4 * (int64_t)a.n_mu + 6 * (int64_t)glen;
  for (int ul = blockIdx.x; ul < a.n_units; ul += gridDim.x) {
    const int64_t unit = a.units[ul];
    if (t < 16 * B) {
      const int b = t / 8, k = t % 8;
      double s = 0.0;
      for (int c = 0; c < a.cpu; ++c)
        s += a.chunk_sums[(((int64_t)ul * a.cpu + c) * 2 * B + b) * 8 + k];
      S[b][k] = s;
    }
    __syncthreads();
    const double* un = a.unit_norm + kNormStrideD * unit;
    const double z = un[0], ez = un[1], tr = un[2];
    const bool point = un[3] != 0.0;
    // One element's average and error along block b from its sums (s0, e0: the values';
    // sb, eb: the block's).
    auto avg = [&](int b, double s0, double e0, double sb, double eb, double* v, double* e) {
      const double v0 = s0 / z, av0 = fabs(v0);
      const double er0 = (e0 + av0 * ez) / z + tr * av0;
      if (b == 0) {
        *v = v0;
        *e = er0;
      } else if (b <= nth) {
        const double dz = un[8 + b - 1], edz = un[11 + b - 1];
        const double dv = (sb - v0 * dz) / z;
        *v = dv;
        *e = (eb + av0 * edz + fabs(dv) * ez + er0 * fabs(dz)) / z + tr * fabs(dv);
      } else {
        const double dv = sb / z;
        *v = dv;
        *e = (eb + fabs(dv) * ez) / z + tr * fabs(dv);
      }
    };
    double* out = a.avg + 2 * B * row * unit;
    for (int idx = t; idx < 8 * B; idx += NT) {
      const int b = idx / 8, k = idx % 8;
      double v, e;
      avg(b, S[0][k], S[B][k], S[b][k], S[B + b][k], &v, &e);
      if (!point && k >= 6) {
        const int m = k - 6;
        if (b == 0) {
          v = un[4 + 2 * m];
          e = un[5 + 2 * m];
        } else if (b <= nth) {
          v = un[14 + 4 * (b - 1) + 2 * m];
          e = un[15 + 4 * (b - 1) + 2 * m];
        } else {
          v = 0.0;
          e = 0.0;
        }
      }
      out[2 * b * row + k] = v;
      out[(2 * b + 1) * row + k] = e;
    }
    const double* acc_user = a.acc + a.unit_acc[ul];
    const int64_t tl = 4 * (int64_t)a.n_mu;
    for (int64_t idx = t; idx < tl * B; idx += NT) {
      const int b = (int)(idx / tl);
      const int64_t j = idx % tl;
      double v, e;
      avg(b, acc_user[j], acc_user[B * tl + j], acc_user[b * tl + j], acc_user[(B + b) * tl + j],
          &v, &e);
      out[2 * b * row + 8 + j] = v;
      out[(2 * b + 1) * row + 8 + j] = e;
    }
    if (glen > 0) {
      // The unit's slots per band: B value slots, then B error slots.
      const int2 sl = a.unit_slots[ul];
      for (int64_t idx = t; idx < 6 * (int64_t)glen * B; idx += NT) {
        const int b = (int)(idx / (6 * glen));
        const int g = (int)(idx % (6 * glen)), e = g / glen, l = g % glen;
        double gv = 0.0, ge = 0.0;
        for (int k = 0; k + 2 * B <= sl.y; k += 2 * B) {
          const BandSlot bs = a.slots[sl.x + k];
          if (l <= a.bands[bs.band].order) {
            gv += a.slot_greek[(int64_t)(sl.x + k + b) * 6 * glen + (int64_t)e * glen + l];
            ge += a.slot_greek[(int64_t)(sl.x + k + B + b) * 6 * glen + (int64_t)e * glen + l];
          }
        }
        out[2 * b * row + 8 + tl + g] = gv;
        out[(2 * b + 1) * row + 8 + tl + g] = ge;
      }
    }
    __syncthreads();
  }
}

// Stage 2: each output unit (o, wavelength i) mixes its parts' averages with their number
// fractions f (engine.rs:2121-2176: values and errors alike, in part order) and assembles the
// outputs: ratios, normalizations and bounds of ensemble/lin.rs, Greek normalized by the
// mixture's alpha1_0 (engine.rs:2396-2497).
__global__ void __launch_bounds__(NT) mix_assemble_kernel(MixArgs a) {
  __shared__ double V[16];
  __shared__ LinE a0s;
  const int t = threadIdx.x;
  const int glen = a.greek_order >= 0 ? a.greek_order + 1 : 0;
  const int64_t stride = 16 + 8 * (int64_t)a.n_mu + 12 * (int64_t)glen;
  const int64_t n_out = (int64_t)a.n_out * a.n_wl;
  auto mixed = [&](int64_t o, int64_t i, int64_t off) {
    double v = 0.0;
    for (int k = a.first[o]; k < a.first[o + 1]; ++k)
      v += a.fraction[k] * a.avg[stride * ((int64_t)a.part[k] * a.n_wl + i) + off];
    return v;
  };
  for (int64_t ou = blockIdx.x; ou < n_out; ou += gridDim.x) {
    const int64_t o = ou / a.n_wl, i = ou % a.n_wl;
    if (t < 16) V[t] = mixed(o, i, t);
    __syncthreads();
    auto lin = [&](int k) { return LinE{V[k], V[8 + k]}; };
    const LinE ext = lin(1), sca = lin(2), scag = lin(3), ab = lin(4), back = lin(5), r2 = lin(6),
               r3 = lin(7);
    if (t == 0) {
      const bool bext = !(isfinite(ext.v) && ext.v != 0.0);
      const bool bsca = !(isfinite(sca.v) && sca.v != 0.0);
      const bool bback = !(isfinite(back.v) && back.v != 0.0);
      if (bext || bsca || bback) {
        unsigned long long key = ((unsigned long long)(i * a.n_out + o) << 2) |
                                 (unsigned long long)(bext ? 1 : (bsca ? 2 : 3));
        atomicMin(a.err + 1, key);
      }
      const LinE out[11] = {ext,
                            sca,
                            ab,
                            back,
                            ldiv(sca, ext),
                            ldiv(scag, sca),
                            lscale(ldiv(ext, back), 4.0 * kPi),
                            LinE{0.0, 0.0},
                            ldiv(r3, r2),
                            lscale(r2, kPi),
                            lscale(r3, 4.0 * kPi / 3.0)};
      for (int k = 0; k < 11; ++k) {
        a.values[k * n_out + ou] = out[k].v;
        a.errors[k * n_out + ou] = out[k].e;
      }
    }
    if (a.phase) {
      for (int j = t; j < a.n_mu; j += NT) {
        LinE f[4];
        for (int e = 0; e < 4; ++e) {
          f[e] = LinE{mixed(o, i, 16 + e * a.n_mu + j),
                      mixed(o, i, 16 + (4 + e) * (int64_t)a.n_mu + j)};
          if (a.normalized) f[e] = ldiv(f[e], sca);
        }
        const int src[6] = {0, 1, 0, 2, 3, 2};
        for (int e = 0; e < 6; ++e) {
          a.phase[((int64_t)e * n_out + ou) * a.n_mu + j] = f[src[e]].v;
          a.phase_err[((int64_t)e * n_out + ou) * a.n_mu + j] = f[src[e]].e;
        }
      }
    }
    if (glen > 0 && a.greek) {
      const int64_t g0 = 16 + 8 * (int64_t)a.n_mu;
      if (t == 0) a0s = LinE{mixed(o, i, g0), mixed(o, i, g0 + 6 * glen)};
      __syncthreads();
      const LinE a0 = a0s;
      for (int idx = t; idx < 6 * glen; idx += NT) {
        const int e = idx / glen, l = idx % glen;
        LinE g{mixed(o, i, g0 + idx), mixed(o, i, g0 + 6 * glen + idx)};
        if (a.normalized) g = idx == 0 ? LinE{1.0, 0.0} : ldiv(g, a0);
        a.greek[((int64_t)e * n_out + ou) * glen + l] = g.v;
        a.greek_err[((int64_t)e * n_out + ou) * glen + l] = g.e;
      }
    }
    __syncthreads();
  }
}

void launch_mix(const MixArgs& a, cudaStream_t s) {
  const int64_t n = (int64_t)a.n_out * a.n_wl;
  const int grid = (int)(n < 4096 ? n : 4096);
  if (grid > 0) mix_assemble_kernel<<<grid, NT, 0, s>>>(a);
}

// The unit kernels' stage buffers are dynamic shared memory (above the 48 KB static limit);
// the attribute is per device: set it once on each.
static void configure_units() {
  static bool configured[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 64 && !configured[dev]) {
    for (auto f : {unit_kernel, unit_deriv_kernel, unit_adaptive_kernel, unit_adaptive_deriv_kernel})
      cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(Smem));
    configured[dev] = true;
  }
}

int unit_kernel_blocks_per_sm() {
  configure_units();
  int n = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, unit_kernel, NT, sizeof(Smem));
  return n > 0 ? n : 1;
}

void launch_units(const UnitArgs& a, int grid, cudaStream_t s) {
  configure_units();
  if (a.deriv && a.wdiff)
    unit_adaptive_deriv_kernel<<<grid, NT, sizeof(Smem), s>>>(a);
  else if (a.deriv)
    unit_deriv_kernel<<<grid, NT, sizeof(Smem), s>>>(a);
  else if (a.wdiff)
    unit_adaptive_kernel<<<grid, NT, sizeof(Smem), s>>>(a);
  else
    unit_kernel<<<grid, NT, sizeof(Smem), s>>>(a);
}

void launch_proj(const ProjArgs& a, cudaStream_t s) {
  // The attribute is per device: set it once on each.
  static bool configured[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 64 && !configured[dev]) {
    cudaFuncSetAttribute(proj_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sizeof(ProjSmem));
    configured[dev] = true;
  }
  int grid = a.n_items < 8192 ? a.n_items : 8192;
  if (grid > 0) proj_kernel<<<grid, PT, sizeof(ProjSmem), s>>>(a);
}

void launch_final(const FinalArgs& a, cudaStream_t s) {
  int grid = a.n_units < 4096 ? a.n_units : 4096;
  if (a.ad_blocks > 0)
    final_adaptive_d_kernel<<<grid, NT, 0, s>>>(a);
  else if (a.d_values)
    final_deriv_kernel<<<grid, NT, 0, s>>>(a);
  else if (a.unit_norm)
    final_adaptive_kernel<<<grid, NT, 0, s>>>(a);
  else
    final_kernel<<<grid, NT, 0, s>>>(a);
}

}  // namespace sb
