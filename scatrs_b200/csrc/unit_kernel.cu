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
constexpr int KB = 16;   // orders per GEMM stage
constexpr int TR = 32;   // table rows per tile
constexpr int NT = 128;  // threads: 8 row groups of 4 rows x 16 node groups of 2 nodes

__device__ __forceinline__ void elements4(double s1r, double s1i, double s2r, double s2i,
                                          double e[4]) {
  // (|S1|^2+|S2|^2)/2, (|S2|^2-|S1|^2)/2, Re(S2 S1*), Im(S2 S1*) (scatrs/src/mie/phase.rs:54-59)
  double n1 = s1r * s1r + s1i * s1i, n2 = s2r * s2r + s2i * s2i;
  e[0] = 0.5 * (n1 + n2);
  e[1] = 0.5 * (n2 - n1);
  e[2] = s2r * s1r + s2i * s1i;
  e[3] = s2i * s1r - s2r * s1i;
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
  double ae[KB][TR];
  double ao[KB][TR];
  double xs[KB][128];
  double w[32], cu[32], area[32], sc[32];
  double S[8];
  int slot;
};

// accE/accO[r][c] = sum_k G[r0 + 4 rg + r][k] X[k][4 ng + c (+ 64 for c >= 4)] for k < nc.
__device__ __forceinline__ void gemm_tile(Smem& sm, const double* __restrict__ ge,
                                          const double* __restrict__ go, int ld, int r0, int nc,
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
  for (int k0 = 0; k0 < nc; k0 += KB) {
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      int idx = t + q * NT;
      int row = idx >> 3, kp = (idx & 7) * 2;
      int k = k0 + kp;
      double2 e = make_double2(0.0, 0.0), o = make_double2(0.0, 0.0);
      if (k < nc) {
        int64_t off = (int64_t)(r0 + row) * ld + k;
        e = *reinterpret_cast<const double2*>(ge + off);
        o = *reinterpret_cast<const double2*>(go + off);
        if (k + 1 >= nc) {
          e.y = 0.0;
          o.y = 0.0;
        }
      }
      sm.ae[kp][row] = e.x;
      sm.ae[kp + 1][row] = e.y;
      sm.ao[kp][row] = o.x;
      sm.ao[kp + 1][row] = o.y;
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      int idx = t + q * NT;
      int kr = idx >> 6, cp = (idx & 63) * 2;
      int k = k0 + kr;
      double2 v = make_double2(0.0, 0.0);
      if (k < nc) v = *reinterpret_cast<const double2*>(xc + (int64_t)k * 128 + cp);
      *reinterpret_cast<double2*>(&sm.xs[kr][cp]) = v;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < KB; ++kk) {
      double2 e01 = *reinterpret_cast<const double2*>(&sm.ae[kk][rg * 4]);
      double2 e23 = *reinterpret_cast<const double2*>(&sm.ae[kk][rg * 4 + 2]);
      double2 o01 = *reinterpret_cast<const double2*>(&sm.ao[kk][rg * 4]);
      double2 o23 = *reinterpret_cast<const double2*>(&sm.ao[kk][rg * 4 + 2]);
      double2 x0 = *reinterpret_cast<const double2*>(&sm.xs[kk][ng * 4]);
      double2 x1 = *reinterpret_cast<const double2*>(&sm.xs[kk][ng * 4 + 2]);
      double2 y0 = *reinterpret_cast<const double2*>(&sm.xs[kk][(ng + 16) * 4]);
      double2 y1 = *reinterpret_cast<const double2*>(&sm.xs[kk][(ng + 16) * 4 + 2]);
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
    __syncthreads();
  }
}

// The elements at +mu (P) and -mu (M) of this thread's 4 rows, scaled and weighted per sphere
// and summed over the chunk's 32 spheres; returned in the threads with ng == 0.
template <bool kUser>
__device__ __forceinline__ void chunk_elements(const Smem& sm, const double accE[4][8],
                                               const double accO[4][8], double P[4][4],
                                               double M[4][4]) {
  const int ng = threadIdx.x & 15;
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      P[r][e] = 0.0;
      M[r][e] = 0.0;
    }
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
          P[r][e] += w * ((cu * ep[e]) * ar);
          M[r][e] += w * ((cu * em[e]) * ar);
        } else {
          P[r][e] += w * (sc * ep[e]);
          M[r][e] += w * (sc * em[e]);
        }
      }
    }
  }
#pragma unroll
  for (int off = 8; off > 0; off >>= 1)
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        P[r][e] += __shfl_xor_sync(0xffffffffu, P[r][e], off);
        M[r][e] += __shfl_xor_sync(0xffffffffu, M[r][e], off);
      }
}

// K-d: the band's averaged tables projected and added to the Greek accumulators; the band
// accumulator is cleared for the next band.
__device__ void flush_band(const UnitArgs& a, int b, double z, double* acc_band,
                           double* acc_greek, int glen) {
  __syncthreads();
  const BandDesc B = a.bands[b];
  const int q = B.n_q, len = B.order + 1;
  for (int k = threadIdx.x; k < 4 * q; k += NT) acc_band[k] = acc_band[k] / z;
  __syncthreads();
  const double* D = a.band_d + B.d_off;
  for (int l = threadIdx.x; l < len; l += NT) {
    double a1 = 0.0, a4 = 0.0, p = 0.0, mi = 0.0, b1 = 0.0, b2 = 0.0;
    for (int k = 0; k < q; ++k) {
      const double f11 = acc_band[k], f12 = acc_band[q + k];
      const double f33 = acc_band[2 * q + k], f34 = acc_band[3 * q + k];
      const double d00 = D[(int64_t)k * len + l];
      const double d22 = D[(int64_t)(q + k) * len + l];
      const double d2m2 = D[(int64_t)(2 * q + k) * len + l];
      const double d02 = D[(int64_t)(3 * q + k) * len + l];
      a1 = fma(f11, d00, a1);
      a4 = fma(f33, d00, a4);
      p = fma(f11 + f33, d22, p);
      mi = fma(f11 - f33, d2m2, mi);
      b1 = fma(f12, d02, b1);
      b2 = fma(f34, d02, b2);
    }
    acc_greek[l] += a1;
    acc_greek[glen + l] += (p + mi) * 0.5;
    acc_greek[2 * glen + l] += (p - mi) * 0.5;
    acc_greek[3 * glen + l] += a4;
    acc_greek[4 * glen + l] += b1;
    acc_greek[5 * glen + l] += b2;
  }
  __syncthreads();
  for (int k = threadIdx.x; k < 4 * q; k += NT) acc_band[k] = 0.0;
  __syncthreads();
}

}  // namespace

__global__ void __launch_bounds__(NT) unit_kernel(UnitArgs a) {
  __shared__ __align__(16) Smem sm;
  const int t = threadIdx.x, rg = t >> 4, ng = t & 15;
  double* acc_user = a.acc + (int64_t)blockIdx.x * a.acc_stride;
  double* acc_band = acc_user + 4 * a.n_mu;
  double* acc_greek = acc_band + 4 * a.nq_max;
  const int L = a.greek_order;
  const int glen = L >= 0 ? L + 1 : 0;
  for (;;) {
    if (t == 0) sm.slot = atomicAdd(a.work_counter, 1);
    __syncthreads();
    const int slot = sm.slot;
    if (slot >= a.n_units) break;
    const int ul = a.unit_order ? a.unit_order[slot] : slot;
    const int64_t unit = a.unit0 + ul;
    const int64_t d = unit / a.n_wl, i = unit % a.n_wl;
    const double lam = a.wl[i];
    for (int k = t; k < 4 * a.n_mu; k += NT) acc_user[k] = 0.0;
    for (int k = t; k < 4 * a.nq_max; k += NT) acc_band[k] = 0.0;
    for (int k = t; k < 6 * glen; k += NT) acc_greek[k] = 0.0;
    if (t < 8) {
      double s = 0.0;
      for (int c = 0; c < a.cpu; ++c) s += a.chunk_sums[((int64_t)ul * a.cpu + c) * 8 + t];
      sm.S[t] = s;
    }
    __syncthreads();
    const double z = sm.S[0];
    int prev = -1;
    for (int c = 0; c < a.cpu; ++c) {
      const int nc = a.chunk_n[ul * a.cpu + c];
      if (nc == 0) continue;
      const int b = L >= 0 ? band_of(nc) : -1;
      if (b != prev && prev >= 0) flush_band(a, prev, z, acc_band, acc_greek, glen);
      prev = b;
      if (t < 32) {
        const int j = c * 32 + t;
        double w = 0.0, cu = 0.0, ar = 0.0, sc = 0.0;
        if (j < a.n_nodes) {
          const double r = a.radius[d * a.n_nodes + j];
          const double x = 2.0 * kPi * r / lam;
          w = a.weight[d * a.n_nodes + j];  // w_j u(r_j) r_j
          cu = 4.0 / (x * x);
          ar = kPi * r * r;
          sc = 4.0 / (x * x) * (kPi * r * r);
        }
        sm.w[t] = w;
        sm.cu[t] = cu;
        sm.area[t] = ar;
        sm.sc[t] = sc;
      }
      __syncthreads();
      const double* xc = a.X + a.chunk_row[ul * a.cpu + c] * 128;
      double accE[4][8], accO[4][8], P[4][4], M[4][4];
      for (int r0 = 0; r0 < a.h_u; r0 += TR) {
        gemm_tile(sm, a.ge_u, a.go_u, a.ld_u, r0, nc, xc, accE, accO);
        chunk_elements<true>(sm, accE, accO, P, M);
        if (ng == 0) {
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            const int row = r0 + rg * 4 + r;
            if (row < a.h_u) {
              const int2 mp = a.user_map[row];
#pragma unroll
              for (int e = 0; e < 4; ++e) {
                acc_user[e * a.n_mu + mp.x] += P[r][e];
                if (mp.y >= 0) acc_user[e * a.n_mu + mp.y] += M[r][e];
              }
            }
          }
        }
      }
      if (b >= 0) {
        const BandDesc B = a.bands[b];
        const int q = B.n_q, lo = q / 2;
        for (int r0 = 0; r0 < B.h; r0 += TR) {
          gemm_tile(sm, a.band_ge + B.g_off, a.band_go + B.g_off, B.ld, r0, nc, xc, accE, accO);
          chunk_elements<false>(sm, accE, accO, P, M);
          if (ng == 0) {
#pragma unroll
            for (int r = 0; r < 4; ++r) {
              const int row = r0 + rg * 4 + r;
              if (row < B.h) {
                const int jn = lo + row, mirror = q - 1 - jn;
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                  acc_band[e * q + jn] += P[r][e];
                  if (mirror != jn) acc_band[e * q + mirror] += M[r][e];
                }
              }
            }
          }
        }
      }
      __syncthreads();
    }
    if (prev >= 0) flush_band(a, prev, z, acc_band, acc_greek, glen);
    __syncthreads();
    // Averages and outputs (engine.rs:1782-1836, 2396-2497).
    double v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = sm.S[k] / z;
    const double ext = v[1], sca = v[2], scag = v[3], ab = v[4], back = v[5], r2 = v[6],
                 r3 = v[7];
    const int64_t nu = a.n_units_total;
    if (t == 0) {
      bool bad = !(isfinite(ext) && ext != 0.0) || !(isfinite(sca) && sca != 0.0) ||
                 !(isfinite(back) && back != 0.0);
      if (bad) {
        unsigned long long key =
            ((unsigned long long)(i * a.n_dist + d) << 2) |
            (unsigned long long)(!(isfinite(ext) && ext != 0.0) ? 1 : (!(isfinite(sca) && sca != 0.0) ? 2 : 3));
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
    if (a.greek && glen > 0) {
      const double a0 = acc_greek[0];
      for (int idx = t; idx < 6 * glen; idx += NT) {
        const int e = idx / glen, l = idx % glen;
        double g = acc_greek[idx];
        if (a.normalized) g = idx == 0 ? 1.0 : g / a0;
        a.greek[((int64_t)e * nu + unit) * glen + l] = g;
      }
    }
    __syncthreads();
  }
}

int unit_kernel_blocks_per_sm() {
  int n = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, unit_kernel, NT, 0);
  return n > 0 ? n : 1;
}

void launch_units(const UnitArgs& a, int grid, cudaStream_t s) {
  unit_kernel<<<grid, NT, 0, s>>>(a);
}

}  // namespace sb
