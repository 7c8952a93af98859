// K-a: the Mie recurrences of every size node, one thread per node, one warp per chunk of 32
// consecutive nodes of a (distribution, wavelength) unit. Compiled with -fmad=false (see
// mie_device.cuh). The coefficients leave in the layout the angle GEMM reads: for each chunk a
// row per order n (n = 1..N_c, N_c the chunk's largest number of terms) of 128 doubles,
// 4 per lane: u.re, u.im, v.re, v.im with (u, v) = (a_n, b_n) for odd n and (b_n, a_n) for even
// n (scatrs/src/ensemble/fast.rs:95-137), zero above the node's own N.
#include "kernels.h"
#include "layered_deriv.cuh"
#include "mie_device.cuh"

namespace sb {

// Error word: the smallest (wavelength, distribution, radius) key of a node whose inputs fail,
// with its status in the low 2 bits.
__device__ __forceinline__ void record_error(unsigned long long* err, long long i_wl,
                                             long long d, long long j, long long n_dist,
                                             long long n_nodes, int status) {
  unsigned long long key = (unsigned long long)(((i_wl * n_dist + d) * n_nodes + j) << 2) |
                           (unsigned long long)status;
  atomicMin(err, key);
}

// Each chunk's largest number of terms (the band selector, engine.rs:961-978).
__global__ void plan_chunks_kernel(PlanArgs a) {
  int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (warp >= a.n_chunks) return;
  int64_t unit = warp / a.cpu;
  int c = warp % a.cpu;
  int64_t d = unit / a.n_wl, i = unit % a.n_wl;
  int j = c * 32 + lane;
  int64_t n = 0;
  if (j < a.n_nodes) {
    double r = a.radius[(a.per_unit ? unit : d) * a.n_nodes + j];
    if (r > 0.0) {
      double x = 2.0 * kPi * r / a.wl[i];
      n = default_n_max(x);
      if (n > (1 << 20)) n = 1 << 20;
    }
  }
  int nn = (int)n;
  for (int off = 16; off > 0; off >>= 1) {
    int o = __shfl_xor_sync(0xffffffffu, nn, off);
    nn = o > nn ? o : nn;
  }
  if (lane == 0) a.chunk_n[warp] = nn;
}

template <bool kLayered, bool kAdaptive>
__device__ __forceinline__ void mie_chunk(const MieFixedArgs& a) {
  int wslot = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (wslot >= a.n_chunks) return;
  int chunk = wslot;
  int64_t unit = a.units[chunk / a.cpu];
  int c = chunk % a.cpu;
  int64_t d = unit / a.n_wl, i = unit % a.n_wl;
  int j = c * 32 + lane;
  int nc = a.chunk_n[chunk];
  int64_t row0 = a.chunk_row[chunk];
  double* X = a.X + row0 * 128 + lane * 4;
  // Scratch: 2L - 1 complex ratio arrays (one for a sphere) of nc + 2 rows, and u_k(x).
  const int n_arr = kLayered ? 2 * a.n_layers - 1 : 1;
  Scratch s;
  s.uz = a.uz + (row0 + 2 * (int64_t)chunk) * n_arr * 32 + lane;
  s.ux = a.ux + (row0 + 2 * (int64_t)chunk) * 32 + lane;
  s.stride = 32;
  double q[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  double qe[kAdaptive ? 8 : 1] = {};  // adaptive: weighted by w_K - w_G
  double cm[4] = {0.0, 0.0, 0.0, 0.0};  // the largest |X| of this lane's four columns
  int64_t n = 0;
  const int64_t node = (a.per_unit ? unit : d) * a.n_nodes + j;
  if (j < a.n_nodes && a.radius[node] > 0.0) {
    const double r = a.radius[node];
    const double w = a.weight[node];
    const double x = 2.0 * kPi * r / a.wl[i];
    n = default_n_max(x);
    auto emit = [&](int64_t k, cplx an, cplx bn) {
      const bool odd = (k & 1) != 0;
      const cplx u = odd ? an : bn, v = odd ? bn : an;
      *reinterpret_cast<double4*>(X + (k - 1) * 128) = make_double4(u.re, u.im, v.re, v.im);
      cm[0] = fmax(cm[0], fabs(u.re));
      cm[1] = fmax(cm[1], fabs(u.im));
      cm[2] = fmax(cm[2], fabs(v.re));
      cm[3] = fmax(cm[3], fabs(v.im));
    };
    ValueSums vs;
    double asum = 0.0;
    int st;
    if (!kLayered) {
      const double2 mv = a.m[unit];
      const cplx m = mk(mv.x, mv.y);
      st = check_node(x, m, n, a.allow_unvalidated != 0);
      if (st == 0 && n <= nc) {
        mie_prepare(x, m, n, s);
        asum = mie_finish(x, m, n, s, vs, emit);
      }
    } else {
      // A layered sphere: x_l = f_l x, the outer surface's x last (ensemble/particle.rs:186-195).
      const int L = a.n_layers;
      double xs[kMaxLayers];
      cplx ms[kMaxLayers];
      bool lossless = true;
      for (int l = 0; l < L; ++l) {
        xs[l] = l < L - 1 ? a.fractions[d * (L - 1) + l] * x : x;
        const double2 mv = a.m_layers[(d * L + l) * a.n_wl + i];
        ms[l] = mk(mv.x, mv.y);
        lossless = lossless && mv.y == 0.0;
      }
      st = check_layered(xs, ms, L, n, a.allow_unvalidated != 0);
      if (st == 0 && n <= nc) {
        mie_prepare(x, ms[L - 1], n, s);
        Layered lay;
        lay.layers = L;
        lay.x = xs;
        lay.m = ms;
        lay.arr.base = s.uz;
        lay.arr.astride = (int64_t)(nc + 2) * 32;
        lay.arr.stride = 32;
        lay.prepare(n);
        asum = mie_finish(x, ms[L - 1], n, s, vs, emit, lay);
        // A lossless particle absorbs nothing (layered/kernel.rs:455-464).
        if (lossless) asum = 0.0;
      }
    }
    if (st != 0 || n > nc) {
      record_error(a.err, i, d, j, a.n_dist, a.n_nodes, st != 0 ? st : 1);
      n = 0;
    } else {
      const Eff e = efficiencies_from(x, asum, vs);
      // The per-particle quantities of pass 2 (engine.rs:1047-1057), weighted.
      const double area = kPi * r * r;
      const double qv[8] = {1.0,           area * e.q_ext, area * e.q_sca, area * e.q_sca * e.g,
                            area * e.q_abs, area * e.q_back, r * r,         r * r * r};
      for (int k = 0; k < 8; ++k) q[k] = w * qv[k];
      if constexpr (kAdaptive) {
        const double wd = a.wdiff[node];
        for (int k = 0; k < 8; ++k) qe[k] = wd * qv[k];
      }
    }
  }
  // Orders above the node's own N are zero up to the chunk's.
  for (int64_t k = n + 1; k <= nc; ++k)
    *reinterpret_cast<double4*>(X + (k - 1) * 128) = make_double4(0.0, 0.0, 0.0, 0.0);
  if (a.colmax != nullptr)
    *reinterpret_cast<double4*>(a.colmax + (int64_t)chunk * 128 + lane * 4) =
        make_double4(cm[0], cm[1], cm[2], cm[3]);
  // The chunk's weighted sums, in a fixed tree order.
  const int stride = kAdaptive ? 16 : 8;
  for (int k = 0; k < 8; ++k) {
    double v = q[k];
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if (lane == 0) a.chunk_sums[(int64_t)chunk * stride + k] = v;
  }
  if constexpr (kAdaptive) {
    // |Kronrod - Gauss| of each of the chunk's two panels (lanes 0-15, 16-31), then added.
    for (int k = 0; k < 8; ++k) {
      double v = qe[k];
      for (int off = 8; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
      const double other = __shfl_sync(0xffffffffu, v, 16);
      if (lane == 0) a.chunk_sums[(int64_t)chunk * 16 + 8 + k] = fabs(v) + fabs(other);
    }
  }
}

// Homogeneous spheres with the derivatives along the distribution's parameters and m. The
// chunk's coefficient rows are two halves of 16 nodes, nc rows each (lanes 0-15, then 16-31);
// a row holds the 16 nodes' (u, v) in its first 64 doubles and their derivatives along m,
// (du/dm, dv/dm), in the last 64, so that one 128-column GEMM tile carries both. The chunk's
// sums are per block: values, then each parameter of the distribution (weights
// w_j (du/dtheta)(r_j) r_j), then Re m and Im m (engine.rs:1047-1109).
__device__ __forceinline__ void mie_chunk_deriv(const MieFixedArgs& a) {
  int wslot = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (wslot >= a.n_chunks) return;
  int chunk = wslot;
  int64_t unit = a.units[chunk / a.cpu];
  int c = chunk % a.cpu;
  int64_t d = unit / a.n_wl, i = unit % a.n_wl;
  int j = c * 32 + lane;
  int nc = a.chunk_n[chunk];
  int64_t row0 = a.chunk_row[chunk];
  double* X = a.X + (row0 + (int64_t)(lane >> 4) * nc) * 128 + (lane & 15) * 4;
  Scratch s;
  s.uz = a.uz + (row0 + 2 * (int64_t)chunk) * 32 + lane;
  s.ux = a.ux + (row0 + 2 * (int64_t)chunk) * 32 + lane;
  s.stride = 32;
  const int P = a.n_theta;
  const int B = 3 + P;
  // The node's quantities, their derivatives along Re m and Im m, and the blocks' weights
  // (adaptive: and their error weights (w_K - w_G) ...).
  double qv[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  double qd[2][8] = {{0, 0, 0, 0, 0, 0, 0, 0}, {0, 0, 0, 0, 0, 0, 0, 0}};
  double wb[4] = {0, 0, 0, 0}, wbd[4] = {0, 0, 0, 0};  // values, then each parameter
  const bool adaptive = a.wdiff != nullptr;
  int64_t n = 0;
  const int64_t node = (a.per_unit ? unit : d) * a.n_nodes + j;
  if (j < a.n_nodes && a.radius[node] > 0.0) {
    const double r = a.radius[node];
    const double x = 2.0 * kPi * r / a.wl[i];
    n = default_n_max(x);
    ValueSums vs;
    DerivSums ds;
    MDeriv md;
    md.along_x = a.deriv_dir == 1;  // the x pass: derivatives along x at fixed m
    const double2 mv = a.m[unit];
    const cplx m = mk(mv.x, mv.y);
    const int st = check_node(x, m, n, a.allow_unvalidated != 0);
    double asum = 0.0;
    if (st == 0 && n <= nc) {
      mie_prepare(x, m, n, s);
      NoLayers none;
      auto emit = [&](int64_t k, cplx an, cplx bn, cplx dan, cplx dbn) {
        const bool odd = (k & 1) != 0;
        const cplx u = odd ? an : bn, v = odd ? bn : an;
        const cplx du = odd ? dan : dbn, dv = odd ? dbn : dan;
        *reinterpret_cast<double4*>(X + (k - 1) * 128) = make_double4(u.re, u.im, v.re, v.im);
        *reinterpret_cast<double4*>(X + (k - 1) * 128 + 64) =
            make_double4(du.re, du.im, dv.re, dv.im);
        ds.add(k, an, bn, dan, dbn);
      };
      asum = mie_finish(x, m, n, s, vs, emit, none, &md);
      ds.close(n);
    }
    if (st != 0 || n > nc) {
      record_error(a.err, i, d, j, a.n_dist, a.n_nodes, st != 0 ? st : 1);
      n = 0;
    } else {
      const Eff e = efficiencies_from(x, asum, vs);
      const double area = kPi * r * r;
      const double q0[8] = {1.0,           area * e.q_ext, area * e.q_sca, area * e.q_sca * e.g,
                            area * e.q_abs, area * e.q_back, r * r,         r * r * r};
      for (int k = 0; k < 8; ++k) qv[k] = q0[k];
      for (int p = 0; p < 2; ++p) {
        const Eff de = efficiency_derivs(x, vs, e, ds, p,
                                         p == 0 ? (md.along_x ? md.abs_x : md.abs_re) : md.abs_im);
        const double q1[8] = {0.0,
                              area * de.q_ext,
                              area * de.q_sca,
                              area * (de.q_sca * e.g + e.q_sca * de.g),
                              area * de.q_abs,
                              area * de.q_back,
                              0.0,
                              0.0};
        for (int k = 0; k < 8; ++k) qd[p][k] = q1[k];
      }
      wb[0] = a.weight[node];
      for (int p = 0; p < P; ++p) wb[1 + p] = a.wtheta[node * 3 + p];
      if (adaptive) {
        wbd[0] = a.wdiff[node];
        for (int p = 0; p < P; ++p) wbd[1 + p] = a.wthdiff[node * 3 + p];
      }
    }
  }
  for (int64_t k = n + 1; k <= nc; ++k) {
    *reinterpret_cast<double4*>(X + (k - 1) * 128) = make_double4(0.0, 0.0, 0.0, 0.0);
    *reinterpret_cast<double4*>(X + (k - 1) * 128 + 64) = make_double4(0.0, 0.0, 0.0, 0.0);
  }
  // Per block: the values and each parameter weight the node's quantities, Re m and Im m
  // weight its derivatives with the values' weight. The chunk's sums in a fixed tree order;
  // adaptive: then |Kronrod - Gauss| of each of the chunk's two panels (lanes 0-15, 16-31),
  // added.
  const int stride = adaptive ? 2 * B : B;
  for (int b = 0; b < B; ++b) {
    const int wi = b <= P ? b : 0;
    for (int k = 0; k < 8; ++k) {
      const double qk = b <= P ? qv[k] : qd[b - 1 - P][k];
      double v = wb[wi] * qk;
      for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
      if (lane == 0) a.chunk_sums[((int64_t)chunk * stride + b) * 8 + k] = v;
      if (adaptive) {
        double e = wbd[wi] * qk;
        for (int off = 8; off > 0; off >>= 1) e += __shfl_xor_sync(0xffffffffu, e, off);
        const double other = __shfl_sync(0xffffffffu, e, 16);
        if (lane == 0)
          a.chunk_sums[((int64_t)chunk * stride + B + b) * 8 + k] = fabs(e) + fabs(other);
      }
    }
  }
}

// Homogeneous spheres.
// 4 CTAs per SM (128 registers, 216 bytes spilled): the recurrences are latency-bound, and 16
// warps per SM hide more of it than 12 (160 registers, no spills) did: 54.4 -> 49.7 ms per step
// of the batched workload (5 CTAs, 96 registers: 60.5 ms).
__global__ void __launch_bounds__(128, 4) mie_fixed_kernel(MieFixedArgs a) {
  mie_chunk<false, false>(a);
}

// Homogeneous spheres on adaptive panels (with the chunk's |Kronrod - Gauss| sums). 4 CTAs per
// SM as mie_fixed_kernel (178 -> 128 registers): 7.8 -> 5.1 ms on a batch of 16 lognormals x 256
// wavelengths (3 CTAs: 6.0 ms).
__global__ void __launch_bounds__(128, 4) mie_adaptive_kernel(MieFixedArgs a) {
  mie_chunk<false, true>(a);
}

// Homogeneous spheres with derivatives.
__global__ void __launch_bounds__(128) mie_deriv_kernel(MieFixedArgs a) { mie_chunk_deriv(a); }

// Layered spheres with derivatives along one parameter direction (a.deriv_dir: 0..L-1 the
// complex derivative along layer l's index, then L..2L-2 along the fraction f_{l-L}): the same
// row layout and chunk sums as mie_chunk_deriv, the blocks "Re" and "Im" being the derivative
// along the direction and along i times it (meaningful for the index directions only).
// Scratch per chunk: 2 (2L - 1) arrays (the ratios and their derivatives) of nc + 2 rows.
template <int kCap>
__device__ __forceinline__ void layered_deriv_chunk(const MieFixedArgs& a) {
  int wslot = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (wslot >= a.n_chunks) return;
  int chunk = wslot;
  int64_t unit = a.units[chunk / a.cpu];
  int c = chunk % a.cpu;
  int64_t d = unit / a.n_wl, i = unit % a.n_wl;
  int j = c * 32 + lane;
  int nc = a.chunk_n[chunk];
  int64_t row0 = a.chunk_row[chunk];
  double* X = a.X + (row0 + (int64_t)(lane >> 4) * nc) * 128 + (lane & 15) * 4;
  const int L = a.n_layers, n_arr = 2 * L - 1;
  Scratch s;
  s.uz = a.uz + (row0 + 2 * (int64_t)chunk) * (2 * n_arr) * 32 + lane;
  s.ux = a.ux + (row0 + 2 * (int64_t)chunk) * 32 + lane;
  s.stride = 32;
  const int P = a.n_theta;
  const int B = 3 + P;
  // The node's quantities, their derivatives along the direction and along i times it, and
  // the blocks' weights (adaptive panels: and their error weights, as mie_chunk_deriv's).
  double qv[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  double qd[2][8] = {{0, 0, 0, 0, 0, 0, 0, 0}, {0, 0, 0, 0, 0, 0, 0, 0}};
  double wb[4] = {0, 0, 0, 0}, wbd[4] = {0, 0, 0, 0};
  const bool adaptive = a.wdiff != nullptr;
  int64_t n = 0;
  const int64_t node = (a.per_unit ? unit : d) * a.n_nodes + j;
  if (j < a.n_nodes && a.radius[node] > 0.0) {
    const double r = a.radius[node];
    const double x = 2.0 * kPi * r / a.wl[i];
    n = default_n_max(x);
    double xs[kCap];
    cplx ms[kCap];
    lder::DR xd[kCap];
    lder::DC md[kCap];
    bool lossless = true;
    const int dir = a.deriv_dir;
    for (int l = 0; l < L; ++l) {
      xs[l] = l < L - 1 ? a.fractions[d * (L - 1) + l] * x : x;
      const double2 mv = a.m_layers[(d * L + l) * a.n_wl + i];
      ms[l] = mk(mv.x, mv.y);
      lossless = lossless && mv.y == 0.0;
      xd[l] = lder::DR{xs[l], dir >= L && l == dir - L ? x : 0.0};
      md[l] = lder::DC{ms[l], rl(dir == l ? 1.0 : 0.0)};
    }
    const int st = check_layered(xs, ms, L, n, a.allow_unvalidated != 0);
    double asum = 0.0, abs_d[2] = {0.0, 0.0};
    ValueSums vs;
    DerivSums ds;
    if (st == 0 && n <= nc) {
      mie_prepare(x, ms[L - 1], n, s);  // u_k(x); array 0 is redone with its derivatives
      lder::LayeredD<kCap> lay;
      lay.layers = L;
      lay.x = xd;
      lay.m = md;
      lay.arr.arr.base = s.uz;
      lay.arr.arr.astride = (int64_t)(nc + 2) * 32;
      lay.arr.arr.stride = 32;
      lay.arr.n_val = n_arr;
      lay.prepare(n, lder::DR{x, 0.0});
      auto emit = [&](int64_t k, cplx an, cplx bn, cplx dan, cplx dbn) {
        const bool odd = (k & 1) != 0;
        const cplx u = odd ? an : bn, v = odd ? bn : an;
        const cplx du = odd ? dan : dbn, dv = odd ? dbn : dan;
        *reinterpret_cast<double4*>(X + (k - 1) * 128) = make_double4(u.re, u.im, v.re, v.im);
        *reinterpret_cast<double4*>(X + (k - 1) * 128 + 64) =
            make_double4(du.re, du.im, dv.re, dv.im);
        ds.add(k, an, bn, dan, dbn);
      };
      asum = lder::layered_finish_d(x, md[L - 1], n, s, vs, emit, lay, abs_d);
      ds.close(n);
      // A lossless particle absorbs nothing (layered/kernel.rs:455-464); its derivatives stand.
      if (lossless) asum = 0.0;
    }
    if (st != 0 || n > nc) {
      record_error(a.err, i, d, j, a.n_dist, a.n_nodes, st != 0 ? st : 1);
      n = 0;
    } else {
      const Eff e = efficiencies_from(x, asum, vs);
      const double area = kPi * r * r;
      const double q0[8] = {1.0,           area * e.q_ext, area * e.q_sca, area * e.q_sca * e.g,
                            area * e.q_abs, area * e.q_back, r * r,         r * r * r};
      for (int k = 0; k < 8; ++k) qv[k] = q0[k];
      for (int p = 0; p < 2; ++p) {
        const Eff de = efficiency_derivs(x, vs, e, ds, p, abs_d[p]);
        const double q1[8] = {0.0,
                              area * de.q_ext,
                              area * de.q_sca,
                              area * (de.q_sca * e.g + e.q_sca * de.g),
                              area * de.q_abs,
                              area * de.q_back,
                              0.0,
                              0.0};
        for (int k = 0; k < 8; ++k) qd[p][k] = q1[k];
      }
      wb[0] = a.weight[node];
      for (int p = 0; p < P; ++p) wb[1 + p] = a.wtheta[node * 3 + p];
      if (adaptive) {
        wbd[0] = a.wdiff[node];
        for (int p = 0; p < P; ++p) wbd[1 + p] = a.wthdiff[node * 3 + p];
      }
    }
  }
  for (int64_t k = n + 1; k <= nc; ++k) {
    *reinterpret_cast<double4*>(X + (k - 1) * 128) = make_double4(0.0, 0.0, 0.0, 0.0);
    *reinterpret_cast<double4*>(X + (k - 1) * 128 + 64) = make_double4(0.0, 0.0, 0.0, 0.0);
  }
  // The chunk's sums per block (values and each parameter on the values' quantities, the
  // direction's blocks on the derivatives with the values' weight) in a fixed tree order;
  // adaptive: then |Kronrod - Gauss| of each of the chunk's two panels, added.
  const int stride = adaptive ? 2 * B : B;
  for (int b = 0; b < B; ++b) {
    const int wi = b <= P ? b : 0;
    for (int k = 0; k < 8; ++k) {
      const double qk = b <= P ? qv[k] : qd[b - 1 - P][k];
      double v = wb[wi] * qk;
      for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
      if (lane == 0) a.chunk_sums[((int64_t)chunk * stride + b) * 8 + k] = v;
      if (adaptive) {
        double e = wbd[wi] * qk;
        for (int off = 8; off > 0; off >>= 1) e += __shfl_xor_sync(0xffffffffu, e, off);
        const double other = __shfl_sync(0xffffffffu, e, 16);
        if (lane == 0)
          a.chunk_sums[((int64_t)chunk * stride + B + b) * 8 + k] = fabs(e) + fabs(other);
      }
    }
  }
}

// Up to 4 layers with the per-shell state sized for them; more through the general form.
__global__ void __launch_bounds__(128) mie_layered_deriv_kernel(MieFixedArgs a) {
  layered_deriv_chunk<4>(a);
}
__global__ void __launch_bounds__(128) mie_layered_deriv16_kernel(MieFixedArgs a) {
  layered_deriv_chunk<kMaxLayers>(a);
}

// Layered spheres (their per-layer state lives in local memory).
__global__ void __launch_bounds__(128) mie_layered_kernel(MieFixedArgs a) {
  mie_chunk<true, false>(a);
}

// Layered spheres on adaptive panels.
__global__ void __launch_bounds__(128) mie_layered_adaptive_kernel(MieFixedArgs a) {
  mie_chunk<true, true>(a);
}

// Independent spheres, one per thread (the batched Mie::compute): coefficients a_1..a_N then
// b_1..b_N per sphere, and the efficiencies.
__global__ void __launch_bounds__(128) mie_nodes_kernel(MieNodesArgs a) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.n) return;
  double x = a.x[t];
  cplx m = mk(a.m[t].x, a.m[t].y);
  int64_t n = default_n_max(x);
  int st = check_node(x, m, n, a.allow_unvalidated != 0);
  if (st != 0) {
    unsigned long long key = ((unsigned long long)t << 2) | (unsigned long long)st;
    atomicMin(a.err, key);
    return;
  }
  if (a.n_terms) a.n_terms[t] = n;
  if (!a.coeffs) return;
  int64_t off = a.coeff_offset[t];
  Scratch s;
  s.uz = a.uz + off + 2 * t;
  s.ux = a.ux + off + 2 * t;
  s.stride = 1;
  mie_prepare(x, m, n, s);
  ValueSums vs;
  double2* out = reinterpret_cast<double2*>(a.coeffs) + 2 * off;
  double asum = mie_finish(x, m, n, s, vs, [&](int64_t k, cplx an, cplx bn) {
    out[k - 1] = make_double2(an.re, an.im);
    out[n + k - 1] = make_double2(bn.re, bn.im);
  });
  Eff e = efficiencies_from(x, asum, vs);
  if (a.eff) {
    a.eff[5 * t] = e.q_ext;
    a.eff[5 * t + 1] = e.q_sca;
    a.eff[5 * t + 2] = e.q_abs;
    a.eff[5 * t + 3] = e.q_back;
    a.eff[5 * t + 4] = e.g;
  }
}

// Pass 1 of the adaptive ensemble: one thread per node (engine.rs:369-449 quantities1 for
// spheres). Scratch rows scratch[t]..scratch[t+1]-1 hold u_k(mx) and u_k(x); a node whose
// number of terms does not fit them reports status 1 (the host sizes them from the same
// truncation rule with a margin).
__global__ void __launch_bounds__(128) pass1_kernel(Pass1Args a) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.n) return;
  const double r = a.radius[t];
  const int wi = a.wl_index[t];
  const double x = 2.0 * kPi * r / a.wl[wi];
  int64_t n = default_n_max(x);
  const int L = a.n_layers > 1 ? a.n_layers : 1;
  double xs[kMaxLayers];
  cplx ms[kMaxLayers];
  bool lossless = true;
  int st;
  if (L == 1) {
    ms[0] = mk(a.m[wi].x, a.m[wi].y);
    st = check_node(x, ms[0], n, a.allow_unvalidated != 0);
  } else {
    // x_l = f_l x, the outer surface's x last (ensemble/particle.rs:186-195).
    const int p = wi / a.n_wl, i = wi % a.n_wl;
    for (int l = 0; l < L; ++l) {
      xs[l] = l < L - 1 ? a.fractions[p * (L - 1) + l] * x : x;
      const double2 mv = a.m_layers[(p * L + l) * a.n_wl + i];
      ms[l] = mk(mv.x, mv.y);
      lossless = lossless && mv.y == 0.0;
    }
    st = check_layered(xs, ms, L, n, a.allow_unvalidated != 0);
  }
  const int64_t off = a.scratch[t], cap = a.scratch[t + 1] - off;
  if (st == 0 && n + 2 > cap) st = 1;
  a.status[t] = st;
  a.n_terms[t] = st == 0 ? n : 0;
  const int nq = a.deriv ? 16 : 6;
  double* q = a.q + nq * t;
  if (st != 0) {
    for (int k = 0; k < nq; ++k) q[k] = 0.0;
    return;
  }
  Scratch s;
  s.uz = a.uz + off * (2 * L - 1);
  s.ux = a.ux + off;
  s.stride = 1;
  mie_prepare(x, ms[L - 1], n, s);
  ValueSums vs;
  double asum;
  if (L == 1 && a.deriv) {
    // The derivatives of the pass-1 quantities along Re m and Im m (engine.rs:447-461).
    DerivSums ds;
    MDeriv md;
    NoLayers none;
    asum = mie_finish(
        x, ms[0], n, s, vs,
        [&](int64_t k, cplx an, cplx bn, cplx dan, cplx dbn) { ds.add(k, an, bn, dan, dbn); },
        none, &md);
    ds.close(n);
    const Eff e = efficiencies_from(x, asum, vs);
    const double area = kPi * r * r;
    for (int p = 0; p < 2; ++p) {
      const Eff d = efficiency_derivs(x, vs, e, ds, p, p == 0 ? md.abs_re : md.abs_im);
      double* o = q + 6 + 5 * p;
      o[0] = area * d.q_ext;
      o[1] = area * d.q_sca;
      o[2] = area * (d.q_sca * e.g + e.q_sca * d.g);
      o[3] = area * d.q_back;
      o[4] = area * d.q_abs;
    }
  } else if (L == 1) {
    asum = mie_finish(x, ms[0], n, s, vs, [](int64_t, cplx, cplx) {});
  } else {
    Layered lay;
    lay.layers = L;
    lay.x = xs;
    lay.m = ms;
    lay.arr.base = s.uz;
    lay.arr.astride = cap;
    lay.arr.stride = 1;
    lay.prepare(n);
    asum = mie_finish(x, ms[L - 1], n, s, vs, [](int64_t, cplx, cplx) {}, lay);
    // A lossless particle absorbs nothing (layered/kernel.rs:455-464).
    if (lossless) asum = 0.0;
  }
  const Eff e = efficiencies_from(x, asum, vs);
  const double area = kPi * r * r;
  q[0] = 1.0;
  q[1] = area * e.q_ext;
  q[2] = area * e.q_sca;
  q[3] = area * e.q_sca * e.g;
  q[4] = area * e.q_back;
  q[5] = area * e.q_abs;
}

// Pass 1 of a layered sphere's derivatives along one direction (engine.rs:447-461 with
// Solved::direction, particle.rs:206-219): one thread per node, the layered recursion in
// forward mode (layered_deriv.cuh) along a.deriv_dir; q[t] gets the node's 6 quantities and
// the derivatives of pi r^2 (Q_ext, Q_sca, Q_sca g, Q_back, Q_abs) along the direction, then
// along i times it (meaningful for an index direction only).
__global__ void __launch_bounds__(128) pass1_layered_deriv_kernel(Pass1Args a) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.n) return;
  const double r = a.radius[t];
  const int wi = a.wl_index[t];
  const double x = 2.0 * kPi * r / a.wl[wi];
  int64_t n = default_n_max(x);
  const int L = a.n_layers;
  double xs[kMaxLayers];
  cplx ms[kMaxLayers];
  bool lossless = true;
  const int p = wi / a.n_wl, i = wi % a.n_wl;
  for (int l = 0; l < L; ++l) {
    xs[l] = l < L - 1 ? a.fractions[p * (L - 1) + l] * x : x;
    const double2 mv = a.m_layers[(p * L + l) * a.n_wl + i];
    ms[l] = mk(mv.x, mv.y);
    lossless = lossless && mv.y == 0.0;
  }
  int st = check_layered(xs, ms, L, n, a.allow_unvalidated != 0);
  // The derivatives are validated up to x_L = 1000 (layered/domain.rs:39-70).
  if (st == 0 && a.allow_unvalidated == 0 && xs[L - 1] > 1e3) st = 3;
  const int64_t off = a.scratch[t], cap = a.scratch[t + 1] - off;
  if (st == 0 && n + 2 > cap) st = 1;
  a.status[t] = st;
  a.n_terms[t] = st == 0 ? n : 0;
  double* q = a.q + 16 * t;
  if (st != 0) {
    for (int k = 0; k < 16; ++k) q[k] = 0.0;
    return;
  }
  const int n_arr = 2 * L - 1, dir = a.deriv_dir;
  Scratch s;
  s.uz = a.uz + off * (2 * n_arr);
  s.ux = a.ux + off;
  s.stride = 1;
  lder::DR xd[kMaxLayers];
  lder::DC md[kMaxLayers];
  for (int l = 0; l < L; ++l) {
    xd[l] = lder::DR{xs[l], dir >= L && l == dir - L ? x : 0.0};
    md[l] = lder::DC{ms[l], rl(dir == l ? 1.0 : 0.0)};
  }
  mie_prepare(x, ms[L - 1], n, s);  // u_k(x); array 0 is redone with its derivatives
  lder::LayeredD<kMaxLayers> lay;
  lay.layers = L;
  lay.x = xd;
  lay.m = md;
  lay.arr.arr.base = s.uz;
  lay.arr.arr.astride = cap;
  lay.arr.arr.stride = 1;
  lay.arr.n_val = n_arr;
  lay.prepare(n, lder::DR{x, 0.0});
  ValueSums vs;
  DerivSums ds;
  double abs_d[2];
  double asum = lder::layered_finish_d(
      x, md[L - 1], n, s, vs,
      [&](int64_t k, cplx an, cplx bn, cplx dan, cplx dbn) { ds.add(k, an, bn, dan, dbn); }, lay,
      abs_d);
  ds.close(n);
  // A lossless particle absorbs nothing (layered/kernel.rs:455-464); its derivatives stand.
  if (lossless) asum = 0.0;
  const Eff e = efficiencies_from(x, asum, vs);
  const double area = kPi * r * r;
  q[0] = 1.0;
  q[1] = area * e.q_ext;
  q[2] = area * e.q_sca;
  q[3] = area * e.q_sca * e.g;
  q[4] = area * e.q_back;
  q[5] = area * e.q_abs;
  for (int c = 0; c < 2; ++c) {
    const Eff d = efficiency_derivs(x, vs, e, ds, c, abs_d[c]);
    double* o = q + 6 + 5 * c;
    o[0] = area * d.q_ext;
    o[1] = area * d.q_sca;
    o[2] = area * (d.q_sca * e.g + e.q_sca * d.g);
    o[3] = area * d.q_back;
    o[4] = area * d.q_abs;
  }
}

void launch_pass1_layered_deriv(const Pass1Args& a, cudaStream_t s) {
  const int threads = 128;
  const int64_t blocks = (a.n + threads - 1) / threads;
  if (blocks > 0) pass1_layered_deriv_kernel<<<(unsigned)blocks, threads, 0, s>>>(a);
}

void launch_pass1(const Pass1Args& a, cudaStream_t s) {
  const int threads = 128;
  const int64_t blocks = (a.n + threads - 1) / threads;
  if (blocks > 0) pass1_kernel<<<(unsigned)blocks, threads, 0, s>>>(a);
}

void launch_plan_chunks(const PlanArgs& a, cudaStream_t s) {
  int threads = 128;
  int blocks = (int)((a.n_chunks * 32 + threads - 1) / threads);
  plan_chunks_kernel<<<blocks, threads, 0, s>>>(a);
}

void launch_mie_fixed(const MieFixedArgs& a, cudaStream_t s) {
  int threads = 128;
  int blocks = (a.n_chunks * 32 + threads - 1) / threads;
  if (a.deriv && a.n_layers > 4)
    mie_layered_deriv16_kernel<<<blocks, threads, 0, s>>>(a);
  else if (a.deriv && a.n_layers > 1)
    mie_layered_deriv_kernel<<<blocks, threads, 0, s>>>(a);
  else if (a.deriv)
    mie_deriv_kernel<<<blocks, threads, 0, s>>>(a);
  else if (a.n_layers > 1 && a.wdiff)
    mie_layered_adaptive_kernel<<<blocks, threads, 0, s>>>(a);
  else if (a.n_layers > 1)
    mie_layered_kernel<<<blocks, threads, 0, s>>>(a);
  else if (a.wdiff)
    mie_adaptive_kernel<<<blocks, threads, 0, s>>>(a);
  else
    mie_fixed_kernel<<<blocks, threads, 0, s>>>(a);
}

void launch_mie_nodes(const MieNodesArgs& a, cudaStream_t s) {
  int threads = 128;
  int blocks = (int)((a.n + threads - 1) / threads);
  mie_nodes_kernel<<<blocks, threads, 0, s>>>(a);
}

}  // namespace sb
