// The T-matrix of spheroids by the extended boundary condition method on the GPU
// (scatrs/src/tmatrix: kernel.rs for Q and P = RgQ of each azimuthal mode by Gauss-Legendre
// quadrature over the surface, solve.rs for T = -P Q^{-1} with residual refinement,
// kernel.rs:985-1010 for the orientation-averaged cross sections), batched over spheroids
// (geometries) and their modes (jobs) in four kernels:
//
//   tm_geom_kernel     one thread per (spheroid, node): r(theta), 1/r, the normal's
//                      theta-component, the weight factor, s r, and the radial functions
//                      j_n(r), y_n(r), j_n(s r) with their [z z_n]'/z, orders 0..N;
//   tm_angular_kernel  one thread per (mode, node): the normalized d, pi, tau, orders 0..N;
//   tm_series_kernel   one thread per (spheroid, node, order): the power series of y_n(r) and
//                      j_n(s r) with their partial sums (regular.rs);
//   tm_surface_kernel  one thread per (mode, i, k): the surface integrals
//                      J[a][b]_{ik} = sum_nodes w r^2 2 pi n . (A_i x B_k) of the regular
//                      and inner vector spherical wave functions, and the y-part of the outgoing
//                      ones in the cleanest of three exact forms per element of Q;
//   tm_solve_kernel    one block per mode: Q^T and -P^T from J, an FP64 LU factorization of Q^T
//                      with partial pivoting, the solve, and residual sweeps X += LU^{-1}
//                      (-P^T - Q^T X) with the residual in double-double; then the mode's
//                      -Re tr T and sum |T|^2.
//
// Everything before the factorization is double-double (dd.cuh): the EBCM's outgoing integrals
// cancel exactly in their singular (electrostatic) terms, by up to 1e16 and more at the sizes
// and aspect ratios of the spheroid workloads (research/tmatrix/README.md, findings 1-3), and
// any pointwise error of the sampled functions or the rule is amplified by that factor.
// The y-part's singular terms are removed as the reference removes them (regular.rs:1-24,
// kernel.rs:468-490): the terms of power <= 0 (or < 0) of each radial product's Laurent series
// integrate to zero over an element, so each element keeps the form without them whose
// magnitude sum is the smallest. Carrying the functions, the Gauss-Legendre rule and the sums
// in about 106 bits leaves the elements accurate to about 1e-32 times what cancellation
// remains; the residual refinement then removes the FP64 factorization's floor (Skeel(Q)
// 2^-53, finding 4), which is what the reference's refinement (solve.rs:249-385) does. The
// vector products of the integrands are the classical ones from the definition (Mishchenko,
// Travis & Lacis 2002, section 5.8; research/tmatrix/ebcm.py).
#include <cuda_runtime.h>

#include <cstdint>

#include "dd.cuh"
#include "kernels.h"

namespace sb {

using ddm::cdd;
using ddm::dd;
using ddm::mkc;
using ddm::mkdd;

namespace {

constexpr int kNodeD = 16;  // doubles per node
constexpr int kRadD = 20;   // doubles per (node, order): j, j', y, y' (dd), w, w', w/(s r) (cdd)
constexpr int kAngD = 6;    // doubles per (node, order): d, pi, tau (dd)
constexpr double kPiHi = 3.141592653589793, kPiLo = 1.2246467991473532e-16;

__device__ __forceinline__ dd ld(const double* p) { return dd{p[0], p[1]}; }
__device__ __forceinline__ void st(double* p, dd v) {
  p[0] = v.hi;
  p[1] = v.lo;
}
__device__ __forceinline__ cdd ldc(const double* p) { return cdd{dd{p[0], p[1]}, dd{p[2], p[3]}}; }
__device__ __forceinline__ void stc(double* p, cdd v) {
  p[0] = v.re.hi;
  p[1] = v.re.lo;
  p[2] = v.im.hi;
  p[3] = v.im.lo;
}

// The largest index i in [0, n) with first(i) <= t (first ascending, first(0) = 0).
template <class F>
__device__ __forceinline__ int owner(int n, int64_t t, F first) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    if (first(mid) <= t) lo = mid; else hi = mid - 1;
  }
  return lo;
}

}  // namespace

__global__ void __launch_bounds__(128) tm_geom_kernel(TmArgs a) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.n_node_total) return;
  const int gi = owner(a.n_geoms, t, [&](int i) { return a.geoms[i].node0; });
  const TmGeom g = a.geoms[gi];
  const int q = (int)(t - g.node0), N = g.N;
  const double* rl = a.rule + 4 * (g.rule + q);
  const dd ct = ld(rl), wq = ld(rl + 2);
  const dd stt = ddm::dd_sqrt(mkdd(1.0) - ct * ct);
  // r(theta) and dr/dtheta of the spheroid with semi-axes a (equatorial) and c (ebcm.py:53-65).
  const dd A = mkdd(g.a), Cc = mkdd(g.c);
  const dd den = Cc * Cc * (stt * stt) + A * A * (ct * ct);
  const dd sden = ddm::dd_sqrt(den);
  const dd r = (A * Cc) / sden;
  const dd dr = -((A * Cc) * (Cc * Cc - A * A) * stt * ct) / (den * sden);
  const dd ir = mkdd(1.0) / r;
  double* ns = a.node + t * kNodeD;
  st(ns + 0, r);
  st(ns + 2, ir);
  st(ns + 4, -(dr * ir));
  st(ns + 6, wq * (r * r) * dd{2.0 * kPiHi, 2.0 * kPiLo});
  const cdd s = mkc(g.s_re, g.s_im);
  const cdd sr = s * r;
  stc(ns + 8, sr);
  st(ns + 12, ct);
  st(ns + 14, stt);
  double* f = a.rad + g.rad0 + (int64_t)q * (N + 1) * kRadD;
  // j_n(r): ratios rho_n = j_n / j_{n-1} = r / (2n + 1 - r rho_{n+1}) downward from far above
  // N (kept in the j slots), then values upward from j_0 = sin r / r, j_{-1} = cos r / r;
  // der_n = j_{n-1} - n j_n / r.
  dd sn, cs;
  ddm::dd_sincos(r, &sn, &cs);
  {
    const int start = N + 60 + (int)(2.0 * r.hi);
    dd rho = mkdd(0.0);
    for (int n = start; n >= 1; --n) {
      rho = r / (mkdd(2.0 * n + 1) - r * rho);
      if (n <= N) st(f + n * kRadD + 0, rho);
    }
    dd jm1 = cs * ir, j = sn * ir;
    for (int n = 0; n <= N; ++n) {
      if (n > 0) {
        const dd rn = ld(f + n * kRadD + 0);
        jm1 = j;
        j = rn * j;
      }
      st(f + n * kRadD + 0, j);
      st(f + n * kRadD + 2, jm1 - (j * ir) * (double)n);
    }
  }
  // y_n(r) upward from y_{-1} = sin r / r, y_0 = -cos r / r.
  {
    dd ym1 = sn * ir, y = -(cs * ir);
    for (int n = 0; n <= N; ++n) {
      if (n > 0) {
        const dd yn = (y * ir) * (double)(2 * n - 1) - ym1;
        ym1 = y;
        y = yn;
      }
      st(f + n * kRadD + 4, y);
      st(f + n * kRadD + 6, ym1 - (y * ir) * (double)n);
    }
  }
  // j_n(s r), its derivative term, and j_n(s r) / (s r).
  {
    const cdd isr = ddm::inv(sr);
    const double mag = fmax(fabs(sr.re.hi), fabs(sr.im.hi));
    const int start = N + 60 + (int)(2.0 * mag);
    cdd rho = mkc(0.0);
    for (int n = start; n >= 1; --n) {
      rho = sr * ddm::inv(mkc(2.0 * n + 1) - sr * rho);
      if (n <= N) stc(f + n * kRadD + 8, rho);
    }
    cdd sz, cz;
    ddm::c_sincos(sr, &sz, &cz);
    cdd jm1 = cz * isr, j = sz * isr;
    for (int n = 0; n <= N; ++n) {
      if (n > 0) {
        const cdd rn = ldc(f + n * kRadD + 8);
        jm1 = j;
        j = rn * j;
      }
      const cdd ji = j * isr;
      stc(f + n * kRadD + 8, j);
      stc(f + n * kRadD + 12, jm1 - ji * (double)n);
      stc(f + n * kRadD + 16, ji);
    }
  }
}

// Normalized d_{mn}(theta), pi = m d / sin, tau = dd/dtheta, n = 0..N, m >= 0 (ebcm.py:68-100).
__global__ void __launch_bounds__(128) tm_angular_kernel(TmArgs a) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.n_ang_total) return;
  const int ji = owner(a.n_jobs, t, [&](int i) { return a.jobs[i].ang_node0; });
  const TmJob jb = a.jobs[ji];
  const TmGeom g = a.geoms[jb.geom];
  const int q = (int)(t - jb.ang_node0), N = g.N, m = jb.m;
  const double* ns = a.node + (g.node0 + q) * kNodeD;
  const dd ct = ld(ns + 12), stt = ld(ns + 14);
  const dd ist = mkdd(1.0) / stt;
  double* f = a.ang + jb.ang0 + (int64_t)q * (N + 1) * kAngD;
  dd am = mkdd(1.0);
  for (int k = 1; k <= m; ++k) am = am * ddm::dd_sqrt(mkdd((double)(2 * k - 1)) / (double)(2 * k));
  dd sp = mkdd(1.0);
  for (int k = 0; k < m; ++k) sp = sp * stt;
  dd dprev = mkdd(0.0), dcur = mkdd(0.0);
  for (int n = 0; n <= N; ++n) {
    dd dn;
    if (n < m) dn = mkdd(0.0);
    else if (n == m) dn = am * sp;
    else if (n == m + 1) dn = ddm::dd_sqrt((double)(2 * m + 1)) * ct * dcur;
    else
      dn = ((ct * dcur) * (double)(2 * n - 1) -
            ddm::dd_sqrt((double)(n - 1) * (n - 1) - (double)m * m) * dprev) /
           ddm::dd_sqrt((double)n * n - (double)m * m);
    dd tau = mkdd(0.0), pi = mkdd(0.0);
    if (n >= (m > 1 ? m : 1)) {
      const dd prev = n - 1 >= m ? dcur : mkdd(0.0);
      tau = ((ct * dn) * (double)n - ddm::dd_sqrt((double)n * n - (double)m * m) * prev) * ist;
      pi = (dn * (double)m) * ist;
    }
    st(f + n * kAngD + 0, dn);
    st(f + n * kAngD + 2, pi);
    st(f + n * kAngD + 4, tau);
    dprev = dcur;
    dcur = dn;
  }
}

namespace {

constexpr int kMaxSeriesTerms = 4000;
// The plain form is kept only when its magnitude sum is below 2^-20 of the regularized forms':
// its integrand comes from the radial functions' recurrences, whose accumulated rounding its
// magnitude sum does not see, while the regularized forms within 2^20 of it still hold about 86
// bits against it. (At x = 25, aspect ratio 0.4 the unbiased choice left the mode-0 T-matrix's
// unitarity at 1e-3 to 1e-2, the biased one at 1e-5; at x = 21 and x = 25, aspect ratio 3,
// 5e-9 became 5e-11 and 1e-10 became 2e-12.)
constexpr double kPlainBias = 0x1p20;
constexpr double kSeriesTol = 0x1p-112;  // a term negligible against the largest at r_max

// The series table of one spheroid (tm_series_slot): j-slots of JS = 30 G + 17 doubles per
// (node h, order n), then the y-table, per (node h, kind c, index l <= G) five fields (the term
// hi, lo, the suffix sum hi, lo, the suffix magnitude sum), each over the orders 0..N.
__device__ __forceinline__ int64_t j_slot_size(int G) { return 30 * (int64_t)G + 17; }
struct JSlot {
  const double* p;
  int G;
  __device__ const double* jk(int c) const { return p + 2 + c * (10 * G + 5); }
};
struct YTab {  // the y-table of one (node, kind)
  const double* p;
  int n1;
  __device__ dd term(int l, int n) const {
    const double* q = p + (int64_t)l * 5 * n1 + n;
    return dd{q[0], q[n1]};
  }
  __device__ dd sum(int l, int n) const {
    const double* q = p + ((int64_t)l * 5 + 2) * n1 + n;
    return dd{q[0], q[n1]};
  }
  __device__ double mag(int l, int n) const { return p[((int64_t)l * 5 + 4) * n1 + n]; }
};
__device__ __forceinline__ const double* y_table(const double* ser0, int n_theta, int N, int G,
                                                 int h, int c) {
  const int n1 = N + 1;
  return ser0 + (int64_t)n_theta * n1 * j_slot_size(G) + (int64_t)(h * 3 + c) * (G + 1) * 5 * n1;
}
// The forms table after the y-table: per (node h, column order k, product slot ts < 4) ten
// fields over the row orders 0..N: the form without the powers <= 0 (re hi, lo, im hi, lo), its
// magnitude sum, the form without the powers < 0 (the same five).
__device__ __forceinline__ double* forms_slot(const double* ser0, int n_theta, int N, int G, int h,
                                              int k, int ts) {
  const int64_t n1 = N + 1;
  return const_cast<double*>(ser0) + (int64_t)n_theta * n1 * (j_slot_size(G) + 15 * (int64_t)(G + 1)) +
         (((int64_t)h * n1 + k) * 4 + ts) * 10 * n1;
}

// The number of terms of a series with term ratios x^2 / den(l), l >= 1, until the terms at
// r_max are past their peak (after l_min) and below kSeriesTol of it (regular.rs:97-124, 140-150).
template <class Den>
__device__ int series_length(double x2max, int l_min, Den den) {
  double at = 1.0, peak = 1.0;
  for (int l = 1; l < kMaxSeriesTerms; ++l) {
    const double ratio = x2max / fabs(den(l));
    at *= ratio;
    peak = fmax(peak, at);
    if (l > l_min && ratio < 0.5 && at < kSeriesTol * peak) return l + 1;
  }
  return -1;
}

}  // namespace

// The power series of the radial factors at the nodes of one half of the surface (the
// integrands of the nonzero elements are even in cos theta), one thread per (spheroid, node,
// order n >= 1) (regular.rs:1-31, 155-211, in the unscaled functions of tm_geom_kernel):
//   y_n(r) = sum_l Y_l,      Y_l = a_l r^(2l - n - 1), a_0 = -(2n - 1)!!, a_l = -a_{l-1} / (2l (2l - 2n - 1));
//   j_n(s r) = sum_i t_i,    t_i = b_i (s r)^(n + 2i), b_0 = 1 / (2n + 1)!!, b_i = -b_{i-1} / (2i (2i + 2n + 1));
// with [r y]'/r = sum (2l - n) Y_l / r, y / r = sum Y_l / r, [z j]'/z = sum (n + 2i + 1) t_i / z and
// j / z = sum t_i / z (z = s r). Kept: the y terms l < G with their suffix sums (and the sums of
// their magnitudes) l <= G, the j prefix sums i < G and suffix sums i <= G, G = N/2 + 2, which
// is every index the surface kernel's forms reach. Each suffix sum is accumulated from the
// series' far end (its terms by the backward recurrence), so that it is accurate against its
// own terms.
__global__ void __launch_bounds__(128) tm_series_kernel(TmArgs a) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.n_ser_total) return;
  const int gi = owner(a.n_geoms, t, [&](int i) { return a.geoms[i].sth0; });
  const TmGeom g = a.geoms[gi];
  const int N = g.N, G = N / 2 + 2;
  const int64_t local = t - g.sth0;
  const int h = (int)(local / N), n = 1 + (int)(local % N);
  const int64_t JS = j_slot_size(G), n1 = N + 1;
  double* p = a.ser + g.ser0 + ((int64_t)h * n1 + n) * JS;
  for (int64_t j = 0; j < JS; ++j) p[j] = 0.0;
  double* yb[3];
  for (int c = 0; c < 3; ++c) {
    yb[c] = const_cast<double*>(y_table(a.ser + g.ser0, g.n_theta, N, G, h, c)) + n;
    for (int64_t j = 0; j < 5 * (int64_t)(G + 1); ++j) yb[c][j * n1] = 0.0;
  }
  const double* ns = a.node + (g.node0 + g.n_theta + h) * kNodeD;
  const dd r = ld(ns), ir = ld(ns + 2);
  const cdd sr = ldc(ns + 8);
  const double xmax = fmax(g.a, g.c), smag2 = g.s_re * g.s_re + g.s_im * g.s_im;
  const int Ly = series_length(xmax * xmax, n, [&](int l) { return 2.0 * l * (2.0 * l - 2.0 * n - 1.0); });
  const int Lj = series_length(xmax * xmax * smag2, 0, [&](int i) { return 2.0 * i * (2.0 * i + 2.0 * n + 1.0); });
  if (Ly < 0 || Lj < 0) {
    atomicOr(a.err, 2u);
    return;
  }
  p[0] = Ly;
  p[1] = Lj;
  double* jb[3];
  for (int c = 0; c < 3; ++c) jb[c] = p + 2 + c * (10 * G + 5);
  // y: the first term, forward to the last, then back with the suffix sums.
  {
    const dd r2 = r * r, ir2 = ir * ir;
    dd v = -ir;
    for (int i = 1; i <= n; ++i) v = (v * (double)(2 * i - 1)) * ir;
    for (int l = 1; l < Ly; ++l) v = -(v * r2) / (2.0 * l * (2.0 * l - 2.0 * n - 1.0));
    dd sum[3] = {mkdd(0.0), mkdd(0.0), mkdd(0.0)};
    double mag[3] = {0.0, 0.0, 0.0};
    for (int l = Ly - 1; l >= 0; --l) {
      const dd over = v * ir;
      const dd term[3] = {v, over * (double)(2 * l - n), over};
      for (int c = 0; c < 3; ++c) {
        sum[c] = sum[c] + term[c];
        mag[c] += fabs(term[c].hi);
        if (l <= G) {
          double* e = yb[c] + (int64_t)l * 5 * n1;
          if (l < G) {
            e[0] = term[c].hi;
            e[n1] = term[c].lo;
          }
          e[2 * n1] = sum[c].hi;
          e[3 * n1] = sum[c].lo;
          e[4 * n1] = mag[c];
        }
      }
      if (l > 0) v = -(v * (2.0 * l * (2.0 * l - 2.0 * n - 1.0))) * ir2;
    }
  }
  // j(s r): the first term, forward with the prefix sums, then back with the suffix sums.
  {
    const cdd sr2 = sr * sr, isr = ddm::inv(sr), isr2 = isr * isr;
    cdd v = mkc(1.0);
    for (int i = 1; i <= n; ++i) {
      v = v * sr;
      v = cdd{v.re / (double)(2 * i + 1), v.im / (double)(2 * i + 1)};
    }
    cdd sum[3] = {mkc(0.0), mkc(0.0), mkc(0.0)};
    double mag[3] = {0.0, 0.0, 0.0};
    for (int i = 0; i < Lj; ++i) {
      if (i > 0) {
        const double den = 2.0 * i * (2.0 * i + 2.0 * n + 1.0);
        v = -(v * sr2);
        v = cdd{v.re / den, v.im / den};
      }
      if (i < G) {
        const cdd over = v * isr;
        const cdd term[3] = {v, over * (double)(n + 2 * i + 1), over};
        for (int c = 0; c < 3; ++c) {
          sum[c] = sum[c] + term[c];
          mag[c] += fabs(term[c].re.hi) + fabs(term[c].im.hi);
          stc(jb[c] + 4 * i, sum[c]);
          jb[c][4 * G + i] = mag[c];
        }
      }
    }
    for (int c = 0; c < 3; ++c) {
      sum[c] = mkc(0.0);
      mag[c] = 0.0;
    }
    for (int i = Lj - 1; i >= 0; --i) {
      const cdd over = v * isr;
      const cdd term[3] = {v, over * (double)(n + 2 * i + 1), over};
      for (int c = 0; c < 3; ++c) {
        sum[c] = sum[c] + term[c];
        mag[c] += fabs(term[c].re.hi) + fabs(term[c].im.hi);
        if (i <= G) {
          stc(jb[c] + 5 * G + 4 * i, sum[c]);
          jb[c][9 * G + 4 + i] = mag[c];
        }
      }
      if (i > 0) v = -((v * isr2) * (2.0 * i * (2.0 * i + 2.0 * n + 1.0)));
    }
  }
}

namespace {

// R+ of one radial product R_t = r^e Y_t(r) J_t(s r) of the y-part at one node: R minus the
// terms of its Laurent series in r of power <= cut, by the series of its higher powers or as
// R minus the lower ones, whichever adds less in magnitude (regular.rs:255-311). yk, jk: the
// kinds of the y_n and j_k factors (0 f, 1 [z f]'/z, 2 f/z); full = R_t at the node, xe = r^e.
__device__ __forceinline__ void reg_form(const YTab& yt, int Ly, const JSlot& sk, int Lj, int yk,
                                         int jk, int e, int n, int k, int cut, dd xe, cdd full,
                                         cdd* out, double* out_abs) {
  const double* jb = sk.jk(jk);
  const int G = sk.G;
  const int base0 = (-n - 1 - (yk > 0)) + (k - (jk > 0)) + e;
  int l_end = cut >= base0 ? (cut - base0) / 2 + 1 : 0;
  l_end = min(min(l_end, Ly), G - 1);
  cdd neg = mkc(0.0), pos = mkc(0.0);
  double neg_abs = 0.0, pos_abs = 0.0;
  for (int l = 0; l < l_end; ++l) {
    const int i_max = (cut - base0 - 2 * l) / 2;
    const dd yv = yt.term(l, n) * xe;
    const double ya = fabs(yv.hi);
    const int ii = max(min(min(i_max, Lj - 1), G - 1), 0);
    neg = ddm::add_terms(neg, ldc(jb + 4 * ii) * yv);
    neg_abs += jb[4 * G + ii] * ya;
    const int from = min(min(i_max + 1, Lj), G);
    pos = ddm::add_terms(pos, ldc(jb + 5 * G + 4 * from) * yv);
    pos_abs += jb[9 * G + 4 + from] * ya;
  }
  const dd ysum = yt.sum(l_end, n) * xe;
  pos = ddm::add_terms(pos, ldc(jb + 5 * G) * ysum);
  pos_abs += jb[9 * G + 4] * yt.mag(l_end, n) * fabs(xe.hi);
  const double sub_abs = fabs(full.re.hi) + fabs(full.im.hi) + neg_abs;
  if (pos_abs <= sub_abs) {
    *out = pos;
    *out_abs = pos_abs;
  } else {
    *out = ddm::sub_terms(full, neg);
    *out_abs = sub_abs;
  }
}

// One term c R_t of a y-part integrand (c = alpha or i alpha, im) in the three forms: plain,
// minus the powers < 0 (|n - k| >= 3) and minus the powers <= 0 (n != k), each with the sum of
// the magnitudes it adds (kernel.rs:418-442).
struct Forms3 {
  cdd v0, v1, v2;
  double a0, a1, a2;
};
// The series' view at one node for a row order n and a column order k.
struct SerView {
  YTab yt[3];  // y-table of the node per kind
  JSlot sk;    // j-slot of (node, k)
  int Ly, Lj;
};

// The radial products of an (n, k) pair's nonzero elements, by the parity of n + k, as (y kind,
// j kind, e): even (MN, NM): R_1, R_4, R_6, R_2; odd (MM, NN): R_0, R_3, R_5, R_7.
__device__ __forceinline__ void product_kind(bool even, int ts, int* yk, int* jk, int* e) {
  constexpr int kEven[4][3] = {{0, 1, 2}, {0, 2, 4}, {2, 0, 4}, {1, 0, 2}};
  constexpr int kOdd[4][3] = {{0, 0, 2}, {1, 1, 2}, {1, 2, 4}, {2, 1, 4}};
  const int* v = even ? kEven[ts] : kOdd[ts];
  *yk = v[0];
  *jk = v[1];
  *e = v[2];
}

// One term c R_t of a y-part integrand (c = alpha or i alpha, im) in the three forms: plain,
// minus the powers < 0 (|n - k| >= 3) and minus the powers <= 0 (n != k), each with the sum of
// the magnitudes it adds (kernel.rs:418-442); the regularized forms from the forms table
// (fs: the pair's slot at the node, row n at offset 0).
__device__ __forceinline__ void add_type(Forms3& f, const double* fs, int n1, int n, int k,
                                         cdd full, dd alpha, bool im, dd W) {
  const dd cw = alpha * W;
  const double ca = fabs(cw.hi);
  auto scaled = [&](cdd v) {
    const cdd x = v * cw;
    return im ? ddm::times_i(x) : x;
  };
  f.v0 = ddm::add_terms(f.v0, scaled(full));
  f.a0 += ca * (fabs(full.re.hi) + fabs(full.im.hi));
  if (n == k) return;
  auto field = [&](int j) { return fs[(int64_t)j * n1]; };
  f.v2 = ddm::add_terms(f.v2, scaled(cdd{dd{field(0), field(1)}, dd{field(2), field(3)}}));
  f.a2 += ca * field(4);
  if (abs(n - k) >= 3) {
    f.v1 = ddm::add_terms(f.v1, scaled(cdd{dd{field(5), field(6)}, dd{field(7), field(8)}}));
    f.a1 += ca * field(9);
  }
}

}  // namespace

// The regularized forms of the radial products of the y-part, which do not depend on the
// azimuthal mode: one thread per (spheroid, node of the half surface, column order k, row order
// n != k), rows fastest (the reference computes them once per node before its mode loop,
// kernel.rs:327-342). Per product of the pair's nonzero elements the forms without the powers
// <= 0 and (|n - k| >= 3) without those < 0, with their magnitude sums, into the forms table.
__global__ void __launch_bounds__(128) tm_forms_kernel(TmArgs a) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.n_forms_total) return;
  const int gi = owner(a.n_geoms, t, [&](int i) { return a.geoms[i].fth0; });
  const TmGeom g = a.geoms[gi];
  const int N = g.N, G = N / 2 + 2, nh = g.n_theta;
  const int64_t local = t - g.fth0, NN = (int64_t)N * N;
  const int h = (int)(local / NN), rem = (int)(local % NN);
  const int k = 1 + rem / N, n = 1 + rem % N;
  if (n == k) return;
  const int q = nh + h;
  const double* ser = a.ser + g.ser0;
  const int64_t JS = j_slot_size(G);
  SerView sv;
#pragma unroll
  for (int c = 0; c < 3; ++c) sv.yt[c] = YTab{y_table(ser, nh, N, G, h, c), N + 1};
  sv.sk = JSlot{ser + ((int64_t)h * (N + 1) + k) * JS, G};
  sv.Ly = (int)ser[(int64_t)n * JS];
  sv.Lj = (int)ser[(int64_t)k * JS + 1];
  const double* ns = a.node + (g.node0 + q) * kNodeD;
  const dd r = ld(ns), ir = ld(ns + 2), r2 = r * r, r4 = r2 * r2;
  const double* ri = a.rad + g.rad0 + ((int64_t)q * (N + 1) + n) * kRadD;
  const double* rk = a.rad + g.rad0 + ((int64_t)q * (N + 1) + k) * kRadD;
  const dd yr = ld(ri + 4), ydr = ld(ri + 6), yo = yr * ir;
  const cdd w = ldc(rk + 8), wd = ldc(rk + 12), u = ldc(rk + 16);
  const bool even = ((n + k) & 1) == 0;
  const int n1 = N + 1;
#pragma unroll
  for (int ts = 0; ts < 4; ++ts) {
    int yk, jk, e;
    product_kind(even, ts, &yk, &jk, &e);
    const dd yv = yk == 0 ? yr : (yk == 1 ? ydr : yo);
    const cdd jv = jk == 0 ? w : (jk == 1 ? wd : u);
    const dd xe = e == 2 ? r2 : r4;
    const cdd full = jv * (yv * xe);
    double* fs = forms_slot(ser, nh, N, G, h, k, ts) + n;
    cdd v;
    double va;
    reg_form(sv.yt[yk], sv.Ly, sv.sk, sv.Lj, yk, jk, e, n, k, 0, xe, full, &v, &va);
    fs[0] = v.re.hi;
    fs[n1] = v.re.lo;
    fs[2 * n1] = v.im.hi;
    fs[3 * n1] = v.im.lo;
    fs[4 * n1] = va;
    if (abs(n - k) >= 3) {
      reg_form(sv.yt[yk], sv.Ly, sv.sk, sv.Lj, yk, jk, e, n, k, -1, xe, full, &v, &va);
      fs[5 * n1] = v.re.hi;
      fs[6 * n1] = v.re.lo;
      fs[7 * n1] = v.im.hi;
      fs[8 * n1] = v.im.lo;
      fs[9 * n1] = va;
    }
  }
}

// The surface integrals of one (mode, i, k) (ebcm.py:103-186, pi -> -pi for the outgoing
// functions' phi-factor convention, g_i g_k taken out of the sum). With z = j_i(r) or
// i y_i(r), zeta = z or [r z]'/r, and the inner w, w' = [s r w]'/(s r), u = w/(s r) at s r, the
// triple products n . (A_i x B_k) are
//   MM = i z w (pi_i tau_k + tau_i pi_k)
//   MN = z w' (pi_i pi_k + tau_i tau_k) - nu k(k+1) z u tau_i d_k
//   NM = -z' w (tau_i tau_k + pi_i pi_k) + nu i(i+1) (z/r) w d_i tau_k
//   NN = i [z' w' (tau_i pi_k + pi_i tau_k) - nu (k(k+1) z' u pi_i d_k + i(i+1) (z/r) w' d_i pi_k)]
// where nu = -r'/r = nu' r^2, nu' = -beta sin cos (1/r^2 = alpha + beta cos^2). MN and NM are even
// in cos theta when i + k is even and odd otherwise, MM and NN the reverse: each (i, k) has two
// nonzero integrals, taken over the half cos theta > 0 of the rule and doubled; the other two
// are exactly zero.
//
// Out: J[0..3] = the regular (z = j) MM, MN, NM, NN; J[4 + 2 bi + bk] = the y-part (z = i y) of
// the element (bi, bk) of Q, -i s J_a - i J_b (tm_solve_kernel's pairs), in the cleanest of its
// three exact forms (kernel.rs:468-490): per type t the radial product R_t = r^e Y_t J_t has
// powers of r whose terms <= 0 integrate, over the element's four types together, to zero when
// i != k, and those < 0 when |i - k| >= 3 (the spheroid's 1/r^2 is a polynomial in cos theta);
// removing them removes the catastrophic cancellation of the plain integrals. The form whose
// magnitude sum is the smallest is kept.
__global__ void __launch_bounds__(128) tm_surface_kernel(TmArgs a) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.n_pair_total) return;
  const int ji = owner(a.n_jobs, t, [&](int i) { return a.jobs[i].pair0; });
  const TmJob jb = a.jobs[ji];
  const TmGeom g = a.geoms[jb.geom];
  const int N = g.N, m = jb.m, n0 = m > 1 ? m : 1, K = jb.K;
  // Rows fastest: a warp's threads share the column order k, so its j-slot, and read the
  // y-table's consecutive orders.
  const int pr = (int)(t - jb.pair0), i = n0 + pr % K, k = n0 + pr / K;
  const bool even = ((i + k) & 1) == 0;
  const int G = N / 2 + 2;
  const double* ser = a.ser + g.ser0;
  cdd R0 = mkc(0.0), R1 = mkc(0.0);  // regular: MN, NM (even) or MM, NN (odd)
  Forms3 Y0, Y1;                     // y-part: the same two
  Y0.v0 = Y0.v1 = Y0.v2 = Y1.v0 = Y1.v1 = Y1.v2 = mkc(0.0);
  Y0.a0 = Y0.a1 = Y0.a2 = Y1.a0 = Y1.a1 = Y1.a2 = 0.0;

  const double cki = (double)i * (i + 1), ckk = (double)k * (k + 1);
  const int nh = g.n_theta;
  for (int h = 0; h < nh; ++h) {
    const int q = nh + h;
    const double* ns = a.node + (g.node0 + q) * kNodeD;
    const dd ir = ld(ns + 2), nu = ld(ns + 4), fac = ld(ns + 6) * 2.0;
    const dd r = ld(ns), r2 = r * r, r4 = r2 * r2, ir2 = ir * ir;
    const dd W = fac * ir2, nup = nu * ir2;
    const double* ri = a.rad + g.rad0 + ((int64_t)q * (N + 1) + i) * kRadD;
    const double* rk = a.rad + g.rad0 + ((int64_t)q * (N + 1) + k) * kRadD;
    const double* ai = a.ang + jb.ang0 + ((int64_t)q * (N + 1) + i) * kAngD;
    const double* ak = a.ang + jb.ang0 + ((int64_t)q * (N + 1) + k) * kAngD;
    const dd di = ld(ai), pii = ld(ai + 2), ti = ld(ai + 4);
    const dd dk = ld(ak), pik = ld(ak + 2), tk = ld(ak + 4);
    const cdd w = ldc(rk + 8), wd = ldc(rk + 12), u = ldc(rk + 16);
    const dd jr = ld(ri), jdr = ld(ri + 2), yr = ld(ri + 4), ydr = ld(ri + 6);
    const dd yo = yr * ir;  // y / r
    const int n1 = N + 1;
    const double* fs = forms_slot(ser, nh, N, G, h, k, 0) + i;  // product slot ts at ts 10 n1
    if (even) {
      const dd A2 = ddm::add_terms(pii * pik, ti * tk), A3 = ti * dk, A4 = di * tk;
      // Regular: MN = j w' A2 - nu k(k+1) j u A3, NM = nu i(i+1) (j/r) w A4 - j' w A2.
      const cdd mn = ddm::sub_terms(wd * (jr * A2), u * ((jr * A3) * (nu * ckk)));
      const cdd nm = ddm::sub_terms(w * (((jr * ir) * A4) * (nu * cki)), w * (jdr * A2));
      R0 = ddm::add_terms(R0, mn * fac);
      R1 = ddm::add_terms(R1, nm * fac);
      // y-part: MN = i A2 R_1 - i k(k+1) A3 nu' R_4, NM = i i(i+1) A4 nu' R_6 - i A2 R_2.
      add_type(Y0, fs, n1, i, k, wd * (yr * r2), A2, true, W);
      add_type(Y0, fs + 10 * n1, n1, i, k, u * (yr * r4), -((A3 * nup) * ckk), true, W);
      add_type(Y1, fs + 20 * n1, n1, i, k, w * (yo * r4), (A4 * nup) * cki, true, W);
      add_type(Y1, fs + 30 * n1, n1, i, k, w * (ydr * r2), -A2, true, W);
    } else {
      const dd A1 = ddm::add_terms(pii * tk, ti * pik), A5 = pii * dk, A6 = di * pik;
      // Regular: MM = i j w A1, NN = i [j' w' A1 - nu (k(k+1) j' u A5 + i(i+1) (j/r) w' A6)].
      const cdd mm = ddm::times_i(w * (jr * A1));
      const cdd nn = ddm::times_i(ddm::sub_terms(
          wd * (jdr * A1),
          ddm::add_terms(u * ((jdr * A5) * ckk), wd * (((jr * ir) * A6) * cki)) * nu));
      R0 = ddm::add_terms(R0, mm * fac);
      R1 = ddm::add_terms(R1, nn * fac);
      // y-part: MM = -A1 R_0, NN = -A1 R_3 + k(k+1) A5 nu' R_5 + i(i+1) A6 nu' R_7.
      add_type(Y0, fs, n1, i, k, w * (yr * r2), -A1, false, W);
      add_type(Y1, fs + 10 * n1, n1, i, k, wd * (ydr * r2), -A1, false, W);
      add_type(Y1, fs + 20 * n1, n1, i, k, u * (ydr * r4), (A5 * nup) * ckk, false, W);
      add_type(Y1, fs + 30 * n1, n1, i, k, wd * (yo * r4), (A6 * nup) * cki, false, W);
    }
  }
  // g_i g_k = sqrt((2i+1)(2k+1) / (16 pi^2 i(i+1) k(k+1))).
  const dd pi2 = dd{kPiHi, kPiLo} * dd{kPiHi, kPiLo};
  const dd gg = ddm::dd_sqrt((mkdd((double)(2 * i + 1) * (2 * k + 1)) / (pi2 * 16.0)) /
                             (cki * ckk));
  // The two elements of Q this (i, k) feeds, with s on the first of their pair:
  // even: (0, 0) = -i s MN - i NM, (1, 1) = -i s NM - i MN; odd: (0, 1) = -i s MM - i NN,
  // (1, 0) = -i s NN - i MM.
  const cdd s = mkc(g.s_re, g.s_im), mis = -ddm::times_i(s);
  const double sa = fabs(g.s_re) + fabs(g.s_im);
  auto element = [&](const Forms3& first, const Forms3& second) {
    int best = 0;
    if (a.form >= 0) {
      if (a.form == 2 && i != k) best = 2;
      if (a.form == 1 && abs(i - k) >= 3) best = 1;
    } else if (i != k) {
      const double m2 = sa * first.a2 + second.a2;
      double mb = kPlainBias * (sa * first.a0 + second.a0);
      if (m2 < mb) {
        best = 2;
        mb = m2;
      }
      if (abs(i - k) >= 3 && sa * first.a1 + second.a1 < mb) best = 1;
    }
    const cdd fv = best == 0 ? first.v0 : (best == 1 ? first.v1 : first.v2);
    const cdd sv = best == 0 ? second.v0 : (best == 1 ? second.v1 : second.v2);
    return ddm::add_terms(mis * fv, ddm::times_i(sv) * -1.0) * gg;
  };
  cdd out[8];
#pragma unroll
  for (int c = 0; c < 8; ++c) out[c] = mkc(0.0);
  if (even) {
    out[1] = R0 * gg;
    out[2] = R1 * gg;
    out[4 + 0] = element(Y0, Y1);
    out[4 + 3] = element(Y1, Y0);
  } else {
    out[0] = R0 * gg;
    out[3] = R1 * gg;
    out[4 + 1] = element(Y0, Y1);
    out[4 + 2] = element(Y1, Y0);
  }
  double* o = a.J + 4 * jb.J0;
  const int64_t KK = (int64_t)K * K, e = (int64_t)(i - n0) * K + (k - n0);
#pragma unroll
  for (int c = 0; c < 8; ++c) stc(o + 4 * (c * KK + e), out[c]);
}
namespace {

struct Cd {  // complex double
  double re, im;
};
__device__ __forceinline__ Cd cmul(Cd a, Cd b) {
  return Cd{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
__device__ __forceinline__ Cd csub(Cd a, Cd b) { return Cd{a.re - b.re, a.im - b.im}; }
__device__ __forceinline__ Cd cdiv(Cd a, Cd b) {
  const double s = fmax(fabs(b.re), fabs(b.im));
  const Cd bs{b.re / s, b.im / s};
  const double d = bs.re * bs.re + bs.im * bs.im;
  const Cd as{a.re / s, a.im / s};
  return Cd{(as.re * bs.re + as.im * bs.im) / d, (as.im * bs.re - as.re * bs.im) / d};
}

// Block-wide max of v (blockDim.x = 256) through red; every thread gets the result.
__device__ double block_max(double v, double* red) {
  const int t = threadIdx.x;
  red[t] = v;
  __syncthreads();
  for (int off = 128; off > 0; off >>= 1) {
    if (t < off) red[t] = fmax(red[t], red[t + off]);
    __syncthreads();
  }
  const double r = red[0];
  __syncthreads();
  return r;
}

// Applies the LU factors (row swaps piv in order, unit L, U) to column c of X (row-major n2 x n2
// complex doubles), one column per thread.
__device__ void lu_apply(const Cd* A, const int* piv, Cd* X, int n2, int c) {
  for (int k = 0; k < n2; ++k) {
    const int p = piv[k];
    if (p != k) {
      const Cd x = X[(int64_t)k * n2 + c];
      X[(int64_t)k * n2 + c] = X[(int64_t)p * n2 + c];
      X[(int64_t)p * n2 + c] = x;
    }
  }
  for (int i = 1; i < n2; ++i) {
    Cd v = X[(int64_t)i * n2 + c];
    for (int j = 0; j < i; ++j) v = csub(v, cmul(A[(int64_t)i * n2 + j], X[(int64_t)j * n2 + c]));
    X[(int64_t)i * n2 + c] = v;
  }
  for (int i = n2 - 1; i >= 0; --i) {
    Cd v = X[(int64_t)i * n2 + c];
    for (int j = i + 1; j < n2; ++j)
      v = csub(v, cmul(A[(int64_t)i * n2 + j], X[(int64_t)j * n2 + c]));
    X[(int64_t)i * n2 + c] = cdiv(v, A[(int64_t)i * n2 + i]);
  }
}

}  // namespace

// One mode per block of 256 threads. Workspace (doubles): Q^T and -P^T as complex double-double
// (4 (2K)^2 each), the LU factors, X and the residual as complex doubles (2 (2K)^2 each).
__global__ void __launch_bounds__(256) tm_solve_kernel(TmArgs a) {
  __shared__ double red_v[256];
  __shared__ int red_i[256];
  __shared__ double sums[2][256];
  const TmJob jb = a.jobs[blockIdx.x];
  const TmGeom g = a.geoms[jb.geom];
  const int t = threadIdx.x;
  const int K = jb.K, n2 = 2 * K;
  const int64_t KK = (int64_t)K * K, NN = (int64_t)n2 * n2;
  const double* J = a.J + 4 * jb.J0;
  double* Qd = a.work + jb.W0;  // Q^T, dd complex
  double* Bd = Qd + 4 * NN;     // -P^T, dd complex
  Cd* A = reinterpret_cast<Cd*>(Bd + 4 * NN);
  Cd* X = A + NN;
  Cd* R = X + NN;
  int* piv = a.piv + jb.piv0;
  const cdd s = mkc(g.s_re, g.s_im);
  const cdd mis = -ddm::times_i(s), mi = mkc(0.0, -1.0);
  auto Jv = [&](int o, int p, int b, int64_t e) { return ldc(J + 4 * (((o * 2 + p) * 2 + b) * KK + e)); };
  // RgQ11 = -i s J12 - i J21, RgQ12 = -i s J11 - i J22, RgQ21 = -i s J22 - i J11,
  // RgQ22 = -i s J21 - i J12 (ebcm.py:189-195) of the regular J, and Q = RgQ + its y-part
  // (tm_surface_kernel); element (row, col) of Q goes to (col, row).
  for (int64_t idx = t; idx < NN; idx += blockDim.x) {
    const int row = (int)(idx / n2), col = (int)(idx % n2);
    const int bi = row >= K, bk = col >= K;
    const int64_t e = (int64_t)(row - bi * K) * K + (col - bk * K);
    cdd q[2];
    if (!bi && !bk) q[0] = mis * Jv(0, 0, 1, e) + mi * Jv(0, 1, 0, e);
    else if (!bi && bk) q[0] = mis * Jv(0, 0, 0, e) + mi * Jv(0, 1, 1, e);
    else if (bi && !bk) q[0] = mis * Jv(0, 1, 1, e) + mi * Jv(0, 0, 0, e);
    else q[0] = mis * Jv(0, 1, 0, e) + mi * Jv(0, 0, 1, e);
    q[1] = q[0] + Jv(1, bi, bk, e);
    const int64_t tr = (int64_t)col * n2 + row;
    stc(Qd + 4 * tr, q[1]);
    stc(Bd + 4 * tr, -q[0]);
    A[tr] = Cd{q[1].re.hi + q[1].re.lo, q[1].im.hi + q[1].im.lo};
    X[tr] = Cd{-(q[0].re.hi + q[0].re.lo), -(q[0].im.hi + q[0].im.lo)};
  }
  __syncthreads();
  // Each equation scaled by the power of two that brings its largest coefficient to [1, 2):
  // the unscaled radial functions give the rows magnitudes over hundreds of decades, and
  // partial pivoting is only as good as the rows' balance. Exact, and the solution is unchanged.
  for (int r = t; r < n2; r += blockDim.x) {
    double mx = 0.0;
    for (int c = 0; c < n2; ++c) {
      const Cd v = A[(int64_t)r * n2 + c];
      mx = fmax(mx, fmax(fabs(v.re), fabs(v.im)));
    }
    if (!(mx > 0.0) || !isfinite(mx)) continue;
    const int e = -ilogb(mx);
    for (int c = 0; c < n2; ++c) {
      const int64_t idx = (int64_t)r * n2 + c;
      A[idx] = Cd{ldexp(A[idx].re, e), ldexp(A[idx].im, e)};
      X[idx] = Cd{ldexp(X[idx].re, e), ldexp(X[idx].im, e)};
      for (int p = 0; p < 4; ++p) {
        Qd[4 * idx + p] = ldexp(Qd[4 * idx + p], e);
        Bd[4 * idx + p] = ldexp(Bd[4 * idx + p], e);
      }
    }
  }
  __syncthreads();
  // LU of A with partial pivoting (the largest modulus, the first row on ties).
  for (int kk = 0; kk < n2; ++kk) {
    double best = -1.0;
    int bi = kk;
    for (int r = kk + t; r < n2; r += blockDim.x) {
      const Cd v = A[(int64_t)r * n2 + kk];
      const double mag = hypot(v.re, v.im);
      if (mag > best) {
        best = mag;
        bi = r;
      }
    }
    red_v[t] = best;
    red_i[t] = bi;
    __syncthreads();
    for (int off = 128; off > 0; off >>= 1) {
      if (t < off) {
        const double ov = red_v[t + off];
        const int oi = red_i[t + off];
        if (ov > red_v[t] || (ov == red_v[t] && oi < red_i[t])) {
          red_v[t] = ov;
          red_i[t] = oi;
        }
      }
      __syncthreads();
    }
    const int p = red_i[0];
    const bool singular = !(red_v[0] > 0.0);
    __syncthreads();
    if (singular) {
      if (t == 0) atomicExch(a.err, 1u);
      return;
    }
    if (t == 0) piv[kk] = p;
    if (p != kk)
      for (int c = t; c < n2; c += blockDim.x) {
        const Cd x = A[(int64_t)kk * n2 + c];
        A[(int64_t)kk * n2 + c] = A[(int64_t)p * n2 + c];
        A[(int64_t)p * n2 + c] = x;
      }
    __syncthreads();
    const Cd pv = A[(int64_t)kk * n2 + kk];
    for (int r = kk + 1 + t; r < n2; r += blockDim.x)
      A[(int64_t)r * n2 + kk] = cdiv(A[(int64_t)r * n2 + kk], pv);
    __syncthreads();
    const int w = n2 - kk - 1;
    for (int idx = t; idx < w * w; idx += blockDim.x) {
      const int r = kk + 1 + idx / w, c = kk + 1 + idx % w;
      A[(int64_t)r * n2 + c] =
          csub(A[(int64_t)r * n2 + c], cmul(A[(int64_t)r * n2 + kk], A[(int64_t)kk * n2 + c]));
    }
    __syncthreads();
  }
  for (int c = t; c < n2; c += blockDim.x) lu_apply(A, piv, X, n2, c);
  __syncthreads();
  // Residual sweeps: R = -P^T - Q^T X with the products and sums in double-double.
  double rel = 0.0;
  for (int sweep = 0; sweep < a.max_sweeps; ++sweep) {
    double xm = 0.0, rm = 0.0;
    for (int64_t idx = t; idx < NN; idx += blockDim.x) {
      const int i = (int)(idx / n2), c = (int)(idx % n2);
      cdd acc = ldc(Bd + 4 * idx);
      const double* qrow = Qd + 4 * (int64_t)i * n2;
      for (int j = 0; j < n2; ++j) {
        const cdd qv = ldc(qrow + 4 * j);
        const Cd x = X[(int64_t)j * n2 + c];
        // The residual's accuracy is measured against its terms (2^-106 of |Q^T| |X|), as
        // mixed-precision refinement needs.
        acc = ddm::sub_terms(acc, cdd{ddm::add_terms(qv.re * x.re, -(qv.im * x.im)),
                                      ddm::add_terms(qv.re * x.im, qv.im * x.re)});
      }
      const Cd rv{acc.re.hi + acc.re.lo, acc.im.hi + acc.im.lo};
      R[idx] = rv;
      const Cd xv = X[idx];
      xm = fmax(xm, fmax(fabs(xv.re), fabs(xv.im)));
    }
    __syncthreads();
    for (int c = t; c < n2; c += blockDim.x) lu_apply(A, piv, R, n2, c);
    __syncthreads();
    for (int64_t idx = t; idx < NN; idx += blockDim.x) {
      const Cd d = R[idx];
      rm = fmax(rm, fmax(fabs(d.re), fabs(d.im)));
      X[idx] = Cd{X[idx].re + d.re, X[idx].im + d.im};
    }
    xm = block_max(xm, red_v);
    rm = block_max(rm, red_v);
    rel = xm > 0.0 ? rm / xm : 0.0;
    if (!(rel > 0x1p-54)) break;
  }
  // T[i][k] = X[k][i].
  double ext = 0.0, sca = 0.0;
  double* T = a.T ? a.T + 2 * jb.T0 : nullptr;
  for (int64_t idx = t; idx < NN; idx += blockDim.x) {
    const int i = (int)(idx / n2), k = (int)(idx % n2);
    const Cd v = X[(int64_t)k * n2 + i];
    if (T) {
      T[2 * idx] = v.re;
      T[2 * idx + 1] = v.im;
    }
    if (i == k) ext -= v.re;
    sca += v.re * v.re + v.im * v.im;
  }
  sums[0][t] = ext;
  sums[1][t] = sca;
  __syncthreads();
  for (int off = 128; off > 0; off >>= 1) {
    if (t < off) {
      sums[0][t] += sums[0][t + off];
      sums[1][t] += sums[1][t + off];
    }
    __syncthreads();
  }
  if (t == 0) {
    a.sums[3 * blockIdx.x] = sums[0][0];
    a.sums[3 * blockIdx.x + 1] = sums[1][0];
    a.sums[3 * blockIdx.x + 2] = rel;
  }
}

void launch_tm_tables(const TmArgs& a, cudaStream_t s) {
  if (a.n_jobs <= 0) return;
  tm_geom_kernel<<<(unsigned)((a.n_node_total + 127) / 128), 128, 0, s>>>(a);
  tm_angular_kernel<<<(unsigned)((a.n_ang_total + 127) / 128), 128, 0, s>>>(a);
  if (a.n_ser_total > 0)
    tm_series_kernel<<<(unsigned)((a.n_ser_total + 127) / 128), 128, 0, s>>>(a);
  if (a.n_forms_total > 0)
    tm_forms_kernel<<<(unsigned)((a.n_forms_total + 127) / 128), 128, 0, s>>>(a);
}
void launch_tm_surface(const TmArgs& a, cudaStream_t s) {
  if (a.n_jobs <= 0) return;
  tm_surface_kernel<<<(unsigned)((a.n_pair_total + 127) / 128), 128, 0, s>>>(a);
}
void launch_tm_solve(const TmArgs& a, cudaStream_t s) {
  if (a.n_jobs <= 0) return;
  tm_solve_kernel<<<a.n_jobs, 256, 0, s>>>(a);
}
void launch_tmatrix(const TmArgs& a, cudaStream_t s) {
  launch_tm_tables(a, s);
  launch_tm_surface(a, s);
  launch_tm_solve(a, s);
}

}  // namespace sb
