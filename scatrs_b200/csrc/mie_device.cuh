// Device-side Mie arithmetic for one size node per thread: complex numbers in num-complex's
// operation order, the reference's complex reciprocal, the start index of the downward
// recurrences and the truncation rule. Translation units including this header are compiled
// with -fmad=false, so every a*b+c rounds twice as the reference's Rust does; the coefficients
// then match the reference's bit for bit wherever the device's sin, cos, cbrt, log2 and pow
// return the same doubles as the host's libm.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace sb {

constexpr double kPi = 3.14159265358979323846264338327950288;
constexpr double kEps = 2.220446049250313e-16;  // 2^-52

struct cplx {
  double re, im;
};
__device__ __forceinline__ cplx mk(double r, double i) { return {r, i}; }
__device__ __forceinline__ cplx rl(double v) { return {v, 0.0}; }
__device__ __forceinline__ cplx operator+(cplx a, cplx b) { return {a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ cplx operator-(cplx a, cplx b) { return {a.re - b.re, a.im - b.im}; }
__device__ __forceinline__ cplx operator-(cplx a) { return {-a.re, -a.im}; }
__device__ __forceinline__ cplx operator*(cplx a, cplx b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
__device__ __forceinline__ cplx scl(cplx a, double t) { return {a.re * t, a.im * t}; }
// i u (complex.rs:43-45).
__device__ __forceinline__ cplx cti(cplx u) { return {-u.im, u.re}; }
__device__ __forceinline__ double nsq(cplx a) { return a.re * a.re + a.im * a.im; }
__device__ __forceinline__ double cabs_(cplx a) { return hypot(a.re, a.im); }
__device__ __forceinline__ double re_mul_conj(cplx u, cplx v) { return u.re * v.re + u.im * v.im; }

// 1/z as scatrs/src/complex.rs:21-38: one division where 1e-300 < |z|^2 < 1e300 and
// Im z != 0, Smith's algorithm otherwise.
__device__ __forceinline__ cplx cinv(cplx z) {
  double c = z.re, d = z.im;
  double s = c * c + d * d;
  if (s > 1e-300 && s < 1e300 && d != 0.0) {
    double t = 1.0 / s;
    return {c * t, -(d * t)};
  }
  if (fabs(d) <= fabs(c)) {
    double r = d / c;
    double t = 1.0 / (c + d * r);
    return {t, -(r * t)};
  }
  double r = c / d;
  double t = 1.0 / (c * r + d);
  return {r * t, -t};
}

// ceil(x + 6 x^(1/3) + 3), the f64 truncation (scatrs/src/mie/mod.rs:122-145).
__device__ __forceinline__ int64_t default_n_max(double x) {
  double n = ceil(x + 6.0 * cbrt(x) + 3.0);
  if (isfinite(n) && n < 9007199254740992.0) return (int64_t)n;
  return INT64_MAX;
}

// The start of a downward ratio recurrence that reaches n_top with its start value forgotten
// to rounding level (scatrs/src/mie/kernel.rs:99-112), 52 bits, margin 30.
__device__ __forceinline__ int64_t start_index(int64_t n_top, double rho_abs) {
  const double bits = 52.0;
  double c15 = ceil(1.5 * rho_abs);
  int64_t k0 = n_top > (int64_t)c15 ? n_top : (int64_t)c15;
  double q = (double)(2 * k0 + 1) / rho_abs - 0.5;
  int64_t enclosed = k0 + (int64_t)ceil(bits / (2.0 * log2(q))) + 2;
  if ((double)n_top >= 1.5 * rho_abs) return enclosed;
  double s0 = (double)n_top - rho_abs;
  double s0_32 = s0 > 0.0 ? s0 * sqrt(s0) : 0.0;
  double s = pow(s0_32 + 1.4 * 0.37 * bits * sqrt(rho_abs), 2.0 / 3.0);
  int64_t asymptotic = (int64_t)ceil(rho_abs + s) + 30;
  return asymptotic < enclosed ? asymptotic : enclosed;
}

// One downward step u_k = 1/((2k+1)/z - u_{k+1}) (kernel.rs:116-125).
__device__ __forceinline__ cplx step_complex(int64_t k, cplx inv_z, cplx u) {
  cplx c = scl(inv_z, (double)(2 * k + 1));
  cplx den = c - u;
  if (den.re == 0.0 && den.im == 0.0) den = rl(kEps * (cabs_(c) + cabs_(u)));
  return cinv(den);
}

// The real form (kernel.rs:129-136).
__device__ __forceinline__ double step_real(int64_t k, double inv_rho, double u) {
  double c = inv_rho * (double)(2 * k + 1);
  double den = c - u;
  if (den == 0.0) den = kEps * (fabs(c) + fabs(u));
  return 1.0 / den;
}

// The last order of the upward psi/chi recurrences (kernel.rs:208-215).
__device__ __forceinline__ int64_t upward_orders(double x, int64_t n) {
  if (x >= 1.0) {
    int64_t f = (int64_t)floor(x);
    return f < n ? f : n;
  }
  return 0;
}

// Input checks of Mie::compute (scatrs/src/mie/mod.rs:274-320) with the default truncation:
// 0 when accepted, else the status (1 invalid input, 3 outside the validated domain).
__device__ __forceinline__ int check_node(double x, cplx m, int64_t n, bool allow_unvalidated) {
  if (!(x >= 1e-30 && x <= 1e6)) return 1;
  if (!(isfinite(m.re) && isfinite(m.im))) return 1;
  if (m.re < 0.0 || m.im < 0.0) return 1;
  double abs_m = hypot(m.re, m.im);
  if (!(abs_m >= 1e-6 && abs_m <= 1e3)) return 1;
  if (n == 0 || n > (1 << 20)) return 1;
  if (!allow_unvalidated) {
    bool in = x >= 1e-6 && x <= 2e4 && m.re > 0.0 && m.re <= 10.0 && m.im >= 0.0 &&
              m.im <= 10.0 && abs_m >= 0.1;
    if (!in) return 3;
  }
  return 0;
}

// Per-node scratch of the downward recurrences: u_k(mx) and u_k(x) at order k, strided so that
// the lanes of a warp touch consecutive addresses.
struct Scratch {
  double2* uz;
  double* ux;
  int stride;  // lanes sharing the rows
  __device__ __forceinline__ void put_z(int64_t k, cplx v) const {
    uz[k * stride] = make_double2(v.re, v.im);
  }
  __device__ __forceinline__ cplx get_z(int64_t k) const {
    double2 v = uz[k * stride];
    return {v.x, v.y};
  }
  __device__ __forceinline__ void put_x(int64_t k, double v) const { ux[k * stride] = v; }
  __device__ __forceinline__ double get_x(int64_t k) const { return ux[k * stride]; }
};

// State::prepare (kernel.rs:249-313): u_k(mx) for k = 1..n+1 and u_k(x) for the orders above
// the upward recurrences. The two recurrences are independent; they run one after the other.
__device__ __forceinline__ void mie_prepare(double x, cplx m, int64_t n, const Scratch& s) {
  int64_t n_s = upward_orders(x, n);
  int64_t top = n + 1;
  if (n_s < n) {
    int64_t start = start_index(top, fabs(x));
    int64_t lo = n_s + 1 > 1 ? n_s + 1 : 1;
    double inv_x = 1.0 / x;
    double ux = 0.0;
    for (int64_t k = start; k >= lo; --k) {
      ux = step_real(k, inv_x, ux);
      if (k <= top) s.put_x(k, ux);
    }
  }
  cplx z = scl(m, x);
  if (m.im == 0.0) {
    double inv_rho = 1.0 / z.re;
    double u = 0.0;
    int64_t start = start_index(top, fabs(z.re));
    for (int64_t k = start; k >= 1; --k) {
      u = step_real(k, inv_rho, u);
      if (k <= top) s.put_z(k, rl(u));
    }
  } else {
    cplx inv_z = cinv(z);
    cplx u = rl(0.0);
    int64_t start = start_index(top, cabs_(z));
    for (int64_t k = start; k >= 1; --k) {
      u = step_complex(k, inv_z, u);
      if (k <= top) s.put_z(k, u);
    }
  }
}

// Running sums of value_sums (scatrs/src/mie/efficiencies.rs:64-84), fed one order at a time
// in the reference's order of operations.
struct ValueSums {
  double sca = 0.0, g = 0.0;
  cplx back = {0.0, 0.0};
  cplx a_prev = {0.0, 0.0}, b_prev = {0.0, 0.0};
  // Order k's coefficients arrive; the pair and own terms of order k-1 follow.
  __device__ __forceinline__ void add(int64_t k, cplx ak, cplx bk) {
    if (k > 1) {
      double kf = (double)(k - 1);
      double w1 = (double)(2 * (k - 1) + 1);
      g += kf * (kf + 2.0) / (kf + 1.0) * (re_mul_conj(a_prev, ak) + re_mul_conj(b_prev, bk));
      g += w1 / (kf * (kf + 1.0)) * re_mul_conj(a_prev, b_prev);
    }
    double w = (double)(2 * k + 1);
    sca += w * (nsq(ak) + nsq(bk));
    cplx t = scl(ak - bk, w);
    back = (k % 2 == 0) ? back + t : back - t;
    a_prev = ak;
    b_prev = bk;
  }
  // After the last order n: its own term.
  __device__ __forceinline__ void close(int64_t n) {
    if (n >= 1) {
      double kf = (double)n;
      double w = (double)(2 * n + 1);
      g += w / (kf * (kf + 1.0)) * re_mul_conj(a_prev, b_prev);
    }
  }
};

struct Eff {
  double q_ext, q_sca, q_abs, q_back, g;
};

// Running sums of derivative_sums (efficiencies.rs:89-146) along Re m (p = 0) and Im m (p = 1,
// where d/d(Im m) = i d/dm), fed one order at a time like ValueSums.
struct DerivSums {
  double sca[2] = {0.0, 0.0}, g[2] = {0.0, 0.0};
  cplx back[2] = {{0.0, 0.0}, {0.0, 0.0}};
  cplx a_prev = {0.0, 0.0}, b_prev = {0.0, 0.0}, da_prev = {0.0, 0.0}, db_prev = {0.0, 0.0};
  __device__ __forceinline__ void add(int64_t k, cplx ak, cplx bk, cplx dak, cplx dbk) {
    const cplx dA[2] = {dak, cti(dak)}, dB[2] = {dbk, cti(dbk)};
    if (k > 1) {
      const double kf = (double)(k - 1);
      const double pair = kf * (kf + 2.0) / (kf + 1.0);
      const double own = (double)(2 * (k - 1) + 1) / (kf * (kf + 1.0));
      const cplx pA[2] = {da_prev, cti(da_prev)}, pB[2] = {db_prev, cti(db_prev)};
#pragma unroll
      for (int p = 0; p < 2; ++p) {
        g[p] += pair * (re_mul_conj(pA[p], ak) + re_mul_conj(a_prev, dA[p]) +
                        re_mul_conj(pB[p], bk) + re_mul_conj(b_prev, dB[p]));
        g[p] += own * (re_mul_conj(pA[p], b_prev) + re_mul_conj(a_prev, pB[p]));
      }
    }
    const double w = (double)(2 * k + 1);
#pragma unroll
    for (int p = 0; p < 2; ++p) {
      sca[p] += w * 2.0 * (re_mul_conj(dA[p], ak) + re_mul_conj(dB[p], bk));
      const cplx t = scl(dA[p] - dB[p], w);
      back[p] = (k % 2 == 0) ? back[p] + t : back[p] - t;
    }
    a_prev = ak;
    b_prev = bk;
    da_prev = dak;
    db_prev = dbk;
  }
  __device__ __forceinline__ void close(int64_t n) {
    if (n >= 1) {
      const double kf = (double)n;
      const double own = (double)(2 * n + 1) / (kf * (kf + 1.0));
      const cplx pA[2] = {da_prev, cti(da_prev)}, pB[2] = {db_prev, cti(db_prev)};
#pragma unroll
      for (int p = 0; p < 2; ++p)
        g[p] += own * (re_mul_conj(pA[p], b_prev) + re_mul_conj(a_prev, pB[p]));
    }
  }
};

// efficiencies_from (efficiencies.rs:169-187).
__device__ __forceinline__ Eff efficiencies_from(double x, double abs_sum, const ValueSums& s) {
  double inv_x = 1.0 / x;
  double inv_x2 = inv_x * inv_x;
  double two_x2 = 2.0 * inv_x2;
  double q_sca = two_x2 * s.sca;
  double q_abs = two_x2 * abs_sum;
  double g = s.sca == 0.0 ? 0.0 : 2.0 * s.g / s.sca;
  return {q_sca + q_abs, q_sca, q_abs, nsq(s.back) * inv_x2, g};
}

// The efficiencies' derivatives along Re m (p = 0) or Im m (p = 1) of a homogeneous sphere
// (efficiencies_jacobian, efficiencies.rs:192-230; no x term along m).
__device__ __forceinline__ Eff efficiency_derivs(double x, const ValueSums& vs, const Eff& q,
                                                 const DerivSums& ds, int p, double abs_d) {
  double inv_x = 1.0 / x;
  double inv_x2 = inv_x * inv_x;
  double two_x2 = 2.0 * inv_x2;
  double q_sca = two_x2 * ds.sca[p];
  double q_abs = two_x2 * abs_d;
  double q_back = 2.0 * re_mul_conj(ds.back[p], vs.back) * inv_x2;
  double g = vs.sca == 0.0 ? 0.0 : (2.0 * ds.g[p] - q.g * ds.sca[p]) / vs.sca;
  return {q_sca + q_abs, q_sca, q_abs, q_back, g};
}

// One coefficient's effective log-derivative H at a layered sphere's outer surface at one order
// (kernel.rs:16-24): the correction delta = H - D_n(mx), or H itself near D_n's poles.
struct Side {
  bool direct;
  cplx v;
};

// No layers: D_n(mx) itself.
struct NoLayers {
  static constexpr bool kLayered = false;
  __device__ __forceinline__ void order(int64_t, Side&, Side&) {}
};

// No derivatives.
struct NoDeriv {
  static constexpr bool kOn = false;
};

// The derivatives along the refractive index of a homogeneous sphere (kernel.rs:486-532):
// da/dm, db/dm per order go to emit(k, a_k, b_k, da_k/dm, db_k/dm), and the absorption sum's
// derivatives along Re m and Im m (d/d(Im m) = i d/dm) accumulate here.
// With along_x, emit receives the derivatives along the size parameter x at fixed m instead,
// and abs_x the absorption sum's (kernel.rs:501-518, 509-516).
struct MDeriv {
  static constexpr bool kOn = true;
  double abs_re = 0.0, abs_im = 0.0;
  bool along_x = false;
  double abs_x = 0.0;
};

// State::finish (kernel.rs:324-559): calls emit(k, a_k, b_k) for k = 1..n and returns the
// absorption sum (x^2/2) Q_abs, feeding the value sums on the way. With a layered sphere's
// `layers`, its H_a, H_b replace D_n(mx) at each order (kernel.rs:382-476); they are computed
// order by order in the same upward loop. With MDeriv (homogeneous spheres only) emit also
// receives the coefficients' derivatives along m.
template <class Emit, class Layers, class Deriv = NoDeriv>
__device__ __forceinline__ double mie_finish(double x, cplx m, int64_t n, const Scratch& s,
                                             ValueSums& vs, Emit emit, Layers& layers,
                                             Deriv* deriv = nullptr) {
  const double one = 1.0;
  cplx z = scl(m, x);
  int64_t n_s = upward_orders(x, n);
  double inv_x = 1.0 / x;
  cplx inv_z = cinv(z);
  cplx inv_m = cinv(m);
  cplx inv_m2 = inv_m * inv_m;
  cplx m2_minus_1 = (m - rl(one)) * (m + rl(one));
  cplx c_a = -(m2_minus_1 * inv_m2);
  double sin_x, cos_x;
  sincos(x, &sin_x, &cos_x);
  double psi_prev = cos_x, psi = sin_x;
  double chi_prev = -sin_x, chi = cos_x;
  cplx t = rl(0.0), inv_xi = rl(0.0), r = rl(0.0);
  if (n_s == 0) {
    cplx xi0 = mk(sin_x, -cos_x);
    t = rl(sin_x) * cinv(xi0);
    inv_xi = mk(sin_x, cos_x);
    r = mk(0.0, one);
  }
  double asum = 0.0;
  cplx u_next = s.get_z(1 + 1);
  for (int64_t k = 1; k <= n; ++k) {
    double kf = (double)k;
    double k_x = kf * inv_x;
    cplx u_z1 = u_next;
    if (k < n) u_next = s.get_z(k + 2);
    cplx d = scl(inv_z, (double)(k + 1)) - u_z1;
    Side sa{false, rl(0.0)}, sb{false, rl(0.0)};
    cplx hh_a = d, hh_b = d;
    if (Layers::kLayered) {
      layers.order(k, sa, sb);
      hh_a = sa.direct ? sa.v : d + sa.v;
      hh_b = sb.direct ? sb.v : d + sb.v;
    }
    cplx d_m = hh_a * inv_m;
    cplx md = hh_b * m;
    cplx big_a = d_m + rl(k_x);
    cplx big_b = md + rl(k_x);
    cplx an, bn, inv_da, inv_db, g_a, g_b, h_a, h_b;
    if (k <= n_s) {
      double c = (double)(2 * k - 1) * inv_x;
      double psi_next = c * psi - psi_prev;
      psi_prev = psi;
      psi = psi_next;
      double chi_next = c * chi - chi_prev;
      chi_prev = chi;
      chi = chi_next;
      cplx xi = mk(psi, -chi);
      cplx xi_prev = mk(psi_prev, -chi_prev);
      inv_da = cinv(big_a * xi - xi_prev);
      inv_db = cinv(big_b * xi - xi_prev);
      if (!Layers::kLayered) {
        an = (scl(big_a, psi) - rl(psi_prev)) * inv_da;
        bn = (scl(big_b, psi) - rl(psi_prev)) * inv_db;
      } else {
        // The outer layer's own numerator plus delta/m psi_n and m delta psi_n
        // (kernel.rs:412-435); the own numerator is exactly 0 for m = 1.
        const bool unit_m = m.re == 1.0 && m.im == 0.0;
        cplx own_a = unit_m ? rl(0.0) : scl(d * inv_m + rl(k_x), psi) - rl(psi_prev);
        cplx own_b = unit_m ? rl(0.0) : scl(d * m + rl(k_x), psi) - rl(psi_prev);
        an = sa.direct ? (scl(big_a, psi) - rl(psi_prev)) * inv_da
                       : (own_a + scl(sa.v * inv_m, psi)) * inv_da;
        bn = sb.direct ? (scl(big_b, psi) - rl(psi_prev)) * inv_db
                       : (own_b + scl(m * sb.v, psi)) * inv_db;
      }
      if (Deriv::kOn) {
        g_a = xi * inv_da;
        g_b = xi * inv_db;
        h_a = xi_prev * inv_da;
        h_b = xi_prev * inv_db;
      }
      if (k == n_s) {
        inv_xi = cinv(xi);
        t = rl(psi) * inv_xi;
        r = xi_prev * inv_xi;
      }
    } else {
      r = cinv(rl((double)(2 * k - 1) * inv_x) - r);
      t = scl(t * r, s.get_x(k));
      inv_xi = inv_xi * r;
      cplx u_x1 = rl(s.get_x(k + 1));
      cplx num_a = scl(c_a, (double)(k + 1) * inv_x) + u_x1 - u_z1 * inv_m;
      cplx num_b = u_x1 - m * u_z1;
      if (Layers::kLayered) {
        // kernel.rs:456-466.
        cplx d_x = rl((double)(k + 1) * inv_x) - u_x1;
        num_a = sa.direct ? d_m - d_x : num_a + sa.v * inv_m;
        num_b = sb.direct ? md - d_x : num_b + m * sb.v;
      }
      cplx ia = cinv(big_a - r);
      cplx ib = cinv(big_b - r);
      an = t * num_a * ia;
      bn = t * num_b * ib;
      inv_da = inv_xi * ia;
      inv_db = inv_xi * ib;
      g_a = ia;
      g_b = ib;
      if (Deriv::kOn) {
        h_a = r * ia;
        h_b = r * ib;
      }
    }
    vs.add(k, an, bn);
    double na = nsq(inv_da);
    double nb = nsq(inv_db);
    double weight = (double)(2 * k + 1);
    asum += weight * (-(d_m.im * na) - md.im * nb);
    if constexpr (Deriv::kOn) {
      // d_plus = D + z D' and d_minus = D - z D' in terms of u = u_{k+1}(mx) (kernel.rs:
      // 490-500); d(D/m)/dm and d(mD)/dm and the absorption terms (kernel.rs:507-532).
      const double two = 2.0;
      cplx one_u2 = rl(one) + u_z1 * u_z1;
      cplx d_plus = scl(u_z1, weight) - z * one_u2;
      cplx d_minus = scl(d, two) - d_plus;
      cplx ida2 = inv_da * inv_da;
      cplx idb2 = inv_db * inv_db;
      if (deriv->along_x) {
        // da/dx and db/dx at fixed m (kernel.rs:501-504); D' = n(n+1)/z^2 - 1 - D^2 in terms
        // of u, and the absorption sum's x term (kernel.rs:509-516).
        const double kk1 = kf * (double)(k + 1);
        cplx dan = cti(m2_minus_1) * (d * d + rl(kk1 * inv_x * inv_x)) * inv_m2 * ida2;
        cplx dbn = cti(m2_minus_1) * idb2;
        emit(k, an, bn, dan, dbn);
        cplx dp = scl(scl(u_z1, two) * inv_z - inv_z * inv_z, (double)(k + 1)) - one_u2;
        const cplx m2 = m * m;
        const double k_x2 = k_x * inv_x;
        cplx la_x = g_a * (dp - rl(k_x2) - scl(big_a, k_x) + rl(one)) + h_a * d_m;
        cplx lb_x = g_b * (m2 * dp - rl(k_x2) - scl(big_b, k_x) + rl(one)) + h_b * md;
        auto term = [&](cplx f, cplx df, cplx l, double n2) {
          return -((df.im - two * f.im * l.re) * n2);
        };
        deriv->abs_x += weight * (term(d_m, dp, la_x, na) + term(md, m2 * dp, lb_x, nb));
        continue;
      }
      cplx dan = cti(d_minus) * inv_m2 * ida2;
      cplx dbn = -(cti(d_plus) * idb2);
      emit(k, an, bn, dan, dbn);
      cplx fa_m = -(d_minus * inv_m2);
      cplx fb_m = d_plus;
      cplx la_m = fa_m * g_a;
      cplx lb_m = fb_m * g_b;
      auto term = [&](cplx f, cplx df, cplx l, double n2) {
        return -((df.im - two * f.im * l.re) * n2);
      };
      deriv->abs_re += weight * (term(d_m, fa_m, la_m, na) + term(md, fb_m, lb_m, nb));
      deriv->abs_im += weight * (term(d_m, cti(fa_m), cti(la_m), na) +
                                 term(md, cti(fb_m), cti(lb_m), nb));
    } else {
      emit(k, an, bn);
    }
  }
  vs.close(n);
  return asum;
}

template <class Emit>
__device__ __forceinline__ double mie_finish(double x, cplx m, int64_t n, const Scratch& s,
                                             ValueSums& vs, Emit emit) {
  NoLayers none;
  return mie_finish(x, m, n, s, vs, emit, none);
}

// ---------------------------------------------------------------------------------------------
// Layered spheres (scatrs/src/layered/kernel.rs), values only.
// ---------------------------------------------------------------------------------------------
constexpr int kMaxLayers = 16;

// num-complex's sin, cos, and complex::exp_m1 (scatrs/src/complex.rs:51-56).
__device__ __forceinline__ cplx csin(cplx z) {
  return {sin(z.re) * cosh(z.im), cos(z.re) * sinh(z.im)};
}
__device__ __forceinline__ cplx ccos(cplx z) {
  return {cos(z.re) * cosh(z.im), -sin(z.re) * sinh(z.im)};
}
__device__ __forceinline__ cplx cexp_m1(cplx w) {
  double sb, cb;
  sincos(w.im, &sb, &cb);
  double h = sin(w.im * 0.5);
  return {expm1(w.re) * cb - h * h * 2.0, exp(w.re) * sb};
}
__device__ __forceinline__ cplx two_i(cplx z) { return {-(z.im * 2.0), z.re * 2.0}; }
__device__ __forceinline__ double norm1(cplx z) { return fabs(z.re) + fabs(z.im); }

// Pi_n(z) and w_{n+1}(z) of one argument (layered/kernel.rs:33-103).
struct LArg {
  cplx z, inv_z, pi, w, w_n;
  __device__ __forceinline__ void init(cplx zz, bool chi) {
    z = zz;
    inv_z = cinv(z);
    if (chi) {
      cplx sz = csin(z), cz = ccos(z);
      pi = sz * cz;
      w = inv_z + sz * cinv(cz);
    } else {
      pi = -scl(cexp_m1(two_i(z)), 0.5);
      w = inv_z - mk(0.0, 1.0);
    }
    w_n = rl(0.0);
  }
  __device__ __forceinline__ void step(int64_t n, cplx u_n) {
    w_n = w;
    pi = pi * u_n * w;
    w = scl(inv_z, (double)(2 * n + 1)) - cinv(w);
  }
  __device__ __forceinline__ cplx d1(int64_t n, cplx u_next) const {
    return scl(inv_z, (double)(n + 1)) - u_next;
  }
  __device__ __forceinline__ cplx d3(int64_t n) const {
    return scl(inv_z, (double)(n + 1)) - w;
  }
};

// Ratio arrays of one lane: array 0 is the outer layer's u_k(m x) (the sphere's u_z), then the
// core's, then per layer l >= 1 those of m_l x_{l-1} and (but for the outermost) m_l x_l.
struct LayerArrays {
  double2* base;
  int64_t astride;  // elements between arrays
  int stride;       // lanes
  __device__ __forceinline__ cplx get(int a, int64_t k) const {
    double2 v = base[a * astride + k * stride];
    return {v.x, v.y};
  }
  __device__ __forceinline__ void put(int a, int64_t k, cplx v) const {
    base[a * astride + k * stride] = make_double2(v.re, v.im);
  }
};

// ratios (kernel.rs:159-205): u_k(m x) for k = 1..n+1 into array a.
__device__ __forceinline__ void ratios_into(cplx m, double x, int64_t n, const LayerArrays& L,
                                            int a) {
  cplx z = scl(m, x);
  int64_t top = n + 1;
  if (m.im == 0.0) {
    double inv_rho = 1.0 / z.re, u = 0.0;
    int64_t start = start_index(top, fabs(z.re));
    for (int64_t k = start; k >= 1; --k) {
      u = step_real(k, inv_rho, u);
      if (k <= top) L.put(a, k, rl(u));
    }
  } else {
    cplx inv_z = cinv(z), u = rl(0.0);
    int64_t start = start_index(top, cabs_(z));
    for (int64_t k = start; k >= 1; --k) {
      u = step_complex(k, inv_z, u);
      if (k <= top) L.put(a, k, u);
    }
  }
}

// side (layered/kernel.rs:158-183) for the values.
__device__ __forceinline__ Side layer_side(cplx mi, cplx mo, Side prev, cplx h, cplx lead,
                                           cplx u_prev, cplx u1, cplx d1i, cplx d3i, cplx d1o,
                                           cplx d3o, cplx pio, cplx p, cplx w, cplx* h_out) {
  cplx mh = mi * h;
  cplx g1 = prev.direct ? mh - mo * d1i : lead - mi * u_prev + mo * u1 + mi * prev.v;
  cplx g2 = mh - mo * d3i;
  cplx inv_den = cinv(pio * g2 - p * g1);
  cplx delta = -(w * p * g1 * inv_den * cinv(pio));
  cplx hd = d1o + delta;
  if (norm1(hd) * 4.0 >= fmax(norm1(d1o), norm1(delta))) {
    *h_out = hd;
    return {false, delta};
  }
  cplx hp = d3o - w * g2 * inv_den;
  *h_out = hp;
  return {true, hp};
}

// Kernel::solve's recursion (layered/kernel.rs:308-465) for `layers` layers of interface size
// parameters x[0..layers) and indices m, its H_a, H_b produced one order at a time.
struct Layered {
  static constexpr bool kLayered = true;
  int layers;
  const double* x;
  const cplx* m;
  LayerArrays arr;
  LArg inner[kMaxLayers - 1], outer[kMaxLayers - 1], core;
  cplx p[kMaxLayers - 1], lead[kMaxLayers - 1];
  bool chi[kMaxLayers - 1];

  // Array index of the ratios of layer l's outer argument (l < layers - 1), of m_l x_{l-1}, and
  // of the core.
  __device__ __forceinline__ int a_outer(int l) const { return l == layers - 1 ? 0 : 2 * l + 1; }
  __device__ __forceinline__ int a_inner(int l) const { return 2 * l; }
  static constexpr int kCore = 1;

  // The ratio arrays and the initial state; the outer argument's own ratios (array 0) come from
  // mie_prepare.
  __device__ void prepare(int64_t n) {
    const int last = layers - 1;
    ratios_into(m[0], x[0], n, arr, kCore);
    for (int l = 1; l < layers; ++l) {
      ratios_into(m[l], x[l - 1], n, arr, a_inner(l));
      if (l < last) ratios_into(m[l], x[l], n, arr, a_outer(l));
    }
    for (int l = 1; l < layers; ++l) {
      const bool c = m[l].im * x[l] < 0.5;
      chi[l - 1] = c;
      const cplx a = m[l], b = m[l - 1];
      lead[l - 1] = (a - b) * (a + b) * cinv(a * b);
      const cplx z1 = scl(m[l], x[l - 1]), z2 = scl(m[l], x[l]);
      inner[l - 1].init(z1, c);
      outer[l - 1].init(z2, c);
      if (c) {
        const cplx c2 = ccos(z2);
        p[l - 1] = csin(z1) * cinv(ccos(z1)) * c2 * c2;
      } else {
        const double dx = x[l] - x[l - 1];
        const double ea = -(m[l].im * dx * 2.0), eb = m[l].re * dx * 2.0;
        double sb, cb;
        sincos(eb, &sb, &cb);
        const cplx e = scl(mk(cb, sb), exp(ea));
        p[l - 1] = -scl(e * cexp_m1(two_i(z1)), 0.5);
      }
    }
    core.init(scl(m[0], x[0]), false);
  }

  __device__ __forceinline__ void order(int64_t k, Side& sa, Side& sb) {
    for (int l = 1; l < layers; ++l) {
      LArg& ai = inner[l - 1];
      LArg& ao = outer[l - 1];
      const cplx u1k = arr.get(a_inner(l), k);
      ai.step(k, u1k);
      ao.step(k, arr.get(a_outer(l), k));
      p[l - 1] = p[l - 1] * u1k * cinv(ai.w_n) * ao.w_n * ao.w_n;
    }
    cplx ha = core.d1(k, arr.get(kCore, k + 1));
    cplx hb = ha;
    Side a{false, rl(0.0)}, b{false, rl(0.0)};
    for (int l = 1; l < layers; ++l) {
      const LArg& ai = inner[l - 1];
      const LArg& ao = outer[l - 1];
      const cplx u_prev = arr.get(l == 1 ? kCore : a_outer(l - 1), k + 1);
      const cplx u1 = arr.get(a_inner(l), k + 1);
      const cplx u2 = arr.get(a_outer(l), k + 1);
      const cplx d1i = ai.d1(k, u1), d3i = ai.d3(k);
      const cplx d1o = ao.d1(k, u2), d3o = ao.d3(k);
      const cplx w = chi[l - 1] ? rl(-1.0) : mk(0.0, 1.0);
      const cplx ld = scl(lead[l - 1], (double)(k + 1) / x[l - 1]);
      cplx na, nb;
      const Side a2 = layer_side(m[l], m[l - 1], a, ha, ld, u_prev, u1, d1i, d3i, d1o, d3o,
                                 ao.pi, p[l - 1], w, &na);
      const Side b2 = layer_side(m[l - 1], m[l], b, hb, rl(0.0), u_prev, u1, d1i, d3i, d1o, d3o,
                                 ao.pi, p[l - 1], w, &nb);
      ha = na;
      hb = nb;
      a = a2;
      b = b2;
    }
    sa = a;
    sb = b;
  }
};

// Layered::check_inputs (layered/mod.rs:233-305) with the default truncation: 0 when accepted,
// else the status (1 invalid input, 3 outside the validated domain, layered/domain.rs:76-92).
__device__ __forceinline__ int check_layered(const double* x, const cplx* m, int layers,
                                             int64_t n, bool allow_unvalidated) {
  for (int l = 0; l < layers; ++l)
    if (!isfinite(x[l]) || (l > 0 && x[l] < x[l - 1])) return 1;
  const double outer = x[layers - 1];
  if (x[0] < 1e-30 || outer > 1e6) return 1;
  for (int l = 0; l < layers; ++l) {
    if (!(isfinite(m[l].re) && isfinite(m[l].im)) || m[l].re < 0.0 || m[l].im < 0.0) return 1;
    const double a = hypot(m[l].re, m[l].im);
    if (!(a >= 1e-6 && a <= 1e3)) return 1;
  }
  if (n == 0 || n > (1 << 20)) return 1;
  if (!allow_unvalidated) {
    if (layers > 16 || !(outer >= 1e-6 && outer <= 1e4)) return 3;
    for (int l = 0; l < layers; ++l) {
      const double a = hypot(m[l].re, m[l].im);
      if (!(a * outer <= 3e4 && m[l].re > 0.0 && m[l].re <= 10.0 && m[l].im >= 0.0 &&
            m[l].im <= 10.0 && a >= 0.1))
        return 3;
    }
  }
  return 0;
}

}  // namespace sb
