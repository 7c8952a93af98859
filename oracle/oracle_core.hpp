// CPU oracle: a plain double-precision restatement of the reference's algorithms on the
// size-distribution ensemble path. TEST INFRASTRUCTURE ONLY: the parity tests, the smoke check
// and the CPU-baseline leg of the benchmark use it as the checker; the product path never links
// it. Compile with -ffp-contract=off so that every a*b+c rounds twice, as the reference's Rust
// does (it never fuses on its own).
//
// Each function names the reference file:line it follows (paths inside usask-arg/scatrs).
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>
#include <algorithm>
#include <limits>
#include <stdexcept>

namespace orc {

constexpr double PI = 3.14159265358979323846264338327950288;
constexpr double EPS = 2.220446049250313e-16;  // f64::EPSILON = 2^-52

// ---------------------------------------------------------------------------------------
// Complex arithmetic with num-complex 0.4's operation order (a*b = (ac - bd) + i(ad + bc)).
// ---------------------------------------------------------------------------------------
struct cplx {
  double re, im;
};
inline cplx C(double r, double i) { return {r, i}; }
inline cplx real(double v) { return {v, 0.0}; }
inline cplx operator+(cplx a, cplx b) { return {a.re + b.re, a.im + b.im}; }
inline cplx operator-(cplx a, cplx b) { return {a.re - b.re, a.im - b.im}; }
inline cplx operator-(cplx a) { return {-a.re, -a.im}; }
inline cplx operator*(cplx a, cplx b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
inline cplx scale(cplx a, double t) { return {a.re * t, a.im * t}; }
inline double norm_sqr(cplx a) { return a.re * a.re + a.im * a.im; }
inline double cnorm(cplx a) { return std::hypot(a.re, a.im); }
inline cplx conj(cplx a) { return {a.re, -a.im}; }
inline bool is_zero(cplx a) { return a.re == 0.0 && a.im == 0.0; }

// complex::inv (scatrs/src/complex.rs:21-38): the plain formula where 1e-300 < c^2+d^2 <
// 1e300 and d != 0, Smith's algorithm otherwise.
inline cplx inv(cplx z) {
  double c = z.re, d = z.im;
  double s = c * c + d * d;
  if (s > 1e-300 && s < 1e300 && d != 0.0) {
    double t = 1.0 / s;
    return {c * t, -(d * t)};
  }
  if (std::fabs(d) <= std::fabs(c)) {
    double r = d / c;
    double t = 1.0 / (c + d * r);
    return {t, -(r * t)};
  }
  double r = c / d;
  double t = 1.0 / (c * r + d);
  return {r * t, -t};
}

// complex::times_i (complex.rs:43-45).
inline cplx times_i(cplx u) { return {-u.im, u.re}; }

// ---------------------------------------------------------------------------------------
// Truncation and input checks (scatrs/src/mie/mod.rs:101-155, 274-320; domain.rs:124-140).
// ---------------------------------------------------------------------------------------
constexpr int64_t MAX_MIE_ORDER = 1 << 20;
constexpr double MIN_SIZE_PARAMETER = 1e-30;
constexpr double MAX_SIZE_PARAMETER = 1e6;
constexpr double MIN_REFRACTIVE_INDEX = 1e-6;
constexpr double MAX_REFRACTIVE_INDEX = 1e3;

// terms (mie/mod.rs:138-145): ceil(x + c x^(1/3) + d), SIZE_MAX when not finite.
inline int64_t terms(double x, double c, double d) {
  double n = std::ceil(x + c * std::cbrt(x) + d);
  if (std::isfinite(n) && n < 9007199254740992.0) return (int64_t)n;
  return INT64_MAX;
}
inline int64_t default_n_max(double x) { return terms(x, 6.0, 3.0); }

// VALIDATED_DOMAIN.contains (mie/domain.rs:124-140).
inline bool in_validated_domain(double x, cplx m) {
  return x >= 1e-6 && x <= 2e4 && m.re > 0.0 && m.re <= 10.0 && m.im >= 0.0 && m.im <= 10.0 &&
         cnorm(m) >= 0.1;
}

enum Status { OK = 0, INVALID_INPUT = 1, NOT_CONVERGED = 2, OUTSIDE_VALIDATED_DOMAIN = 3 };

// check_inputs (mie/mod.rs:274-320). Returns the status; n_out receives the number of terms.
inline int check_inputs(double x, double m_re, double m_im, int64_t n_max_opt,
                        bool allow_unvalidated, int64_t* n_out, std::string* msg) {
  if (!(x >= MIN_SIZE_PARAMETER && x <= MAX_SIZE_PARAMETER)) {
    if (msg) *msg = "the size parameter x must be in [1e-30, 1e6]";
    return INVALID_INPUT;
  }
  if (!(std::isfinite(m_re) && std::isfinite(m_im))) {
    if (msg) *msg = "the refractive index must be finite";
    return INVALID_INPUT;
  }
  if (m_re < 0.0 || m_im < 0.0) {
    if (msg) *msg = "the refractive index must have Re m >= 0 and Im m >= 0";
    return INVALID_INPUT;
  }
  double abs_m = std::hypot(m_re, m_im);
  if (!(abs_m >= MIN_REFRACTIVE_INDEX && abs_m <= MAX_REFRACTIVE_INDEX)) {
    if (msg) *msg = "|m| must be in [1e-6, 1e3]";
    return INVALID_INPUT;
  }
  int64_t def = default_n_max(x);
  int64_t n = n_max_opt > 0 ? n_max_opt : def;
  if (n == 0 || n > MAX_MIE_ORDER) {
    if (msg) *msg = "the number of terms must be in [1, 1048576]";
    return INVALID_INPUT;
  }
  if (!allow_unvalidated) {
    if (!in_validated_domain(x, C(m_re, m_im))) {
      if (msg) *msg = "outside the validated domain";
      return OUTSIDE_VALIDATED_DOMAIN;
    }
    if (n < def) {
      if (msg) *msg = "n_max is below the default truncation";
      return OUTSIDE_VALIDATED_DOMAIN;
    }
  }
  *n_out = n;
  return OK;
}

// ---------------------------------------------------------------------------------------
// The Mie recurrences (scatrs/src/mie/kernel.rs).
// ---------------------------------------------------------------------------------------
constexpr double BITS = 52.0;   // bits::<f64>() = -log2(2^-52) (kernel.rs:76-78)
constexpr int64_t MARGIN = 30;  // margin::<f64>() = ceil(52/2) + 4 (kernel.rs:82-84)

// start_index (kernel.rs:99-112).
inline int64_t start_index(int64_t n_top, double rho_abs) {
  double c15 = std::ceil(1.5 * rho_abs);
  int64_t k0 = std::max<int64_t>(n_top, (int64_t)c15);
  double q = (double)(2 * k0 + 1) / rho_abs - 0.5;
  int64_t enclosed = k0 + (int64_t)std::ceil(BITS / (2.0 * std::log2(q))) + 2;
  if ((double)n_top >= 1.5 * rho_abs) return enclosed;
  double s0 = (double)n_top - rho_abs;
  double s0_32 = s0 > 0.0 ? s0 * std::sqrt(s0) : 0.0;
  double s = std::pow(s0_32 + 1.4 * 0.37 * BITS * std::sqrt(rho_abs), 2.0 / 3.0);
  int64_t asymptotic = (int64_t)std::ceil(rho_abs + s) + MARGIN;
  return std::min(asymptotic, enclosed);
}

// step_complex (kernel.rs:116-125).
inline cplx step_complex(int64_t k, cplx inv_z, cplx u) {
  cplx c = scale(inv_z, (double)(2 * k + 1));
  cplx den = c - u;
  if (den.re == 0.0 && den.im == 0.0) den = real(EPS * (cnorm(c) + cnorm(u)));
  return inv(den);
}

// step_real (kernel.rs:129-136).
inline double step_real(int64_t k, double inv_rho, double u) {
  double c = inv_rho * (double)(2 * k + 1);
  double den = c - u;
  if (den == 0.0) den = EPS * (std::fabs(c) + std::fabs(u));
  return 1.0 / den;
}

// upward_orders (kernel.rs:208-215).
inline int64_t upward_orders(double x, int64_t n) {
  if (x >= 1.0) return std::min<int64_t>((int64_t)std::floor(x), n);
  return 0;
}

// One coefficient's effective log-derivative H at a layered sphere's outer surface at one order
// (mie/kernel.rs:16-24): as the correction delta = H - D_n(mx), or as H itself near the poles.
enum SideKind { SIDE_DELTA = 0, SIDE_DIRECT = 1 };
struct Side {
  int kind;
  cplx v;
};
struct Outer {
  Side a, b;
};

struct MieState {
  double x = 0;
  cplx m{0, 0};
  std::vector<cplx> a, b;
  bool derivatives = false;
  std::vector<cplx> da_dx, da_dm, db_dx, db_dm;
  double abs_sum = 0;
  double abs_sum_jacobian[3] = {0, 0, 0};
  std::vector<cplx> u_z;
  std::vector<double> u_x;

  // State::prepare (kernel.rs:249-313). The two downward recurrences are independent; their
  // interleaving in the reference only overlaps latencies, so they run one after the other.
  void prepare(double xv, cplx mv, int64_t n) {
    int64_t n_s = upward_orders(xv, n);
    int64_t top = n + 1;
    u_x.assign(n + 2, 0.0);
    if (n_s < n) {
      int64_t start = start_index(top, std::fabs(xv));
      int64_t lo = std::max<int64_t>(n_s + 1, 1);
      double inv_x = 1.0 / xv;
      double ux = 0.0;
      for (int64_t k = start; k >= lo; --k) {
        ux = step_real(k, inv_x, ux);
        if (k <= top) u_x[k] = ux;
      }
    }
    cplx z = scale(mv, xv);
    u_z.assign(n + 2, real(0.0));
    if (mv.im == 0.0) {
      double inv_rho = 1.0 / z.re;
      double u = 0.0;
      int64_t start = start_index(top, std::fabs(z.re));
      for (int64_t k = start; k >= 1; --k) {
        u = step_real(k, inv_rho, u);
        if (k <= top) u_z[k] = real(u);
      }
    } else {
      cplx inv_z = inv(z);
      cplx u = real(0.0);
      int64_t start = start_index(top, cnorm(z));
      for (int64_t k = start; k >= 1; --k) {
        u = step_complex(k, inv_z, u);
        if (k <= top) u_z[k] = u;
      }
    }
  }

  // State::finish (kernel.rs:324-559), homogeneous sphere (no layered outer hooks).
  void finish(double xv, cplx mv, int64_t n, bool derivs, const Outer* outer = nullptr) {
    const double one = 1.0, two = 2.0;
    x = xv;
    m = mv;
    derivatives = derivs;
    cplx z = scale(mv, xv);
    int64_t n_s = upward_orders(xv, n);
    a.clear();
    b.clear();
    da_dx.clear();
    da_dm.clear();
    db_dx.clear();
    db_dm.clear();
    double inv_x = 1.0 / xv;
    cplx inv_z = inv(z);
    cplx inv_m = inv(mv);
    cplx m2 = mv * mv;
    cplx inv_m2 = inv_m * inv_m;
    cplx m2_minus_1 = (mv - real(one)) * (mv + real(one));
    cplx c_a = -(m2_minus_1 * inv_m2);
    double sin_x = std::sin(xv), cos_x = std::cos(xv);
    double psi_prev = cos_x, psi = sin_x;
    double chi_prev = -sin_x, chi = cos_x;
    cplx t = real(0.0), inv_xi = real(0.0), r = real(0.0);
    if (n_s == 0) {
      cplx xi0 = C(sin_x, -cos_x);
      t = real(sin_x) * inv(xi0);
      inv_xi = C(sin_x, cos_x);
      r = C(0.0, one);
    }
    double asum = 0.0;
    double jac[3] = {0, 0, 0};
    for (int64_t k = 1; k <= n; ++k) {
      double kf = (double)k;
      double k_x = kf * inv_x;
      cplx d = scale(inv_z, (double)(k + 1)) - u_z[k + 1];
      // H of a layered sphere in place of D_n(mx) (kernel.rs:382-388).
      auto hsel = [&](const Side* sd) {
        if (!sd) return d;
        return sd->kind == SIDE_DELTA ? d + sd->v : sd->v;
      };
      const Outer* side = outer ? &outer[k - 1] : nullptr;
      cplx hh_a = hsel(side ? &side->a : nullptr), hh_b = hsel(side ? &side->b : nullptr);
      cplx d_m = hh_a * inv_m;
      cplx md = hh_b * mv;
      cplx big_a = d_m + real(k_x);
      cplx big_b = md + real(k_x);
      cplx an, bn, inv_da, inv_db, g_a, g_b, h_a, h_b;
      if (k <= n_s) {
        double c = (double)(2 * k - 1) * inv_x;
        double psi_next = c * psi - psi_prev;
        psi_prev = psi;
        psi = psi_next;
        double chi_next = c * chi - chi_prev;
        chi_prev = chi;
        chi = chi_next;
        cplx xi = C(psi, -chi);
        cplx xi_prev = C(psi_prev, -chi_prev);
        inv_da = inv(big_a * xi - xi_prev);
        inv_db = inv(big_b * xi - xi_prev);
        if (!side) {
          an = (scale(big_a, psi) - real(psi_prev)) * inv_da;
          bn = (scale(big_b, psi) - real(psi_prev)) * inv_db;
        } else {
          // kernel.rs:412-435: the outer layer's own numerator plus delta/m psi_n, m delta psi_n.
          auto own = [&](cplx f) {
            if (mv.re == 1.0 && mv.im == 0.0) return real(0.0);
            return scale(f + real(k_x), psi) - real(psi_prev);
          };
          an = side->a.kind == SIDE_DELTA
                   ? (own(d * inv_m) + scale(side->a.v * inv_m, psi)) * inv_da
                   : (scale(big_a, psi) - real(psi_prev)) * inv_da;
          bn = side->b.kind == SIDE_DELTA ? (own(d * mv) + scale(mv * side->b.v, psi)) * inv_db
                                          : (scale(big_b, psi) - real(psi_prev)) * inv_db;
        }
        g_a = xi * inv_da;
        g_b = xi * inv_db;
        h_a = xi_prev * inv_da;
        h_b = xi_prev * inv_db;
        if (k == n_s) {
          inv_xi = inv(xi);
          t = real(psi) * inv_xi;
          r = xi_prev * inv_xi;
        }
      } else {
        r = inv(real((double)(2 * k - 1) * inv_x) - r);
        t = scale(t * r, u_x[k]);
        inv_xi = inv_xi * r;
        cplx u_z1 = u_z[k + 1];
        cplx u_x1 = real(u_x[k + 1]);
        cplx num_a = scale(c_a, (double)(k + 1) * inv_x) + u_x1 - u_z1 * inv_m;
        cplx num_b = u_x1 - mv * u_z1;
        if (side) {
          // kernel.rs:456-466.
          cplx d_x = real((double)(k + 1) * inv_x) - u_x1;
          num_a = side->a.kind == SIDE_DELTA ? num_a + side->a.v * inv_m : d_m - d_x;
          num_b = side->b.kind == SIDE_DELTA ? num_b + mv * side->b.v : md - d_x;
        }
        cplx ia = inv(big_a - r);
        cplx ib = inv(big_b - r);
        an = t * num_a * ia;
        bn = t * num_b * ib;
        inv_da = inv_xi * ia;
        inv_db = inv_xi * ib;
        g_a = ia;
        g_b = ib;
        h_a = r * ia;
        h_b = r * ib;
      }
      a.push_back(an);
      b.push_back(bn);
      double na = norm_sqr(inv_da);
      double nb = norm_sqr(inv_db);
      double weight = (double)(2 * k + 1);
      asum += weight * (-(d_m.im * na) - md.im * nb);
      if (derivs && !outer) {
        cplx u = u_z[k + 1];
        cplx one_u2 = real(one) + u * u;
        cplx dp = scale(scale(u, two) * inv_z - inv_z * inv_z, (double)(k + 1)) - one_u2;
        cplx d_plus = scale(u, weight) - z * one_u2;
        cplx d_minus = scale(d, two) - d_plus;
        double kk1 = (double)k * (double)(k + 1);
        cplx ida2 = inv_da * inv_da;
        cplx idb2 = inv_db * inv_db;
        da_dm.push_back(times_i(d_minus) * inv_m2 * ida2);
        db_dm.push_back(-(times_i(d_plus) * idb2));
        da_dx.push_back(times_i(m2_minus_1) * (d * d + real(kk1 * inv_x * inv_x)) * inv_m2 * ida2);
        db_dx.push_back(times_i(m2_minus_1) * idb2);
        cplx fa_m = -(d_minus * inv_m2);
        cplx fb_m = d_plus;
        double k_x2 = k_x * inv_x;
        cplx la_x = g_a * (dp - real(k_x2) - scale(big_a, k_x) + real(one)) + h_a * d_m;
        cplx lb_x = g_b * (m2 * dp - real(k_x2) - scale(big_b, k_x) + real(one)) + h_b * md;
        cplx la_m = fa_m * g_a;
        cplx lb_m = fb_m * g_b;
        auto term = [&](cplx f, cplx df, cplx l, double n2) {
          return -((df.im - two * f.im * l.re) * n2);
        };
        jac[0] += weight * (term(d_m, dp, la_x, na) + term(md, m2 * dp, lb_x, nb));
        jac[1] += weight * (term(d_m, fa_m, la_m, na) + term(md, fb_m, lb_m, nb));
        jac[2] += weight * (term(d_m, times_i(fa_m), times_i(la_m), na) +
                            term(md, times_i(fb_m), times_i(lb_m), nb));
      }
    }
    abs_sum = asum;
    abs_sum_jacobian[0] = jac[0];
    abs_sum_jacobian[1] = jac[1];
    abs_sum_jacobian[2] = jac[2];
  }

  void solve(double xv, cplx mv, int64_t n, bool derivs) {
    prepare(xv, mv, n);
    finish(xv, mv, n, derivs);
  }
};

// ---------------------------------------------------------------------------------------
// Layered spheres (scatrs/src/layered/kernel.rs), values only.
// ---------------------------------------------------------------------------------------
// num-complex's sin, cos: sin(a+ib) = sin a cosh b + i cos a sinh b, cos(a+ib) = cos a cosh b
// - i sin a sinh b.
inline cplx csin(cplx z) { return {std::sin(z.re) * std::cosh(z.im), std::cos(z.re) * std::sinh(z.im)}; }
inline cplx ccos(cplx z) { return {std::cos(z.re) * std::cosh(z.im), -std::sin(z.re) * std::sinh(z.im)}; }
// complex::exp_m1 (complex.rs:51-56).
inline cplx cexp_m1(cplx w) {
  double a = w.re, b = w.im;
  double sb = std::sin(b), cb = std::cos(b);
  double h = std::sin(b * 0.5);
  return {std::expm1(a) * cb - h * h * 2.0, std::exp(a) * sb};
}
// 2iz (layered/kernel.rs:45-47).
inline cplx two_i(cplx z) { return {-(z.im * 2.0), z.re * 2.0}; }

// ratios (mie/kernel.rs:159-205): u_k(mx) for k = 1..n+1.
inline std::vector<cplx> ratios(cplx m, double x, int64_t n) {
  std::vector<cplx> out(n + 2, real(0.0));
  cplx z = scale(m, x);
  if (m.im == 0.0) {
    double inv_rho = 1.0 / z.re, u = 0.0;
    int64_t start = start_index(n + 1, std::fabs(z.re));
    for (int64_t k = start; k >= 1; --k) {
      u = step_real(k, inv_rho, u);
      if (k <= n + 1) out[k] = real(u);
    }
  } else {
    cplx inv_z = inv(z), u = real(0.0);
    int64_t start = start_index(n + 1, cnorm(z));
    for (int64_t k = start; k >= 1; --k) {
      u = step_complex(k, inv_z, u);
      if (k <= n + 1) out[k] = u;
    }
  }
  return out;
}

// Arg (layered/kernel.rs:33-103): Pi_n(z) and w_{n+1}(z), advanced order by order.
struct Arg {
  cplx z, inv_z, pi, w, w_n;
  Arg() = default;
  Arg(cplx zz, bool chi) {
    z = zz;
    inv_z = inv(z);
    if (chi) {
      cplx sz = csin(z), cz = ccos(z);
      pi = sz * cz;
      w = inv_z + sz * inv(cz);
    } else {
      pi = -scale(cexp_m1(two_i(z)), 0.5);
      w = inv_z - C(0.0, 1.0);
    }
    w_n = real(0.0);
  }
  void step(int64_t n, cplx u_n) {
    w_n = w;
    pi = pi * u_n * w;
    w = scale(inv_z, (double)(2 * n + 1)) - inv(w);
  }
  cplx d1(int64_t n, cplx u_next) const { return scale(inv_z, (double)(n + 1)) - u_next; }
  cplx d3(int64_t n) const { return scale(inv_z, (double)(n + 1)) - w; }
};

inline double norm1(cplx z) { return std::fabs(z.re) + std::fabs(z.im); }

struct LayerStep {
  cplx u_prev, u1, d1i, d3i, d1o, d3o, pio, p, w;
};

// side (layered/kernel.rs:158-183) without the derivatives' sensitivities.
inline Side layer_side(cplx mi, cplx mo, Side prev, cplx h, cplx lead, const LayerStep& s,
                       cplx* h_out) {
  cplx mh = mi * h;
  cplx g1 = prev.kind == SIDE_DELTA ? lead - mi * s.u_prev + mo * s.u1 + mi * prev.v
                                    : mh - mo * s.d1i;
  cplx g2 = mh - mo * s.d3i;
  cplx inv_den = inv(s.pio * g2 - s.p * g1);
  cplx delta = -(s.w * s.p * g1 * inv_den * inv(s.pio));
  cplx hd = s.d1o + delta;
  if (norm1(hd) * 4.0 >= std::max(norm1(s.d1o), norm1(delta))) {
    *h_out = hd;
    return {SIDE_DELTA, delta};
  }
  cplx hp = s.d3o - s.w * g2 * inv_den;
  *h_out = hp;
  return {SIDE_DIRECT, hp};
}

// Kernel::solve (layered/kernel.rs:308-465) for values: x[l] the interface size parameters (the
// outer one last), m[l] the layers' indices; a_n, b_n and the absorption sum into `mie`.
inline void layered_solve(const std::vector<double>& x, const std::vector<cplx>& m, int64_t n,
                          MieState& mie) {
  const size_t layers = x.size(), last = layers - 1;
  if (last == 0) {
    mie.solve(x[0], m[0], n, false);
    return;
  }
  mie.prepare(x[last], m[last], n);
  std::vector<std::vector<cplx>> u(2 * last);
  u[0] = ratios(m[0], x[0], n);
  for (size_t l = 1; l < layers; ++l) {
    u[2 * l - 1] = ratios(m[l], x[l - 1], n);
    if (l < last) u[2 * l] = ratios(m[l], x[l], n);
  }
  std::vector<Arg> inner, outer_args;
  std::vector<cplx> p, lead;
  std::vector<bool> chi;
  for (size_t l = 1; l < layers; ++l) {
    bool c = m[l].im * x[l] < 0.5;
    chi.push_back(c);
    cplx a = m[l], b = m[l - 1];
    lead.push_back((a - b) * (a + b) * inv(a * b));
    cplx z1 = scale(m[l], x[l - 1]), z2 = scale(m[l], x[l]);
    inner.emplace_back(z1, c);
    outer_args.emplace_back(z2, c);
    cplx p0;
    if (c) {
      cplx c2 = ccos(z2);
      p0 = csin(z1) * inv(ccos(z1)) * c2 * c2;
    } else {
      double dx = x[l] - x[l - 1];
      double ea = -(m[l].im * dx * 2.0), eb = m[l].re * dx * 2.0;
      double sb = std::sin(eb), cb = std::cos(eb);
      cplx e = scale(C(cb, sb), std::exp(ea));
      p0 = -scale(e * cexp_m1(two_i(z1)), 0.5);
    }
    p.push_back(p0);
  }
  Arg core(scale(m[0], x[0]), false);
  std::vector<Outer> outer(n);
  for (int64_t k = 1; k <= n; ++k) {
    auto u_of = [&](size_t l) -> const std::vector<cplx>& {
      return l == last ? mie.u_z : u[2 * l];
    };
    for (size_t l = 1; l < layers; ++l) {
      Arg& ai = inner[l - 1];
      Arg& ao = outer_args[l - 1];
      ai.step(k, u[2 * l - 1][k]);
      ao.step(k, u_of(l)[k]);
      p[l - 1] = p[l - 1] * u[2 * l - 1][k] * inv(ai.w_n) * ao.w_n * ao.w_n;
    }
    cplx ha = core.d1(k, u[0][k + 1]);
    cplx hb = ha;
    Side sa{SIDE_DELTA, real(0.0)}, sb{SIDE_DELTA, real(0.0)};
    for (size_t l = 1; l < layers; ++l) {
      const Arg& ai = inner[l - 1];
      const Arg& ao = outer_args[l - 1];
      const std::vector<cplx>& up = l == 1 ? u[0] : u[2 * (l - 1)];
      LayerStep st;
      st.u_prev = up[k + 1];
      st.u1 = u[2 * l - 1][k + 1];
      st.d1i = ai.d1(k, u[2 * l - 1][k + 1]);
      st.d3i = ai.d3(k);
      st.d1o = ao.d1(k, u_of(l)[k + 1]);
      st.d3o = ao.d3(k);
      st.pio = ao.pi;
      st.p = p[l - 1];
      st.w = chi[l - 1] ? real(-1.0) : C(0.0, 1.0);
      cplx ld = scale(lead[l - 1], (double)(k + 1) / x[l - 1]);
      cplx na, nb;
      Side a2 = layer_side(m[l], m[l - 1], sa, ha, ld, st, &na);
      Side b2 = layer_side(m[l - 1], m[l], sb, hb, real(0.0), st, &nb);
      ha = na;
      hb = nb;
      sa = a2;
      sb = b2;
    }
    outer[k - 1] = {sa, sb};
  }
  mie.finish(x[last], m[last], n, false, outer.data());
  bool lossless = true;
  for (auto& v : m) lossless = lossless && v.im == 0.0;
  if (lossless) mie.abs_sum = 0.0;
}

// ---------------------------------------------------------------------------------------
// Efficiencies (scatrs/src/mie/efficiencies.rs:64-84, 169-187).
// ---------------------------------------------------------------------------------------
struct Efficiencies {
  double q_ext, q_sca, q_abs, q_back, g;
};
struct Sums {
  double sca;
  cplx back;
  double g;
};
inline double re_mul_conj(cplx u, cplx v) { return u.re * v.re + u.im * v.im; }

inline Sums value_sums(const cplx* a, const cplx* b, int64_t n) {
  Sums s{0.0, real(0.0), 0.0};
  for (int64_t k = 1; k <= n; ++k) {
    cplx ak = a[k - 1], bk = b[k - 1];
    double w = (double)(2 * k + 1);
    s.sca += w * (norm_sqr(ak) + norm_sqr(bk));
    cplx t = scale(ak - bk, w);
    s.back = (k % 2 == 0) ? s.back + t : s.back - t;
    double kf = (double)k;
    if (k < n) {
      cplx a1 = a[k], b1 = b[k];
      s.g += kf * (kf + 2.0) / (kf + 1.0) * (re_mul_conj(ak, a1) + re_mul_conj(bk, b1));
    }
    s.g += w / (kf * (kf + 1.0)) * re_mul_conj(ak, bk);
  }
  return s;
}

inline Efficiencies efficiencies_from(double x, double abs_sum, const Sums& s) {
  double inv_x = 1.0 / x;
  double inv_x2 = inv_x * inv_x;
  double two_x2 = 2.0 * inv_x2;
  double q_sca = two_x2 * s.sca;
  double q_abs = two_x2 * abs_sum;
  double g = s.sca == 0.0 ? 0.0 : 2.0 * s.g / s.sca;
  return {q_sca + q_abs, q_sca, q_abs, norm_sqr(s.back) * inv_x2, g};
}

inline Efficiencies efficiencies(const MieState& st) {
  return efficiencies_from(st.x, st.abs_sum, value_sums(st.a.data(), st.b.data(), st.a.size()));
}

// The efficiencies' derivatives along the size parameter x at fixed m of a sphere solved with
// derivatives: derivative_sums along da/dx, db/dx and efficiencies_jacobian's x column with its
// -(2/x) Q term (efficiencies.rs:89-146, 192-230).
inline Efficiencies efficiency_x(const MieState& st, const Efficiencies& q) {
  const int64_t n = (int64_t)st.a.size();
  const Sums vs = value_sums(st.a.data(), st.b.data(), n);
  double sca = 0.0, g = 0.0;
  cplx back = real(0.0);
  for (int64_t k = 1; k <= n; ++k) {
    const cplx ak = st.a[k - 1], bk = st.b[k - 1], dak = st.da_dx[k - 1], dbk = st.db_dx[k - 1];
    const double w = (double)(2 * k + 1), kf = (double)k;
    const double pair = kf * (kf + 2.0) / (kf + 1.0);
    const double own = w / (kf * (kf + 1.0));
    sca += w * 2.0 * (re_mul_conj(dak, ak) + re_mul_conj(dbk, bk));
    const cplx t = scale(dak - dbk, w);
    back = (k % 2 == 0) ? back + t : back - t;
    if (k < n) {
      const cplx a1 = st.a[k], b1 = st.b[k], da1 = st.da_dx[k], db1 = st.db_dx[k];
      g += pair * (re_mul_conj(dak, a1) + re_mul_conj(ak, da1) + re_mul_conj(dbk, b1) +
                   re_mul_conj(bk, db1));
    }
    g += own * (re_mul_conj(dak, bk) + re_mul_conj(ak, dbk));
  }
  const double inv_x = 1.0 / st.x, inv_x2 = inv_x * inv_x, two_x2 = 2.0 * inv_x2;
  const double dsca = two_x2 * sca - 2.0 * inv_x * q.q_sca;
  const double dabs = two_x2 * st.abs_sum_jacobian[0] - 2.0 * inv_x * q.q_abs;
  const double dback = 2.0 * re_mul_conj(back, vs.back) * inv_x2 - 2.0 * inv_x * q.q_back;
  const double dg = vs.sca == 0.0 ? 0.0 : (2.0 * g - q.g * sca) / vs.sca;
  return {dsca + dabs, dsca, dabs, dback, dg};
}

// The efficiencies' derivatives along direction p (0: Re m, 1: Im m, with d/d(Im m) = i d/dm)
// of a sphere solved with derivatives: derivative_sums (efficiencies.rs:89-146) and
// efficiencies_jacobian (192-230). q are the sphere's efficiencies.
inline Efficiencies efficiency_dir(const MieState& st, int p, const Efficiencies& q) {
  const int64_t n = (int64_t)st.a.size();
  const Sums vs = value_sums(st.a.data(), st.b.data(), n);
  double sca = 0.0, g = 0.0;
  cplx back = real(0.0);
  auto dA = [&](int64_t i) { return p == 0 ? st.da_dm[i] : times_i(st.da_dm[i]); };
  auto dB = [&](int64_t i) { return p == 0 ? st.db_dm[i] : times_i(st.db_dm[i]); };
  for (int64_t k = 1; k <= n; ++k) {
    const cplx ak = st.a[k - 1], bk = st.b[k - 1], dak = dA(k - 1), dbk = dB(k - 1);
    const double w = (double)(2 * k + 1), kf = (double)k;
    const double pair = kf * (kf + 2.0) / (kf + 1.0);
    const double own = w / (kf * (kf + 1.0));
    sca += w * 2.0 * (re_mul_conj(dak, ak) + re_mul_conj(dbk, bk));
    const cplx t = scale(dak - dbk, w);
    back = (k % 2 == 0) ? back + t : back - t;
    if (k < n) {
      const cplx a1 = st.a[k], b1 = st.b[k], da1 = dA(k), db1 = dB(k);
      g += pair * (re_mul_conj(dak, a1) + re_mul_conj(ak, da1) + re_mul_conj(dbk, b1) +
                   re_mul_conj(bk, db1));
    }
    g += own * (re_mul_conj(dak, bk) + re_mul_conj(ak, dbk));
  }
  const double inv_x = 1.0 / st.x, inv_x2 = inv_x * inv_x, two_x2 = 2.0 * inv_x2;
  const double dsca = two_x2 * sca;
  const double dabs = two_x2 * st.abs_sum_jacobian[1 + p];
  const double dback = 2.0 * re_mul_conj(back, vs.back) * inv_x2;
  const double dg = vs.sca == 0.0 ? 0.0 : (2.0 * g - q.g * sca) / vs.sca;
  return {dsca + dabs, dsca, dabs, dback, dg};
}

// ---------------------------------------------------------------------------------------
// Angular functions, amplitudes and the phase matrix (mie/amplitudes.rs:52-65, 328-344;
// mie/phase.rs:54-59, 151-158, 204-219).
// ---------------------------------------------------------------------------------------
// for_each_order: calls f(n, w*pi_n, w*tau_n), w = (2n+1)/(n(n+1)).
template <class F>
inline void for_each_order(double mu, int64_t n_max, F f) {
  double pi_prev = 0.0, pi = 1.0;
  for (int64_t n = 1; n <= n_max; ++n) {
    double nf = (double)n;
    double n1 = nf + 1.0;
    double tau = nf * mu * pi - n1 * pi_prev;
    double w = (double)(2 * n + 1) / (nf * n1);
    f(n, w * pi, w * tau);
    double pi_next = ((double)(2 * n + 1) * mu * pi - n1 * pi_prev) / nf;
    pi_prev = pi;
    pi = pi_next;
  }
}

inline void amplitudes(const cplx* a, const cplx* b, int64_t n, double mu, cplx* s1o, cplx* s2o) {
  cplx s1 = real(0.0), s2 = real(0.0);
  for_each_order(mu, n, [&](int64_t k, double p, double t) {
    cplx an = a[k - 1], bn = b[k - 1];
    s1 = s1 + scale(an, p) + scale(bn, t);
    s2 = s2 + scale(an, t) + scale(bn, p);
  });
  *s1o = s1;
  *s2o = s2;
}

// elements (phase.rs:54-59): (|S1|^2+|S2|^2)/2, (|S2|^2-|S1|^2)/2, Re(S2 S1*), Im(S2 S1*).
inline void elements(cplx s1, cplx s2, double out[4]) {
  double n1 = norm_sqr(s1), n2 = norm_sqr(s2);
  cplx p = s2 * conj(s1);
  out[0] = 0.5 * (n1 + n2);
  out[1] = 0.5 * (n2 - n1);
  out[2] = p.re;
  out[3] = p.im;
}

// element_derivatives (phase.rs:62-73): the elements' derivatives for amplitude derivatives
// (d1, d2).
inline void element_derivs(cplx s1, cplx s2, cplx d1, cplx d2, double out[4]) {
  double r1 = (conj(s1) * d1).re;
  double r2 = (conj(s2) * d2).re;
  cplx p = d2 * conj(s1) + s2 * conj(d1);
  out[0] = r1 + r2;
  out[1] = r2 - r1;
  out[2] = p.re;
  out[3] = p.im;
}

// ---------------------------------------------------------------------------------------
// Gauss-Legendre rules (special/gauss_legendre.rs). Restated with Newton iteration on P_n in
// 80-bit extended precision from Tricomi's starting guess (the same guess as
// gauss_legendre.rs:128-137), rounded once to double. The reference rounds a double-double
// rule for n <= 100 and uses Bogaert's expansions above; both are within a few ulps of the
// exact rule, which the golden tests pin.
// ---------------------------------------------------------------------------------------
// The iteration runs on the angle theta (x = cos theta), so that 1 - x^2 = sin^2 theta keeps
// its relative accuracy next to +-1, where the weights are ill-conditioned in the nodes.
inline void gauss_legendre(int64_t n, double* nodes, double* weights) {
  typedef long double ld;
  int64_t half = (n + 1) / 2;
  for (int64_t i = 0; i < half; ++i) {
    // P_n(x) and P_{n-1}(x) by the three-term recurrence.
    auto eval = [&](ld xv, ld* p_out, ld* pm_out) {
      ld p_prev = 1.0L, p = xv;
      for (int64_t j = 2; j <= n; ++j) {
        ld next = ((ld)(2 * j - 1) * xv * p - (ld)(j - 1) * p_prev) / (ld)j;
        p_prev = p;
        p = next;
      }
      *p_out = p;
      *pm_out = p_prev;
    };
    ld x, s2, dp;
    if (2 * i + 1 == n) {
      x = 0.0L;
      ld p, pm;
      eval(x, &p, &pm);
      s2 = 1.0L;
      dp = (ld)n * pm;
    } else {
      double nf = (double)n;
      double k = (double)(i + 1);
      double theta0 = PI * (4.0 * k - 1.0) / (4.0 * nf + 2.0);
      double guess = (1.0 - (nf - 1.0) / (8.0 * nf * nf * nf)) * std::cos(theta0);
      ld th = acosl((ld)guess);
      // Newton on f(theta) = P_n(cos theta), f' = -sin theta P_n'(cos theta), until the step is
      // below 1e-17, then two polishing steps.
      int polish = 0;
      for (int it = 0; it < 100 && polish < 2; ++it) {
        ld c = cosl(th), s = sinl(th);
        ld p, pm;
        eval(c, &p, &pm);
        ld dpx = (ld)n * (pm - c * p) / (s * s);
        ld step = p / (s * dpx);
        th += step;
        if (std::fabs((double)step) <= 1e-17) ++polish;
      }
      x = cosl(th);
      ld s = sinl(th);
      s2 = s * s;
      ld p, pm;
      eval(x, &p, &pm);
      dp = (ld)n * (pm - x * p) / s2;
    }
    ld w = 2.0L / (s2 * dp * dp);
    // Ascending nodes: the (i+1)-th largest root sits at n-1-i, its mirror at i.
    nodes[n - 1 - i] = (double)x;
    nodes[i] = -(double)x;
    weights[n - 1 - i] = (double)w;
    weights[i] = (double)w;
    if (2 * i + 1 == n) {
      nodes[i] = 0.0;
    }
  }
}

// ---------------------------------------------------------------------------------------
// Wigner d functions for |m|, |n| <= 2 (special/wigner.rs:152-520). The scaled phase for
// start values below 2^-900 (wigner.rs:268-301) is never entered for |m|, |n| <= 2 at
// double-precision cosines: the start value is at least ((1-x)/2)^2 >= 2^-108.
// ---------------------------------------------------------------------------------------
inline void start_value(uint64_t a, uint64_t b, double x, double* v_out) {
  double half_sin = std::sqrt((1.0 - x) * 0.5);
  double half_cos = std::sqrt((1.0 + x) * 0.5);
  if (a >= 2 && half_sin == 0.0) {
    if (a > 2) {
      *v_out = 0.0;
      return;
    }
    double b1 = (double)b + 1.0, b2 = (double)b + 2.0;
    double v = (1.0 - x) * 0.5 * std::sqrt(b1 * b2 * 0.5);
    for (uint64_t i = 0; i < b; ++i) v *= half_cos;
    *v_out = v;
    return;
  }
  double v = 1.0;
  uint64_t top = std::max(a, b);
  for (uint64_t k = 1; k <= top; ++k) {
    if (k <= a) v = v * std::sqrt((double)(b + k) / (double)k) * half_sin;
    if (k <= b) v *= half_cos;
  }
  *v_out = v;
}

// wigner_d (wigner.rs:152-184) with three_term (232-248), difference_form (251-266),
// general_difference_form (269-290) and the steps of ThreeTerm (330-346), Difference
// (360-379) and GeneralDifference (400-415).
inline void wigner_d(int m, int n, double x, double* out, int64_t len) {
  int64_t lm = std::max(std::abs(m), std::abs(n));
  if (lm >= len) {
    for (int64_t l = 0; l < len; ++l) out[l] = 0.0;
    return;
  }
  for (int64_t l = 0; l < lm; ++l) out[l] = 0.0;
  int64_t l_min = lm;
  bool reflect = x < 0.0 && (m == -n || -x >= 0.9);
  int64_t nn = n;
  double xx = x;
  if (reflect) {
    nn = -n;
    xx = -x;
  }
  int64_t mm = m;
  auto run_state = [&](auto step, int64_t s, double st0, double st1) {
    double state[2] = {st0, st1};
    out[s] = state[1];
    while (s + 1 < len) {
      step(s, state);
      s += 1;
      out[s] = state[1];
    }
  };
  if (mm == nn && xx >= 0.0) {
    uint64_t b = 2 * (uint64_t)std::llabs(mm);
    double start;
    start_value(0, b, xx, &start);
    double w = xx - 1.0;
    double mf = (double)mm;
    auto step = [&](int64_t s, double* state) {
      double delta = state[0], cur = state[1];
      double sf = (double)s;
      double s1 = sf + 1.0;
      double k = (2.0 * sf + 1.0) * sf * s1;
      double bb = s1 * ((sf - mf) * (sf + mf));
      double c = sf * ((s1 - mf) * (s1 + mf));
      double next = (w * k * cur + delta * bb) * (1.0 / c);
      state[0] = next;
      state[1] = cur + next;
    };
    if (l_min == 0) {
      out[0] = start;
      if (len > 1) run_state(step, 1, w, xx);
    } else {
      run_state(step, l_min, start, start);
    }
  } else if (xx >= 0.9) {
    uint64_t a = (uint64_t)std::llabs(mm - nn), b = (uint64_t)std::llabs(mm + nn);
    double mag;
    start_value(a, b, xx, &mag);
    double start = (nn >= mm || (mm - nn) % 2 == 0) ? mag : -mag;
    double mf = (double)mm, nf = (double)nn, lf = (double)l_min;
    double w = xx - 1.0;
    double q = 0.0;
    double u = lf * (lf + 1.0) - mf * nf;
    auto step = [&](int64_t s, double* state) {
      double delta = state[0], cur = state[1];
      double sf = (double)s;
      double s1 = sf + 1.0;
      double q1 = std::sqrt(((s1 - mf) * (s1 + mf)) * ((s1 - nf) * (s1 + nf)));
      double alpha = sf * s1 - mf * nf;
      double dmn = mf - nf;
      double numer = s1 * s1 * (1.0 + dmn * dmn - 2.0 * s1) + (2.0 * s1) * (mf * nf);
      double v = numer / (alpha + q1);
      double k = w * ((2.0 * sf + 1.0) * sf * s1) + u * s1 + v * sf;
      double next = (k * cur + delta * (q * s1)) * (1.0 / (q1 * sf));
      q = q1;
      u = v + 2.0 * s1;
      state[0] = next;
      state[1] = cur + next;
    };
    run_state(step, l_min, start, start);
  } else {
    uint64_t a = (uint64_t)std::llabs(mm - nn), b = (uint64_t)std::llabs(mm + nn);
    double mag;
    start_value(a, b, xx, &mag);
    double start = (nn >= mm || (mm - nn) % 2 == 0) ? mag : -mag;
    double mf = (double)mm, nf = (double)nn;
    double q = 0.0;
    auto step = [&](int64_t s, double* state) {
      double prev = state[0], cur = state[1];
      double sf = (double)s;
      double c_prev = q * (sf + 1.0);
      double numer = (xx * (sf * (sf + 1.0)) - mf * nf) * (2.0 * sf + 1.0) * cur - c_prev * prev;
      double s1 = sf + 1.0;
      q = std::sqrt((s1 - mf) * (s1 + mf)) * std::sqrt((s1 - nf) * (s1 + nf));
      state[0] = cur;
      state[1] = numer / (q * sf);
    };
    run_state(step, l_min, 0.0, start);
  }
  if (reflect) {
    int64_t parity = ((l_min + mm) % 2 + 2) % 2;
    int64_t first_odd = 1 - parity;
    for (int64_t l = l_min + first_odd; l < len; l += 2) out[l] = -out[l];
  }
}

// ---------------------------------------------------------------------------------------
// Greek projection (mie/greek.rs:161-220, 386-447, 501-509).
// ---------------------------------------------------------------------------------------
struct Greek {
  std::vector<double> c[6];  // alpha1, alpha2, alpha3, alpha4, beta1, beta2
  void zeros(int64_t len) {
    for (auto& v : c) v.assign(len, 0.0);
  }
};

// GreekProjector::project for one table at the rule (nodes, weights), orders 0..order.
inline Greek project(const double* nodes, const double* weights, int64_t n_q, int64_t order,
                     const double* f11, const double* f12, const double* f33, const double* f34) {
  int64_t len = order + 1;
  Greek g;
  g.zeros(len);
  std::vector<double> d00(len), d22(len), d2m2(len), d02(len);
  for (int64_t k = 0; k < n_q; ++k) {
    double mu = nodes[k], w = weights[k];
    wigner_d(0, 0, mu, d00.data(), len);
    wigner_d(2, 2, mu, d22.data(), len);
    wigner_d(2, -2, mu, d2m2.data(), len);
    wigner_d(0, 2, mu, d02.data(), len);
    double a11 = w * f11[k];
    double a33 = w * f33[k];
    double sum = a11 + a33, diff = a11 - a33;
    double a12 = w * f12[k], a34 = w * f34[k];
    for (int64_t l = 0; l < len; ++l) {
      g.c[0][l] += a11 * d00[l];
      g.c[3][l] += a33 * d00[l];
      g.c[1][l] += sum * d22[l];
      g.c[2][l] += diff * d2m2[l];
      g.c[4][l] += a12 * d02[l];
      g.c[5][l] += a34 * d02[l];
    }
  }
  for (int64_t l = 0; l < len; ++l) {
    double s = (double)(2 * l + 1) * 0.5;
    double plus = g.c[1][l], minus = g.c[2][l];
    g.c[0][l] *= s;
    g.c[3][l] *= s;
    g.c[1][l] = s * 0.5 * (plus + minus);
    g.c[2][l] = s * 0.5 * (plus - minus);
    g.c[4][l] *= s;
    g.c[5][l] *= s;
  }
  return g;
}

// ---------------------------------------------------------------------------------------
// Size distributions (scatrs/src/ensemble/distribution.rs:15-468).
// ---------------------------------------------------------------------------------------
enum DistKind { LOGNORMAL = 1, GAMMA = 2, MODIFIED_GAMMA = 3, POWER_LAW = 4, TABULATED = 6 };

struct Density {
  int kind;
  double p0, p1, p2;
  double reference;
  double log_width;
  // TABULATED: table_len radii (increasing) followed by their table_len densities.
  const double* table = nullptr;
  int64_t table_len = 0;
};

// interpolate (distribution.rs:458-468): linear through the points, 0 outside them.
inline double table_interpolate(const double* r_tab, const double* n_tab, int64_t n, double r) {
  if (r < r_tab[0] || r > r_tab[n - 1]) return 0.0;
  int64_t i = std::upper_bound(r_tab, r_tab + n, r) - r_tab;  // first radius above r
  i = std::min<int64_t>(std::max<int64_t>(i, 1), n - 1);
  const double t = (r - r_tab[i - 1]) / (r_tab[i] - r_tab[i - 1]);
  return n_tab[i - 1] + t * (n_tab[i] - n_tab[i - 1]);
}

// SizeDistribution::validate for Tabulated (distribution.rs:149-172).
inline bool table_valid(const double* table, int64_t n, std::string* msg) {
  if (table == nullptr || n < 2) {
    *msg = "a tabulated distribution needs at least 2 points and as many densities as radii";
    return false;
  }
  const double* dens = table + n;
  bool any = false;
  for (int64_t i = 0; i < n; ++i) {
    if (!(std::isfinite(table[i]) && table[i] > 0.0)) {
      *msg = "radius must be finite and > 0";
      return false;
    }
    if (i > 0 && !(table[i - 1] < table[i])) {
      *msg = "tabulated radii must increase";
      return false;
    }
    if (!(std::isfinite(dens[i]) && dens[i] >= 0.0)) {
      *msg = "tabulated densities must be finite and >= 0";
      return false;
    }
    any = any || dens[i] != 0.0;
  }
  if (!any) *msg = "tabulated densities must not all be 0";
  return any;
}

// SizeDistribution::prepare (distribution.rs:296-355).
inline Density prepare(int kind, double p0, double p1, double p2) {
  Density d{kind, p0, p1, p2, 1.0, std::numeric_limits<double>::infinity()};
  switch (kind) {
    case LOGNORMAL:
      d.reference = p0;
      d.log_width = std::log(p1);
      break;
    case GAMMA: {
      double a = p0, b = p1;
      double alpha = (1.0 - 3.0 * b) / b;
      d.reference = alpha > 0.0 ? alpha * a * b : a;
      d.log_width = std::sqrt(b / (1.0 - 2.0 * b));
      break;
    }
    case MODIFIED_GAMMA: {
      double alpha = p0, b = p1, gamma = p2;
      d.reference = std::pow(std::max(alpha, 1.0) / (b * gamma), 1.0 / gamma);
      d.log_width = alpha > 0.0 ? 1.0 / std::sqrt(alpha * gamma) : 1.0 / gamma;
      break;
    }
    case POWER_LAW:
      d.reference = p0 >= 0.0 ? p1 : p2;
      break;
  }
  return d;
}

// A tabulated density: reference radius 1, no width limit on the steps.
inline Density prepare_table(const double* table, int64_t n) {
  Density d = prepare(TABULATED, 0.0, 0.0, 0.0);
  d.table = table;
  d.table_len = n;
  return d;
}

// Density::eval (distribution.rs:370-441): u(r) and its gradient (up to 3 parameters).
inline double density_eval(const Density& d, double r, double* grad) {
  double r0 = d.reference;
  double ln_u = 0.0, dln[3] = {0, 0, 0};
  switch (d.kind) {
    case LOGNORMAL: {
      double median = d.p0, width = d.p1;
      double mu = std::log(median), s = std::log(width);
      double z = std::log(r) - mu;
      ln_u = -z * z / (2.0 * s * s) - std::log(s) - std::log(r / r0);
      dln[0] = z / (s * s * median);
      dln[1] = (z * z / (s * s * s) - 1.0 / s) / width;
      break;
    }
    case GAMMA: {
      double a = d.p0, b = d.p1;
      double alpha = (1.0 - 3.0 * b) / b;
      double sc = a * b;
      double l = std::log(r / r0);
      ln_u = alpha * l - (r - r0) / sc;
      dln[0] = (r - r0) * b / (sc * sc);
      dln[1] = -l / (b * b) + (r - r0) * a / (sc * sc);
      break;
    }
    case MODIFIED_GAMMA: {
      double alpha = d.p0, b = d.p1, gamma = d.p2;
      double rg = std::pow(r, gamma), r0g = std::pow(r0, gamma);
      double l = std::log(r / r0);
      ln_u = alpha * l - b * (rg - r0g);
      dln[0] = l;
      dln[1] = -(rg - r0g);
      dln[2] = -b * (rg * std::log(r) - r0g * std::log(r0));
      break;
    }
    case TABULATED: {
      if (grad) grad[0] = grad[1] = grad[2] = 0.0;
      return table_interpolate(d.table, d.table + d.table_len, d.table_len, r);
    }
    case POWER_LAW: {
      double ex = d.p0, lo = d.p1, hi = d.p2;
      if (r < lo || r > hi) {
        if (grad) grad[0] = grad[1] = grad[2] = 0.0;
        return 0.0;
      }
      double l = std::log(r / r0);
      ln_u = -ex * l;
      dln[0] = -l;
      break;
    }
  }
  double u = std::exp(ln_u);
  if (grad)
    for (int i = 0; i < 3; ++i) grad[i] = u * dln[i];
  return u;
}

// ---------------------------------------------------------------------------------------
// Bands (scatrs/src/ensemble/engine.rs:951-957, 2034-2072).
// ---------------------------------------------------------------------------------------
inline int64_t bucket(int64_t n) {
  int64_t u = 1;
  while (u < n) u = (int64_t)std::ceil((double)u * 1.25);
  return u;
}

// Layered::check_inputs (layered/mod.rs:233-305) with the default truncation.
inline int check_layered(const std::vector<double>& x, const std::vector<cplx>& m,
                         bool allow_unvalidated, std::string* msg) {
  const size_t L = x.size();
  for (size_t l = 0; l < L; ++l)
    if (!std::isfinite(x[l]) || (l > 0 && x[l] < x[l - 1])) {
      *msg = "the size parameters must be finite and nondecreasing from the core out";
      return INVALID_INPUT;
    }
  const double outer = x[L - 1];
  if (x[0] < MIN_SIZE_PARAMETER || outer > MAX_SIZE_PARAMETER) {
    *msg = "the size parameters must be in [1e-30, 1e6]";
    return INVALID_INPUT;
  }
  for (auto& v : m) {
    if (!(std::isfinite(v.re) && std::isfinite(v.im)) || v.re < 0.0 || v.im < 0.0 ||
        !(cnorm(v) >= MIN_REFRACTIVE_INDEX && cnorm(v) <= MAX_REFRACTIVE_INDEX)) {
      *msg = "invalid refractive index of a layer";
      return INVALID_INPUT;
    }
  }
  if (!allow_unvalidated) {
    bool in = L <= 16 && outer >= 1e-6 && outer <= 1e4;
    for (auto& v : m)
      in = in && cnorm(v) * outer <= 3e4 && v.re > 0.0 && v.re <= 10.0 && v.im >= 0.0 &&
           v.im <= 10.0 && cnorm(v) >= 0.1;
    if (!in) {
      *msg = "outside the validated domain of layered spheres";
      return OUTSIDE_VALIDATED_DOMAIN;
    }
  }
  return OK;
}


// ---------------------------------------------------------------------------------------
// Distributions as the C ABI passes them, and a projector band's tables (engine.rs:2034-2072,
// fast.rs:22-50, 210-235).
// ---------------------------------------------------------------------------------------
struct FixedDist {
  int32_t kind;
  int32_t pad;
  double p[3];
  double r_lo, r_hi;
  const double* table;  // TABULATED: radii then densities, table_len of each
  int64_t table_len;
};

inline Density prepare(const FixedDist& d) {
  return d.kind == TABULATED ? prepare_table(d.table, d.table_len)
                             : prepare(d.kind, d.p[0], d.p[1], d.p[2]);
}

constexpr int NODES_PER_CHUNK = 32;

struct BandData {
  int64_t upper;
  int64_t order;  // L_b
  int64_t n_q;
  std::vector<double> nodes, weights;
  std::vector<double> ge, go;  // h x upper, row-major
  std::vector<double> dmat[4];  // n_q x (L_b+1): (2l+1)/2 w_k d_l(mu_k)
};

inline BandData make_band(int64_t upper, int64_t order) {
  BandData b;
  b.upper = upper;
  b.order = std::min(order, 2 * upper);
  b.n_q = upper + (b.order + 2) / 2;
  b.nodes.resize(b.n_q);
  b.weights.resize(b.n_q);
  gauss_legendre(b.n_q, b.nodes.data(), b.weights.data());
  int64_t lo = b.n_q / 2, h = b.n_q - lo;
  b.ge.assign(h * upper, 0.0);
  b.go.assign(h * upper, 0.0);
  for (int64_t i = 0; i < h; ++i) {
    for_each_order(b.nodes[lo + i], upper, [&](int64_t k, double pi, double tau) {
      bool odd = k % 2 == 1;
      b.ge[i * upper + (k - 1)] = odd ? pi : tau;
      b.go[i * upper + (k - 1)] = odd ? tau : pi;
    });
  }
  int64_t len = b.order + 1;
  std::vector<double> buf(len);
  const int mn[4][2] = {{0, 0}, {2, 2}, {2, -2}, {0, 2}};
  for (int i = 0; i < 4; ++i) b.dmat[i].assign(b.n_q * len, 0.0);
  for (int64_t k = 0; k < b.n_q; ++k) {
    for (int i = 0; i < 4; ++i) {
      wigner_d(mn[i][0], mn[i][1], b.nodes[k], buf.data(), len);
      for (int64_t l = 0; l < len; ++l)
        b.dmat[i][k * len + l] = (double)(2 * l + 1) * 0.5 * b.weights[k] * buf[l];
    }
  }
  return b;
}

}  // namespace orc
