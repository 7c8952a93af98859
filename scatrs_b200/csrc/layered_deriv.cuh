// Derivatives of a layered sphere's Mie coefficients along one parameter (layered/kernel.rs's
// solve with its derivatives, restated in forward mode): every quantity of the value recursion
// of mie_device.cuh (Layered, LArg, layer_side, the outer part of mie_finish) carries its
// derivative along a real parameter t, or the complex derivative along a layer's index m_l (the
// coefficients are holomorphic in each m_l, so the derivative along Im m_l is i times it).
// Values are computed by the same expressions as the value path; branches (the chi / xi choice
// per shell, the direct form near D_n's poles, the upward and ratio regimes) follow the values.
// The ratio arrays u_k(m_l x) are differentiated through their downward recurrences.
#pragma once

#include "mie_device.cuh"

namespace sb {
namespace lder {

struct DR {  // a real value and its derivative
  double v, d;
};
struct DC {  // a complex value and its derivative
  cplx v, d;
};

__device__ __forceinline__ DC dc(cplx v) { return DC{v, rl(0.0)}; }
__device__ __forceinline__ DC operator+(DC a, DC b) { return DC{a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ DC operator-(DC a, DC b) { return DC{a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ DC operator-(DC a) { return DC{-a.v, -a.d}; }
__device__ __forceinline__ DC operator*(DC a, DC b) { return DC{a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ __forceinline__ DC operator*(DC a, cplx b) { return DC{a.v * b, a.d * b}; }
__device__ __forceinline__ DC operator*(cplx a, DC b) { return DC{a * b.v, a * b.d}; }
__device__ __forceinline__ DC operator+(DC a, cplx b) { return DC{a.v + b, a.d}; }
__device__ __forceinline__ DC operator-(DC a, cplx b) { return DC{a.v - b, a.d}; }
__device__ __forceinline__ DC operator-(cplx a, DC b) { return DC{a - b.v, -b.d}; }
__device__ __forceinline__ DC dinv(DC a) {
  const cplx iv = cinv(a.v);
  return DC{iv, -(a.d * iv * iv)};
}
__device__ __forceinline__ DC dscl(DC a, double s) { return DC{scl(a.v, s), scl(a.d, s)}; }
__device__ __forceinline__ DC dscl(DC a, DR s) {
  return DC{scl(a.v, s.v), scl(a.d, s.v) + scl(a.v, s.d)};
}
__device__ __forceinline__ DC dsin(DC z) { return DC{csin(z.v), ccos(z.v) * z.d}; }
__device__ __forceinline__ DC dcos(DC z) { return DC{ccos(z.v), -(csin(z.v) * z.d)}; }
__device__ __forceinline__ DC dexp_m1(DC w) {
  const cplx e = cexp_m1(w.v);
  return DC{e, (e + rl(1.0)) * w.d};
}
__device__ __forceinline__ DC dtwo_i(DC z) { return DC{two_i(z.v), two_i(z.d)}; }

// Ratio arrays with their derivatives: value array a at a, its derivative at a + n_val.
struct ArraysD {
  LayerArrays arr;
  int n_val;
  __device__ __forceinline__ DC get(int a, int64_t k) const {
    return DC{arr.get(a, k), arr.get(a + n_val, k)};
  }
  __device__ __forceinline__ void put(int a, int64_t k, DC v) const {
    arr.put(a, k, v.v);
    arr.put(a + n_val, k, v.d);
  }
};

// ratios_into with derivatives: u_k(m x), k = 1..n+1, of the downward recurrence
// u_k = 1/((2k+1)/z - u_{k+1}) (kernel.rs:116-136, 159-205).
__device__ __forceinline__ void ratios_d(DC m, DR x, int64_t n, const ArraysD& A, int a) {
  const DC z = dscl(m, x);
  const int64_t top = n + 1;
  if (m.v.im == 0.0) {
    // The real form; z and its derivative are real here.
    const double inv_rho = 1.0 / z.v.re;
    const double d_inv_rho = -z.d.re * inv_rho * inv_rho;
    double u = 0.0, du = 0.0;
    const int64_t start = start_index(top, fabs(z.v.re));
    for (int64_t k = start; k >= 1; --k) {
      const double c = inv_rho * (double)(2 * k + 1);
      const double dcv = d_inv_rho * (double)(2 * k + 1);
      double den = c - u, dden = dcv - du;
      if (den == 0.0) {
        den = kEps * (fabs(c) + fabs(u));
        dden = 0.0;
      }
      u = 1.0 / den;
      du = -dden * u * u;
      if (k <= top) A.put(a, k, DC{rl(u), rl(du)});
    }
  } else {
    const DC inv_z = dinv(z);
    DC u = dc(rl(0.0));
    const int64_t start = start_index(top, cabs_(z.v));
    for (int64_t k = start; k >= 1; --k) {
      const DC c = dscl(inv_z, (double)(2 * k + 1));
      DC den = c - u;
      if (den.v.re == 0.0 && den.v.im == 0.0) den = dc(rl(kEps * (cabs_(c.v) + cabs_(u.v))));
      u = dinv(den);
      if (k <= top) A.put(a, k, u);
    }
  }
}

// LArg (layered/kernel.rs:33-103) with derivatives.
struct LArgD {
  DC z, inv_z, pi, w, w_n;
  __device__ __forceinline__ void init(DC zz, bool chi) {
    z = zz;
    inv_z = dinv(z);
    if (chi) {
      const DC sz = dsin(z), cz = dcos(z);
      pi = sz * cz;
      w = inv_z + sz * dinv(cz);
    } else {
      pi = -dscl(dexp_m1(dtwo_i(z)), 0.5);
      w = inv_z - mk(0.0, 1.0);
    }
    w_n = dc(rl(0.0));
  }
  __device__ __forceinline__ void step(int64_t n, DC u_n) {
    w_n = w;
    pi = pi * u_n * w;
    w = dscl(inv_z, (double)(2 * n + 1)) - dinv(w);
  }
  __device__ __forceinline__ DC d1(int64_t n, DC u_next) const {
    return dscl(inv_z, (double)(n + 1)) - u_next;
  }
  __device__ __forceinline__ DC d3(int64_t n) const { return dscl(inv_z, (double)(n + 1)) - w; }
};

struct SideD {
  bool direct;
  DC v;
};

// layer_side (layered/kernel.rs:158-183) with derivatives; the branch follows the values.
__device__ __forceinline__ SideD layer_side_d(DC mi, DC mo, SideD prev, DC h, DC lead, DC u_prev,
                                              DC u1, DC d1i, DC d3i, DC d1o, DC d3o, DC pio, DC p,
                                              cplx w, DC* h_out) {
  const DC mh = mi * h;
  const DC g1 = prev.direct ? mh - mo * d1i : lead - mi * u_prev + mo * u1 + mi * prev.v;
  const DC g2 = mh - mo * d3i;
  const DC inv_den = dinv(pio * g2 - p * g1);
  const DC delta = -(w * p * g1 * inv_den * dinv(pio));
  const DC hd = d1o + delta;
  if (norm1(hd.v) * 4.0 >= fmax(norm1(d1o.v), norm1(delta.v))) {
    *h_out = hd;
    return {false, delta};
  }
  const DC hp = d3o - w * g2 * inv_den;
  *h_out = hp;
  return {true, hp};
}

// Layered (mie_device.cuh) with derivatives: interface sizes x[l] and indices m[l] with their
// derivatives along the parameter, for at most kCap layers (the per-shell state sized at
// compile time, so that a few layers stay out of local memory).
template <int kCap>
struct LayeredD {
  int layers;
  const DR* x;
  const DC* m;
  ArraysD arr;
  LArgD inner[kCap - 1], outer[kCap - 1], core;
  DC p[kCap - 1], lead[kCap - 1];
  bool chi[kCap - 1];

  __device__ __forceinline__ int a_outer(int l) const { return l == layers - 1 ? 0 : 2 * l + 1; }
  __device__ __forceinline__ int a_inner(int l) const { return 2 * l; }
  static constexpr int kCore = 1;

  // Every ratio array (the outer argument's, array 0, included) and the initial state.
  __device__ void prepare(int64_t n, DR x_outer) {
    const int last = layers - 1;
    ratios_d(m[last], x_outer, n, arr, 0);
    ratios_d(m[0], x[0], n, arr, kCore);
    for (int l = 1; l < layers; ++l) {
      ratios_d(m[l], x[l - 1], n, arr, a_inner(l));
      if (l < last) ratios_d(m[l], x[l], n, arr, a_outer(l));
    }
    for (int l = 1; l < layers; ++l) {
      const bool c = m[l].v.im * x[l].v < 0.5;
      chi[l - 1] = c;
      const DC a = m[l], b = m[l - 1];
      lead[l - 1] = (a - b) * (a + b) * dinv(a * b);
      const DC z1 = dscl(m[l], x[l - 1]), z2 = dscl(m[l], x[l]);
      inner[l - 1].init(z1, c);
      outer[l - 1].init(z2, c);
      if (c) {
        const DC c2 = dcos(z2);
        p[l - 1] = dsin(z1) * dinv(dcos(z1)) * c2 * c2;
      } else {
        const DR dx{x[l].v - x[l - 1].v, x[l].d - x[l - 1].d};
        const DR ea{-(m[l].v.im * dx.v * 2.0), -(m[l].d.im * dx.v + m[l].v.im * dx.d) * 2.0};
        const DR eb{m[l].v.re * dx.v * 2.0, (m[l].d.re * dx.v + m[l].v.re * dx.d) * 2.0};
        double sb, cb;
        sincos(eb.v, &sb, &cb);
        const double ex = exp(ea.v);
        const DC e{scl(mk(cb, sb), ex), scl(mk(-sb * eb.d, cb * eb.d), ex) +
                                            scl(mk(cb, sb), ex * ea.d)};
        p[l - 1] = -dscl(e * dexp_m1(dtwo_i(z1)), 0.5);
      }
    }
    core.init(dscl(m[0], x[0]), false);
  }

  __device__ __forceinline__ void order(int64_t k, SideD& sa, SideD& sb) {
    for (int l = 1; l < layers; ++l) {
      LArgD& ai = inner[l - 1];
      LArgD& ao = outer[l - 1];
      const DC u1k = arr.get(a_inner(l), k);
      ai.step(k, u1k);
      ao.step(k, arr.get(a_outer(l), k));
      p[l - 1] = p[l - 1] * u1k * dinv(ai.w_n) * ao.w_n * ao.w_n;
    }
    DC ha = core.d1(k, arr.get(kCore, k + 1));
    DC hb = ha;
    SideD a{false, dc(rl(0.0))}, b{false, dc(rl(0.0))};
    for (int l = 1; l < layers; ++l) {
      const LArgD& ai = inner[l - 1];
      const LArgD& ao = outer[l - 1];
      const DC u_prev = arr.get(l == 1 ? kCore : a_outer(l - 1), k + 1);
      const DC u1 = arr.get(a_inner(l), k + 1);
      const DC u2 = arr.get(a_outer(l), k + 1);
      const DC d1i = ai.d1(k, u1), d3i = ai.d3(k);
      const DC d1o = ao.d1(k, u2), d3o = ao.d3(k);
      const cplx w = chi[l - 1] ? rl(-1.0) : mk(0.0, 1.0);
      const DR q{(double)(k + 1) / x[l - 1].v,
                 -(double)(k + 1) * x[l - 1].d / (x[l - 1].v * x[l - 1].v)};
      const DC ld = dscl(lead[l - 1], q);
      DC na, nb;
      const SideD a2 = layer_side_d(m[l], m[l - 1], a, ha, ld, u_prev, u1, d1i, d3i, d1o, d3o,
                                    ao.pi, p[l - 1], w, &na);
      const SideD b2 = layer_side_d(m[l - 1], m[l], b, hb, dc(rl(0.0)), u_prev, u1, d1i, d3i,
                                    d1o, d3o, ao.pi, p[l - 1], w, &nb);
      ha = na;
      hb = nb;
      a = a2;
      b = b2;
    }
    sa = a;
    sb = b;
  }
};

// The outer part of mie_finish for a layered sphere (kernel.rs:324-559) with derivatives: x is
// the particle's size parameter (fixed), m its outer index (with its derivative). emit(k, a_k,
// b_k, da_k, db_k); the absorption sum's derivatives along the parameter (abs_d[0]) and, for a
// complex-derivative direction, along i times it (abs_d[1]). Returns the absorption sum.
template <class Emit, class Lay>
__device__ double layered_finish_d(double x, DC m, int64_t n, const Scratch& s, ValueSums& vs,
                                   Emit emit, Lay& layers, double abs_d[2]) {
  const double one = 1.0;
  const DC z = dscl(m, x);
  const int64_t n_s = upward_orders(x, n);
  const double inv_x = 1.0 / x;
  const DC inv_z = dinv(z);
  const DC inv_m = dinv(m);
  const DC inv_m2 = inv_m * inv_m;
  const DC m2_minus_1 = (m - rl(one)) * (m + rl(one));
  const DC c_a = -(m2_minus_1 * inv_m2);
  const bool unit_m = m.v.re == 1.0 && m.v.im == 0.0;
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
  abs_d[0] = abs_d[1] = 0.0;
  for (int64_t k = 1; k <= n; ++k) {
    const double k_x = (double)k * inv_x;
    const DC u_z1 = layers.arr.get(0, k + 1);
    const DC d = dscl(inv_z, (double)(k + 1)) - u_z1;
    SideD sa, sb;
    layers.order(k, sa, sb);
    const DC hh_a = sa.direct ? sa.v : d + sa.v;
    const DC hh_b = sb.direct ? sb.v : d + sb.v;
    const DC d_m = hh_a * inv_m;
    const DC md = hh_b * m;
    const DC big_a = d_m + rl(k_x);
    const DC big_b = md + rl(k_x);
    DC an, bn, inv_da, inv_db;
    if (k <= n_s) {
      const double c = (double)(2 * k - 1) * inv_x;
      const double psi_next = c * psi - psi_prev;
      psi_prev = psi;
      psi = psi_next;
      const double chi_next = c * chi - chi_prev;
      chi_prev = chi;
      chi = chi_next;
      const cplx xi = mk(psi, -chi);
      const cplx xi_prev = mk(psi_prev, -chi_prev);
      inv_da = dinv(big_a * xi - xi_prev);
      inv_db = dinv(big_b * xi - xi_prev);
      // The outer layer's own numerator (exactly 0 in value for m = 1, kernel.rs:412-435).
      DC own_a = dscl(d * inv_m + rl(k_x), psi) - rl(psi_prev);
      DC own_b = dscl(d * m + rl(k_x), psi) - rl(psi_prev);
      if (unit_m) {
        own_a.v = rl(0.0);
        own_b.v = rl(0.0);
      }
      an = sa.direct ? (dscl(big_a, psi) - rl(psi_prev)) * inv_da
                     : (own_a + dscl(sa.v * inv_m, psi)) * inv_da;
      bn = sb.direct ? (dscl(big_b, psi) - rl(psi_prev)) * inv_db
                     : (own_b + dscl(m * sb.v, psi)) * inv_db;
      if (k == n_s) {
        inv_xi = cinv(xi);
        t = rl(psi) * inv_xi;
        r = xi_prev * inv_xi;
      }
    } else {
      r = cinv(rl((double)(2 * k - 1) * inv_x) - r);
      t = scl(t * r, s.get_x(k));
      inv_xi = inv_xi * r;
      const cplx u_x1 = rl(s.get_x(k + 1));
      const cplx d_x = rl((double)(k + 1) * inv_x) - u_x1;
      const DC num_a = sa.direct ? d_m - d_x
                                 : dscl(c_a, (double)(k + 1) * inv_x) + u_x1 - u_z1 * inv_m +
                                       sa.v * inv_m;
      const DC num_b = sb.direct ? md - d_x : (dc(u_x1) - m * u_z1) + m * sb.v;
      const DC ia = dinv(big_a - r);
      const DC ib = dinv(big_b - r);
      an = t * num_a * ia;
      bn = t * num_b * ib;
      inv_da = inv_xi * ia;
      inv_db = inv_xi * ib;
    }
    vs.add(k, an.v, bn.v);
    const double na = nsq(inv_da.v), nb = nsq(inv_db.v);
    const double weight = (double)(2 * k + 1);
    asum += weight * (-(d_m.v.im * na) - md.v.im * nb);
    // |g|^2 and Im f along the parameter, and along i times it (holomorphic f and g).
    const cplx pa = mk(inv_da.v.re, -inv_da.v.im) * inv_da.d;
    const cplx pb = mk(inv_db.v.re, -inv_db.v.im) * inv_db.d;
    abs_d[0] += weight * (-(d_m.d.im * na + d_m.v.im * 2.0 * pa.re) -
                          (md.d.im * nb + md.v.im * 2.0 * pb.re));
    abs_d[1] += weight * (-(d_m.d.re * na - d_m.v.im * 2.0 * pa.im) -
                          (md.d.re * nb - md.v.im * 2.0 * pb.im));
    emit(k, an.v, bn.v, an.d, bn.d);
  }
  return asum;
}

}  // namespace lder
}  // namespace sb
