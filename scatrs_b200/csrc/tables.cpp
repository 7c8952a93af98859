// Host-side tables (see tables.h). Every routine follows the reference's arithmetic so that
// the tables hold the same doubles; the Gauss-Legendre rule is computed by Newton iteration on
// the angle in x87 extended precision and rounded once.
#include "tables.h"

#include <algorithm>
#include <cmath>
#include <limits>

namespace sb {

void gauss_legendre(int64_t n, double* nodes, double* weights) {
  typedef long double ld;
  const double pi = 3.14159265358979323846264338327950288;
  // P_n and P_{n-1} at x by the three-term recurrence.
  auto legendre = [n](ld x, ld* p, ld* pm) {
    ld a = 1.0L, b = x;
    for (int64_t j = 2; j <= n; ++j) {
      ld c = ((ld)(2 * j - 1) * x * b - (ld)(j - 1) * a) / (ld)j;
      a = b;
      b = c;
    }
    *p = b;
    *pm = a;
  };
  for (int64_t i = 0; i < (n + 1) / 2; ++i) {
    ld x, s2, p, pm;
    if (2 * i + 1 == n) {
      x = 0.0L;
      s2 = 1.0L;
      legendre(x, &p, &pm);
    } else {
      // Tricomi's approximation of the (i+1)-th largest root (gauss_legendre.rs:128-137),
      // then Newton on theta: theta += P_n(cos theta) / (sin theta P_n'(cos theta)).
      double nf = (double)n, k = (double)(i + 1);
      double th0 = pi * (4.0 * k - 1.0) / (4.0 * nf + 2.0);
      ld th = acosl((ld)((1.0 - (nf - 1.0) / (8.0 * nf * nf * nf)) * std::cos(th0)));
      for (int it = 0, small = 0; it < 100 && small < 2; ++it) {
        ld c = cosl(th), s = sinl(th);
        legendre(c, &p, &pm);
        ld step = p * s / ((ld)n * (pm - c * p));
        th += step;
        if (std::fabs((double)step) <= 1e-17) ++small;
      }
      x = cosl(th);
      ld s = sinl(th);
      s2 = s * s;
      legendre(x, &p, &pm);
    }
    ld dp = (ld)n * (pm - x * p) / s2;
    ld w = 2.0L / (s2 * dp * dp);
    nodes[n - 1 - i] = (double)x;
    nodes[i] = 2 * i + 1 == n ? 0.0 : -(double)x;
    weights[n - 1 - i] = (double)w;
    weights[i] = (double)w;
  }
}

namespace {

// sqrt(C(a+b, a)) sin^a(theta/2) cos^b(theta/2) (wigner.rs:423-460); for |m|, |n| <= 2 the
// value never leaves the normal range, so no exponent is carried.
double start_value(int a, int b, double x) {
  double hs = std::sqrt((1.0 - x) * 0.5);
  double hc = std::sqrt((1.0 + x) * 0.5);
  if (a >= 2 && hs == 0.0) {
    if (a > 2) return 0.0;
    double v = (1.0 - x) * 0.5 * std::sqrt(((double)b + 1.0) * ((double)b + 2.0) * 0.5);
    for (int i = 0; i < b; ++i) v *= hc;
    return v;
  }
  double v = 1.0;
  for (int k = 1; k <= std::max(a, b); ++k) {
    if (k <= a) v = v * std::sqrt((double)(b + k) / (double)k) * hs;
    if (k <= b) v *= hc;
  }
  return v;
}

}  // namespace

void wigner_d(int m, int n, double x, double* out, int64_t len) {
  const int64_t l0 = std::max(std::abs(m), std::abs(n));
  for (int64_t l = 0; l < std::min(l0, len); ++l) out[l] = 0.0;
  if (l0 >= len) return;
  // d^l_{mn}(x) = (-1)^{l+m} d^l_{m,-n}(-x) maps x = -1 onto x = 1 (wigner.rs:170-183).
  const bool flip = x < 0.0 && (m == -n || -x >= 0.9);
  if (flip) {
    n = -n;
    x = -x;
  }
  const double mf = m, nf = n;
  double st[2];
  int64_t s = l0;
  auto emit_and_run = [&](auto&& step) {
    out[s] = st[1];
    while (s + 1 < len) {
      step(s, st);
      ++s;
      out[s] = st[1];
    }
  };
  if (m == n && x >= 0.0) {
    // Reinsch's difference form for m = n (wigner.rs:351-380).
    const double w = x - 1.0;
    auto step = [&](int64_t si, double* v) {
      double sf = (double)si, s1 = sf + 1.0;
      double k = (2.0 * sf + 1.0) * sf * s1;
      double bb = s1 * ((sf - mf) * (sf + mf));
      double c = sf * ((s1 - mf) * (s1 + mf));
      double nx = (w * k * v[1] + v[0] * bb) * (1.0 / c);
      v[0] = nx;
      v[1] = v[1] + nx;
    };
    double start = start_value(0, 2 * std::abs(m), x);
    if (l0 == 0) {
      out[0] = start;
      if (len > 1) {
        s = 1;
        st[0] = w;
        st[1] = x;
        emit_and_run(step);
      }
    } else {
      st[0] = start;
      st[1] = start;
      emit_and_run(step);
    }
  } else {
    const int a = std::abs(m - n), b = std::abs(m + n);
    const double mag = start_value(a, b, x);
    const double start = (n >= m || (m - n) % 2 == 0) ? mag : -mag;
    if (x >= 0.9) {
      // The general difference form (wigner.rs:382-416).
      const double w = x - 1.0;
      double q = 0.0, u = (double)l0 * ((double)l0 + 1.0) - mf * nf;
      auto step = [&](int64_t si, double* v) {
        double sf = (double)si, s1 = sf + 1.0;
        double q1 = std::sqrt(((s1 - mf) * (s1 + mf)) * ((s1 - nf) * (s1 + nf)));
        double alpha = sf * s1 - mf * nf;
        double dmn = mf - nf;
        double numer = s1 * s1 * (1.0 + dmn * dmn - 2.0 * s1) + (2.0 * s1) * (mf * nf);
        double vv = numer / (alpha + q1);
        double k = w * ((2.0 * sf + 1.0) * sf * s1) + u * s1 + vv * sf;
        double nx = (k * v[1] + v[0] * (q * s1)) * (1.0 / (q1 * sf));
        q = q1;
        u = vv + 2.0 * s1;
        v[0] = nx;
        v[1] = v[1] + nx;
      };
      st[0] = start;
      st[1] = start;
      emit_and_run(step);
    } else {
      // The three-term recurrence, MTL Eq. B.22 (wigner.rs:315-346).
      double q = 0.0;
      auto step = [&](int64_t si, double* v) {
        double sf = (double)si;
        double c_prev = q * (sf + 1.0);
        double numer = (x * (sf * (sf + 1.0)) - mf * nf) * (2.0 * sf + 1.0) * v[1] - c_prev * v[0];
        double s1 = sf + 1.0;
        q = std::sqrt((s1 - mf) * (s1 + mf)) * std::sqrt((s1 - nf) * (s1 + nf));
        v[0] = v[1];
        v[1] = numer / (q * sf);
      };
      st[0] = 0.0;
      st[1] = start;
      emit_and_run(step);
    }
  }
  if (flip) {
    int64_t first = ((l0 + m) % 2 + 2) % 2 == 0 ? l0 + 1 : l0;
    for (int64_t l = first; l < len; l += 2) out[l] = -out[l];
  }
}

void pi_tau_row(double mu, int64_t n_max, double* ge, double* go) {
  double pi_prev = 0.0, pi = 1.0;
  for (int64_t n = 1; n <= n_max; ++n) {
    double nf = (double)n, n1 = nf + 1.0;
    double tau = nf * mu * pi - n1 * pi_prev;
    double w = (double)(2 * n + 1) / (nf * n1);
    double wp = w * pi, wt = w * tau;
    if (n & 1) {
      ge[n - 1] = wp;
      go[n - 1] = wt;
    } else {
      ge[n - 1] = wt;
      go[n - 1] = wp;
    }
    double next = ((double)(2 * n + 1) * mu * pi - n1 * pi_prev) / nf;
    pi_prev = pi;
    pi = next;
  }
}

int64_t bucket(int64_t n) {
  int64_t u = 1;
  while (u < n) u = (int64_t)std::ceil((double)u * 1.25);
  return u;
}

int band_index(int64_t n) {
  int64_t u = 1;
  int i = 0;
  while (u < n) {
    u = (int64_t)std::ceil((double)u * 1.25);
    ++i;
  }
  return i;
}

int64_t band_upper(int index) {
  int64_t u = 1;
  for (int i = 0; i < index; ++i) u = (int64_t)std::ceil((double)u * 1.25);
  return u;
}

static bool positive(double v) { return std::isfinite(v) && v > 0.0; }

bool validate_distribution(int kind, const double* p, std::string* msg) {
  switch (kind) {
    case 1:
      if (!positive(p[0])) return *msg = "median_radius must be finite and > 0", false;
      if (!(std::isfinite(p[1]) && p[1] > 1.0))
        return *msg = "the lognormal width must be finite and > 1", false;
      return true;
    case 2:
      if (!positive(p[0])) return *msg = "effective_radius must be finite and > 0", false;
      if (!(p[1] > 0.0 && p[1] < 0.5)) return *msg = "effective_variance must be in (0, 0.5)", false;
      return true;
    case 3:
      if (!(std::isfinite(p[0]) && p[0] > -1.0)) return *msg = "alpha must be finite and > -1", false;
      if (!positive(p[1])) return *msg = "b must be finite and > 0", false;
      if (!positive(p[2])) return *msg = "gamma must be finite and > 0", false;
      return true;
    case 4:
      if (!std::isfinite(p[0])) return *msg = "exponent must be finite", false;
      if (!positive(p[1]) || !positive(p[2]))
        return *msg = "min_radius and max_radius must be finite and > 0", false;
      if (p[1] >= p[2]) return *msg = "min_radius must be < max_radius", false;
      return true;
  }
  *msg = "unknown distribution kind";
  return false;
}

// Density::eval (distribution.rs:370-441) without the gradient, with prepare's reference
// radius (296-336).
double density(int kind, const double* p, double r) {
  double ln_u = 0.0;
  switch (kind) {
    case 1: {
      double r0 = p[0];
      double mu = std::log(p[0]), s = std::log(p[1]);
      double z = std::log(r) - mu;
      ln_u = -z * z / (2.0 * s * s) - std::log(s) - std::log(r / r0);
      break;
    }
    case 2: {
      double a = p[0], b = p[1];
      double alpha = (1.0 - 3.0 * b) / b;
      double r0 = alpha > 0.0 ? alpha * a * b : a;
      double l = std::log(r / r0);
      ln_u = alpha * l - (r - r0) / (a * b);
      break;
    }
    case 3: {
      double alpha = p[0], b = p[1], g = p[2];
      double r0 = std::pow(std::max(alpha, 1.0) / (b * g), 1.0 / g);
      ln_u = alpha * std::log(r / r0) - b * (std::pow(r, g) - std::pow(r0, g));
      break;
    }
    case 4: {
      if (r < p[1] || r > p[2]) return 0.0;
      double r0 = p[0] >= 0.0 ? p[1] : p[2];
      ln_u = -p[0] * std::log(r / r0);
      break;
    }
  }
  return std::exp(ln_u);
}

int parameter_count(int kind) { return kind == 3 ? 3 : kind == 4 ? 1 : kind == kTabulated ? 0 : 2; }

double table_density(const double* t, int64_t n, double r) {
  const double* xs = t;
  const double* ys = t + n;
  if (r < xs[0] || r > xs[n - 1]) return 0.0;
  // The first point above r (partition_point of v <= r), kept in 1..n-1.
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    const int64_t mid = (lo + hi) / 2;
    if (xs[mid] <= r) lo = mid + 1; else hi = mid;
  }
  const int64_t i = std::min<int64_t>(std::max<int64_t>(lo, 1), n - 1);
  const double w = (r - xs[i - 1]) / (xs[i] - xs[i - 1]);
  return ys[i - 1] + w * (ys[i] - ys[i - 1]);
}

bool validate_table(const double* t, int64_t n, std::string* msg) {
  if (!t || n < 2) {
    *msg = "a tabulated distribution needs at least 2 points and as many densities as radii";
    return false;
  }
  for (int64_t k = 0; k < n; ++k)
    if (!(std::isfinite(t[k]) && t[k] > 0.0)) return *msg = "radius must be finite and > 0", false;
  for (int64_t k = 1; k < n; ++k)
    if (!(t[k - 1] < t[k])) return *msg = "tabulated radii must increase", false;
  bool any = false;
  for (int64_t k = 0; k < n; ++k) {
    const double u = t[n + k];
    if (!(std::isfinite(u) && u >= 0.0))
      return *msg = "tabulated densities must be finite and >= 0", false;
    any = any || u != 0.0;
  }
  if (!any) return *msg = "tabulated densities must not all be 0", false;
  return true;
}

double density_gradient(int kind, const double* p, double r, double grad[3]) {
  const double u = density(kind, p, r);
  double dln[3] = {0.0, 0.0, 0.0};
  switch (kind) {
    case 1: {
      // ln u = -z^2 / (2 s^2) - ln s - ln(r/r0), z = ln r - ln median, s = ln width.
      const double s = std::log(p[1]);
      const double z = std::log(r) - std::log(p[0]);
      dln[0] = z / (s * s * p[0]);
      dln[1] = (z * z / (s * s * s) - 1.0 / s) / p[1];
      break;
    }
    case 2: {
      // ln u = alpha ln(r/r0) - (r - r0)/(a b), alpha = (1 - 3b)/b.
      const double a = p[0], b = p[1];
      const double alpha = (1.0 - 3.0 * b) / b;
      const double r0 = alpha > 0.0 ? alpha * a * b : a;
      const double sc = a * b;
      dln[0] = (r - r0) * b / (sc * sc);
      dln[1] = -std::log(r / r0) / (b * b) + (r - r0) * a / (sc * sc);
      break;
    }
    case 3: {
      // ln u = alpha ln(r/r0) - b (r^gamma - r0^gamma).
      const double alpha = p[0], b = p[1], g = p[2];
      const double r0 = std::pow(std::max(alpha, 1.0) / (b * g), 1.0 / g);
      const double rg = std::pow(r, g), r0g = std::pow(r0, g);
      dln[0] = std::log(r / r0);
      dln[1] = -(rg - r0g);
      dln[2] = -b * (rg * std::log(r) - r0g * std::log(r0));
      break;
    }
    case 4: {
      // ln u = -exponent ln(r/r0) on [min, max], 0 outside.
      const double r0 = p[0] >= 0.0 ? p[1] : p[2];
      if (r >= p[1] && r <= p[2]) dln[0] = -std::log(r / r0);
      break;
    }
  }
  for (int k = 0; k < 3; ++k) grad[k] = u * dln[k];
  return u;
}

DensityInfo density_info(int kind, const double* p) {
  DensityInfo d{1.0, std::numeric_limits<double>::infinity()};
  switch (kind) {
    case 1:
      d.reference = p[0];
      d.log_width = std::log(p[1]);
      break;
    case 2: {
      const double b = p[1], alpha = (1.0 - 3.0 * b) / b;
      d.reference = alpha > 0.0 ? alpha * p[0] * b : p[0];
      d.log_width = std::sqrt(b / (1.0 - 2.0 * b));
      break;
    }
    case 3: {
      const double alpha = p[0], b = p[1], g = p[2];
      d.reference = std::pow(std::max(alpha, 1.0) / (b * g), 1.0 / g);
      d.log_width = alpha > 0.0 ? 1.0 / std::sqrt(alpha * g) : 1.0 / g;
      break;
    }
    case 4:
      d.reference = p[0] >= 0.0 ? p[1] : p[2];
      break;
  }
  return d;
}

}  // namespace sb
