// TEST INFRASTRUCTURE ONLY: the T-matrix of a spheroid by the extended boundary condition
// method, restated on the CPU in double precision from its definition, as the reference's own
// research EBCM states it (research/tmatrix/ebcm.py: Q and RgQ of one azimuthal mode as surface
// integrals of cross products of vector spherical wave functions, Mishchenko, Travis & Lacis
// 2002 section 5.8, at Gauss-Legendre nodes in cos theta), and the orientation-averaged cross
// sections of scatrs/src/tmatrix/kernel.rs:985-1010. The checker of the GPU T-matrix.
//
// Conventions (ebcm.py:8-11): e^{-i w t}; relative index s; k = 1, lengths are size parameters
// and x is the equal-volume sphere's; aspect ratio eps = a/c, > 1 oblate.
#include "oracle_core.hpp"
#include "oracle_spheroid.hpp"

#include <array>
#include <cmath>
#include <vector>

using namespace orc;

namespace {

// r(theta) and dr/dtheta (ebcm.py:53-65).
struct Shape {
  double a, c;
  void at(double ct, double st, double* r, double* dr) const {
    const double den = c * c * st * st + a * a * ct * ct;
    *r = a * c / std::sqrt(den);
    *dr = -a * c * (c * c - a * a) * st * ct / (den * std::sqrt(den));
  }
};

// Normalized d_{mn}(theta), pi_{mn} = m d / sin, tau_{mn} = dd/dtheta for n = 0..N, m >= 0
// (ebcm.py:68-100).
void angular(int m, int N, double ct, double st, std::vector<double>& d, std::vector<double>& pi,
             std::vector<double>& tau) {
  d.assign(N + 1, 0.0);
  pi.assign(N + 1, 0.0);
  tau.assign(N + 1, 0.0);
  if (m <= N) {
    double am = 1.0;
    for (int k = 1; k <= m; ++k) am *= std::sqrt((double)(2 * k - 1) / (2 * k));
    d[m] = am * std::pow(st, m);
    if (m + 1 <= N) d[m + 1] = std::sqrt(2.0 * m + 1) * ct * d[m];
    for (int n = m + 1; n < N; ++n)
      d[n + 1] = ((2 * n + 1) * ct * d[n] - std::sqrt((double)n * n - (double)m * m) * d[n - 1]) /
                 std::sqrt((double)(n + 1) * (n + 1) - (double)m * m);
  }
  for (int n = std::max(m, 1); n <= N; ++n) {
    const double prev = n - 1 >= m ? d[n - 1] : 0.0;
    tau[n] = (n * ct * d[n] - std::sqrt((double)n * n - (double)m * m) * prev) / st;
    pi[n] = m * d[n] / st;
  }
}

// Spherical Bessel j_n(z), n = -1..N (index n + 1), of a complex argument: j_0 = sin z / z and
// j_{-1} = cos z / z, the ratios j_n / j_{n-1} by the downward recurrence
// rho_n = z / (2n + 1 - z rho_{n+1}) from far above N.
void sph_j(cplx z, int N, std::vector<cplx>& j) {
  j.assign(N + 2, real(0.0));
  const int start = N + 40 + (int)(2.0 * cnorm(z));
  std::vector<cplx> rho(start + 2, real(0.0));
  for (int n = start; n >= 1; --n) rho[n] = z * inv(real(2.0 * n + 1) - z * rho[n + 1]);
  const cplx iz = inv(z);
  cplx s, c;
  s = C(std::sin(z.re) * std::cosh(z.im), std::cos(z.re) * std::sinh(z.im));
  c = C(std::cos(z.re) * std::cosh(z.im), -std::sin(z.re) * std::sinh(z.im));
  j[0] = c * iz;
  j[1] = s * iz;
  for (int n = 1; n <= N; ++n) j[n + 1] = rho[n] * j[n];
}

// y_n(x) of a real argument, n = -1..N, by the upward recurrence (y_{-1} = sin x / x).
void sph_y(double x, int N, std::vector<double>& y) {
  y.assign(N + 2, 0.0);
  y[0] = std::sin(x) / x;
  y[1] = -std::cos(x) / x;
  for (int n = 0; n < N; ++n) y[n + 2] = (2 * n + 1) / x * y[n + 1] - y[n];
}

struct Vswf {
  // (r, theta, phi) components of M and N per order, the phi factor dropped.
  std::vector<std::array<cplx, 3>> M, Nv;
};

// ebcm.py:103-142: z_n and [z z_n]'/z = z_{n-1} - n z_n / z, and the components.
void vswf(int m, int N, cplx z, const std::vector<cplx>& zn, const std::vector<double>& d,
          const std::vector<double>& pi, const std::vector<double>& tau, bool flip, Vswf& out) {
  out.M.assign(N + 1, {real(0.0), real(0.0), real(0.0)});
  out.Nv.assign(N + 1, {real(0.0), real(0.0), real(0.0)});
  const cplx iz = inv(z);
  const double sgn = flip ? -1.0 : 1.0;
  for (int n = std::max(m, 1); n <= N; ++n) {
    const double g = std::sqrt((double)(2 * n + 1) / (4.0 * PI * n * (n + 1)));
    const double p = sgn * pi[n];
    const cplx zz = zn[n + 1];
    const cplx der = zn[n] - scale(zz * iz, (double)n);
    out.M[n] = {real(0.0), times_i(scale(zz, g * p)), scale(zz, -g * tau[n])};
    out.Nv[n] = {scale(zz * iz, g * n * (n + 1) * d[n]), scale(der, g * tau[n]),
                 times_i(scale(der, g * p))};
  }
}

// Complex LU with partial pivoting of an n x n row-major matrix; false if singular.
bool lu(std::vector<cplx>& a, int n, std::vector<int>& piv) {
  piv.resize(n);
  for (int k = 0; k < n; ++k) {
    int p = k;
    double best = cnorm(a[k * n + k]);
    for (int i = k + 1; i < n; ++i)
      if (cnorm(a[i * n + k]) > best) {
        best = cnorm(a[i * n + k]);
        p = i;
      }
    if (best == 0.0) return false;
    piv[k] = p;
    if (p != k)
      for (int j = 0; j < n; ++j) std::swap(a[k * n + j], a[p * n + j]);
    const cplx ipv = inv(a[k * n + k]);
    for (int i = k + 1; i < n; ++i) {
      const cplx f = a[i * n + k] * ipv;
      a[i * n + k] = f;
      for (int j = k + 1; j < n; ++j) a[i * n + j] = a[i * n + j] - f * a[k * n + j];
    }
  }
  return true;
}

void lu_solve(const std::vector<cplx>& a, int n, const std::vector<int>& piv, cplx* b) {
  for (int k = 0; k < n; ++k)
    if (piv[k] != k) std::swap(b[k], b[piv[k]]);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < i; ++j) b[i] = b[i] - a[i * n + j] * b[j];
  for (int i = n - 1; i >= 0; --i) {
    for (int j = i + 1; j < n; ++j) b[i] = b[i] - a[i * n + j] * b[j];
    b[i] = b[i] * inv(a[i * n + i]);
  }
}

// Q (outgoing) and RgQ (regular) of mode m >= 0, 2K x 2K row-major with blocks
// [11 12; 21 22] (ebcm.py:145-199), and T = -RgQ Q^{-1} (ebcm.py:202-204).
bool mode_tmatrix(double x, double eps, cplx s, int m, int N, int n_theta, std::vector<cplx>& T) {
  const double a = x * std::cbrt(eps);
  Shape shape{a, a / eps};
  // n_theta nodes in 0 < theta < pi/2 (kernel.rs:100, 260): the 2 n_theta-point rule on
  // [-1, 1], whose nodes are those and their mirror images.
  const int n_nodes = 2 * n_theta;
  std::vector<double> nodes(n_nodes), weights(n_nodes);
  gauss_legendre(n_nodes, nodes.data(), weights.data());
  const int n0 = std::max(m, 1), K = N - n0 + 1;
  if (K <= 0) return false;
  // J[out][a][b]: K x K.
  std::vector<cplx> J[2][2][2];
  for (auto& o : J)
    for (auto& p : o)
      for (auto& q : p) q.assign((size_t)K * K, real(0.0));
  std::vector<double> d, pi, tau, yv;
  std::vector<cplx> jin, jr, h;
  Vswf inner, outv;
  for (int q = 0; q < n_nodes; ++q) {
    const double ct = nodes[q], st = std::sqrt(1.0 - ct * ct);
    double r, dr;
    shape.at(ct, st, &r, &dr);
    angular(m, N, ct, st, d, pi, tau);
    const double nv[2] = {1.0, -dr / r};
    const double fac = weights[q] * r * r * 2.0 * PI;
    const cplx zi = s * real(r);
    sph_j(zi, N, jin);
    vswf(m, N, zi, jin, d, pi, tau, false, inner);
    sph_j(real(r), N, jr);
    sph_y(r, N, yv);
    for (int out = 0; out < 2; ++out) {
      std::vector<cplx> zn(N + 2);
      for (int n = 0; n <= N + 1; ++n) zn[n] = out ? jr[n] + times_i(real(yv[n])) : jr[n];
      vswf(m, N, real(r), zn, d, pi, tau, true, outv);
      for (int aa = 0; aa < 2; ++aa) {
        const auto& A = aa == 0 ? outv.M : outv.Nv;
        for (int bb = 0; bb < 2; ++bb) {
          const auto& B = bb == 0 ? inner.M : inner.Nv;
          std::vector<cplx>& mat = J[out][aa][bb];
          for (int i = n0; i <= N; ++i)
            for (int k = n0; k <= N; ++k) {
              const auto& X = A[i];
              const auto& Y = B[k];
              const cplx trip = scale(X[1] * Y[2] - X[2] * Y[1], nv[0]) +
                                scale(X[2] * Y[0] - X[0] * Y[2], nv[1]);
              mat[(size_t)(i - n0) * K + (k - n0)] =
                  mat[(size_t)(i - n0) * K + (k - n0)] + scale(trip, fac);
            }
        }
      }
    }
  }
  auto assemble = [&](int out, std::vector<cplx>& Q) {
    const int n2 = 2 * K;
    Q.assign((size_t)n2 * n2, real(0.0));
    const cplx mis = times_i(s) * real(-1.0), mi = C(0.0, -1.0);
    for (int i = 0; i < K; ++i)
      for (int k = 0; k < K; ++k) {
        const size_t e = (size_t)i * K + k;
        // Q11 = -i s J12 - i J21, Q12 = -i s J11 - i J22, Q21 = -i s J22 - i J11,
        // Q22 = -i s J21 - i J12.
        Q[(size_t)i * n2 + k] = mis * J[out][0][1][e] + mi * J[out][1][0][e];
        Q[(size_t)i * n2 + K + k] = mis * J[out][0][0][e] + mi * J[out][1][1][e];
        Q[(size_t)(K + i) * n2 + k] = mis * J[out][1][1][e] + mi * J[out][0][0][e];
        Q[(size_t)(K + i) * n2 + K + k] = mis * J[out][1][0][e] + mi * J[out][0][1][e];
      }
  };
  std::vector<cplx> Q, RgQ;
  assemble(1, Q);
  assemble(0, RgQ);
  // T Q = -RgQ: Q^T T^T = -RgQ^T, one row of T per solve.
  const int n2 = 2 * K;
  std::vector<cplx> QT((size_t)n2 * n2);
  for (int i = 0; i < n2; ++i)
    for (int k = 0; k < n2; ++k) QT[(size_t)k * n2 + i] = Q[(size_t)i * n2 + k];
  std::vector<int> piv;
  if (!lu(QT, n2, piv)) return false;
  T.assign((size_t)n2 * n2, real(0.0));
  std::vector<cplx> rhs(n2);
  for (int i = 0; i < n2; ++i) {
    for (int k = 0; k < n2; ++k) rhs[k] = real(0.0) - RgQ[(size_t)i * n2 + k];
    lu_solve(QT, n2, piv, rhs.data());
    for (int k = 0; k < n2; ++k) T[(size_t)i * n2 + k] = rhs[k];
  }
  return true;
}

// The cross sections of one mode (kernel.rs:985-1010 without the 2 pi): -Re tr T and sum |T|^2.
void mode_sums(const std::vector<cplx>& T, double* ext, double* sca) {
  const int n2 = (int)std::lround(std::sqrt((double)T.size()));
  *ext = 0.0;
  *sca = 0.0;
  for (int i = 0; i < n2; ++i) {
    *ext -= T[(size_t)i * n2 + i].re;
    for (int k = 0; k < n2; ++k) *sca += norm_sqr(T[(size_t)i * n2 + k]);
  }
}

double rel_change(double e0, double s0, double e1, double s1) {
  return std::max(std::fabs(e1 - e0) / std::fabs(e1), std::fabs(s1 - s0) / std::fabs(s1));
}

// driver.rs:166-214 (x_max, Wiscombe's start, the cap, n_theta tied to N and to the shape).
double x_max(double x, double eps) {
  const double a = x * std::cbrt(eps);
  return std::max(a, a / eps);
}
int wiscombe(double xm) { return std::max((int)std::ceil(xm + 4.0 * std::cbrt(xm)) + 2, 4); }
int shape_theta(double eps, double rtol) {
  const double h = std::max(eps, 1.0 / eps);
  if (h <= 1.0) return 0;
  return (int)std::ceil(std::log(1e4 / rtol) / (2.0 * std::log((h + 1.0) / (h - 1.0))));
}
int theta_of(int n, double eps, double rtol) { return std::max(2 * n, shape_theta(eps, rtol)); }

// The N and n_theta loops of driver.rs:343-420 on mode 0 (double precision): returns 0, 1
// (invalid or singular) or 2 (not converged within the caps).
int converge(double x, double eps, double s_re, double s_im, double rtol, int* n_out,
             int* nth_out) {
  const cplx s = C(s_re, s_im);
  const int cap = 2 * wiscombe(x_max(x, eps) * std::max(cnorm(s), 1.0)) + 20;
  const int start = std::min(wiscombe(x_max(x, eps)), cap);
  // mod.rs:293-300: n_theta's cap is 4 theta(start) + 40.
  const int th_cap = 4 * theta_of(start, eps, rtol) + 40;
  auto theta = [&](int nn) { return std::min(theta_of(nn, eps, rtol), th_cap); };
  int n = start, nth = theta(n);
  std::vector<cplx> T;
  double e0, s0, e1, s1;
  if (!mode_tmatrix(x, eps, s, 0, n, nth, T)) return INVALID_INPUT;
  mode_sums(T, &e0, &s0);
  bool ok = false;
  while (n < cap) {
    const int next = std::min(n + std::max(n / 8, 2), cap);
    if (!mode_tmatrix(x, eps, s, 0, next, theta(next), T)) return INVALID_INPUT;
    mode_sums(T, &e1, &s1);
    const double c = rel_change(e0, s0, e1, s1);
    n = next;
    nth = theta(next);
    e0 = e1;
    s0 = s1;
    if (c < rtol) {
      ok = true;
      break;
    }
  }
  if (!ok) return NOT_CONVERGED;
  for (;;) {
    if (nth >= th_cap) return NOT_CONVERGED;
    const int next = std::min(nth + std::max(nth / 10, 2), th_cap);
    if (!mode_tmatrix(x, eps, s, 0, n, next, T)) return INVALID_INPUT;
    mode_sums(T, &e1, &s1);
    const double c = rel_change(e0, s0, e1, s1);
    nth = next;
    e0 = e1;
    s0 = s1;
    if (c < rtol) break;
  }
  *n_out = n;
  *nth_out = nth;
  return OK;
}

}  // namespace

extern "C" {

// Orientation-averaged Q_ext, Q_sca, Q_abs with N and n_theta grown until the cross sections of
// mode 0 settle to rtol (driver.rs:343-420: N by max(N/8, 2), then n_theta by a tenth), then
// every mode at the final N and n_theta. out: q[3], n_terms, n_theta. Returns 0, 1 (invalid or
// singular) or 2 (not converged within the cap).
int orc_spheroid_converged(double x, double eps, double s_re, double s_im, double rtol,
                           double* q, int* n_out, int* nth_out) {
  const cplx s = C(s_re, s_im);
  int n = 0, nth = 0;
  const int st = converge(x, eps, s_re, s_im, rtol, &n, &nth);
  if (st != OK) return st;
  std::vector<cplx> T;
  double ext = 0.0, sca = 0.0;
  for (int m = 0; m <= n; ++m) {
    if (!mode_tmatrix(x, eps, s, m, n, nth, T)) return INVALID_INPUT;
    double em, sm;
    mode_sums(T, &em, &sm);
    const double w = m == 0 ? 1.0 : 2.0;
    ext += w * em;
    sca += w * sm;
  }
  const double area = PI * x * x;
  q[0] = 2.0 * PI * ext / area;
  q[1] = 2.0 * PI * sca / area;
  q[2] = q[0] - q[1];
  *n_out = n;
  *nth_out = nth;
  return OK;
}


// One mode's T-matrix (2K x 2K complex, row-major, K = N - max(m, 1) + 1) into t (2 (2K)^2
// doubles). Returns 0, or 1 for an invalid input or a singular Q.
int orc_tmatrix_mode(double x, double eps, double s_re, double s_im, int m, int N, int n_theta,
                     double* t) {
  if (!(x > 0 && eps > 0 && N >= 1 && n_theta >= 2 && m >= 0 && m <= N)) return INVALID_INPUT;
  std::vector<cplx> T;
  if (!mode_tmatrix(x, eps, C(s_re, s_im), m, N, n_theta, T)) return INVALID_INPUT;
  for (size_t i = 0; i < T.size(); ++i) {
    t[2 * i] = T[i].re;
    t[2 * i + 1] = T[i].im;
  }
  return OK;
}

// Orientation-averaged Q_ext and Q_sca (kernel.rs:985-1010 over modes 0..N, divided by the
// equal-volume sphere's area pi x^2).
int orc_spheroid_q(double x, double eps, double s_re, double s_im, int N, int n_theta,
                   double* q) {
  double ext = 0.0, sca = 0.0;
  for (int m = 0; m <= N; ++m) {
    std::vector<cplx> T;
    if (!mode_tmatrix(x, eps, C(s_re, s_im), m, N, n_theta, T)) return INVALID_INPUT;
    const int n2 = (int)std::lround(std::sqrt((double)T.size()));
    const double w = m == 0 ? 1.0 : 2.0;
    for (int i = 0; i < n2; ++i) {
      ext -= w * T[(size_t)i * n2 + i].re;
      for (int k = 0; k < n2; ++k) sca += w * norm_sqr(T[(size_t)i * n2 + k]);
    }
  }
  const double area = PI * x * x;
  q[0] = 2.0 * PI * ext / area;
  q[1] = 2.0 * PI * sca / area;
  return OK;
}

}  // extern "C"

extern "C" int orc_random_greek(int N, const double* t_all, int order, double* out);

namespace orc {

int spheroid_node(double x, double eps, cplx s, double rtol, SpheroidNode* out) {
  int n = 0, nth = 0;
  const int st = converge(x, eps, s.re, s.im, rtol, &n, &nth);
  if (st != OK) return st;
  std::vector<double> t_all;
  double ext = 0.0, sca = 0.0;
  for (int m = 0; m <= n; ++m) {
    std::vector<cplx> T;
    if (!mode_tmatrix(x, eps, s, m, n, nth, T)) return INVALID_INPUT;
    double e, sc;
    mode_sums(T, &e, &sc);
    const double w = m == 0 ? 1.0 : 2.0;
    ext += w * e;
    sca += w * sc;
    for (const cplx& v : T) {
      t_all.push_back(v.re);
      t_all.push_back(v.im);
    }
  }
  const int len = 2 * n + 1;
  std::vector<double> raw(6 * len);
  orc_random_greek(n, t_all.data(), 2 * n, raw.data());
  const double area = PI * x * x, un = 4.0 / (x * x);
  out->n = n;
  out->nth = nth;
  out->q_ext = 2.0 * PI * ext / area;
  out->q_sca = 2.0 * PI * sca / area;
  out->q_abs = out->q_ext - out->q_sca;
  out->g = raw[0] > 0.0 ? raw[1] / (3.0 * raw[0]) : 0.0;
  double f11 = 0.0, dep = 0.0;
  for (int l = 0; l < len; ++l) {
    const double sg = l % 2 ? -1.0 : 1.0;
    f11 += sg * raw[l];
    dep += sg * un * (raw[l] - 0.5 * (raw[len + l] - raw[2 * len + l]));
  }
  out->q_back = 4.0 * PI * f11 / area;
  out->depol = dep;
  out->greek.resize(6 * len);
  for (int k = 0; k < 6 * len; ++k) out->greek[k] = un * raw[k];
  return OK;
}

}  // namespace orc

extern "C" {

// One spheroid node of the ensemble's direct path (oracle_spheroid.hpp): q[5] = Q_ext, Q_sca,
// Q_abs, Q_back, g; n[2] = N, n_theta. Returns the status.
int orc_spheroid_node(double x, double eps, double s_re, double s_im, double rtol, double* q,
                      int* n) {
  orc::SpheroidNode v;
  const int st = orc::spheroid_node(x, eps, C(s_re, s_im), rtol, &v);
  if (st != OK) return st;
  q[0] = v.q_ext;
  q[1] = v.q_sca;
  q[2] = v.q_abs;
  q[3] = v.q_back;
  q[4] = v.g;
  n[0] = v.n;
  n[1] = v.nth;
  return OK;
}

}  // extern "C"
