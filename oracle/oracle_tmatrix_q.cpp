// TEST INFRASTRUCTURE ONLY: the spheroid T-matrix by the extended boundary condition method in
// quadruple precision (__float128 with libquadmath's elementary functions): the same
// definition as the double-precision restatement beside it (research/tmatrix/ebcm.py; Q and RgQ
// of one azimuthal mode as surface integrals of cross products of vector spherical wave
// functions at Gauss-Legendre nodes in cos theta), with every function, node, weight, sum and
// the LU solve carried in 113-bit arithmetic. The EBCM's outgoing integrals cancel by up to
// 1e16 and more (research/tmatrix/README.md, findings 1-3); in quadruple precision that leaves
// about 1e-18 of relative error, so this is the high-precision checker of the GPU T-matrix
// (whose double-double assembly targets the same cancellation) where plain double fails.
//
// Inputs are doubles; the semi-axes are a = x cbrt(eps) and c = a / eps rounded to double, as
// the reference's Spheroid computes them (scatrs/src/tmatrix/kernel.rs:40-98), then exact.
#include <quadmath.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "oracle_core.hpp"

namespace {

typedef __float128 Q;

struct CQ {
  Q re, im;
};
inline CQ cq(Q r, Q i = 0) { return CQ{r, i}; }
inline CQ operator+(CQ a, CQ b) { return cq(a.re + b.re, a.im + b.im); }
inline CQ operator-(CQ a, CQ b) { return cq(a.re - b.re, a.im - b.im); }
inline CQ operator*(CQ a, CQ b) { return cq(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
inline CQ operator*(CQ a, Q s) { return cq(a.re * s, a.im * s); }
inline CQ ti(CQ a) { return cq(-a.im, a.re); }  // i a
inline Q norm2(CQ a) { return a.re * a.re + a.im * a.im; }
inline CQ cinvq(CQ a) {
  const Q d = norm2(a);
  return cq(a.re / d, -a.im / d);
}
inline Q absq(CQ a) { return sqrtq(norm2(a)); }

const Q PIQ = 4 * atanq((Q)1);

// The 2 n-point Gauss-Legendre rule on [-1, 1] in quadruple precision: double starting points
// refined by Newton's method on P_n (three-term recurrence), weights 2 / ((1 - x^2) P_n'^2).
void gauss_legendre_q(int n, std::vector<Q>& x, std::vector<Q>& w) {
  std::vector<double> xd(n), wd(n);
  orc::gauss_legendre(n, xd.data(), wd.data());
  x.resize(n);
  w.resize(n);
  for (int i = 0; i < n; ++i) {
    Q t = xd[i], dp = 0;
    for (int it = 0; it < 3; ++it) {
      Q p0 = 1, p1 = t;
      for (int k = 2; k <= n; ++k) {
        const Q p2 = ((2 * k - 1) * t * p1 - (k - 1) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      dp = n * (t * p1 - p0) / (t * t - 1);
      t -= p1 / dp;
    }
    Q p0 = 1, p1 = t;
    for (int k = 2; k <= n; ++k) {
      const Q p2 = ((2 * k - 1) * t * p1 - (k - 1) * p0) / k;
      p0 = p1;
      p1 = p2;
    }
    dp = n * (t * p1 - p0) / (t * t - 1);
    x[i] = t;
    w[i] = 2 / ((1 - t * t) * dp * dp);
  }
}

void angular_q(int m, int N, Q ct, Q st, std::vector<Q>& d, std::vector<Q>& pi,
               std::vector<Q>& tau) {
  d.assign(N + 1, 0);
  pi.assign(N + 1, 0);
  tau.assign(N + 1, 0);
  if (m <= N) {
    Q am = 1;
    for (int k = 1; k <= m; ++k) am *= sqrtq((Q)(2 * k - 1) / (2 * k));
    Q sp = 1;
    for (int k = 0; k < m; ++k) sp *= st;
    d[m] = am * sp;
    if (m + 1 <= N) d[m + 1] = sqrtq((Q)(2 * m + 1)) * ct * d[m];
    for (int n = m + 1; n < N; ++n)
      d[n + 1] = ((2 * n + 1) * ct * d[n] - sqrtq((Q)n * n - (Q)m * m) * d[n - 1]) /
                 sqrtq((Q)(n + 1) * (n + 1) - (Q)m * m);
  }
  for (int n = std::max(m, 1); n <= N; ++n) {
    const Q prev = n - 1 >= m ? d[n - 1] : 0;
    tau[n] = (n * ct * d[n] - sqrtq((Q)n * n - (Q)m * m) * prev) / st;
    pi[n] = m * d[n] / st;
  }
}

// j_n(z), n = -1..N (index n + 1), by downward ratios from far above N.
void sph_j_q(CQ z, int N, std::vector<CQ>& j) {
  j.assign(N + 2, cq(0));
  const int start = N + 60 + (int)(2.0 * (double)absq(z));
  std::vector<CQ> rho(start + 2, cq(0));
  for (int n = start; n >= 1; --n) rho[n] = z * cinvq(cq((Q)(2 * n + 1)) - z * rho[n + 1]);
  const CQ iz = cinvq(z);
  const CQ s = cq(sinq(z.re) * coshq(z.im), cosq(z.re) * sinhq(z.im));
  const CQ c = cq(cosq(z.re) * coshq(z.im), -(sinq(z.re) * sinhq(z.im)));
  j[0] = c * iz;
  j[1] = s * iz;
  for (int n = 1; n <= N; ++n) j[n + 1] = rho[n] * j[n];
}

void sph_y_q(Q x, int N, std::vector<Q>& y) {
  y.assign(N + 2, 0);
  y[0] = sinq(x) / x;
  y[1] = -cosq(x) / x;
  for (int n = 0; n < N; ++n) y[n + 2] = (2 * n + 1) / x * y[n + 1] - y[n];
}

struct V3 {
  CQ c[3];
};

void vswf_q(int m, int N, CQ z, const std::vector<CQ>& zn, const std::vector<Q>& d,
            const std::vector<Q>& pi, const std::vector<Q>& tau, bool flip, std::vector<V3>& M,
            std::vector<V3>& Nv) {
  M.assign(N + 1, V3{{cq(0), cq(0), cq(0)}});
  Nv.assign(N + 1, V3{{cq(0), cq(0), cq(0)}});
  const CQ iz = cinvq(z);
  for (int n = std::max(m, 1); n <= N; ++n) {
    const Q g = sqrtq((Q)(2 * n + 1) / (4 * PIQ * n * (n + 1)));
    const Q p = flip ? -pi[n] : pi[n];
    const CQ zz = zn[n + 1];
    const CQ der = zn[n] - (zz * iz) * (Q)n;
    M[n] = V3{{cq(0), ti(zz * (g * p)), zz * (-g * tau[n])}};
    Nv[n] = V3{{(zz * iz) * (g * n * (n + 1) * d[n]), der * (g * tau[n]), ti(der * (g * p))}};
  }
}

bool mode_tmatrix_q(double x, double eps, double s_re, double s_im, int m, int N, int n_theta,
                    std::vector<CQ>& T) {
  const double ad = x * std::cbrt(eps), cd = ad / eps;
  const Q a = ad, c = cd;
  const CQ s = cq(s_re, s_im);
  const int n_nodes = 2 * n_theta;
  std::vector<Q> nodes, weights;
  gauss_legendre_q(n_nodes, nodes, weights);
  const int n0 = std::max(m, 1), K = N - n0 + 1;
  if (K <= 0) return false;
  std::vector<CQ> J[2][2][2];
  for (auto& o : J)
    for (auto& p : o)
      for (auto& q : p) q.assign((size_t)K * K, cq(0));
  std::vector<Q> d, pi, tau, yv;
  std::vector<CQ> jin, jr, zn(N + 2);
  std::vector<V3> iM, iN, oM, oN;
  for (int q = 0; q < n_nodes; ++q) {
    const Q ct = nodes[q], st = sqrtq(1 - ct * ct);
    const Q den = c * c * st * st + a * a * ct * ct;
    const Q r = a * c / sqrtq(den);
    const Q dr = -a * c * (c * c - a * a) * st * ct / (den * sqrtq(den));
    angular_q(m, N, ct, st, d, pi, tau);
    const Q nv1 = -dr / r;
    const Q fac = weights[q] * r * r * 2 * PIQ;
    const CQ zi = s * r;
    sph_j_q(zi, N, jin);
    vswf_q(m, N, zi, jin, d, pi, tau, false, iM, iN);
    sph_j_q(cq(r), N, jr);
    sph_y_q(r, N, yv);
    for (int out = 0; out < 2; ++out) {
      for (int n = 0; n <= N + 1; ++n) zn[n] = out ? jr[n] + ti(cq(yv[n])) : jr[n];
      vswf_q(m, N, cq(r), zn, d, pi, tau, true, oM, oN);
      for (int aa = 0; aa < 2; ++aa) {
        const auto& A = aa == 0 ? oM : oN;
        for (int bb = 0; bb < 2; ++bb) {
          const auto& B = bb == 0 ? iM : iN;
          std::vector<CQ>& mat = J[out][aa][bb];
          for (int i = n0; i <= N; ++i)
            for (int k = n0; k <= N; ++k) {
              const CQ* X = A[i].c;
              const CQ* Y = B[k].c;
              const CQ trip = (X[1] * Y[2] - X[2] * Y[1]) + (X[2] * Y[0] - X[0] * Y[2]) * nv1;
              CQ& e = mat[(size_t)(i - n0) * K + (k - n0)];
              e = e + trip * fac;
            }
        }
      }
    }
  }
  const int n2 = 2 * K;
  auto assemble = [&](int out, std::vector<CQ>& M) {
    M.assign((size_t)n2 * n2, cq(0));
    const CQ mis = ti(s) * (Q)-1, mi = cq(0, -1);
    for (int i = 0; i < K; ++i)
      for (int k = 0; k < K; ++k) {
        const size_t e = (size_t)i * K + k;
        M[(size_t)i * n2 + k] = mis * J[out][0][1][e] + mi * J[out][1][0][e];
        M[(size_t)i * n2 + K + k] = mis * J[out][0][0][e] + mi * J[out][1][1][e];
        M[(size_t)(K + i) * n2 + k] = mis * J[out][1][1][e] + mi * J[out][0][0][e];
        M[(size_t)(K + i) * n2 + K + k] = mis * J[out][1][0][e] + mi * J[out][0][1][e];
      }
  };
  std::vector<CQ> Qm, P;
  assemble(1, Qm);
  assemble(0, P);
  // Q^T X = -P^T with X = T^T: LU with partial pivoting of Q^T.
  std::vector<CQ> A((size_t)n2 * n2);
  for (int i = 0; i < n2; ++i)
    for (int k = 0; k < n2; ++k) A[(size_t)k * n2 + i] = Qm[(size_t)i * n2 + k];
  std::vector<int> piv(n2);
  for (int k = 0; k < n2; ++k) {
    int p = k;
    Q best = absq(A[(size_t)k * n2 + k]);
    for (int i = k + 1; i < n2; ++i)
      if (absq(A[(size_t)i * n2 + k]) > best) {
        best = absq(A[(size_t)i * n2 + k]);
        p = i;
      }
    if (best == 0) return false;
    piv[k] = p;
    if (p != k)
      for (int j = 0; j < n2; ++j) std::swap(A[(size_t)k * n2 + j], A[(size_t)p * n2 + j]);
    const CQ ipv = cinvq(A[(size_t)k * n2 + k]);
    for (int i = k + 1; i < n2; ++i) {
      const CQ f = A[(size_t)i * n2 + k] * ipv;
      A[(size_t)i * n2 + k] = f;
      for (int j = k + 1; j < n2; ++j)
        A[(size_t)i * n2 + j] = A[(size_t)i * n2 + j] - f * A[(size_t)k * n2 + j];
    }
  }
  T.assign((size_t)n2 * n2, cq(0));
  std::vector<CQ> b(n2);
  for (int i = 0; i < n2; ++i) {
    for (int k = 0; k < n2; ++k) b[k] = cq(0) - P[(size_t)i * n2 + k];
    for (int k = 0; k < n2; ++k)
      if (piv[k] != k) std::swap(b[k], b[piv[k]]);
    for (int r = 0; r < n2; ++r)
      for (int j = 0; j < r; ++j) b[r] = b[r] - A[(size_t)r * n2 + j] * b[j];
    for (int r = n2 - 1; r >= 0; --r) {
      for (int j = r + 1; j < n2; ++j) b[r] = b[r] - A[(size_t)r * n2 + j] * b[j];
      b[r] = b[r] * cinvq(A[(size_t)r * n2 + r]);
    }
    for (int k = 0; k < n2; ++k) T[(size_t)i * n2 + k] = b[k];
  }
  return true;
}

void sums_q(const std::vector<CQ>& T, Q* ext, Q* sca) {
  const int n2 = (int)std::lround(std::sqrt((double)T.size()));
  *ext = 0;
  *sca = 0;
  for (int i = 0; i < n2; ++i) {
    *ext -= T[(size_t)i * n2 + i].re;
    for (int k = 0; k < n2; ++k) *sca += norm2(T[(size_t)i * n2 + k]);
  }
}

}  // namespace

extern "C" {

// One mode's T-matrix in quadruple precision, rounded to double into t (2 (2K)^2 doubles,
// row-major complex, K = N - max(m, 1) + 1). Returns 0, or 1 for an invalid input or a
// singular Q.
int orc_tmatrix_mode_q(double x, double eps, double s_re, double s_im, int m, int N, int n_theta,
                       double* t) {
  if (!(x > 0 && eps > 0 && N >= 1 && n_theta >= 2 && m >= 0 && m <= N)) return 1;
  std::vector<CQ> T;
  if (!mode_tmatrix_q(x, eps, s_re, s_im, m, N, n_theta, T)) return 1;
  for (size_t i = 0; i < T.size(); ++i) {
    t[2 * i] = (double)T[i].re;
    t[2 * i + 1] = (double)T[i].im;
  }
  return 0;
}

// Orientation-averaged Q_ext, Q_sca at fixed N and n_theta in quadruple precision (every mode
// 0..N; kernel.rs:985-1010): q[2].
int orc_spheroid_q_q(double x, double eps, double s_re, double s_im, int N, int n_theta,
                     double* q) {
  Q ext = 0, sca = 0;
  std::vector<CQ> T;
  for (int m = 0; m <= N; ++m) {
    if (!mode_tmatrix_q(x, eps, s_re, s_im, m, N, n_theta, T)) return 1;
    Q e, s;
    sums_q(T, &e, &s);
    const Q w = m == 0 ? 1 : 2;
    ext += w * e;
    sca += w * s;
  }
  const Q area = PIQ * (Q)x * (Q)x;
  q[0] = (double)(2 * PIQ * ext / area);
  q[1] = (double)(2 * PIQ * sca / area);
  return 0;
}

}  // extern "C"
