// TEST INFRASTRUCTURE ONLY: the orientation-averaged phase matrix of an axisymmetric particle
// from its T-matrix by the rank decomposition (scatrs/src/tmatrix/random.rs:85-280, after
// research/tmatrix/ranks.py), its Mueller form (random.rs:295-335) and its Greek coefficients
// (greek_raw, random.rs:283-292), restated on the CPU in double precision. The checker of the
// GPU's random-orientation kernels.
//
// In the helicity basis W^p = (M + p N)/sqrt 2 the T-matrix blocks are
// T^{p sigma}_m = (T11 + sigma T12 + p T21 + p sigma T22)/2, with T^{p sigma}_{-m} = T^{-p,-sigma}_m.
// Rank components t^(s)(n, n') = sum_mu (-1)^(n'-mu) C^{s 0}_{n mu; n' -mu} T^{p sigma}_mu(n, n');
// for incident helicity sigma and scattered helicity p at Theta,
// Phi_{sq} = sum_n far_n(q + sigma, p; Theta) w_n, w_n = sum_n' inc_n' (-1)^(n'-sigma)
// C^{s q}_{n, q+sigma; n', -sigma} t^(s)(n, n'), and <A_{p sigma} A*_{p' sigma'}> =
// sum_{s,q} Phi Phi'* / (2s + 1); inc_n = 2 i^(n-1) sqrt(pi (2n+1)), far_n(m, p) =
// gamma_n (-i)^n (pi_mn + p tau_mn). The Clebsch-Gordan coefficients here come from Racah's
// closed formula evaluated in quadruple precision (exact enough for the small truncations the
// tests use), independently of the recursion the GPU evaluates.
#include <quadmath.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <unordered_map>
#include <vector>

#include "oracle_core.hpp"

using namespace orc;

namespace {

typedef __float128 Q;

// n! for n <= 600 (the table built once).
Q fact(int n) {
  static std::vector<Q> t = [] {
    std::vector<Q> v(601);
    v[0] = 1;
    for (int k = 1; k <= 600; ++k) v[k] = v[k - 1] * k;
    return v;
  }();
  return t[n];
}

double cg_racah(int j1, int m1, int j2, int m2, int J);

// C^{J M}_{j1 m1; j2 m2}, memoized per thread (the values depend on the indices alone).
double cg(int j1, int m1, int j2, int m2, int J) {
  thread_local std::unordered_map<uint64_t, double> memo;
  // Five 12-bit fields (every index below 2048 in magnitude here).
  const uint64_t key = ((uint64_t)j1 << 48) | ((uint64_t)(m1 + 2048) << 36) |
                       ((uint64_t)j2 << 24) | ((uint64_t)(m2 + 2048) << 12) | (uint64_t)J;
  auto it = memo.find(key);
  if (it != memo.end()) return it->second;
  const double v = cg_racah(j1, m1, j2, m2, J);
  memo.emplace(key, v);
  return v;
}

// C^{J M}_{j1 m1; j2 m2} by Racah's formula (Condon-Shortley phases).
double cg_racah(int j1, int m1, int j2, int m2, int J) {
  const int M = m1 + m2;
  if (J < std::abs(j1 - j2) || J > j1 + j2 || std::abs(m1) > j1 || std::abs(m2) > j2 ||
      std::abs(M) > J)
    return 0.0;
  const Q pre = sqrtq((Q)(2 * J + 1) * fact(J + j1 - j2) * fact(J - j1 + j2) * fact(j1 + j2 - J) /
                      fact(j1 + j2 + J + 1)) *
                sqrtq(fact(J + M) * fact(J - M) * fact(j1 - m1) * fact(j1 + m1) * fact(j2 - m2) *
                      fact(j2 + m2));
  Q sum = 0;
  for (int k = 0; k <= j1 + j2 + J; ++k) {
    const int a[6] = {k, j1 + j2 - J - k, j1 - m1 - k, j2 + m2 - k, J - j2 + m1 + k, J - j1 - m2 + k};
    bool ok = true;
    for (int v : a) ok = ok && v >= 0;
    if (!ok) continue;
    Q den = 1;
    for (int v : a) den *= fact(v);
    sum += (k % 2 ? -1 : 1) / den;
  }
  return (double)(pre * sum);
}

double sgn(int k) { return (k % 2 + 2) % 2 ? -1.0 : 1.0; }
cplx ipow(int k) {  // i^k
  switch ((k % 4 + 4) % 4) {
    case 0: return C(1, 0);
    case 1: return C(0, 1);
    case 2: return C(-1, 0);
    default: return C(0, -1);
  }
}

// The four blocks T^{ij}_m(n, n') of mode m, dense over orders 0..N (zero where absent), from
// the mode's 2K x 2K matrix (blocks [T11 T12; T21 T22] over orders max(m, 1)..N).
void dense(const cplx* t, int m, int N, std::vector<cplx> out[4]) {
  const int n0 = std::max(m, 1), K = N - n0 + 1, n1 = N + 1;
  for (int b = 0; b < 4; ++b) out[b].assign((size_t)n1 * n1, C(0, 0));
  for (int bi = 0; bi < 2; ++bi)
    for (int bj = 0; bj < 2; ++bj)
      for (int i = 0; i < K; ++i)
        for (int j = 0; j < K; ++j)
          out[bi * 2 + bj][(size_t)(n0 + i) * n1 + (n0 + j)] =
              t[(size_t)(bi * K + i) * (2 * K) + (bj * K + j)];
}

// The normalized d, pi, tau of mode m >= 0 (functions.rs:192-239).
void angular(int m, int N, double ct, double st, std::vector<double>& d, std::vector<double>& pi,
             std::vector<double>& tau) {
  d.assign(N + 1, 0.0);
  pi.assign(N + 1, 0.0);
  tau.assign(N + 1, 0.0);
  if (m > N) return;
  double am = 1.0;
  for (int k = 1; k <= m; ++k) am *= std::sqrt((double)(2 * k - 1) / (2 * k));
  d[m] = am * std::pow(st, m);
  if (m < N) d[m + 1] = std::sqrt(2.0 * m + 1) * ct * d[m];
  for (int k = m + 1; k < N; ++k)
    d[k + 1] = ((2 * k + 1) * ct * d[k] - std::sqrt((double)k * k - (double)m * m) * d[k - 1]) /
               std::sqrt((double)(k + 1) * (k + 1) - (double)m * m);
  for (int k = std::max(m, 1); k <= N; ++k) {
    const double prev = k > m ? d[k - 1] : 0.0;
    tau[k] = (k * ct * d[k] - std::sqrt((double)k * k - (double)m * m) * prev) / st;
    pi[k] = m * d[k] / st;
  }
}

// F11, F12, F22, F33, F34, F44 (f[6][nq]) of the average at the cosines mu.
void random_orientation(const cplx* t_all, int N, const double* mu, int nq, double* f) {
  const int n1 = N + 1;
  // hel[key = pi * 2 + si][mu + N][n * n1 + n'].
  std::vector<std::vector<std::vector<cplx>>> hel(
      4, std::vector<std::vector<cplx>>(2 * N + 1, std::vector<cplx>((size_t)n1 * n1, C(0, 0))));
  size_t off = 0;
  for (int m = 0; m <= N; ++m) {
    const int K = N - std::max(m, 1) + 1;
    std::vector<cplx> b[4];
    dense(t_all + off, m, N, b);
    off += (size_t)4 * K * K;
    for (int pi = 0; pi < 2; ++pi)
      for (int si = 0; si < 2; ++si) {
        const double p = pi ? -1.0 : 1.0, s = si ? -1.0 : 1.0;
        for (size_t k = 0; k < (size_t)n1 * n1; ++k) {
          hel[pi * 2 + si][N + m][k] =
              scale(b[0][k] + scale(b[1][k], s) + scale(b[2][k], p) + scale(b[3][k], p * s), 0.5);
          if (m > 0)
            hel[pi * 2 + si][N - m][k] = scale(
                b[0][k] + scale(b[1][k], -s) + scale(b[2][k], -p) + scale(b[3][k], p * s), 0.5);
        }
      }
  }
  // t_rank[key][n * n1 + n'][s - |n - n'|].
  std::vector<std::vector<std::vector<cplx>>> tr(4, std::vector<std::vector<cplx>>((size_t)n1 * n1));
  for (int n = 1; n <= N; ++n)
    for (int np = 1; np <= N; ++np) {
      const int smin = std::abs(n - np), len = n + np - smin + 1;
      for (int k = 0; k < 4; ++k) tr[k][(size_t)n * n1 + np].assign(len, C(0, 0));
      for (int u = -std::min(n, np); u <= std::min(n, np); ++u)
        for (int s = smin; s <= n + np; ++s) {
          const double c = sgn(np - u) * cg(n, u, np, -u, s);
          if (c == 0.0) continue;
          for (int k = 0; k < 4; ++k)
            tr[k][(size_t)n * n1 + np][s - smin] =
                tr[k][(size_t)n * n1 + np][s - smin] + scale(hel[k][N + u][(size_t)n * n1 + np], c);
        }
    }
  std::vector<cplx> inc(n1, C(0, 0));
  std::vector<double> gam(n1, 0.0);
  for (int k = 1; k <= N; ++k) {
    inc[k] = scale(ipow(k - 1), 2.0 * std::sqrt(PI * (2 * k + 1)));
    gam[k] = std::sqrt((2.0 * k + 1) / (PI * 4.0 * k * (k + 1)));
  }
  const int smax = 2 * N;
  std::vector<cplx> prod((size_t)16 * nq, C(0, 0));
  std::vector<double> d, pi_, tau;
  for (int q = -N - 1; q <= N + 1; ++q) {
    std::vector<std::vector<cplx>> phi(4, std::vector<cplx>((size_t)(smax + 1) * nq, C(0, 0)));
    bool active[4] = {false, false, false, false};
    for (int si = 0; si < 2; ++si) {
      const int sigma = si ? -1 : 1, m = q + sigma, am = std::abs(m);
      if (am > N) continue;
      std::vector<cplx> far((size_t)2 * n1 * nq, C(0, 0));
      for (int j = 0; j < nq; ++j) {
        const double ct = mu[j], st = std::sqrt(1.0 - ct * ct);
        angular(am, N, ct, st, d, pi_, tau);
        const double flip = m < 0 ? sgn(am) : 1.0;
        for (int k = std::max(am, 1); k <= N; ++k) {
          const double tk = tau[k] * flip, pk = m < 0 ? -(pi_[k] * flip) : pi_[k];
          const cplx f = scale(ipow(-k), gam[k]);
          far[(size_t)k * nq + j] = scale(f, pk + tk);
          far[(size_t)(n1 + k) * nq + j] = scale(f, pk - tk);
        }
      }
      for (int pi = 0; pi < 2; ++pi) {
        const int key = pi * 2 + si;
        std::vector<cplx> w((size_t)(smax + 1) * n1, C(0, 0));
        for (int n = std::max(am, 1); n <= N; ++n)
          for (int np = 1; np <= N; ++np) {
            const std::vector<cplx>& t = tr[key][(size_t)n * n1 + np];
            const int smin = std::abs(n - np);
            const cplx pre = scale(inc[np], sgn(np - sigma));
            for (int s = std::max(smin, std::abs(q)); s <= n + np; ++s) {
              const double c = cg(n, m, np, -sigma, s);
              if (c == 0.0) continue;
              w[(size_t)s * n1 + n] = w[(size_t)s * n1 + n] + pre * scale(t[s - smin], c);
            }
          }
        for (int s = 0; s <= smax; ++s)
          for (int n = std::max(am, 1); n <= N; ++n) {
            const cplx wv = w[(size_t)s * n1 + n];
            if (wv.re == 0.0 && wv.im == 0.0) continue;
            for (int j = 0; j < nq; ++j)
              phi[key][(size_t)s * nq + j] =
                  phi[key][(size_t)s * nq + j] + wv * far[(size_t)(pi * n1 + n) * nq + j];
          }
        active[key] = true;
      }
    }
    for (int a = 0; a < 4; ++a)
      for (int b = 0; b < 4; ++b) {
        if (!active[a] || !active[b]) continue;
        const int slot = a * 4 + b;
        for (int s = 0; s <= smax; ++s)
          for (int j = 0; j < nq; ++j) {
            const cplx x = phi[a][(size_t)s * nq + j], y = phi[b][(size_t)s * nq + j];
            prod[(size_t)slot * nq + j] =
                prod[(size_t)slot * nq + j] + scale(x * C(y.re, -y.im), 1.0 / (2 * s + 1));
          }
      }
  }
  // Mueller form: S = U A U^{-1}, U = [[1, 1], [i, -i]]/sqrt 2, S = [[S2, S3], [S4, S1]].
  const double r = std::sqrt(0.5);
  const cplx U[2][2] = {{C(r, 0), C(r, 0)}, {C(0, r), C(0, -r)}};
  const cplx Ui[2][2] = {{C(r, 0), C(0, -r)}, {C(r, 0), C(0, r)}};
  for (int j = 0; j < nq; ++j) {
    auto ss = [&](int i, int jj, int k, int l) {
      cplx acc = C(0, 0);
      for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b)
          for (int c = 0; c < 2; ++c)
            for (int e = 0; e < 2; ++e) {
              const cplx g = U[k][c] * Ui[e][l];
              const cplx fct = U[i][a] * Ui[b][jj] * C(g.re, -g.im);
              acc = acc + fct * prod[(size_t)(((a * 2 + b) * 2 + c) * 2 + e) * nq + j];
            }
      return acc;
    };
    const double s22 = ss(0, 0, 0, 0).re, s11 = ss(1, 1, 1, 1).re, s33 = ss(0, 1, 0, 1).re,
                 s44 = ss(1, 0, 1, 0).re;
    const cplx s12 = ss(1, 1, 0, 0), s34 = ss(0, 1, 1, 0);
    f[0 * nq + j] = 0.5 * (s11 + s22 + s33 + s44);
    f[1 * nq + j] = 0.5 * (s22 - s11 + s44 - s33);
    f[2 * nq + j] = 0.5 * (s22 + s11 - s44 - s33);
    f[3 * nq + j] = s12.re + s34.re;
    f[4 * nq + j] = -s12.im - s34.im;
    f[5 * nq + j] = s12.re - s34.re;
  }
}

}  // namespace

extern "C" {

// The averaged phase matrix (f[6 nq]: F11, F12, F22, F33, F34, F44 in 1/k^2 per steradian) at
// the cosines mu of a particle with the T-matrix modes t_all (modes 0..N concatenated, each the
// row-major 2K x 2K complex matrix of scatrs_spheroid_tmatrix). Returns 0.
int orc_random_orientation(int N, const double* t_all, const double* mu, int nq, double* f) {
  random_orientation(reinterpret_cast<const cplx*>(t_all), N, mu, nq, f);
  return 0;
}

// The unnormalized Greek coefficients of the average (greek_raw, random.rs:283-292): order
// L = min(order, 2N) on N + ceil((L + 1)/2) Gauss-Legendre nodes, projected as six elements
// (greek.rs:227-266). out[6 (L + 1)]: alpha1..alpha4, beta1, beta2. Returns L.
int orc_random_greek(int N, const double* t_all, int order, double* out) {
  const int L = std::min(order, 2 * N), len = L + 1;
  const int nq = N + (L + 2) / 2;
  std::vector<double> x(nq), w(nq), f((size_t)6 * nq);
  gauss_legendre(nq, x.data(), w.data());
  random_orientation(reinterpret_cast<const cplx*>(t_all), N, x.data(), nq, f.data());
  std::vector<double> a1(len, 0.0), a4(len, 0.0), pl(len, 0.0), mn(len, 0.0), b1(len, 0.0),
      b2(len, 0.0), d00(len), d22(len), d2m2(len), d02(len);
  for (int k = 0; k < nq; ++k) {
    wigner_d(0, 0, x[k], d00.data(), len);
    wigner_d(2, 2, x[k], d22.data(), len);
    wigner_d(2, -2, x[k], d2m2.data(), len);
    wigner_d(0, 2, x[k], d02.data(), len);
    const double f11 = w[k] * f[k], f12 = w[k] * f[nq + k], f22 = w[k] * f[2 * nq + k],
                 f33 = w[k] * f[3 * nq + k], f34 = w[k] * f[4 * nq + k], f44 = w[k] * f[5 * nq + k];
    for (int l = 0; l < len; ++l) {
      a1[l] += f11 * d00[l];
      a4[l] += f44 * d00[l];
      pl[l] += (f22 + f33) * d22[l];
      mn[l] += (f22 - f33) * d2m2[l];
      b1[l] += f12 * d02[l];
      b2[l] += f34 * d02[l];
    }
  }
  for (int l = 0; l < len; ++l) {
    const double s = (2 * l + 1) * 0.5;
    out[0 * len + l] = s * a1[l];
    out[1 * len + l] = s * 0.5 * (pl[l] + mn[l]);
    out[2 * len + l] = s * 0.5 * (pl[l] - mn[l]);
    out[3 * len + l] = s * a4[l];
    out[4 * len + l] = s * b1[l];
    out[5 * len + l] = s * b2[l];
  }
  return L;
}

}  // extern "C"
