// The orientation-averaged phase matrix of a spheroid from its T-matrix by the rank
// decomposition of T (scatrs/src/tmatrix/random.rs:85-335, after research/tmatrix/ranks.py),
// and its Greek coefficients (greek_raw, random.rs:283-292), batched over spheroids in five
// kernels:
//
//   ro_rank_kernel   one thread per (spheroid, n, n'), the modes u and -u together: the helicity
//                    blocks
//                    T^{p sigma}_mu(n, n') = (T11 + sigma T12 + p T21 + p sigma T22)/2 of every
//                    mode mu (T^{p sigma}_{-m} = T^{-p,-sigma}_m) and their rank components
//                    t^(s)(n, n') = sum_mu (-1)^(n'-mu) C^{s 0}_{n mu; n' -mu} T^{p sigma}_mu(n, n');
//   ro_w_kernel      one thread per (spheroid, q, sigma, n): w_n = sum_n' inc_n' (-1)^(n'-sigma)
//                    C^{s q}_{n, q+sigma; n', -sigma} t^(s)(n, n') for both scattered helicities,
//                    times the cosine-independent part gamma_n (-i)^n of the far field;
//   ro_phi_kernel    one block per (spheroid, q, tile of 32 cosines), one thread per (cosine,
//                    helicity key): Phi_{sq} = sum_n w_n (pi_mn + p tau_mn) (the far field's
//                    angular part, in shared memory for the tile), and the q-th share of
//                    <A_a A_b*> = sum_s Phi_a Phi_b* / (2s + 1) for the 16 helicity pairs, the
//                    four keys of a cosine exchanged between adjacent lanes;
//   ro_f_kernel      one thread per (spheroid, cosine): the shares summed over q in order, and
//                    the Mueller form F11, F12, F22, F33, F34, F44 (S = U A U^{-1});
//   ro_greek_kernel  one thread per (spheroid, l): the six projections on the
//                    N + ceil((L+1)/2)-point Gauss rule (greek.rs:227-266).
//
// Clebsch-Gordan coefficients come from the three-term recursion of the 3j symbol in its first
// angular momentum (Schulten & Gordon, J. Math. Phys. 16, 1961 (1975)), run down from the
// largest J and up from the smallest, joined where the downward solution peaks, normalized by
// sum (2J + 1) f^2 = 1 and signed by the closed form at the largest J. All sums run in a fixed
// order, so the results are bitwise reproducible.
#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.h"

namespace sb {

namespace {

constexpr int kS = 2 * kRoMaxN + 2;  // the longest Clebsch-Gordan vector
constexpr double kPi = 3.14159265358979323846;

struct C2 {
  double re, im;
};
__device__ __forceinline__ C2 c_add(C2 a, C2 b) { return C2{a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ C2 c_mul(C2 a, C2 b) {
  return C2{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
__device__ __forceinline__ C2 c_scale(C2 a, double s) { return C2{a.re * s, a.im * s}; }
__device__ __forceinline__ C2 c_conj(C2 a) { return C2{a.re, -a.im}; }
__device__ __forceinline__ C2 ipow(int k) {  // i^k
  switch (((k % 4) + 4) % 4) {
    case 0: return C2{1, 0};
    case 1: return C2{0, 1};
    case 2: return C2{-1, 0};
    default: return C2{0, -1};
  }
}
__device__ __forceinline__ double sgn(int k) { return (k & 1) ? -1.0 : 1.0; }

// The recursion's coefficients for f(J) = (J ja jb; -M ma mb).
__device__ __forceinline__ double rec_a(int J, int ja, int jb, int M) {
  const double v = ((double)J * J - (double)(ja - jb) * (ja - jb)) *
                   ((double)(ja + jb + 1) * (ja + jb + 1) - (double)J * J) *
                   ((double)J * J - (double)M * M);
  return v > 0.0 ? sqrt(v) : 0.0;
}
__device__ __forceinline__ double rec_b(int J, int ja, int jb, int ma, int mb) {
  const int M = ma + mb;
  return -(2.0 * J + 1) * ((double)ja * (ja + 1) * (-M) - (double)jb * (jb + 1) * (-M) -
                           (double)J * (J + 1) * (mb - ma));
}

// C^{J, ma+mb}_{ja ma; jb mb} for J = J_min..ja+jb into out (at most kS values); returns J_min,
// or -1 when |ma| > ja or |mb| > jb. scratch holds kS doubles.
__device__ int cg_vector(int ja, int ma, int jb, int mb, double* out, double* scratch) {
  if (abs(ma) > ja || abs(mb) > jb) return -1;
  const int M = ma + mb;
  const int jmin = max(abs(ja - jb), abs(M)), jmax = ja + jb;
  if (jmin > jmax) return -1;
  const int len = jmax - jmin + 1;
  double* back = scratch;
  // Downward from f(J_max) = 1.
  back[len - 1] = 1.0;
  for (int J = jmax; J > jmin; --J) {
    const double aj = rec_a(J, ja, jb, M), aj1 = rec_a(J + 1, ja, jb, M);
    const double next = J < jmax ? back[J + 1 - jmin] : 0.0;
    const double den = (J + 1) * aj;
    back[J - 1 - jmin] =
        den == 0.0 ? 0.0 : -(J * aj1 * next + rec_b(J, ja, jb, ma, mb) * back[J - jmin]) / den;
  }
  int peak = 0;
  double pv = -1.0;
  for (int p = 0; p < len; ++p)
    if (fabs(back[p]) > pv) {
      pv = fabs(back[p]);
      peak = p;
    }
  for (int p = 0; p < len; ++p) out[p] = back[p];
  if (peak > 0 && jmin > 0) {
    // Upward from f(J_min) = 1 to the peak, scaled to meet the downward solution there.
    out[0] = 1.0;
    for (int p = 0; p < peak; ++p) {
      const int J = jmin + p;
      const double aj = rec_a(J, ja, jb, M), aj1 = rec_a(J + 1, ja, jb, M);
      const double prev = p > 0 ? out[p - 1] : 0.0;
      const double den = J * aj1;
      out[p + 1] = den == 0.0 ? 0.0 : -(rec_b(J, ja, jb, ma, mb) * out[p] + (J + 1) * aj * prev) / den;
    }
    // out[peak] now holds the upward value; rescale the upward part to the downward one.
    if (out[peak] != 0.0) {
      const double sc = back[peak] / out[peak];
      for (int p = 0; p < peak; ++p) out[p] *= sc;
    }
    out[peak] = back[peak];
  }
  double norm = 0.0;
  for (int p = 0; p < len; ++p) norm += (2.0 * (jmin + p) + 1) * out[p] * out[p];
  double sc = 1.0 / sqrt(norm);
  const bool negative = ((ja - jb + M) % 2 + 2) % 2 == 1;
  if ((out[len - 1] < 0.0) != negative) sc = -sc;
  const double phase = negative ? -1.0 : 1.0;
  for (int p = 0; p < len; ++p) out[p] = phase * sqrt(2.0 * (jmin + p) + 1) * out[p] * sc;
  return jmin;
}

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

__global__ void __launch_bounds__(128) ro_rank_kernel(RoArgs a) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.n_rank) return;
  const int si = owner(a.n_sph, t, [&](int i) { return a.sph[i].t_rank; });
  const RoSph sp = a.sph[si];
  const int N = sp.N, n1 = N + 1, S = 2 * N + 1;
  const int idx = (int)(t - sp.t_rank), n = 1 + idx / N, np = 1 + idx % N;
  const int smin = abs(n - np), len = n + np - smin + 1;
  C2* acc[4];
  for (int k = 0; k < 4; ++k) {
    acc[k] = reinterpret_cast<C2*>(a.rank + sp.rank0) + ((int64_t)(k * n1 + n) * n1 + np) * S;
    for (int p = 0; p < len; ++p) acc[k][p] = C2{0, 0};
  }
  double cgv[kS], scratch[kS];
  const int umax = min(n, np);
  // Modes u and -u together: T^{p sigma}_{-u} = T^{-p,-sigma}_u and
  // C^{s 0}_{n,-u; n',u} = (-1)^{n+n'-s} C^{s 0}_{n,u; n',-u}, with the same (-1)^{n'-u}.
  for (int u = 0; u <= umax; ++u) {
    const int n0 = max(u, 1);
    if (n < n0 || np < n0) continue;
    const TmJob& jb = a.jobs[sp.job0 + u];
    const int K = jb.K;
    const C2* T = reinterpret_cast<const C2*>(a.T) + jb.T0;
    const int r = n - n0, c = np - n0;
    const C2 t11 = T[(int64_t)r * 2 * K + c], t12 = T[(int64_t)r * 2 * K + K + c];
    const C2 t21 = T[(int64_t)(K + r) * 2 * K + c], t22 = T[(int64_t)(K + r) * 2 * K + K + c];
    const int j0 = cg_vector(n, u, np, -u, cgv, scratch);
    if (j0 < 0) continue;
    const double ph = sgn(np - u);
    C2 h[2][2];
    for (int pi = 0; pi < 2; ++pi)
      for (int sg = 0; sg < 2; ++sg) {
        const double p = pi ? -1.0 : 1.0, s = sg ? -1.0 : 1.0;
        h[pi][sg] = c_scale(c_add(c_add(t11, c_scale(t12, s)), c_add(c_scale(t21, p), c_scale(t22, p * s))), 0.5);
      }
    for (int pi = 0; pi < 2; ++pi)
      for (int sg = 0; sg < 2; ++sg) {
        C2* dst = acc[pi * 2 + sg];
        const C2 hp = h[pi][sg], hm = h[1 - pi][1 - sg];
        for (int q = 0; q + j0 <= n + np; ++q) {
          const int J = j0 + q;
          const C2 hh = u == 0 ? hp : c_add(hp, c_scale(hm, sgn(n + np - J)));
          dst[J - smin] = c_add(dst[J - smin], c_scale(hh, ph * cgv[q]));
        }
      }
  }
}

__global__ void __launch_bounds__(128) ro_w_kernel(RoArgs a) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.n_w) return;
  const int si = owner(a.n_sph, t, [&](int i) { return a.sph[i].t_w; });
  const RoSph sp = a.sph[si];
  const int N = sp.N, n1 = N + 1, S = 2 * N + 1;
  const int idx = (int)(t - sp.t_w);
  const int qi = idx / (2 * N), sg = (idx / N) % 2, n = 1 + idx % N;
  const int q = qi - N - 1, sigma = sg ? -1 : 1, m = q + sigma;
  C2* w = reinterpret_cast<C2*>(a.w + sp.w0);
  // w[qi][sg][p][s][n]
  auto at = [&](int p, int s) -> C2& { return w[(((int64_t)(qi * 2 + sg) * 2 + p) * S + s) * n1 + n]; };
  for (int p = 0; p < 2; ++p)
    for (int s = 0; s < S; ++s) at(p, s) = C2{0, 0};
  if (abs(m) > N || n < max(abs(m), 1)) return;
  double cgv[kS], scratch[kS];
  const C2* rank = reinterpret_cast<const C2*>(a.rank + sp.rank0);
  for (int np = 1; np <= N; ++np) {
    const int j0 = cg_vector(n, m, np, -sigma, cgv, scratch);
    if (j0 < 0) continue;
    const int smin = abs(n - np);
    const C2 pre = c_scale(ipow(np - 1), 2.0 * sqrt(kPi * (2 * np + 1)) * sgn(np - sigma));
    for (int p = 0; p < 2; ++p) {
      const C2* tr = rank + ((int64_t)((p * 2 + sg) * n1 + n) * n1 + np) * S;
      for (int k = 0; j0 + k <= n + np; ++k) {
        const int s = j0 + k;
        if (s < smin) continue;
        at(p, s) = c_add(at(p, s), c_mul(pre, c_scale(tr[s - smin], cgv[k])));
      }
    }
  }
  // The far field's cosine-independent factor gamma_n (-i)^n (functions.rs:192-239).
  const C2 fn = c_scale(ipow(-n), sqrt((2.0 * n + 1) / (kPi * 4.0 * n * (n + 1))));
  for (int p = 0; p < 2; ++p)
    for (int s = 0; s < S; ++s) at(p, s) = c_mul(at(p, s), fn);
}

__global__ void __launch_bounds__(128) ro_phi_kernel(RoArgs a) {
  extern __shared__ double ro_pt[];  // [2 sigma][N + 1][32 cosines][2]: pi_mn, tau_mn
  const int b = blockIdx.x, t = threadIdx.x;
  const int si = owner(a.n_sph, b, [&](int i) { return a.sph[i].t_phi; });
  const RoSph sp = a.sph[si];
  const int N = sp.N, n1 = N + 1, S = 2 * N + 1, nq = sp.nq, tiles = (nq + 31) / 32;
  const int idx = b - (int)sp.t_phi, qi = idx / tiles, q = qi - N - 1;
  const int key = t & 3, p = key >> 1, sg = key & 1, jl = t >> 2, j = (idx % tiles) * 32 + jl;
  const bool valid = j < nq;
  // The angular parts at this thread's cosine for both sigma (threads of key 0 and 1):
  // normalized d_{|m| n}, pi and tau (functions.rs:192-239), m = q + sigma, zero where |m| > N.
  if (p == 0) {
    double* pt = ro_pt + (int64_t)sg * n1 * 64;
    for (int k = 0; k <= N; ++k) {
      pt[(k * 32 + jl) * 2] = 0.0;
      pt[(k * 32 + jl) * 2 + 1] = 0.0;
    }
    const int m = q + (sg ? -1 : 1), am = abs(m);
    if (valid && am <= N) {
      const double ct = a.mu[sp.mu0 + j], st = sqrt(1.0 - ct * ct);
      double am_ = 1.0;
      for (int k = 1; k <= am; ++k) am_ *= sqrt((double)(2 * k - 1) / (2 * k));
      double sp_ = 1.0;
      for (int k = 0; k < am; ++k) sp_ *= st;
      const double flip = m < 0 ? sgn(am) : 1.0;
      double dprev = 0.0, dk = am_ * sp_;  // d_{am - 1} = 0, d_{am}
      for (int k = am; k <= N; ++k) {
        if (k >= 1) {
          const double tau = (k * ct * dk - sqrt((double)k * k - (double)am * am) * dprev) / st;
          const double pi = am * dk / st;
          pt[(k * 32 + jl) * 2] = m < 0 ? -(pi * flip) : pi;
          pt[(k * 32 + jl) * 2 + 1] = tau * flip;
        }
        double dnext;
        if (k == am)
          dnext = sqrt(2.0 * am + 1) * ct * dk;
        else
          dnext = ((2 * k + 1) * ct * dk - sqrt((double)k * k - (double)am * am) * dprev) /
                  sqrt((double)(k + 1) * (k + 1) - (double)am * am);
        dprev = dk;
        dk = dnext;
      }
    }
  }
  __syncthreads();
  // Phi over s for this key; the 16 products with the other keys of the same cosine.
  const C2* wr = reinterpret_cast<const C2*>(a.w + sp.w0) + ((int64_t)(qi * 2 + sg) * 2 + p) * S * n1;
  const double* pt = ro_pt + (int64_t)sg * n1 * 64 + jl * 2;
  const double sign = p ? -1.0 : 1.0;
  C2 prod[4] = {C2{0, 0}, C2{0, 0}, C2{0, 0}, C2{0, 0}};
  for (int s = 0; s < S; ++s) {
    C2 v{0, 0};
    const C2* ws = wr + (int64_t)s * n1;
    for (int n = 1; n <= N; ++n) v = c_add(v, c_scale(ws[n], pt[n * 64] + sign * pt[n * 64 + 1]));
    const double inv = 1.0 / (2 * s + 1);
    C2 other[4];
    for (int y = 0; y < 4; ++y) {
      other[y].re = __shfl_sync(0xffffffffu, v.re, y, 4);
      other[y].im = __shfl_sync(0xffffffffu, v.im, y, 4);
    }
    for (int y = 0; y < 4; ++y) prod[y] = c_add(prod[y], c_scale(c_mul(v, c_conj(other[y])), inv));
  }
  if (valid) {
    C2* part = reinterpret_cast<C2*>(a.part + sp.part0);
    for (int y = 0; y < 4; ++y) part[((int64_t)qi * 16 + key * 4 + y) * nq + j] = prod[y];
  }
}

__global__ void __launch_bounds__(128) ro_f_kernel(RoArgs a) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.n_f) return;
  const int si = owner(a.n_sph, t, [&](int i) { return a.sph[i].t_f; });
  const RoSph sp = a.sph[si];
  const int N = sp.N, nq = sp.nq, j = (int)(t - sp.t_f);
  const C2* part = reinterpret_cast<const C2*>(a.part + sp.part0);
  C2 prod[16];
  for (int k = 0; k < 16; ++k) prod[k] = C2{0, 0};
  for (int qi = 0; qi < 2 * N + 3; ++qi)
    for (int k = 0; k < 16; ++k) prod[k] = c_add(prod[k], part[((int64_t)qi * 16 + k) * nq + j]);
  // <S_ij S*_kl> = sum U_ia U^-1_bj conj(U_kc U^-1_dl) <A_ab A*_cd> (random.rs:295-335).
  const double r = sqrt(0.5);
  const C2 U[2][2] = {{C2{r, 0}, C2{r, 0}}, {C2{0, r}, C2{0, -r}}};
  const C2 Ui[2][2] = {{C2{r, 0}, C2{0, -r}}, {C2{r, 0}, C2{0, r}}};
  auto ss = [&](int i, int jj, int k, int l) {
    C2 acc{0, 0};
    for (int x = 0; x < 2; ++x)
      for (int b = 0; b < 2; ++b)
        for (int c = 0; c < 2; ++c)
          for (int e = 0; e < 2; ++e) {
            const C2 fct = c_mul(c_mul(U[i][x], Ui[b][jj]), c_conj(c_mul(U[k][c], Ui[e][l])));
            acc = c_add(acc, c_mul(fct, prod[((x * 2 + b) * 2 + c) * 2 + e]));
          }
    return acc;
  };
  const double s22 = ss(0, 0, 0, 0).re, s11 = ss(1, 1, 1, 1).re, s33 = ss(0, 1, 0, 1).re,
               s44 = ss(1, 0, 1, 0).re;
  const C2 s12 = ss(1, 1, 0, 0), s34 = ss(0, 1, 1, 0);
  double* f = a.f + sp.f0;
  f[0 * nq + j] = 0.5 * (s11 + s22 + s33 + s44);
  f[1 * nq + j] = 0.5 * (s22 - s11 + s44 - s33);
  f[2 * nq + j] = 0.5 * (s22 + s11 - s44 - s33);
  f[3 * nq + j] = s12.re + s34.re;
  f[4 * nq + j] = -s12.im - s34.im;
  f[5 * nq + j] = s12.re - s34.re;
}

__global__ void __launch_bounds__(128) ro_greek_kernel(RoArgs a) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.n_g) return;
  const int si = owner(a.n_sph, t, [&](int i) { return a.sph[i].t_g; });
  const RoSph sp = a.sph[si];
  const int nq = sp.nq, len = sp.L + 1, l = (int)(t - sp.t_g);
  const double* f = a.f + sp.f0;
  const double* D = a.proj[si];
  double a1 = 0, a4 = 0, pl = 0, mn = 0, b1 = 0, b2 = 0;
  for (int k = 0; k < nq; ++k) {
    const double d00 = D[((int64_t)0 * nq + k) * len + l], d22 = D[((int64_t)1 * nq + k) * len + l];
    const double d2m2 = D[((int64_t)2 * nq + k) * len + l], d02 = D[((int64_t)3 * nq + k) * len + l];
    a1 += f[k] * d00;
    b1 += f[nq + k] * d02;
    pl += (f[2 * nq + k] + f[3 * nq + k]) * d22;
    mn += (f[2 * nq + k] - f[3 * nq + k]) * d2m2;
    b2 += f[4 * nq + k] * d02;
    a4 += f[5 * nq + k] * d00;
  }
  double* g = a.greek + sp.g0;
  g[0 * len + l] = a1;
  g[1 * len + l] = 0.5 * (pl + mn);
  g[2 * len + l] = 0.5 * (pl - mn);
  g[3 * len + l] = a4;
  g[4 * len + l] = b1;
  g[5 * len + l] = b2;
}

void launch_random(const RoArgs& a, cudaStream_t s) {
  if (a.n_sph <= 0) return;
  auto grid = [](int64_t n) { return (unsigned)((n + 127) / 128); };
  ro_rank_kernel<<<grid(a.n_rank), 128, 0, s>>>(a);
  ro_w_kernel<<<grid(a.n_w), 128, 0, s>>>(a);
  // Shared memory: pi and tau of both sigma at a tile of 32 cosines for the batch's largest N.
  const size_t pt_bytes = (size_t)2 * (a.max_n + 1) * 32 * 2 * sizeof(double);
  static bool configured[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 64 && !configured[dev]) {
    cudaFuncSetAttribute(ro_phi_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)((size_t)2 * (kRoMaxN + 1) * 32 * 2 * sizeof(double)));
    configured[dev] = true;
  }
  ro_phi_kernel<<<(unsigned)a.n_phi, 128, pt_bytes, s>>>(a);
  ro_f_kernel<<<grid(a.n_f), 128, 0, s>>>(a);
  ro_greek_kernel<<<grid(a.n_g), 128, 0, s>>>(a);
}

}  // namespace sb
