// The T-matrix of spheroids by the extended boundary condition method on the GPU
// (scatrs/src/tmatrix: kernel.rs for Q and P = RgQ of each azimuthal mode by Gauss-Legendre
// quadrature over the surface, solve.rs for T = -RgQ Q^{-1}, kernel.rs:985-1010 for the
// orientation-averaged cross sections), batched over (spheroid, mode) jobs in three kernels:
//
//   tm_functions_kernel  one thread per (job, node): the node's r(theta), the normal, the
//                        weight, the angular functions d, pi, tau and the radial functions
//                        h_n(r), j_n(r), j_n(s r) with their [z z_n]'/z, orders 0..N;
//   tm_surface_kernel    one thread per (job, i, k): the eight surface integrals
//                        J[out][a][b]_{ik} = sum_nodes w r^2 2 pi n . (A_i x B_k) of the outgoing
//                        (h or j) and inner vector spherical wave functions;
//   tm_solve_kernel      one block per job: Q and RgQ from J, the LU factorization of Q^T with
//                        partial pivoting and the solve for T (in global memory, L2-resident),
//                        and the mode's -Re tr T and sum |T|^2.
//
// The formulation is the classical one from the definition (Mishchenko, Travis & Lacis 2002,
// section 5.8; as research/tmatrix/ebcm.py states it), in FP64. It is accurate where the EBCM's
// own cancellation in the outgoing integrals is mild (moderate aspect ratios and sizes); the
// reference's cancellation-free forms and double-double refinement are not restated here.
#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.h"
#include "mie_device.cuh"

namespace sb {

namespace {

constexpr int kFun = 13;  // doubles per (node, order): d, pi, tau, h (2), h' (2), j, j', w (2), w' (2)
constexpr int kNode = 5;  // doubles per node: r, nu_theta, fac, (s r) (2)

__device__ __forceinline__ cplx csin_(cplx z) {
  return mk(sin(z.re) * cosh(z.im), cos(z.re) * sinh(z.im));
}
__device__ __forceinline__ cplx ccos_(cplx z) {
  return mk(cos(z.re) * cosh(z.im), -(sin(z.re) * sinh(z.im)));
}

}  // namespace

__global__ void __launch_bounds__(128) tm_functions_kernel(TmArgs a) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.n_node_total) return;
  // The job of this node: the largest job whose first node is <= t.
  int lo = 0, hi = a.n_jobs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    if (a.jobs[mid].node0 <= t) lo = mid; else hi = mid - 1;
  }
  const TmJob jb = a.jobs[lo];
  const int q = (int)(t - jb.node0);
  const int N = jb.N, m = jb.m;
  const double ct = a.gl_nodes[jb.rule + q], wq = a.gl_weights[jb.rule + q];
  const double st = sqrt(1.0 - ct * ct);
  // r(theta), dr/dtheta of the spheroid x eps^(1/3) (a), a / eps (c) (ebcm.py:53-65).
  const double ax = jb.x * cbrt(jb.eps), cx = ax / jb.eps;
  const double den = cx * cx * st * st + ax * ax * ct * ct;
  const double r = ax * cx / sqrt(den);
  const double dr = -ax * cx * (cx * cx - ax * ax) * st * ct / (den * sqrt(den));
  double* ns = a.node + t * kNode;
  const cplx s = mk(jb.s_re, jb.s_im);
  const cplx sr = scl(s, r);
  ns[0] = r;
  ns[1] = -dr / r;
  ns[2] = wq * r * r * 2.0 * kPi;
  ns[3] = sr.re;
  ns[4] = sr.im;
  double* f = a.fun + jb.fun0 + (int64_t)q * (N + 1) * kFun;
  // Angular functions (ebcm.py:68-100), normalized, m >= 0.
  {
    double am = 1.0;
    for (int k = 1; k <= m; ++k) am *= sqrt((double)(2 * k - 1) / (2 * k));
    double dprev = 0.0, dcur = 0.0;
    for (int n = 0; n <= N; ++n) {
      double dn;
      if (n < m) dn = 0.0;
      else if (n == m) dn = am * pow(st, (double)m);
      else if (n == m + 1) dn = sqrt(2.0 * m + 1) * ct * dcur;
      else
        dn = ((2 * (n - 1) + 1) * ct * dcur - sqrt((double)(n - 1) * (n - 1) - (double)m * m) * dprev) /
             sqrt((double)n * n - (double)m * m);
      double tau = 0.0, pi = 0.0;
      if (n >= (m > 1 ? m : 1)) {
        const double prev = n - 1 >= m ? dcur : 0.0;
        tau = (n * ct * dn - sqrt((double)n * n - (double)m * m) * prev) / st;
        pi = m * dn / st;
      }
      f[n * kFun + 0] = dn;
      f[n * kFun + 1] = pi;
      f[n * kFun + 2] = tau;
      dprev = dcur;
      dcur = dn;
    }
  }
  // j_n(z) by downward ratios rho_n = j_n / j_{n-1} = z / (2n + 1 - z rho_{n+1}) from far above
  // N; the ratios of orders <= N are kept in the output slots, then turned into values upward
  // from j_0 = sin z / z, j_{-1} = cos z / z. der_n = z_{n-1} - n z_n / z.
  auto bessel_j = [&](cplx z, int slot_re, int slot_im, int dslot_re, int dslot_im) {
    const int start = N + 40 + (int)(2.0 * cabs_(z));
    cplx rho = rl(0.0);
    for (int n = start; n >= 1; --n) {
      rho = z * cinv(rl(2.0 * n + 1) - z * rho);
      if (n <= N) {
        f[n * kFun + slot_re] = rho.re;
        if (slot_im >= 0) f[n * kFun + slot_im] = rho.im;
      }
    }
    const cplx iz = cinv(z);
    cplx jm1 = ccos_(z) * iz, j = csin_(z) * iz;
    for (int n = 0; n <= N; ++n) {
      if (n > 0) {
        const cplx rn = mk(f[n * kFun + slot_re], slot_im >= 0 ? f[n * kFun + slot_im] : 0.0);
        jm1 = j;
        j = rn * j;
      }
      const cplx der = jm1 - scl(j * iz, (double)n);
      f[n * kFun + slot_re] = j.re;
      if (slot_im >= 0) f[n * kFun + slot_im] = j.im;
      f[n * kFun + dslot_re] = der.re;
      if (dslot_im >= 0) f[n * kFun + dslot_im] = der.im;
    }
  };
  bessel_j(rl(r), 7, -1, 8, -1);  // j_n(r), real
  bessel_j(sr, 9, 10, 11, 12);    // j_n(s r)
  // h_n(r) = j_n(r) + i y_n(r), y_n by the upward recurrence (y_{-1} = sin r / r).
  {
    const double ir = 1.0 / r;
    double ym1 = sin(r) * ir, y = -cos(r) * ir;
    for (int n = 0; n <= N; ++n) {
      if (n > 0) {
        const double yn = (2 * (n - 1) + 1) * ir * y - ym1;
        ym1 = y;
        y = yn;
      }
      const double jn = f[n * kFun + 7], jd = f[n * kFun + 8];
      const double yd = ym1 - n * y * ir;
      f[n * kFun + 3] = jn;
      f[n * kFun + 4] = y;
      f[n * kFun + 5] = jd;
      f[n * kFun + 6] = yd;
    }
  }
}

// The eight surface integrals of one (job, i, k): J[out][a][b] with out 0 regular (j_n(r)),
// 1 outgoing (h_n(r)), a, b in {M, N}, summed over the job's nodes in order (ebcm.py:145-186).
__global__ void __launch_bounds__(128) tm_surface_kernel(TmArgs a) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.n_pair_total) return;
  int lo = 0, hi = a.n_jobs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    if (a.jobs[mid].pair0 <= t) lo = mid; else hi = mid - 1;
  }
  const TmJob jb = a.jobs[lo];
  const int N = jb.N, m = jb.m, n0 = m > 1 ? m : 1, K = N - n0 + 1;
  const int pr = (int)(t - jb.pair0), i = n0 + pr / K, k = n0 + pr % K;
  const double gi = sqrt((double)(2 * i + 1) / (4.0 * kPi * i * (i + 1)));
  const double gk = sqrt((double)(2 * k + 1) / (4.0 * kPi * k * (k + 1)));
  cplx J[2][2][2];
#pragma unroll
  for (int o = 0; o < 2; ++o)
#pragma unroll
    for (int p = 0; p < 2; ++p)
#pragma unroll
      for (int b = 0; b < 2; ++b) J[o][p][b] = rl(0.0);
  const int nq = 2 * jb.n_theta;
  for (int q = 0; q < nq; ++q) {
    const double* ns = a.node + (jb.node0 + q) * kNode;
    const double r = ns[0], nut = ns[1], fac = ns[2];
    const cplx sr = mk(ns[3], ns[4]);
    const double* fi = a.fun + jb.fun0 + ((int64_t)q * (N + 1) + i) * kFun;
    const double* fk = a.fun + jb.fun0 + ((int64_t)q * (N + 1) + k) * kFun;
    // Inner functions of order k at s r: M = (0, i g w pi, -g w tau),
    // N = (g k(k+1) w / (s r) d, g w' tau, i g w' pi).
    const cplx w = mk(fk[9], fk[10]), wd = mk(fk[11], fk[12]);
    const double dk = fk[0], pk = fk[1], tk = fk[2];
    const cplx BM[3] = {rl(0.0), cti(scl(w, gk * pk)), scl(w, -gk * tk)};
    const cplx BN[3] = {scl(w * cinv(sr), gk * k * (k + 1) * dk), scl(wd, gk * tk),
                        cti(scl(wd, gk * pk))};
    const double di = fi[0], pi = -fi[1], ti = fi[2];  // outgoing: pi -> -pi
    for (int o = 0; o < 2; ++o) {
      const cplx z = o ? mk(fi[3], fi[4]) : rl(fi[7]);
      const cplx zd = o ? mk(fi[5], fi[6]) : rl(fi[8]);
      const cplx AM[3] = {rl(0.0), cti(scl(z, gi * pi)), scl(z, -gi * ti)};
      const cplx AN[3] = {scl(z, gi * i * (i + 1) * di / r), scl(zd, gi * ti),
                          cti(scl(zd, gi * pi))};
      for (int p = 0; p < 2; ++p) {
        const cplx* A = p ? AN : AM;
        for (int b = 0; b < 2; ++b) {
          const cplx* B = b ? BN : BM;
          const cplx trip = (A[1] * B[2] - A[2] * B[1]) + scl(A[2] * B[0] - A[0] * B[2], nut);
          J[o][p][b] = J[o][p][b] + scl(trip, fac);
        }
      }
    }
  }
  double2* out = reinterpret_cast<double2*>(a.J) + jb.J0;
  const int64_t KK = (int64_t)K * K, e = (int64_t)(i - n0) * K + (k - n0);
#pragma unroll
  for (int o = 0; o < 2; ++o)
#pragma unroll
    for (int p = 0; p < 2; ++p)
#pragma unroll
      for (int b = 0; b < 2; ++b)
        out[((o * 2 + p) * 2 + b) * KK + e] = make_double2(J[o][p][b].re, J[o][p][b].im);
}

// One job per block of 256 threads: Q^T (into the workspace as A) and the right-hand sides
// -RgQ^T (as B), Q^T X = B by LU with partial pivoting (largest modulus, the first on ties)
// applied to B as it goes, back substitution per column, T = X^T; and the mode's sums.
__global__ void __launch_bounds__(256) tm_solve_kernel(TmArgs a) {
  __shared__ double red_v[256];
  __shared__ int red_i[256];
  __shared__ double sums[2][256];
  const TmJob jb = a.jobs[blockIdx.x];
  const int t = threadIdx.x;
  const int N = jb.N, m = jb.m, n0 = m > 1 ? m : 1, K = N - n0 + 1, n2 = 2 * K;
  const int64_t KK = (int64_t)K * K;
  const double2* J = reinterpret_cast<const double2*>(a.J) + jb.J0;
  double2* A = reinterpret_cast<double2*>(a.work) + jb.W0;
  double2* B = A + (int64_t)n2 * n2;
  const cplx s = mk(jb.s_re, jb.s_im);
  const cplx mis = scl(cti(s), -1.0), mi = mk(0.0, -1.0);
  auto Jv = [&](int o, int p, int b, int e) {
    const double2 v = J[((o * 2 + p) * 2 + b) * KK + e];
    return mk(v.x, v.y);
  };
  // Q11 = -i s J12 - i J21, Q12 = -i s J11 - i J22, Q21 = -i s J22 - i J11,
  // Q22 = -i s J21 - i J12 (ebcm.py:189-195); A = Q^T (outgoing), B = -RgQ^T (regular).
  for (int idx = t; idx < n2 * n2; idx += blockDim.x) {
    const int row = idx / n2, col = idx % n2;  // element (row, col) of Q
    const int bi = row >= K, bk = col >= K;
    const int e = (row - bi * K) * K + (col - bk * K);
    cplx q[2];
    for (int o = 0; o < 2; ++o) {
      cplx v;
      if (!bi && !bk) v = mis * Jv(o, 0, 1, e) + mi * Jv(o, 1, 0, e);
      else if (!bi && bk) v = mis * Jv(o, 0, 0, e) + mi * Jv(o, 1, 1, e);
      else if (bi && !bk) v = mis * Jv(o, 1, 1, e) + mi * Jv(o, 0, 0, e);
      else v = mis * Jv(o, 1, 0, e) + mi * Jv(o, 0, 1, e);
      q[o] = v;
    }
    A[(int64_t)col * n2 + row] = make_double2(q[1].re, q[1].im);
    B[(int64_t)col * n2 + row] = make_double2(-q[0].re, -q[0].im);
  }
  __syncthreads();
  auto at = [&](double2* M, int r, int c) -> double2& { return M[(int64_t)r * n2 + c]; };
  for (int kk = 0; kk < n2; ++kk) {
    // Pivot: the largest |A[r][kk]|, r >= kk, the first row on ties.
    double best = -1.0;
    int bi = kk;
    for (int r = kk + t; r < n2; r += blockDim.x) {
      const double2 v = at(A, r, kk);
      const double mag = hypot(v.x, v.y);
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
    if (red_v[0] == 0.0) {
      if (t == 0) atomicExch(a.err, 1u);  // singular Q
      return;
    }
    if (p != kk) {
      for (int c = t; c < n2; c += blockDim.x) {
        const double2 x = at(A, kk, c);
        at(A, kk, c) = at(A, p, c);
        at(A, p, c) = x;
        const double2 y = at(B, kk, c);
        at(B, kk, c) = at(B, p, c);
        at(B, p, c) = y;
      }
    }
    __syncthreads();
    const double2 pv = at(A, kk, kk);
    const cplx ipv = cinv(mk(pv.x, pv.y));
    // Multipliers, then the trailing update of A and of every column of B.
    for (int r = kk + 1 + t; r < n2; r += blockDim.x) {
      const double2 v = at(A, r, kk);
      const cplx fct = mk(v.x, v.y) * ipv;
      at(A, r, kk) = make_double2(fct.re, fct.im);
    }
    __syncthreads();
    const int rows = n2 - kk - 1, cols = (n2 - kk - 1) + n2;
    for (int idx = t; idx < rows * cols; idx += blockDim.x) {
      const int r = kk + 1 + idx / cols, c = idx % cols;
      const double2 fv = at(A, r, kk);
      const cplx fct = mk(fv.x, fv.y);
      if (c < n2 - kk - 1) {
        const int cc = kk + 1 + c;
        const double2 u = at(A, kk, cc), x = at(A, r, cc);
        const cplx y = mk(x.x, x.y) - fct * mk(u.x, u.y);
        at(A, r, cc) = make_double2(y.re, y.im);
      } else {
        const int cc = c - (n2 - kk - 1);
        const double2 u = at(B, kk, cc), x = at(B, r, cc);
        const cplx y = mk(x.x, x.y) - fct * mk(u.x, u.y);
        at(B, r, cc) = make_double2(y.re, y.im);
      }
    }
    __syncthreads();
  }
  // Back substitution, one column per thread.
  for (int c = t; c < n2; c += blockDim.x) {
    for (int i = n2 - 1; i >= 0; --i) {
      const double2 bv = at(B, i, c);
      cplx x = mk(bv.x, bv.y);
      for (int j = i + 1; j < n2; ++j) {
        const double2 u = at(A, i, j), v = at(B, j, c);
        x = x - mk(u.x, u.y) * mk(v.x, v.y);
      }
      const double2 d = at(A, i, i);
      x = x * cinv(mk(d.x, d.y));
      at(B, i, c) = make_double2(x.re, x.im);
    }
  }
  __syncthreads();
  // T[i][k] = X[k][i]: T's rows are B's columns.
  double ext = 0.0, sca = 0.0;
  double2* T = a.T ? reinterpret_cast<double2*>(a.T) + jb.T0 : nullptr;
  for (int idx = t; idx < n2 * n2; idx += blockDim.x) {
    const int i = idx / n2, k = idx % n2;
    const double2 v = at(B, k, i);
    if (T) T[idx] = v;
    if (i == k) ext -= v.x;
    sca += v.x * v.x + v.y * v.y;
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
    a.sums[2 * blockIdx.x] = sums[0][0];
    a.sums[2 * blockIdx.x + 1] = sums[1][0];
  }
}

void launch_tmatrix(const TmArgs& a, cudaStream_t s) {
  if (a.n_jobs <= 0) return;
  tm_functions_kernel<<<(unsigned)((a.n_node_total + 127) / 128), 128, 0, s>>>(a);
  tm_surface_kernel<<<(unsigned)((a.n_pair_total + 127) / 128), 128, 0, s>>>(a);
  tm_solve_kernel<<<a.n_jobs, 256, 0, s>>>(a);
}

}  // namespace sb
