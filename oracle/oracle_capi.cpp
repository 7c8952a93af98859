// C entry points of the CPU oracle, for the tests (ctypes) and the CPU baseline of the
// benchmark. TEST INFRASTRUCTURE ONLY: never linked into the product library.
#include "oracle_core.hpp"

#include <cstdio>
#include <omp.h>

using namespace orc;

extern "C" {

int orc_default_n_max(double x) { return (int)default_n_max(x); }

// Mie::compute / compute_with_derivatives (mie/mod.rs:227-271) for one sphere: with a == NULL
// only the number of terms is returned in *n_terms. eff receives Q_ext, Q_sca, Q_abs, Q_back, g.
int orc_mie(double x, double m_re, double m_im, int64_t n_max, int allow_unvalidated,
            int derivatives, int64_t* n_terms, double* a, double* b, double* eff,
            double* abs_sum, double* da_dx, double* da_dm, double* db_dx, double* db_dm,
            double* abs_jac) {
  int64_t n = 0;
  std::string msg;
  int st = check_inputs(x, m_re, m_im, n_max, allow_unvalidated != 0, &n, &msg);
  if (st != OK) return st;
  *n_terms = n;
  if (!a) return OK;
  MieState s;
  s.solve(x, C(m_re, m_im), n, derivatives != 0);
  for (int64_t k = 0; k < n; ++k) {
    a[2 * k] = s.a[k].re;
    a[2 * k + 1] = s.a[k].im;
    b[2 * k] = s.b[k].re;
    b[2 * k + 1] = s.b[k].im;
    if (derivatives) {
      da_dx[2 * k] = s.da_dx[k].re;
      da_dx[2 * k + 1] = s.da_dx[k].im;
      da_dm[2 * k] = s.da_dm[k].re;
      da_dm[2 * k + 1] = s.da_dm[k].im;
      db_dx[2 * k] = s.db_dx[k].re;
      db_dx[2 * k + 1] = s.db_dx[k].im;
      db_dm[2 * k] = s.db_dm[k].re;
      db_dm[2 * k + 1] = s.db_dm[k].im;
    }
  }
  Efficiencies q = efficiencies(s);
  eff[0] = q.q_ext;
  eff[1] = q.q_sca;
  eff[2] = q.q_abs;
  eff[3] = q.q_back;
  eff[4] = q.g;
  *abs_sum = s.abs_sum;
  if (derivatives && abs_jac) {
    abs_jac[0] = s.abs_sum_jacobian[0];
    abs_jac[1] = s.abs_sum_jacobian[1];
    abs_jac[2] = s.abs_sum_jacobian[2];
  }
  return OK;
}

// Layered::compute (layered/mod.rs:137-160): interface size parameters x[0..layers) (the outer
// last) and indices m (re, im pairs); a, b (N complex pairs each) and eff as orc_mie's.
int orc_layered(const double* x, const double* m, int64_t layers, int64_t* n_terms, double* a,
                double* b, double* eff) {
  std::vector<double> xs(x, x + layers);
  std::vector<cplx> ms(layers);
  for (int64_t l = 0; l < layers; ++l) ms[l] = C(m[2 * l], m[2 * l + 1]);
  int64_t n = default_n_max(xs[layers - 1]);
  *n_terms = n;
  if (!a) return OK;
  MieState s;
  layered_solve(xs, ms, n, s);
  for (int64_t k = 0; k < n; ++k) {
    a[2 * k] = s.a[k].re;
    a[2 * k + 1] = s.a[k].im;
    b[2 * k] = s.b[k].re;
    b[2 * k + 1] = s.b[k].im;
  }
  s.x = xs[layers - 1];
  Efficiencies q = efficiencies(s);
  eff[0] = q.q_ext;
  eff[1] = q.q_sca;
  eff[2] = q.q_abs;
  eff[3] = q.q_back;
  eff[4] = q.g;
  return OK;
}

// MieSolution::amplitudes (mie/amplitudes.rs:328-344) of the sphere (x, m) with the default
// truncation (or n_max terms): s1, s2 interleaved re/im, one pair per cosine.
int orc_amplitudes(double x, double m_re, double m_im, int64_t n_max, const double* mu,
                   int64_t n_mu, double* s1, double* s2) {
  int64_t n = 0;
  int st = check_inputs(x, m_re, m_im, n_max, true, &n, nullptr);
  if (st != OK) return st;
  MieState s;
  s.solve(x, C(m_re, m_im), n, false);
  for (int64_t j = 0; j < n_mu; ++j) {
    cplx a1, a2;
    amplitudes(s.a.data(), s.b.data(), n, mu[j], &a1, &a2);
    s1[2 * j] = a1.re;
    s1[2 * j + 1] = a1.im;
    s2[2 * j] = a2.re;
    s2[2 * j + 1] = a2.im;
  }
  return OK;
}

void orc_gauss_legendre(int64_t n, double* nodes, double* weights) {
  gauss_legendre(n, nodes, weights);
}

void orc_wigner_d(int m, int n, double x, int64_t len, double* out) {
  wigner_d(m, n, x, out, len);
}

// MieSolution::greek (mie/greek.rs:386-447, 501-509): out holds alpha1..beta2, each order+1.
int orc_mie_greek(double x, double m_re, double m_im, int64_t order, int normalized,
                  double* out) {
  int64_t n = 0;
  int st = check_inputs(x, m_re, m_im, 0, true, &n, nullptr);
  if (st != OK) return st;
  MieState s;
  s.solve(x, C(m_re, m_im), n, false);
  int64_t projected = std::min(order, 2 * n);
  int64_t nodes = n + (projected + 2) / 2;
  std::vector<double> mu(nodes), w(nodes);
  gauss_legendre(nodes, mu.data(), w.data());
  std::vector<double> f(4 * nodes);
  double c = 4.0 / (x * x);
  for (int64_t k = 0; k < nodes; ++k) {
    cplx a1, a2;
    amplitudes(s.a.data(), s.b.data(), n, mu[k], &a1, &a2);
    double e[4];
    elements(a1, a2, e);
    for (int i = 0; i < 4; ++i) f[i * nodes + k] = c * e[i];
  }
  Greek g = project(mu.data(), w.data(), nodes, projected, f.data(), f.data() + nodes,
                    f.data() + 2 * nodes, f.data() + 3 * nodes);
  double r0 = g.c[0][0];
  for (auto& v : g.c)
    for (auto& e : v) e = e / r0;
  g.c[0][0] = 1.0;
  if (!normalized) {
    double q = efficiencies(s).q_sca;
    for (auto& v : g.c)
      for (auto& e : v) e = e * q;
  }
  for (int i = 0; i < 6; ++i)
    for (int64_t l = 0; l <= order; ++l) out[i * (order + 1) + l] = l <= projected ? g.c[i][l] : 0.0;
  return OK;
}

// Number density u(r) of a distribution (distribution.rs:370-441), with its gradient.
double orc_density(int kind, double p0, double p1, double p2, double r, double* grad) {
  Density d = prepare(kind, p0, p1, p2);
  return density_eval(d, r, grad);
}

int64_t orc_bucket(int64_t n) { return bucket(n); }

// ---------------------------------------------------------------------------------------
// The fixed-grid ensemble (an extension of the reference's pass 2, engine.rs:1025-1202,
// 1423-1766, averages 1782-1836, project 2310-2355 and assemble 2396-2497): every
// (distribution, wavelength) unit is integrated on the same n_nodes Gauss-Legendre nodes in
// t = ln r over [ln r_lo, ln r_hi], weights w_j u(r_j) r_j as in the reference's panels, and
// normalized by the sum of the weights on those nodes. Nodes group into chunks of 32 in
// ascending radius; a chunk's largest number of terms chooses its projector band, as a panel's
// does in the reference. Units are distribution-major: unit = d * n_wl + i.
// ---------------------------------------------------------------------------------------
static int ensemble_impl(const FixedDist* dists, int64_t n_dist, const double* wl, int64_t n_wl,
                         const double* m, int n_layers, const double* fractions,
                         const double* m_layers, int64_t n_nodes, const double* mu,
                         int64_t n_mu, int64_t greek_order, int normalized,
                         int allow_unvalidated, int n_threads, double* values, double* phase,
                         double* greek, char* err, int64_t err_len, int derivs = 0,
                         double* d_values = nullptr, double* d_phase = nullptr,
                         double* d_greek = nullptr);

int orc_ensemble_fixed(const FixedDist* dists, int64_t n_dist, const double* wl, int64_t n_wl,
                       const double* m, int64_t n_nodes, const double* mu, int64_t n_mu,
                       int64_t greek_order, int normalized, int allow_unvalidated,
                       int n_threads, double* values, double* phase, double* greek,
                       char* err, int64_t err_len) {
  return ensemble_impl(dists, n_dist, wl, n_wl, m, 1, nullptr, nullptr, n_nodes, mu, n_mu,
                       greek_order, normalized, allow_unvalidated, n_threads, values, phase,
                       greek, err, err_len);
}

// The fixed-grid ensemble of layered spheres: fractions [n_dist][n_layers - 1], m_layers
// complex [n_dist][n_layers][n_wl].
int orc_ensemble_fixed_layered(const FixedDist* dists, int64_t n_dist, const double* wl,
                               int64_t n_wl, int n_layers, const double* fractions,
                               const double* m_layers, int64_t n_nodes, const double* mu,
                               int64_t n_mu, int64_t greek_order, int normalized,
                               int allow_unvalidated, int n_threads, double* values,
                               double* phase, double* greek, char* err, int64_t err_len) {
  return ensemble_impl(dists, n_dist, wl, n_wl, nullptr, n_layers, fractions, m_layers, n_nodes,
                       mu, n_mu, greek_order, normalized, allow_unvalidated, n_threads, values,
                       phase, greek, err, err_len);
}

// A value with derivatives along P parameters (ensemble/lin.rs:7-68, errors dropped: the fixed
// grid has no error estimates).
struct LinV {
  double v;
  std::vector<double> d;
};
static LinV lin_div(const LinV& a, const LinV& b) {
  LinV o{a.v / b.v, std::vector<double>(a.d.size())};
  for (size_t k = 0; k < a.d.size(); ++k) o.d[k] = (a.d[k] - o.v * b.d[k]) / b.v;
  return o;
}
static LinV lin_scale(const LinV& a, double c) {
  LinV o{c * a.v, std::vector<double>(a.d.size())};
  for (size_t k = 0; k < a.d.size(); ++k) o.d[k] = c * a.d[k];
  return o;
}

// element_derivatives (mie/phase.rs:62-73).
static int theta_count(int kind) {
  return kind == MODIFIED_GAMMA ? 3 : kind == POWER_LAW ? 1 : kind == TABULATED ? 0 : 2;
}

static int ensemble_impl(const FixedDist* dists, int64_t n_dist, const double* wl, int64_t n_wl,
                         const double* m, int n_layers, const double* fractions,
                         const double* m_layers, int64_t n_nodes, const double* mu,
                         int64_t n_mu, int64_t greek_order, int normalized,
                         int allow_unvalidated, int n_threads, double* values, double* phase,
                         double* greek, char* err, int64_t err_len, int derivs,
                         double* d_values, double* d_phase, double* d_greek) {
  const int64_t n_units = n_dist * n_wl;
  std::vector<double> xi(n_nodes), om(n_nodes);
  gauss_legendre(n_nodes, xi.data(), om.data());
  int P_th = 0;
  if (derivs) {
    if (n_layers > 1) {
      if (err && err_len > 0) snprintf(err, err_len, "derivatives of layered spheres: not here");
      return INVALID_INPUT;
    }
    P_th = n_dist > 0 ? theta_count(dists[0].kind) : 0;
    for (int64_t d = 1; d < n_dist; ++d)
      if (theta_count(dists[d].kind) != P_th) {
        if (err && err_len > 0) snprintf(err, err_len, "derivatives need one distribution kind");
        return INVALID_INPUT;
      }
  }
  const int P = derivs ? P_th + 2 : 0;  // theta parameters, then Re m and Im m
  const int B = 1 + P;                  // blocks: values, then one per parameter
  // Node radii and weights per distribution: w u r, and w (du/dtheta) r.
  std::vector<double> radius(n_dist * n_nodes), weight(n_dist * n_nodes);
  std::vector<double> wth(n_dist * n_nodes * 3, 0.0);
  for (int64_t d = 0; d < n_dist; ++d) {
    if (dists[d].kind == TABULATED) {
      std::string msg;
      if (!table_valid(dists[d].table, dists[d].table_len, &msg)) {
        if (err && err_len > 0) snprintf(err, err_len, "%s", msg.c_str());
        return INVALID_INPUT;
      }
    }
    Density den = prepare(dists[d]);
    double a = std::log(dists[d].r_lo), b = std::log(dists[d].r_hi);
    double c = 0.5 * (a + b), h = 0.5 * (b - a);
    for (int64_t j = 0; j < n_nodes; ++j) {
      double t = c + h * xi[j];
      double w = h * om[j];
      double r = std::exp(t);
      double grad[3];
      double u = density_eval(den, r, grad);
      radius[d * n_nodes + j] = r;
      weight[d * n_nodes + j] = w * (u * r);
      for (int p = 0; p < 3; ++p) wth[(d * n_nodes + j) * 3 + p] = w * (grad[p] * r);
    }
  }
  bool want_greek = greek_order >= 0;
  int64_t n_max_all = 0;
  for (int64_t d = 0; d < n_dist; ++d)
    for (int64_t i = 0; i < n_wl; ++i) {
      double r = radius[d * n_nodes + n_nodes - 1];
      double x = 2.0 * PI * r / wl[i];
      n_max_all = std::max(n_max_all, default_n_max(x));
    }
  std::vector<BandData> bands;
  if (want_greek) {
    for (int64_t u = 1;; u = (int64_t)std::ceil((double)u * 1.25)) {
      bands.push_back(make_band(u, greek_order));
      if (u >= n_max_all) break;
    }
  }
  auto band_index = [&](int64_t n) {
    int64_t u = bucket(n);
    for (size_t i = 0; i < bands.size(); ++i)
      if (bands[i].upper == u) return (int64_t)i;
    return (int64_t)-1;
  };
  int64_t L = want_greek ? greek_order : 0;
  int first_status = OK;
  int64_t first_unit = n_units;
  std::string first_msg;
  if (n_threads > 0) omp_set_num_threads(n_threads);
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t unit = 0; unit < n_units; ++unit) {
    int64_t d = unit / n_wl, i = unit % n_wl;
    double lambda = wl[i];
    cplx mv = n_layers > 1 ? C(0.0, 0.0) : C(m[2 * unit], m[2 * unit + 1]);
    std::vector<cplx> mls(n_layers);
    for (int l = 0; n_layers > 1 && l < n_layers; ++l) {
      const double* p = m_layers + 2 * ((d * n_layers + l) * n_wl + i);
      mls[l] = C(p[0], p[1]);
    }
    // Sums per block: 8 per-particle quantities, the cosine tables, each band's tables.
    std::vector<double> S(B * 8, 0.0), Smu(B * 4 * n_mu, 0.0);
    std::vector<std::vector<double>> Sband(bands.size());
    MieState st;
    std::string msg;
    int status = OK;
    for (int64_t c0 = 0; c0 < n_nodes && status == OK; c0 += NODES_PER_CHUNK) {
      int64_t c1 = std::min(n_nodes, c0 + NODES_PER_CHUNK);
      int64_t n_chunk = 0;
      for (int64_t j = c0; j < c1; ++j) {
        double x = 2.0 * PI * radius[d * n_nodes + j] / lambda;
        n_chunk = std::max(n_chunk, default_n_max(x));
      }
      int64_t bi = want_greek ? band_index(n_chunk) : -1;
      for (int64_t j = c0; j < c1; ++j) {
        double r = radius[d * n_nodes + j];
        double W = weight[d * n_nodes + j];
        double Wb[8];  // the weight of each block
        Wb[0] = W;
        for (int p = 0; p < P_th; ++p) Wb[1 + p] = wth[(d * n_nodes + j) * 3 + p];
        for (int k = 0; k < 2 && derivs; ++k) Wb[1 + P_th + k] = W;
        double x = 2.0 * PI * r / lambda;
        int64_t n = 0;
        if (n_layers <= 1) {
          status = check_inputs(x, mv.re, mv.im, 0, allow_unvalidated != 0, &n, &msg);
        } else {
          std::vector<double> xs(n_layers);
          for (int l = 0; l < n_layers - 1; ++l) xs[l] = fractions[d * (n_layers - 1) + l] * x;
          xs[n_layers - 1] = x;
          status = check_layered(xs, mls, allow_unvalidated != 0, &msg);
          n = default_n_max(x);
          if (status == OK) {
            layered_solve(xs, mls, n, st);
            st.x = x;
          }
        }
        if (status != OK) {
          char buf[160];
          snprintf(buf, sizeof buf, "at wavelength %e, radius %e: ", lambda, r);
          msg = buf + msg;
          break;
        }
        if (n_layers <= 1) st.solve(x, mv, n, derivs != 0);
        Efficiencies q = efficiencies(st);
        double area = PI * r * r;
        // Per-block per-particle quantities (engine.rs:1047-1085).
        double qb[8][8] = {};
        {
          double qv[8] = {1.0,            area * q.q_ext, area * q.q_sca, area * q.q_sca * q.g,
                          area * q.q_abs, area * q.q_back, r * r,       r * r * r};
          for (int b = 0; b < 1 + P_th; ++b)
            for (int k = 0; k < 8; ++k) qb[b][k] = qv[k];
        }
        if (derivs) {
          // derivative_sums (efficiencies.rs:89-146) along Re m and Im m, and
          // efficiencies_jacobian (192-230) for those directions.
          for (int p = 0; p < 2; ++p) {
            const Efficiencies de = efficiency_dir(st, p, q);
            double qd[8] = {0.0,          area * de.q_ext, area * de.q_sca,
                            area * (de.q_sca * q.g + q.q_sca * de.g),
                            area * de.q_abs, area * de.q_back, 0.0,        0.0};
            for (int k = 0; k < 8; ++k) qb[1 + P_th + p][k] = qd[k];
          }
        }
        for (int b = 0; b < B; ++b)
          for (int k = 0; k < 8; ++k) S[b * 8 + k] += Wb[b] * qb[b][k];
        // The requested cosines: phase_matrix(_with_derivatives) at each cosine
        // (phase.rs:204-219, 289-341; amplitudes.rs:347-381), times the area.
        double cph = 4.0 / (x * x);
        for (int64_t kk = 0; kk < n_mu; ++kk) {
          cplx s1 = real(0.0), s2 = real(0.0), d1 = real(0.0), d2 = real(0.0);
          for_each_order(mu[kk], n, [&](int64_t k, double pi, double tau) {
            cplx an = st.a[k - 1], bn = st.b[k - 1];
            s1 = s1 + scale(an, pi) + scale(bn, tau);
            s2 = s2 + scale(an, tau) + scale(bn, pi);
            if (derivs) {
              cplx da = st.da_dm[k - 1], db = st.db_dm[k - 1];
              d1 = d1 + scale(da, pi) + scale(db, tau);
              d2 = d2 + scale(da, tau) + scale(db, pi);
            }
          });
          double e[4];
          elements(s1, s2, e);
          for (int b = 0; b < 1 + P_th; ++b)
            for (int t = 0; t < 4; ++t) Smu[(b * 4 + t) * n_mu + kk] += Wb[b] * (cph * e[t] * area);
          if (derivs) {
            double fr[4], fi[4];
            element_derivs(s1, s2, d1, d2, fr);
            element_derivs(s1, s2, times_i(d1), times_i(d2), fi);
            for (int t = 0; t < 4; ++t) {
              Smu[((1 + P_th) * 4 + t) * n_mu + kk] += W * (area * (cph * fr[t] + 0.0 * e[t]));
              Smu[((2 + P_th) * 4 + t) * n_mu + kk] += W * (area * (cph * fi[t] + 0.0 * e[t]));
            }
          }
        }
        if (bi >= 0) {
          BandData& Bd = bands[bi];
          std::vector<double>& sb = Sband[bi];
          if (sb.empty()) sb.assign(B * 4 * Bd.n_q, 0.0);
          int64_t qn = Bd.n_q, lo = qn / 2, h = qn - lo;
          int64_t terms = std::min(n_chunk, Bd.upper);
          double scl = 4.0 / (x * x) * (PI * r * r);
          for (int64_t ii = 0; ii < h; ++ii) {
            // ce = G_E X and co = G_O X over the sphere's 4 columns and, with derivatives, its
            // 4 derivative columns (fast.rs:98-145).
            double ce[8] = {0}, co[8] = {0};
            for (int64_t k = 0; k < terms; ++k) {
              double xr[8] = {0};
              if (k < n) {
                cplx uu = (k % 2 == 0) ? st.a[k] : st.b[k];
                cplx vv = (k % 2 == 0) ? st.b[k] : st.a[k];
                xr[0] = uu.re;
                xr[1] = uu.im;
                xr[2] = vv.re;
                xr[3] = vv.im;
                if (derivs) {
                  cplx du = (k % 2 == 0) ? st.da_dm[k] : st.db_dm[k];
                  cplx dv = (k % 2 == 0) ? st.db_dm[k] : st.da_dm[k];
                  xr[4] = du.re;
                  xr[5] = du.im;
                  xr[6] = dv.re;
                  xr[7] = dv.im;
                }
              }
              double ge = Bd.ge[ii * Bd.upper + k], go = Bd.go[ii * Bd.upper + k];
              for (int t = 0; t < 8; ++t) {
                ce[t] += ge * xr[t];
                co[t] += go * xr[t];
              }
            }
            cplx eu = C(ce[0], ce[1]), ev = C(ce[2], ce[3]);
            cplx ou = C(co[0], co[1]), ov = C(co[2], co[3]);
            cplx deu = C(ce[4], ce[5]), dev = C(ce[6], ce[7]);
            cplx dou = C(co[4], co[5]), dov = C(co[6], co[7]);
            int64_t jn = lo + ii;
            auto write = [&](int64_t node, double sign) {
              cplx s1 = eu + scale(ov, sign), s2 = ev + scale(ou, sign);
              double e[4];
              elements(s1, s2, e);
              for (int b = 0; b < 1 + P_th; ++b)
                for (int t = 0; t < 4; ++t) sb[(b * 4 + t) * qn + node] += Wb[b] * (scl * e[t]);
              if (derivs) {
                cplx d1 = deu + scale(dov, sign), d2 = dev + scale(dou, sign);
                double fr[4], fi[4];
                element_derivs(s1, s2, d1, d2, fr);
                element_derivs(s1, s2, times_i(d1), times_i(d2), fi);
                for (int t = 0; t < 4; ++t) {
                  sb[((1 + P_th) * 4 + t) * qn + node] += W * (scl * fr[t]);
                  sb[((2 + P_th) * 4 + t) * qn + node] += W * (scl * fi[t]);
                }
              }
            };
            write(jn, 1.0);
            int64_t mirror = qn - 1 - jn;
            if (mirror != jn) write(mirror, -1.0);
          }
        }
      }
    }
    if (status == OK) {
      // averages (engine.rs:1782-1836): v = S/Z; theta: (S_t - v dZ)/Z; m: S_m/Z.
      const double z = S[0];
      auto average = [&](std::vector<double>& blk, int64_t len) {
        for (int64_t k = 0; k < len; ++k) blk[k] = blk[k] / z;
        for (int p = 0; p < P_th; ++p) {
          const double dz = S[(1 + p) * 8];
          for (int64_t k = 0; k < len; ++k)
            blk[(1 + p) * len + k] = (blk[(1 + p) * len + k] - blk[k] * dz) / z;
        }
        for (int p = 1 + P_th; p < B; ++p)
          for (int64_t k = 0; k < len; ++k) blk[p * len + k] = blk[p * len + k] / z;
      };
      std::vector<double> Sv = S;
      average(Sv, 8);
      average(Smu, 4 * n_mu);
      for (size_t b2 = 0; b2 < bands.size(); ++b2)
        if (!Sband[b2].empty()) average(Sband[b2], 4 * bands[b2].n_q);
      auto lin = [&](int k) {
        LinV o{Sv[k], std::vector<double>(P)};
        for (int p = 0; p < P; ++p) o.d[p] = Sv[(1 + p) * 8 + k];
        return o;
      };
      LinV ext = lin(1), sca = lin(2), scag = lin(3), ab = lin(4), back = lin(5), r2 = lin(6),
           r3 = lin(7);
      const char* bad = nullptr;
      if (!(std::isfinite(ext.v) && ext.v != 0.0)) bad = "<C_ext>";
      else if (!(std::isfinite(sca.v) && sca.v != 0.0)) bad = "<C_sca>";
      else if (!(std::isfinite(back.v) && back.v != 0.0)) bad = "<C_back>";
      if (bad) {
        status = INVALID_INPUT;
        msg = std::string("the ensemble's ") + bad + " is 0 or not finite, so its ratios are undefined (does m = 1?)";
      } else {
        LinV zero{0.0, std::vector<double>(P, 0.0)};
        LinV out[11] = {ext,
                        sca,
                        ab,
                        back,
                        lin_div(sca, ext),
                        lin_div(scag, sca),
                        lin_scale(lin_div(ext, back), 4.0 * PI),
                        zero,
                        lin_div(r3, r2),
                        lin_scale(r2, PI),
                        lin_scale(r3, 4.0 * PI / 3.0)};
        for (int k = 0; k < 11; ++k) {
          values[k * n_units + unit] = out[k].v;
          for (int p = 0; p < P; ++p) d_values[(p * 11 + k) * n_units + unit] = out[k].d[p];
        }
        if (phase && n_mu > 0) {
          const int src[6] = {0, 1, 0, 2, 3, 2};
          for (int e = 0; e < 6; ++e)
            for (int64_t k = 0; k < n_mu; ++k) {
              LinV f{Smu[src[e] * n_mu + k], std::vector<double>(P)};
              for (int p = 0; p < P; ++p) f.d[p] = Smu[((1 + p) * 4 + src[e]) * n_mu + k];
              if (normalized) f = lin_div(f, sca);
              phase[(e * n_units + unit) * n_mu + k] = f.v;
              for (int p = 0; p < P; ++p)
                d_phase[((p * 6 + e) * n_units + unit) * n_mu + k] = f.d[p];
            }
        }
        if (greek && want_greek) {
          // project (engine.rs:2310-2355) every block of every band, summed over the bands.
          std::vector<double> g(B * 6 * (L + 1), 0.0);
          for (size_t b2 = 0; b2 < bands.size(); ++b2) {
            if (Sband[b2].empty()) continue;
            BandData& Bd = bands[b2];
            int64_t qn = Bd.n_q, len = Bd.order + 1;
            for (int blk = 0; blk < B; ++blk) {
              const double* f = Sband[b2].data() + (int64_t)blk * 4 * qn;
              const double* f11 = f;
              const double* f12 = f + qn;
              const double* f33 = f + 2 * qn;
              const double* f34 = f + 3 * qn;
              for (int64_t l = 0; l < len; ++l) {
                double a1 = 0, a4 = 0, pp = 0, mi = 0, b1 = 0, b2v = 0;
                for (int64_t k = 0; k < qn; ++k) {
                  double d00 = Bd.dmat[0][k * len + l], d22 = Bd.dmat[1][k * len + l];
                  double d2m2 = Bd.dmat[2][k * len + l], d02 = Bd.dmat[3][k * len + l];
                  a1 += f11[k] * d00;
                  a4 += f33[k] * d00;
                  pp += (f11[k] + f33[k]) * d22;
                  mi += (f11[k] - f33[k]) * d2m2;
                  b1 += f12[k] * d02;
                  b2v += f34[k] * d02;
                }
                double c6[6] = {a1, (pp + mi) * 0.5, (pp - mi) * 0.5, a4, b1, b2v};
                for (int e = 0; e < 6; ++e) g[(blk * 6 + e) * (L + 1) + l] += c6[e];
              }
            }
          }
          LinV a0{g[0], std::vector<double>(P)};
          for (int p = 0; p < P; ++p) a0.d[p] = g[((1 + p) * 6) * (L + 1)];
          for (int e = 0; e < 6; ++e)
            for (int64_t l = 0; l <= L; ++l) {
              LinV c{g[e * (L + 1) + l], std::vector<double>(P)};
              for (int p = 0; p < P; ++p) c.d[p] = g[((1 + p) * 6 + e) * (L + 1) + l];
              if (normalized) {
                if (e == 0 && l == 0)
                  c = LinV{1.0, std::vector<double>(P, 0.0)};
                else
                  c = lin_div(c, a0);
              }
              greek[(e * n_units + unit) * (L + 1) + l] = c.v;
              for (int p = 0; p < P; ++p)
                d_greek[((p * 6 + e) * n_units + unit) * (L + 1) + l] = c.d[p];
            }
        }
      }
    }
    if (status != OK) {
#pragma omp critical
      {
        if (unit < first_unit) {
          first_unit = unit;
          first_status = status;
          first_msg = msg;
        }
      }
    }
  }
  if (first_status != OK && err && err_len > 0) {
    snprintf(err, err_len, "%s", first_msg.c_str());
  }
  return first_status;
}

// The fixed-grid ensemble with the derivatives of every output along the distribution's
// parameters, then Re m and Im m (P of them): d_values (P, 11, n), d_phase (P, 6, n, n_mu),
// d_greek (P, 6, n, L + 1).
int orc_ensemble_fixed_d(const FixedDist* dists, int64_t n_dist, const double* wl, int64_t n_wl,
                         const double* m, int64_t n_nodes, const double* mu, int64_t n_mu,
                         int64_t greek_order, int normalized, int allow_unvalidated,
                         int n_threads, double* values, double* phase, double* greek,
                         double* d_values, double* d_phase, double* d_greek, char* err,
                         int64_t err_len) {
  return ensemble_impl(dists, n_dist, wl, n_wl, m, 1, nullptr, nullptr, n_nodes, mu, n_mu,
                       greek_order, normalized, allow_unvalidated, n_threads, values, phase,
                       greek, err, err_len, 1, d_values, d_phase, d_greek);
}

}  // extern "C"
