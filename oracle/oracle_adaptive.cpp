// TEST INFRASTRUCTURE ONLY: the reference's adaptive ensemble engine restated on the CPU, the
// oracle of the GPU adaptive path. Spheres; distributions with unbounded support (lognormal,
// gamma, modified gamma), finite support (power law) or a single radius (monodisperse); one
// distribution per call (`compute`, ensemble/mod.rs:548-606) or a batch sharing panels
// (`compute_batch`, mod.rs:613-686). Values and error estimates; no derivatives.
//
//   ensemble/kronrod.rs   GK15 panels                     (gk_panel)
//   ensemble/range.rs     tail cut-offs                   (masses, cutoffs)
//   ensemble/moments.rs   Z, <r^2>, <r^3>                 (moments)
//   ensemble/engine.rs    parts 141-233, initial_panels 301-354, quantities1/panel1 369-560,
//                         status 620-720, pass1 724-924, panel_terms 961-978, pass2 1363-1766,
//                         averages 1782-1836, monodisperse 1838-1890, wavelength 1964-2250,
//                         project 2310-2355, assemble 2396-2497
//   ensemble/lin.rs       error propagation through the ratios (Lin)
#include "oracle_core.hpp"
#include "oracle_spheroid.hpp"

#include <omp.h>

#include <algorithm>
#include <array>
#include <cstdio>
#include <cstring>
#include <functional>
#include <limits>
#include <map>
#include <set>
#include <string>
#include <vector>

using namespace orc;

namespace {

constexpr double STEP = 0.5;
constexpr int MAX_STEPS = 400;
constexpr int MAX_EXTENSIONS = 100;
constexpr double MIN_WIDTH = 1e-10;
constexpr double MAX_DX = 20.0;
constexpr size_t MOMENT_MAX_PANELS = 100000;
constexpr int MONODISPERSE = 5;
constexpr int64_t GREEK_ALL = -2;  // every order up to 2 N_max at each wavelength

// The Greek coefficients of the last call with GREEK_ALL, per output unit (its own length),
// and with derivatives per parameter.
struct AllOrders {
  std::vector<std::vector<double>> g, ge, dg, dge;
  size_t P = 0;
};
AllOrders g_all_orders;
void keep_all_orders(std::vector<std::vector<double>>& g, std::vector<std::vector<double>>& ge,
                     std::vector<std::vector<double>>& dg, std::vector<std::vector<double>>& dge,
                     size_t P) {
  g_all_orders.g.swap(g);
  g_all_orders.ge.swap(ge);
  g_all_orders.dg.swap(dg);
  g_all_orders.dge.swap(dge);
  g_all_orders.P = P;
}
constexpr double INF = std::numeric_limits<double>::infinity();

// Pass-1 quantities (engine.rs:43-54): 1, C_ext, C_sca, C_sca g, C_back, C_abs.
constexpr int N_BASE = 6;
constexpr int P1_ONE = 0, P1_EXT = 1, P1_SCA = 2, P1_SCAG = 3, P1_BACK = 4, P1_ABS = 5;
// Pass-2 scalars (engine.rs:31-41).
constexpr int S_ONE = 0, S_EXT = 1, S_SCA = 2, S_SCAG = 3, S_ABS = 4, S_BACK = 5, S_R2 = 6,
              S_R3 = 7, SCALARS = 9;

struct Failure {
  int status;
  std::string msg;
};

std::string at(double lambda, double r) {
  char buf[160];
  snprintf(buf, sizeof buf, "at wavelength %e, radius %e: ", lambda, r);
  return buf;
}

// kronrod.rs:5-52.
const double KN[8] = {0.9914553711208126, 0.9491079123427585, 0.8648644233597691,
                      0.7415311855993944, 0.5860872354676911, 0.4058451513773972,
                      0.20778495500789847, 0.0};
const double KW[8] = {0.022935322010529225, 0.06309209262997855, 0.10479001032225018,
                      0.14065325971552592,  0.1690047266392679,  0.1903505780647854,
                      0.2044329400752989,   0.20948214108472783};
const double GW[4] = {0.1294849661688697, 0.2797053914892767, 0.3818300505051189,
                      0.4179591836734694};
struct Node {
  double t, wk, wg;
};
void gk_panel(double a, double b, Node out[15]) {
  const double c = 0.5 * (a + b), h = 0.5 * (b - a);
  for (int i = 0; i < 7; ++i) {
    const double gauss = i % 2 == 1 ? h * GW[i / 2] : 0.0;
    const double k = h * KW[i];
    out[i] = {c - h * KN[i], k, gauss};
    out[14 - i] = {c + h * KN[i], k, gauss};
  }
  out[7] = {c, h * KW[7], h * GW[3]};
}

double powk(double r, int k) { return k == 0 ? 1.0 : k == 2 ? r * r : r * r * r; }

double max_step(const Density& d, double step) { return std::min(step, 0.5 * d.log_width); }

// range.rs:25-36.
void masses(const Density& d, double t0, double t1, const int* powers, int np, double* out) {
  Node nd[15];
  gk_panel(t0, t1, nd);
  for (int k = 0; k < np; ++k) out[k] = 0.0;
  for (auto& n : nd) {
    const double r = std::exp(n.t);
    const double wu = n.wk * r * density_eval(d, r, nullptr);
    for (int k = 0; k < np; ++k) out[k] += wu * powk(r, powers[k]);
  }
}

// range.rs:48-93.
std::pair<double, double> cutoffs(const Density& d, double center, double eps,
                                  std::vector<int> powers) {
  const double t0 = std::log(center);
  const double step = max_step(d, STEP);
  const int np = (int)powers.size();
  std::vector<double> total(np, 0.0);
  double ends[2] = {t0, t0};
  std::vector<double> last[2] = {std::vector<double>(np, INF), std::vector<double>(np, INF)};
  bool done[2] = {false, false};
  std::vector<double> mass(np);
  for (int i = 0; i < MAX_STEPS; ++i) {
    for (int side = 0; side < 2; ++side) {
      if (done[side]) continue;
      const double sign = side == 0 ? -1.0 : 1.0;
      const double a = ends[side], b = a + sign * step;
      masses(d, std::min(a, b), std::max(a, b), powers.data(), np, mass.data());
      for (double m : mass)
        if (!std::isfinite(m)) {
          char buf[160];
          snprintf(buf, sizeof buf,
                   "the size distribution's density is not finite near r = %e", std::exp(b));
          throw Failure{INVALID_INPUT, buf};
        }
      ends[side] = b;
      bool small = i >= 1;
      for (int k = 0; k < np; ++k) {
        total[k] += mass[k];
        const double q = mass[k] / last[side][k];
        last[side][k] = mass[k];
        small = small && (mass[k] == 0.0 || (q < 1.0 && mass[k] / (1.0 - q) <= eps * total[k]));
      }
      done[side] = small;
    }
    if (done[0] && done[1]) return {std::exp(ends[0]), std::exp(ends[1])};
  }
  throw Failure{INVALID_INPUT, "the size distribution is too broad: its tails do not decay"};
}

// moments.rs:15-26: <r^2>, <r^3> and Z with their error estimates, and their derivatives along
// the requested distribution parameters with theirs.
struct Moments {
  double v[2], e[2], z, ez;
  std::vector<std::array<double, 2>> d, de;
  std::vector<double> dz, dez;
};

// moments.rs:62-167: GK15 panels of at most the step (the breaks inside the range as edges),
// split where |Kronrod - Gauss| of any of the 3 (1 + nt) sums is above its share, until each
// meets rtol (of |sum| for the values, of the Kronrod sum of the absolute integrand for the
// derivatives); the averages by the quotient rule with first-order error propagation. `grads`
// are the requested parameters' indices into the density's gradient.
Moments moments(const Density& d, std::pair<double, double> range, double rtol,
                double truncation, const std::vector<double>& breaks = {},
                const std::vector<int>& grads = {}) {
  const double step = max_step(d, STEP);
  const double t_lo = std::log(range.first), t_hi = std::log(range.second);
  const int nt = (int)grads.size(), nq = 3 * (1 + nt);
  std::vector<std::pair<double, double>> panels;
  {
    // moments.rs:71-86: the breaks inside the range are panel edges, each interval in equal
    // panels of at most the step.
    std::vector<double> edges{t_lo};
    for (double r : breaks) {
      const double t = std::log(r);
      if (t > t_lo && t < t_hi) edges.push_back(t);
    }
    edges.push_back(t_hi);
    for (size_t w = 0; w + 1 < edges.size(); ++w) {
      const double a = edges[w], b = edges[w + 1];
      const size_t n = (size_t)std::max(1.0, std::ceil((b - a) / step));
      const double h = (b - a) / (double)n;
      for (size_t i = 0; i < n; ++i) panels.push_back({a + i * h, a + (i + 1) * h});
    }
  }
  // moments.rs:171-212 (averages).
  auto finish = [&](const std::vector<double>& s, const std::vector<double>& e) {
    const double z = s[0], ez = e[0];
    if (!(std::isfinite(z) && z > 0.0)) {
      char buf[128];
      snprintf(buf, sizeof buf,
               "the size distribution has no finite positive mass on its range (got %e)", z);
      throw Failure{INVALID_INPUT, buf};
    }
    Moments m;
    m.z = z;
    m.ez = ez;
    for (int k = 0; k < 2; ++k) {
      m.v[k] = s[1 + k] / z;
      m.e[k] = (e[1 + k] + std::fabs(m.v[k]) * ez) / z + truncation * std::fabs(m.v[k]);
    }
    for (int b = 0; b < nt; ++b) {
      const int o = 3 * (1 + b);
      const double dz = s[o];
      std::array<double, 2> dv, dev;
      for (int k = 0; k < 2; ++k) dv[k] = (s[o + 1 + k] - m.v[k] * dz) / z;
      for (int k = 0; k < 2; ++k)
        dev[k] = (e[o + 1 + k] + std::fabs(m.v[k]) * e[o] + std::fabs(dv[k]) * ez +
                  m.e[k] * std::fabs(dz)) / z +
                 truncation * std::fabs(dv[k]);
      m.d.push_back(dv);
      m.de.push_back(dev);
      m.dz.push_back(dz);
      m.dez.push_back(e[o]);
    }
    return m;
  };
  std::vector<double> grad(3);
  for (;;) {
    // Per panel: Kronrod sums, |K - G| and Kronrod sums of the absolute integrands
    // (moments.rs:31-53).
    const size_t n = panels.size();
    std::vector<double> K(n * nq, 0.0), E(n * nq, 0.0), A(n * nq, 0.0);
    for (size_t i = 0; i < n; ++i) {
      Node nd[15];
      gk_panel(panels[i].first, panels[i].second, nd);
      std::vector<double> g(nq, 0.0);
      for (auto& x : nd) {
        const double r = std::exp(x.t);
        const double u = density_eval(d, r, grad.data());
        const double q[3] = {1.0, r * r, r * r * r};
        for (int j = 0; j < 3; ++j) {
          K[i * nq + j] += x.wk * u * r * q[j];
          g[j] += x.wg * u * r * q[j];
          for (int b = 0; b < nt; ++b) {
            const int o = 3 * (1 + b) + j;
            const double y = grad[grads[b]] * r * q[j];
            K[i * nq + o] += x.wk * y;
            g[o] += x.wg * y;
            A[i * nq + o] += x.wk * std::fabs(y);
          }
        }
      }
      for (int j = 0; j < nq; ++j) E[i * nq + j] = std::fabs(K[i * nq + j] - g[j]);
    }
    std::vector<double> total(nq, 0.0), terr(nq, 0.0), target(nq, 0.0);
    for (size_t i = 0; i < n; ++i)
      for (int j = 0; j < nq; ++j) {
        total[j] += K[i * nq + j];
        terr[j] += E[i * nq + j];
      }
    for (int j = 0; j < nq; ++j) {
      if (j < 3) {
        target[j] = rtol * std::fabs(total[j]);
      } else {
        double abs = 0.0;
        for (size_t i = 0; i < n; ++i) abs += A[i * nq + j];
        target[j] = rtol * abs;
      }
    }
    bool met = true;
    for (int j = 0; j < nq; ++j) met = met && terr[j] <= target[j];
    if (met || n >= MOMENT_MAX_PANELS) return finish(total, terr);
    std::vector<std::pair<double, double>> next;
    for (size_t i = 0; i < n; ++i) {
      bool bad = false;
      for (int j = 0; j < nq; ++j)
        bad = bad || (E[i * nq + j] * (double)n > target[j] && terr[j] > target[j]);
      const auto& p = panels[i];
      if (bad && p.second - p.first > 1e-10) {
        const double mid = 0.5 * (p.first + p.second);
        next.push_back({p.first, mid});
        next.push_back({mid, p.second});
      } else {
        next.push_back(p);
      }
    }
    if (next.size() == n) return finish(total, terr);
    panels.swap(next);
  }
}

enum SupportKind { UNBOUNDED, FINITE, POINT };

struct Part {
  FixedDist dist;
  const double* m = nullptr;  // complex per wavelength: the part's sphere
  // A layered sphere: n_layers > 1, fractions [n_layers - 1], m_layers complex [n_layers][n_wl].
  int n_layers = 1;
  const double* fractions = nullptr;
  const double* m_layers = nullptr;
  int64_t n_wl = 0;
  double eps = 0.0;  // > 0: a spheroid of this aspect ratio (the direct path)
  double f = 1.0;             // the number fraction in its unit (engine.rs:2131)
  // engine.rs:95-115: the component and mode, the component's weight w and the mode's weight
  // v with the component's sum of mode weights (1, 1 without modes); the requested
  // distribution parameters (result column, index into the gradient) and the result columns
  // of the derivatives along Re m and Im m (-1: not requested).
  int component = 0, mode = -1;
  double w = 1.0, v = 1.0, v_total = 1.0;
  std::vector<std::pair<int, int>> theta;
  int dir_col[2] = {-1, -1};
  bool dir_derivatives() const { return dir_col[0] >= 0 || dir_col[1] >= 0; }
  Density den;
  SupportKind support;
  double s_a = 0, s_b = 0;  // center (unbounded), [lo, hi] (finite), radius (point)
  std::pair<double, double> cut;
  Moments mom{};
};

// parts (engine.rs:141-223) for one distribution: its support, cut-offs and moments, the
// moments with the derivatives along `grads` (indices into the density's gradient).
Part make_part(const FixedDist& d, double rtol, const std::vector<int>& grads = {}) {
  Part p;
  p.dist = d;
  if (d.kind == MONODISPERSE) {
    p.den = prepare(LOGNORMAL, 1.0, 2.0, 0.0);  // unused
    p.support = POINT;
    p.s_a = d.p[0];
    p.cut = {d.p[0], d.p[0]};
    return p;
  }
  if (d.kind == TABULATED) {
    // distribution.rs:285-287 and engine.rs:181-185: finite support between the first and
    // last radii, the table's radii as edges of the moment panels.
    std::string msg;
    if (!table_valid(d.table, d.table_len, &msg)) throw Failure{INVALID_INPUT, msg};
    p.den = prepare(d);
    p.support = FINITE;
    p.s_a = d.table[0];
    p.s_b = d.table[d.table_len - 1];
    p.mom = moments(p.den, {p.s_a, p.s_b}, rtol, 0.0,
                    std::vector<double>(d.table, d.table + d.table_len), grads);
    p.cut = {p.s_a, p.s_b};
    return p;
  }
  p.den = prepare(d.kind, d.p[0], d.p[1], d.p[2]);
  if (d.kind == POWER_LAW) {
    p.support = FINITE;
    p.s_a = d.p[1];
    p.s_b = d.p[2];
    p.mom = moments(p.den, {p.s_a, p.s_b}, rtol, 0.0, {}, grads);
    p.cut = {p.s_a, p.s_b};
    return p;
  }
  // distribution.rs:272-290: lognormal about its median, gamma its effective radius,
  // modified gamma its reference radius.
  p.support = UNBOUNDED;
  p.s_a = d.kind == LOGNORMAL ? d.p[0] : d.kind == GAMMA ? d.p[0] : p.den.reference;
  p.cut = cutoffs(p.den, p.s_a, rtol / 10.0, {2});
  const double eps = std::max(1e-3 * rtol, 1e-16);
  auto wide = cutoffs(p.den, p.s_a, eps, {0, 2, 3});
  p.mom = moments(p.den, wide, rtol, 0.2 * rtol, {}, grads);
  return p;
}

double size_param(double r, double lambda) { return 2.0 * PI * r / lambda; }

// engine.rs:301-354.
std::vector<std::pair<double, double>> initial_panels(double t_lo, double t_hi, double lambda,
                                                      const std::vector<double>& breaks,
                                                      const std::function<double(double)>& step_of,
                                                      size_t budget) {
  std::vector<double> edges{t_lo};
  for (double r : breaks) {
    const double t = std::log(r);
    if (t > t_lo && t < t_hi) edges.push_back(t);
  }
  edges.push_back(t_hi);
  std::vector<std::pair<double, double>> out;
  for (size_t e = 0; e + 1 < edges.size() && out.size() <= budget; ++e) {
    double a = edges[e];
    const double b = edges[e + 1];
    while (a < b) {
      const double x = size_param(std::exp(a), lambda);
      const double step = std::min(step_of(a), std::log(1.0 + MAX_DX / x));
      const double n = std::max(1.0, std::ceil((b - a) / step));
      const double h = (b - a) / n;
      const double next = (n <= 1.0 || a + h <= a) ? b : a + h;
      out.push_back({a, next});
      a = next;
      if (out.size() > budget) break;
    }
  }
  if (out.size() <= budget) return out;
  const double width = t_hi - t_lo;
  std::vector<std::pair<double, double>> equal;
  for (size_t e = 0; e + 1 < edges.size(); ++e) {
    const size_t n =
        (size_t)std::max(1.0, std::floor((edges[e + 1] - edges[e]) / width * (double)budget));
    const double h = (edges[e + 1] - edges[e]) / (double)n;
    for (size_t i = 0; i < n; ++i)
      equal.push_back({edges[e] + (double)i * h, edges[e] + (double)(i + 1) * h});
  }
  return equal;
}

struct Options {
  double rtol;
  size_t max_panels;
  bool allow_unvalidated, refine_backscatter;
};

// The particle of a group at one wavelength: a homogeneous sphere (m), or a layered one
// (layered/kernel.rs; particle.rs:186-195: x_l = f_l x, the outer surface's x last).
struct Optics {
  cplx m{0, 0};
  std::vector<double> fr;  // empty for a homogeneous sphere
  std::vector<cplx> ml;
  // A spheroid (eps > 0): its T-matrix tolerance and the wavelength's solved nodes by radius.
  double eps = 0.0, rtol_t = 0.0;
  std::map<double, SpheroidNode>* cache = nullptr;
};

// A spheroid node, solved once (particle.rs:317-366; pass 2 reuses pass 1's values).
const SpheroidNode& sph_node(double r, double lambda, const Optics& op) {
  auto it = op.cache->find(r);
  if (it != op.cache->end()) return it->second;
  SpheroidNode v;
  const int st = spheroid_node(size_param(r, lambda), op.eps, op.m, op.rtol_t, &v);
  if (st != OK)
    throw Failure{st, at(lambda, r) + (st == NOT_CONVERGED ? "the T-matrix did not converge"
                                                           : "invalid spheroid")};
  return op.cache->emplace(r, std::move(v)).first->second;
}

// The node's number of terms after its input checks, or a Failure with the node's context;
// the layered sizes into xs.
int64_t node_terms(double r, double lambda, const Optics& op, bool allow, std::vector<double>& xs) {
  if (op.eps > 0.0) return sph_node(r, lambda, op).n;
  const double x = size_param(r, lambda);
  std::string msg;
  int64_t n = 0;
  int s;
  if (op.fr.empty()) {
    s = check_inputs(x, op.m.re, op.m.im, 0, allow, &n, &msg);
  } else {
    xs.resize(op.ml.size());
    for (size_t l = 0; l + 1 < op.ml.size(); ++l) xs[l] = op.fr[l] * x;
    xs.back() = x;
    s = check_layered(xs, op.ml, allow, &msg);
    n = default_n_max(x);
  }
  if (s != OK) throw Failure{s, at(lambda, r) + msg};
  return n;
}

// A solved particle at radius r (with the derivatives along m if asked: spheres only), or a
// Failure with the node's context.
void solve(double r, double lambda, const Optics& op, bool allow, MieState& st,
           int64_t* n_terms, bool derivs = false) {
  std::vector<double> xs;
  const int64_t n = node_terms(r, lambda, op, allow, xs);
  if (op.fr.empty()) {
    st.solve(size_param(r, lambda), op.m, n, derivs);
  } else {
    layered_solve(xs, op.ml, n, st);
    st.x = xs.back();
  }
  *n_terms = n;
}

// engine.rs:358-373: per part, the Kronrod sums of each refined quantity and then of each
// theta-weighted one (a block of n_refined per requested parameter), |Kronrod - Gauss| of the
// same, the Kronrod sums of |du/dtheta| r |q| (the theta blocks' scales) and of u r |q| (the
// scales of the derivatives along m), the largest number of terms, and the integrands per unit
// ln r at the panel's first and last nodes.
struct Sums1 {
  std::vector<double> k, err, abs, absv;
  int64_t n_terms = 0;
  std::vector<double> edge[2];
};

// The pass-1 quantities (engine.rs:50-55, 464-471): 1, C_ext, C_sca, C_sca g, C_back, C_abs,
// then M_GROUP derivatives per requested direction along m.
constexpr int M_GROUP = 5;
int n_refined(const Part& p) {
  return N_BASE + M_GROUP * ((p.dir_col[0] >= 0) + (p.dir_col[1] >= 0));
}

// quantities1 + panel1 (engine.rs:369-560) for every part of a group: each node's quantities
// (the derivatives of C_ext, C_sca, C_sca g, C_back and C_abs along each direction that the
// group's first part asks for), weighted by each part's u r and du/dtheta r.
std::vector<Sums1> panel1(const std::vector<const Part*>& group, double a, double b,
                          double lambda, const Optics& m, const Options& o) {
  Node nd[15];
  gk_panel(a, b, nd);
  const Part& first = *group.front();
  const int nr = n_refined(first);
  const bool derivs = first.dir_derivatives();
  std::vector<std::vector<double>> q(15, std::vector<double>(nr, 0.0));
  int64_t n_max = 0;
  MieState st;
  for (int i = 0; i < 15; ++i) {
    const double r = std::exp(nd[i].t);
    const double area = PI * r * r;
    if (m.eps > 0.0) {
      const SpheroidNode& v = sph_node(r, lambda, m);
      n_max = std::max<int64_t>(n_max, v.n);
      const double w[N_BASE] = {1.0,           area * v.q_ext,  area * v.q_sca,
                                area * v.q_sca * v.g, area * v.q_back, area * v.q_abs};
      for (int j = 0; j < N_BASE; ++j) q[i][j] = w[j];
      continue;
    }
    int64_t n;
    solve(r, lambda, m, o.allow_unvalidated, st, &n, derivs);
    n_max = std::max(n_max, n);
    const Efficiencies e = efficiencies(st);
    const double v[N_BASE] = {1.0,           area * e.q_ext,  area * e.q_sca,
                              area * e.q_sca * e.g, area * e.q_back, area * e.q_abs};
    for (int j = 0; j < N_BASE; ++j) q[i][j] = v[j];
    int at = N_BASE;
    for (int dir = 0; dir < 2; ++dir) {
      if (first.dir_col[dir] < 0) continue;
      const Efficiencies d = efficiency_dir(st, dir, e);
      const double dq[M_GROUP] = {area * d.q_ext, area * d.q_sca,
                                  area * (d.q_sca * e.g + e.q_sca * d.g), area * d.q_back,
                                  area * d.q_abs};
      for (int j = 0; j < M_GROUP; ++j) q[i][at + j] = dq[j];
      at += M_GROUP;
    }
  }
  std::vector<Sums1> out;
  double grad[3];
  for (const Part* p : group) {
    const int nt = (int)p->theta.size(), nb = (1 + nt) * nr;
    Sums1 s;
    s.k.assign(nb, 0.0);
    s.err.assign(nb, 0.0);
    s.abs.assign(nt * nr, 0.0);
    s.absv.assign(nr, 0.0);
    s.edge[0].assign(nb, 0.0);
    s.edge[1].assign(nb, 0.0);
    std::vector<double> g(nb, 0.0);
    for (int i = 0; i < 15; ++i) {
      const double r = std::exp(nd[i].t);
      const double u = density_eval(p->den, r, grad);
      const double base = u * r;
      const int end = i == 0 ? 0 : (i == 14 ? 1 : -1);
      for (int j = 0; j < nr; ++j) {
        const double qj = q[i][j];
        s.k[j] += nd[i].wk * base * qj;
        g[j] += nd[i].wg * base * qj;
        s.absv[j] += nd[i].wk * std::fabs(base * qj);
        if (end >= 0) s.edge[end][j] = base * qj;
        for (int bi = 0; bi < nt; ++bi) {
          const double dw = grad[p->theta[bi].second] * r;
          const int o2 = (1 + bi) * nr + j;
          s.k[o2] += nd[i].wk * dw * qj;
          g[o2] += nd[i].wg * dw * qj;
          s.abs[bi * nr + j] += nd[i].wk * std::fabs(dw * qj);
          if (end >= 0) s.edge[end][o2] = dw * qj;
        }
      }
    }
    for (int j = 0; j < nb; ++j) s.err[j] = std::fabs(s.k[j] - g[j]);
    s.n_terms = n_max;
    out.push_back(std::move(s));
  }
  return out;
}

struct Status {
  std::vector<double> target, errors;
  bool met;
  bool small[2];
};

// engine.rs:620-720 (no Greek refinement): the targets, errors and ends of one part.
Status status(const Part& part, const std::vector<const Sums1*>& sums, const Options& o,
              double ext) {
  const int nr = n_refined(part), nt = (int)part.theta.size(), nb = (1 + nt) * nr;
  const int n_greek = N_BASE;
  Status s;
  s.target.assign(nb, 0.0);
  auto total = [&](int j) {
    double t = 0.0;
    for (auto* x : sums) t += x->k[j];
    return t;
  };
  auto err = [&](int j) {
    double t = 0.0;
    for (auto* x : sums) t += x->err[j];
    return t;
  };
  auto abs_of = [&](int k) {
    double t = 0.0;
    for (auto* x : sums) t += x->abs[k];
    return t;
  };
  // C_abs and each direction's derivative of C_abs are refined to rtol of C_ext's.
  auto scale_of = [&](int j) {
    if (j == P1_ABS) return P1_EXT;
    if (j >= n_greek && (j - n_greek) % M_GROUP == M_GROUP - 1) return j + 1 - M_GROUP;
    return j;
  };
  const double c_sca = std::fabs(total(P1_SCA));
  for (int j = 0; j < nr; ++j) {
    double scale;
    if (j == P1_SCAG) {
      scale = c_sca;
    } else if (j == P1_BACK) {
      scale = std::max(std::fabs(total(P1_BACK)), c_sca);
    } else if (j >= n_greek) {
      scale = 0.0;
      for (auto* x : sums) scale += x->absv[scale_of(j)];
    } else {
      scale = std::fabs(total(scale_of(j)));
    }
    s.target[j] = o.rtol * scale;
    for (int b = 0; b < nt; ++b) s.target[(1 + b) * nr + j] = o.rtol * abs_of(b * nr + scale_of(j));
  }
  for (int b = 0; b <= nt; ++b) s.target[b * nr + P1_ONE] = INF;
  for (int b = 1; b <= nt; ++b)
    for (int j = n_greek; j < nr; ++j) s.target[b * nr + j] = INF;
  if (!o.refine_backscatter)
    for (int b = 0; b <= nt; ++b) {
      s.target[b * nr + P1_BACK] = INF;
      for (int j = n_greek + 3; j < nr; j += M_GROUP) s.target[b * nr + j] = INF;
    }
  s.errors.assign(nb, 0.0);
  s.met = true;
  for (int j = 0; j < nb; ++j) {
    s.errors[j] = err(j);
    s.met = s.met && s.errors[j] <= s.target[j];
  }
  std::vector<double> end_target(nb);
  for (int o2 = 0; o2 < nb; ++o2) {
    if (o2 < nr || std::isinf(s.target[o2])) {
      end_target[o2] = s.target[o2];
    } else {
      const int b = o2 / nr - 1, j = o2 % nr;
      end_target[o2] = o.rtol * std::max(std::fabs(total(o2)), 1e-3 * abs_of(b * nr + scale_of(j)));
    }
  }
  auto small = [&](const std::vector<double>& density) {
    for (int j = 0; j < nb; ++j)
      if (!(std::fabs(density[j]) * (ext / STEP) <= 0.1 * end_target[j])) return false;
    return true;
  };
  s.small[0] = small(sums.front()->edge[0]);
  s.small[1] = small(sums.back()->edge[1]);
  return s;
}

struct Pass1 {
  std::vector<std::pair<double, double>> panels;
  std::vector<bool> converged;
  int64_t n_terms = 0;
};

// engine.rs:724-924.
Pass1 pass1(const std::vector<const Part*>& group, double lambda, const Optics& m,
            const Options& o) {
  std::vector<double> breaks;
  for (auto* p : group) {
    if (p->support == FINITE) {
      breaks.push_back(p->s_a);
      breaks.push_back(p->s_b);
    }
    // engine.rs:740-752: a table's radii are panel edges too.
    if (p->dist.kind == TABULATED)
      breaks.insert(breaks.end(), p->dist.table, p->dist.table + p->dist.table_len);
  }
  std::sort(breaks.begin(), breaks.end());
  breaks.erase(std::unique(breaks.begin(), breaks.end()), breaks.end());
  double lo = INF, hi = 0.0;
  for (auto* p : group) {
    lo = std::min(lo, p->cut.first);
    hi = std::max(hi, p->cut.second);
  }
  double t_lo = std::log(lo), t_hi = std::log(hi);
  const double x_hi = size_param(hi, lambda);
  if (x_hi > MAX_SIZE_PARAMETER) {
    char buf[200];
    snprintf(buf, sizeof buf,
             "the integration range reaches size parameter %e, above the accepted %e", x_hi,
             MAX_SIZE_PARAMETER);
    throw Failure{INVALID_INPUT, at(lambda, hi) + buf};
  }
  const size_t np = group.size();
  std::vector<bool> extendable(np);
  std::vector<std::array<double, 3>> steps(np);
  std::vector<double> exts(np);
  for (size_t p = 0; p < np; ++p) {
    extendable[p] = group[p]->support == UNBOUNDED;
    steps[p] = {std::log(group[p]->cut.first), std::log(group[p]->cut.second),
                max_step(group[p]->den, STEP)};
    exts[p] = std::min(STEP, group[p]->den.log_width);
  }
  auto step_of = [&](double t) {
    double s = STEP;
    for (auto& st : steps)
      if (st[0] <= t && t < st[1]) s = std::min(s, st[2]);
    return s;
  };
  struct Panel {
    std::pair<double, double> ab;
    bool done = false;
    std::vector<Sums1> sums;
  };
  std::vector<Panel> panels;
  for (auto& ab : initial_panels(t_lo, t_hi, lambda, breaks, step_of, o.max_panels))
    panels.push_back({ab, false, {}});
  int extensions[2] = {0, 0};
  for (;;) {
    // Every panel, then the first error in order.
    const int64_t n_pan = (int64_t)panels.size();
    std::vector<Failure> fails(n_pan, Failure{OK, ""});
    for (int64_t i = 0; i < n_pan; ++i) {
      if (panels[i].done) continue;
      try {
        panels[i].sums = panel1(group, panels[i].ab.first, panels[i].ab.second, lambda, m, o);
        panels[i].done = true;
      } catch (const Failure& f) {
        fails[i] = f;
      }
    }
    for (auto& f : fails)
      if (f.status != OK) throw f;
    const size_t n = panels.size();
    std::vector<Status> statuses;
    for (size_t p = 0; p < np; ++p) {
      std::vector<const Sums1*> sums;
      for (auto& pn : panels) sums.push_back(&pn.sums[p]);
      statuses.push_back(status(*group[p], sums, o, exts[p]));
    }
    auto finish = [&]() {
      Pass1 r;
      for (auto& pn : panels) {
        r.panels.push_back(pn.ab);
        r.n_terms = std::max(r.n_terms, pn.sums.front().n_terms);
      }
      for (size_t p = 0; p < np; ++p)
        r.converged.push_back(statuses[p].met &&
                              (!extendable[p] || (statuses[p].small[0] && statuses[p].small[1])));
      return r;
    };
    bool all_met = true;
    for (auto& s : statuses) all_met = all_met && s.met;
    if (all_met) {
      auto wanting = [&](int end, double* ext, double* step) {
        if (extensions[end] >= MAX_EXTENSIONS) return false;
        bool any = false;
        for (size_t p = 0; p < np; ++p)
          if (extendable[p] && !statuses[p].small[end]) {
            if (!any) {
              *ext = exts[p];
              *step = steps[p][2];
            } else {
              *ext = std::min(*ext, exts[p]);
              *step = std::min(*step, steps[p][2]);
            }
            any = true;
          }
        return any;
      };
      double e0 = 0, s0 = 0, e1 = 0, s1 = 0;
      const bool w0 = wanting(0, &e0, &s0), w1 = wanting(1, &e1, &s1);
      bool extended = false;
      if (w0) {
        auto fresh = initial_panels(t_lo - e0, t_lo, lambda, {}, [&](double) { return s0; },
                                    o.max_panels);
        if (panels.size() + fresh.size() > o.max_panels) return finish();
        t_lo -= e0;
        extensions[0] += 1;
        std::vector<Panel> nw;
        for (auto& ab : fresh) nw.push_back({ab, false, {}});
        for (auto& pn : panels) nw.push_back(std::move(pn));
        panels.swap(nw);
        extended = true;
      }
      if (w1) {
        auto fresh = initial_panels(t_hi, t_hi + e1, lambda, {}, [&](double) { return s1; },
                                    o.max_panels);
        if (panels.size() + fresh.size() > o.max_panels) return finish();
        t_hi += e1;
        extensions[1] += 1;
        for (auto& ab : fresh) panels.push_back({ab, false, {}});
        extended = true;
      }
      if (!extended) return finish();
      continue;
    }
    std::vector<std::pair<double, size_t>> cand;
    for (size_t i = 0; i < n; ++i) {
      if (!(panels[i].ab.second - panels[i].ab.first > MIN_WIDTH)) continue;
      double bad = 0.0;
      for (size_t p = 0; p < np; ++p)
        for (size_t j = 0; j < statuses[p].target.size(); ++j) {
          if (!(statuses[p].errors[j] > statuses[p].target[j])) continue;
          const double t = std::max(statuses[p].target[j], std::numeric_limits<double>::min());
          bad = std::max(bad, panels[i].sums[p].err[j] * (double)n / t);
        }
      if (bad > 1.0) cand.push_back({bad, i});
    }
    const size_t budget = o.max_panels > n ? o.max_panels - n : 0;
    if (cand.empty() || budget == 0) return finish();
    std::sort(cand.begin(), cand.end(), [](const auto& x, const auto& y) {
      return x.first != y.first ? x.first > y.first : x.second < y.second;
    });
    if (cand.size() > budget) cand.resize(budget);
    std::vector<char> split(n, 0);
    for (auto& c : cand) split[c.second] = 1;
    std::vector<Panel> next;
    for (size_t i = 0; i < n; ++i) {
      if (split[i]) {
        const double a = panels[i].ab.first, b = panels[i].ab.second, mid = 0.5 * (a + b);
        next.push_back({{a, mid}, false, {}});
        next.push_back({{mid, b}, false, {}});
      } else {
        next.push_back(std::move(panels[i]));
      }
    }
    panels.swap(next);
  }
}

// panel_terms (engine.rs:961-978).
int64_t panel_terms(double a, double b, double lambda, const Optics& m, bool allow) {
  Node nd[15];
  gk_panel(a, b, nd);
  int64_t most = 0;
  std::vector<double> xs;
  for (auto& n : nd) most = std::max(most, node_terms(std::exp(n.t), lambda, m, allow, xs));
  return most;
}

struct Layout {
  int64_t n_mu = 0;
  std::vector<BandData> bands;
  std::vector<int64_t> start;
  int64_t len = 0;
  int band_of(int64_t n) const {
    const int64_t u = bucket(n);
    for (size_t b = 0; b < bands.size(); ++b)
      if (bands[b].upper == u) return (int)b;
    return -1;
  }
};

// quantities2 (engine.rs:1025-1202): the scalars, the requested cosines' tables (times the
// area) and the band's tables (fast.rs:95-205) of one solved sphere into g; with dm (a sphere
// solved with derivatives), their derivatives along Re m and Im m into dm[0..len) and
// dm[len..2 len) (the amplitudes' derivatives dS/dm and i dS/dm; phase.rs:289-341).
// With dr, the derivatives with respect to r at fixed m go there (engine.rs:1158-1170):
// 2 pi r Q + pi r^2 (2 pi / lambda) dQ/dx for the scalars, 2 r and 3 r^2 for r^2 and r^3, and
// 2 pi r F + pi r^2 (2 pi / lambda) dF/dx for the unnormalized phase tables F.
void quantities2(const MieState& st, int64_t n, double r, double lambda, const Layout& L,
                 const double* mu, int band, int64_t band_terms, double* g,
                 double* dm = nullptr, double* dr = nullptr) {
  const double x = size_param(r, lambda);
  const Efficiencies q = efficiencies(st);
  const double area = PI * r * r;
  const int64_t len = L.len;
  const double sc[SCALARS] = {1.0,           area * q.q_ext, area * q.q_sca, area * q.q_sca * q.g,
                              area * q.q_abs, area * q.q_back, r * r,         r * r * r,
                              0.0};
  for (int k = 0; k < SCALARS; ++k) g[k] = sc[k];
  const double kw = 2.0 * PI / lambda;
  if (dr) {
    const Efficiencies e = efficiency_x(st, q);
    const double values[6] = {0.0, q.q_ext, q.q_sca, q.q_sca * q.g, q.q_abs, q.q_back};
    const double dx[6] = {0.0, area * e.q_ext, area * e.q_sca,
                          area * (e.q_sca * q.g + q.q_sca * e.g), area * e.q_abs, area * e.q_back};
    for (int j = 1; j < 6; ++j) dr[j] = 2.0 * PI * r * values[j] + kw * dx[j];
    dr[S_ONE] = 0.0;
    dr[S_R2] = 2.0 * r;
    dr[S_R3] = 3.0 * r * r;
    dr[SCALARS - 1] = 0.0;
  }
  if (dm) {
    for (int dir = 0; dir < 2; ++dir) {
      const Efficiencies e = efficiency_dir(st, dir, q);
      const double sd[SCALARS] = {0.0,
                                  area * e.q_ext,
                                  area * e.q_sca,
                                  area * (e.q_sca * q.g + q.q_sca * e.g),
                                  area * e.q_abs,
                                  area * e.q_back,
                                  0.0,
                                  0.0,
                                  0.0};
      for (int k = 0; k < SCALARS; ++k) dm[dir * len + k] = sd[k];
    }
  }
  const double cph = 4.0 / (x * x);
  // d(cph F)/dx of the unnormalized tables, cph = 4/x^2.
  auto table_dr = [&](cplx s1, cplx s2, cplx x1, cplx x2, double c, double* out, int64_t stride) {
    double e[4], de[4];
    elements(s1, s2, e);
    element_derivs(s1, s2, x1, x2, de);
    for (int t = 0; t < 4; ++t)
      out[t * stride] = 2.0 * PI * r * (c * e[t]) + area * kw * (c * de[t] - 2.0 / x * (c * e[t]));
  };
  for (int64_t j = 0; j < L.n_mu; ++j) {
    cplx s1 = real(0.0), s2 = real(0.0), d1 = real(0.0), d2 = real(0.0);
    cplx x1 = real(0.0), x2 = real(0.0);
    for_each_order(mu[j], n, [&](int64_t k, double pi, double tau) {
      s1 = s1 + scale(st.a[k - 1], pi) + scale(st.b[k - 1], tau);
      s2 = s2 + scale(st.a[k - 1], tau) + scale(st.b[k - 1], pi);
      if (dm) {
        d1 = d1 + scale(st.da_dm[k - 1], pi) + scale(st.db_dm[k - 1], tau);
        d2 = d2 + scale(st.da_dm[k - 1], tau) + scale(st.db_dm[k - 1], pi);
      }
      if (dr) {
        x1 = x1 + scale(st.da_dx[k - 1], pi) + scale(st.db_dx[k - 1], tau);
        x2 = x2 + scale(st.da_dx[k - 1], tau) + scale(st.db_dx[k - 1], pi);
      }
    });
    if (dr) table_dr(s1, s2, x1, x2, cph, dr + SCALARS + j, L.n_mu);
    double e[4];
    elements(s1, s2, e);
    for (int t = 0; t < 4; ++t) g[SCALARS + t * L.n_mu + j] = cph * e[t] * area;
    if (dm) {
      double fr[4], fi[4];
      element_derivs(s1, s2, d1, d2, fr);
      element_derivs(s1, s2, times_i(d1), times_i(d2), fi);
      for (int t = 0; t < 4; ++t) {
        dm[SCALARS + t * L.n_mu + j] = area * (cph * fr[t]);
        dm[len + SCALARS + t * L.n_mu + j] = area * (cph * fi[t]);
      }
    }
  }
  if (band < 0) return;
  const BandData& B = L.bands[band];
  double* out = g + L.start[band];
  const int64_t qn = B.n_q, lo = qn / 2, h = qn - lo;
  const int64_t terms = std::min(band_terms, B.upper);
  const double scl = 4.0 / (x * x) * (PI * r * r);
  for (int64_t ii = 0; ii < h; ++ii) {
    // ce = G_E X and co = G_O X over the sphere's 4 columns and, with derivatives, its 4
    // derivative columns (fast.rs:98-145).
    double ce[8] = {0, 0, 0, 0, 0, 0, 0, 0}, co[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    double cx[4] = {0, 0, 0, 0}, cy[4] = {0, 0, 0, 0};  // the x derivative columns
    for (int64_t k = 0; k < terms; ++k) {
      double xr[8] = {0, 0, 0, 0, 0, 0, 0, 0}, xx[4] = {0, 0, 0, 0};
      if (k < n) {
        const cplx uu = (k % 2 == 0) ? st.a[k] : st.b[k];
        const cplx vv = (k % 2 == 0) ? st.b[k] : st.a[k];
        xr[0] = uu.re;
        xr[1] = uu.im;
        xr[2] = vv.re;
        xr[3] = vv.im;
        if (dm) {
          const cplx du = (k % 2 == 0) ? st.da_dm[k] : st.db_dm[k];
          const cplx dv = (k % 2 == 0) ? st.db_dm[k] : st.da_dm[k];
          xr[4] = du.re;
          xr[5] = du.im;
          xr[6] = dv.re;
          xr[7] = dv.im;
        }
        if (dr) {
          const cplx du = (k % 2 == 0) ? st.da_dx[k] : st.db_dx[k];
          const cplx dv = (k % 2 == 0) ? st.db_dx[k] : st.da_dx[k];
          xx[0] = du.re;
          xx[1] = du.im;
          xx[2] = dv.re;
          xx[3] = dv.im;
        }
      }
      const double ge = B.ge[ii * B.upper + k], go = B.go[ii * B.upper + k];
      for (int t = 0; t < 8; ++t) {
        ce[t] += ge * xr[t];
        co[t] += go * xr[t];
      }
      for (int t = 0; t < 4; ++t) {
        cx[t] += ge * xx[t];
        cy[t] += go * xx[t];
      }
    }
    const cplx eu = C(ce[0], ce[1]), ev = C(ce[2], ce[3]);
    const cplx ou = C(co[0], co[1]), ov = C(co[2], co[3]);
    const cplx deu = C(ce[4], ce[5]), dev = C(ce[6], ce[7]);
    const cplx dou = C(co[4], co[5]), dov = C(co[6], co[7]);
    const int64_t jn = lo + ii;
    const cplx xeu = C(cx[0], cx[1]), xev = C(cx[2], cx[3]);
    const cplx xou = C(cy[0], cy[1]), xov = C(cy[2], cy[3]);
    auto write = [&](int64_t node, double sign) {
      const cplx s1 = eu + scale(ov, sign), s2 = ev + scale(ou, sign);
      double e[4];
      elements(s1, s2, e);
      for (int t = 0; t < 4; ++t) out[t * qn + node] = scl * e[t];
      if (dr)
        table_dr(s1, s2, xeu + scale(xov, sign), xev + scale(xou, sign), 4.0 / (x * x),
                 dr + L.start[band] + node, qn);
      if (dm) {
        const cplx d1 = deu + scale(dov, sign), d2 = dev + scale(dou, sign);
        double fr[4], fi[4];
        element_derivs(s1, s2, d1, d2, fr);
        element_derivs(s1, s2, times_i(d1), times_i(d2), fi);
        for (int t = 0; t < 4; ++t) {
          dm[L.start[band] + t * qn + node] = scl * fr[t];
          dm[len + L.start[band] + t * qn + node] = scl * fi[t];
        }
      }
    };
    write(jn, 1.0);
    const int64_t mirror = qn - 1 - jn;
    if (mirror != jn) write(mirror, -1.0);
  }
}

struct Lin {
  double v, e;
};
Lin ldiv(Lin a, Lin b) {
  const double v = a.v / b.v;
  return {v, (a.e + std::fabs(v) * b.e) / std::fabs(b.v)};
}
Lin lscale(Lin a, double c) { return {c * a.v, std::fabs(c) * a.e}; }

struct UnitOut {
  double values[11], errors[11];
  std::vector<double> phase, phase_err;  // 6 x n_mu
  std::vector<double> greek, greek_err;  // 6 x (L + 1)
  // The derivatives and their error estimates, a block per requested parameter:
  // [P][11], [P][6 n_mu], [P][6 (L + 1)].
  std::vector<double> d_values, d_errors, d_phase, d_phase_err, d_greek, d_greek_err;
  bool converged = true;
  int64_t panels = 0;
};

// A requested parameter (EnsembleParam, ensemble/mod.rs:180-215): its component, its mode (-1:
// none), its kind and, for a distribution parameter, its index into the distribution's
// gradient.
enum ParamKindId { PK_DIST = 0, PK_REFR_REAL = 1, PK_REFR_IMAG = 2, PK_WEIGHT = 3 };
struct Param {
  int32_t component, mode, kind, index;
};

// Lin (lin.rs:7-68): a value, its error estimate, its derivatives and their error estimates.
struct LinD {
  double v = 0.0, e = 0.0;
  std::vector<double> d, de;
  static LinD constant(double v, size_t n) {
    LinD x;
    x.v = v;
    x.d.assign(n, 0.0);
    x.de.assign(n, 0.0);
    return x;
  }
  LinD div(const LinD& b) const {
    LinD o;
    o.v = v / b.v;
    o.e = (e + std::fabs(o.v) * b.e) / std::fabs(b.v);
    const size_t n = d.size();
    o.d.resize(n);
    o.de.resize(n);
    for (size_t k = 0; k < n; ++k) o.d[k] = (d[k] - o.v * b.d[k]) / b.v;
    for (size_t k = 0; k < n; ++k)
      o.de[k] = (de[k] + std::fabs(o.v) * b.de[k] + std::fabs(o.d[k]) * b.e +
                 o.e * std::fabs(b.d[k])) /
                std::fabs(b.v);
    return o;
  }
  LinD scale(double c) const {
    LinD o = *this;
    o.v = c * v;
    o.e = std::fabs(c) * e;
    for (size_t k = 0; k < d.size(); ++k) {
      o.d[k] = c * d[k];
      o.de[k] = std::fabs(c) * de[k];
    }
    return o;
  }
};

// direct_node (engine.rs:1281-1339) of a solved spheroid node at radius r: the scalars (ONE ...
// DEPOL) into g[0..9) with their declared errors into ge, and its Greek coefficients times the
// area into the direct segment g[dstart + f glen + l] (zero beyond its 2N), each with the
// declared error relative to its largest alpha1; tau the node's T-matrix tolerance.
void fill_direct(const SpheroidNode& v, double r, double tau, double* g, double* ge,
                 int64_t dstart, int64_t glen) {
  const double area = PI * r * r;
  const double c4 = 4.0 * tau, c16 = 16.0 * tau;
  const double sv[9] = {1.0,           area * v.q_ext, area * v.q_sca, area * v.q_sca * v.g,
                        area * v.q_abs, area * v.q_back, r * r,         r * r * r,
                        area * v.depol};
  const double back = area * std::max(std::fabs(v.q_back), std::fabs(v.q_sca));
  const double se[9] = {0.0, c4 * std::fabs(sv[1]), c4 * std::fabs(sv[2]),
                        c4 * std::fabs(sv[2]) * (1.0 + std::fabs(v.g)), c16 * std::fabs(sv[1]),
                        c16 * back, 0.0, 0.0, 2.0 * c16 * back};
  for (int k = 0; k < 9; ++k) {
    g[k] = sv[k];
    ge[k] = se[k];
  }
  if (glen > 0) {
    const int64_t have = 2 * (int64_t)v.n + 1;
    double big = 0.0;
    for (int64_t l = 0; l < have; ++l) big = std::max(big, std::fabs(v.greek[l]));
    for (int f = 0; f < 6; ++f)
      for (int64_t l = 0; l < glen; ++l) {
        g[dstart + f * glen + l] = l < have ? area * v.greek[f * have + l] : 0.0;
        ge[dstart + f * glen + l] = c16 * area * big;
      }
  }
}

// The direct path's pass 2, averages and outputs for spheroids (engine.rs:1207-1339 direct_node,
// 1558-1740 the sums with the declared node errors, 1782-1836 averages, 1896-1961 a single
// radius, 2121-2176 mixing, 2359-2497 assembly: the depolarization ratio, the Greek
// coefficients from the direct segment and the phase matrix from their expansion).
std::vector<UnitOut> direct_outputs(const std::vector<Part>& parts,
                                    const std::vector<std::vector<int>>& groups,
                                    const std::vector<std::vector<int>>& units,
                                    const std::vector<Pass1>& firsts,
                                    const std::vector<int>& group_of, const std::vector<int>& place,
                                    double lambda, const Optics& op, const double* mu,
                                    int64_t n_mu, int64_t order, bool normalized,
                                    const Options& o) {
  const bool keep = order >= 0 || n_mu > 0;
  // N_max over the call's groups, each its final panels' (engine.rs:1987-2030, p1.n_terms).
  int64_t n_direct = 0;
  for (const Pass1& p1 : firsts) n_direct = std::max<int64_t>(n_direct, p1.n_terms);
  const int64_t ld = !keep ? -1 : n_mu == 0 ? std::min<int64_t>(order, 2 * n_direct) : 2 * n_direct;
  const int64_t glen = ld + 1, NS = 9, len = NS + 6 * glen;
  auto node = [&](double r, std::vector<double>& g, std::vector<double>& ge) {
    // max(rtol, estimate) as the declared tolerance: the estimate is below rtol.
    g.assign(len, 0.0);
    ge.assign(len, 0.0);
    fill_direct(sph_node(r, lambda, op), r, op.rtol_t, g.data(), ge.data(), NS, glen);
  };
  std::vector<std::vector<double>> av(parts.size()), ae(parts.size());
  std::vector<double> g, ge;
  for (size_t gi = 0; gi < groups.size(); ++gi) {
    const auto& grp = groups[gi];
    if (parts[grp[0]].support == POINT) {
      node(parts[grp[0]].s_a, g, ge);
      av[grp[0]] = g;
      ae[grp[0]] = ge;
      continue;
    }
    for (size_t p = 0; p < grp.size(); ++p) {
      const Part& part = parts[grp[p]];
      std::vector<double> S(len, 0.0), E(len, 0.0);
      for (auto& ab : firsts[gi].panels) {
        Node nd[15];
        gk_panel(ab.first, ab.second, nd);
        for (int64_t j = 0; j < len; ++j) {
          double K = 0.0, G = 0.0, NE = 0.0;
          for (int i = 0; i < 15; ++i) {
            const double r = std::exp(nd[i].t);
            const double ur = density_eval(part.den, r, nullptr) * r;
            node(r, g, ge);
            K += nd[i].wk * ur * g[j];
            G += nd[i].wg * ur * g[j];
            NE += std::fabs(nd[i].wk * ur) * ge[j];
          }
          S[j] += K;
          E[j] += std::fabs(K - G) + NE;
        }
      }
      const double trunc = part.support == UNBOUNDED ? 0.2 * o.rtol : 0.0;
      const double z = part.mom.z, ez = part.mom.ez;
      std::vector<double> v(len), er(len);
      for (int64_t j = 0; j < len; ++j) {
        v[j] = S[j] / z;
        er[j] = (E[j] + std::fabs(v[j]) * ez) / z + trunc * std::fabs(v[j]);
      }
      for (int k = 0; k < 2; ++k) {
        v[6 + k] = part.mom.v[k];
        er[6 + k] = part.mom.e[k];
      }
      av[grp[p]] = std::move(v);
      ae[grp[p]] = std::move(er);
    }
  }
  std::vector<UnitOut> out;
  std::vector<double> d00, d22, d2m2, d02;
  for (auto& un : units) {
    std::vector<double> v(len, 0.0), e(len, 0.0);
    for (int p : un)
      for (int64_t j = 0; j < len; ++j) {
        v[j] += parts[p].f * av[p][j];
        e[j] += parts[p].f * ae[p][j];
      }
    UnitOut u;
    auto lin = [&](int64_t j) { return Lin{v[j], e[j]}; };
    Lin ext = lin(1), sca = lin(2), scag = lin(3), ab = lin(4), back = lin(5), r2 = lin(6),
        r3 = lin(7), num = lin(8);
    for (Lin* l : {&ext, &sca, &back})
      if (!(std::isfinite(l->v) && l->v != 0.0))
        throw Failure{INVALID_INPUT,
                      "a ratio's denominator (<C_ext>, <C_sca> or <C_back>) is 0 or not finite"};
    const Lin den{2.0 * back.v - num.v, 2.0 * back.e + num.e};
    const Lin sc[11] = {ext, sca, ab, back, ldiv(sca, ext), ldiv(scag, sca),
                        lscale(ldiv(ext, back), 4.0 * PI), ldiv(num, den), ldiv(r3, r2),
                        lscale(r2, PI), lscale(r3, 4.0 * PI / 3.0)};
    for (int k = 0; k < 11; ++k) {
      u.values[k] = sc[k].v;
      u.errors[k] = sc[k].e;
    }
    auto G = [&](int f, int64_t l) { return lin(NS + f * glen + l); };
    if (order >= 0) {
      u.greek.assign(6 * (order + 1), 0.0);
      u.greek_err.assign(6 * (order + 1), 0.0);
      const Lin a0 = G(0, 0);
      for (int f = 0; f < 6; ++f)
        for (int64_t l = 0; l <= order && l < glen; ++l) {
          Lin x = G(f, l);
          if (normalized) x = (f == 0 && l == 0) ? Lin{1.0, 0.0} : ldiv(x, a0);
          u.greek[f * (order + 1) + l] = x.v;
          u.greek_err[f * (order + 1) + l] = x.e;
        }
      if (normalized) u.greek[0] = 1.0;
    }
    if (n_mu > 0) {
      u.phase.assign(6 * n_mu, 0.0);
      u.phase_err.assign(6 * n_mu, 0.0);
      d00.resize(glen);
      d22.resize(glen);
      d2m2.resize(glen);
      d02.resize(glen);
      for (int64_t j = 0; j < n_mu; ++j) {
        wigner_d(0, 0, mu[j], d00.data(), glen);
        wigner_d(2, 2, mu[j], d22.data(), glen);
        wigner_d(2, -2, mu[j], d2m2.data(), glen);
        wigner_d(0, 2, mu[j], d02.data(), glen);
        Lin f[6] = {};
        auto acc = [](Lin& t, double w, const Lin& x) {
          t.v += w * x.v;
          t.e += std::fabs(w) * x.e;
        };
        for (int64_t l = 0; l < glen; ++l) {
          const double pl = 0.5 * (d22[l] + d2m2[l]), mn = 0.5 * (d22[l] - d2m2[l]);
          acc(f[0], d00[l], G(0, l));
          acc(f[1], d02[l], G(4, l));
          acc(f[2], pl, G(1, l));
          acc(f[2], mn, G(2, l));
          acc(f[3], mn, G(1, l));
          acc(f[3], pl, G(2, l));
          acc(f[4], d02[l], G(5, l));
          acc(f[5], d00[l], G(3, l));
        }
        for (int k = 0; k < 6; ++k) {
          const Lin x = normalized ? ldiv(f[k], sca) : f[k];
          u.phase[k * n_mu + j] = x.v;
          u.phase_err[k * n_mu + j] = x.e;
        }
      }
    }
    std::set<int> ug;
    for (int p : un) {
      if (parts[p].support == POINT) continue;
      u.converged = u.converged && firsts[group_of[p]].converged[place[p]];
      ug.insert(group_of[p]);
    }
    for (int gi : ug) u.panels += (int64_t)firsts[gi].panels.size();
    out.push_back(std::move(u));
  }
  return out;
}

// One wavelength (engine.rs:1964-2250): pass 1 per group, bands, pass 2, averages, a unit per
// entry of `units` (each a list of parts with weight 1), the projection and the assembly.
std::vector<UnitOut> wavelength(const std::vector<Part>& parts,
                                const std::vector<std::vector<int>>& groups,
                                const std::vector<std::vector<int>>& units, double lambda,
                                int64_t wi, const double* mu, int64_t n_mu, int64_t order,
                                bool normalized, const Options& o,
                                const std::vector<Param>& params = {}) {
  const int64_t n_wl_all = parts.empty() ? 0 : parts[0].n_wl;
  // Solved spheroid nodes per particle (aspect ratio, indices): a batch's parts share one.
  std::map<std::pair<double, const double*>, std::map<double, SpheroidNode>> caches;
  auto m_of = [&](int p) {
    Optics op;
    const Part& q = parts[p];
    if (q.eps > 0.0) {
      op.m = C(q.m[2 * wi], q.m[2 * wi + 1]);
      op.eps = q.eps;
      op.rtol_t = std::min(std::max(o.rtol / 100.0, 1e-12), 1e-8);  // engine.rs:87
      op.cache = &caches[{q.eps, q.m}];
      return op;
    }
    if (q.n_layers <= 1) {
      op.m = C(q.m[2 * wi], q.m[2 * wi + 1]);
    } else {
      op.fr.assign(q.fractions, q.fractions + q.n_layers - 1);
      for (int l = 0; l < q.n_layers; ++l)
        op.ml.push_back(C(q.m_layers[2 * (l * n_wl_all + wi)], q.m_layers[2 * (l * n_wl_all + wi) + 1]));
    }
    return op;
  };
  std::vector<Pass1> firsts;
  int64_t n_max = 0;
  for (auto& g : groups) {
    std::vector<const Part*> mem;
    for (int p : g) mem.push_back(&parts[p]);
    const Optics m = m_of(g[0]);  // a group shares its particle
    Pass1 p1;
    if (mem[0]->support == POINT) {
      std::vector<double> xs;
      p1.converged = {true};
      p1.n_terms = node_terms(mem[0]->s_a, lambda, m, o.allow_unvalidated, xs);
    } else {
      p1 = pass1(mem, lambda, m, o);
    }
    n_max = std::max(n_max, p1.n_terms);
    firsts.push_back(std::move(p1));
  }
  if (order == GREEK_ALL) order = 2 * n_max;  // GreekOrder::All (engine.rs:2016-2020)
  std::vector<int> group_of(parts.size()), place(parts.size());
  for (size_t gi = 0; gi < groups.size(); ++gi)
    for (size_t k = 0; k < groups[gi].size(); ++k) {
      group_of[groups[gi][k]] = (int)gi;
      place[groups[gi][k]] = (int)k;
    }
  // The groups on the direct path (spheroids, engine.rs:1975-2000).
  std::vector<char> direct(groups.size(), 0);
  bool all_direct = !groups.empty();
  int64_t n_direct = 0;
  for (size_t gi = 0; gi < groups.size(); ++gi) {
    direct[gi] = parts[groups[gi][0]].eps > 0.0;
    all_direct = all_direct && direct[gi];
    if (direct[gi]) n_direct = std::max(n_direct, firsts[gi].n_terms);
  }
  if (all_direct) {
    // Spheroids alone: pass 2 and the outputs on the direct path, from the solved nodes.
    const Optics op = m_of(groups[0][0]);
    return direct_outputs(parts, groups, units, firsts, group_of, place, lambda, op, mu, n_mu,
                          order, normalized, o);
  }
  Layout L;
  L.n_mu = n_mu;
  L.len = SCALARS + 4 * n_mu;
  if (order >= 0) {
    std::set<int64_t> uppers;
    for (size_t gi = 0; gi < groups.size(); ++gi) {
      if (direct[gi]) continue;
      const Optics m = m_of(groups[gi][0]);
      if (parts[groups[gi][0]].support == POINT) {
        uppers.insert(bucket(firsts[gi].n_terms));
        continue;
      }
      for (auto& ab : firsts[gi].panels)
        uppers.insert(bucket(panel_terms(ab.first, ab.second, lambda, m, o.allow_unvalidated)));
    }
    for (int64_t u : uppers) {
      L.bands.push_back(make_band(u, order));
      L.start.push_back(L.len);
      L.len += 4 * L.bands.back().n_q;
    }
  }
  // The spheroids' direct segment (engine.rs:2073-2086): every order to 2 N for the phase
  // matrix, else to the requested one.
  const bool keep = order >= 0 || n_mu > 0;
  int64_t ld = -1, d_start = L.len;
  if (n_direct > 0 && keep) {
    ld = n_mu == 0 ? std::min<int64_t>(order, 2 * n_direct) : 2 * n_direct;
    L.len += 6 * (ld + 1);
  }
  const int64_t len = L.len;
  // Pass 2 and the averages of every part (engine.rs:1423-1766, 1782-1836): blocks of sums,
  // the values (weights u r), each requested distribution parameter (du/dtheta r) and, when
  // the part asks for any derivative along m, Re m and Im m (u r on the nodes' derivatives).
  const size_t n_cols = params.size();
  struct Avg {
    std::vector<double> v, e;
    std::vector<std::pair<int, std::vector<double>>> d, de;  // (column, array)
  };
  std::vector<Avg> avg(parts.size());
  std::vector<double> g(len), dmv(2 * len);
  MieState st;
  double grad[3];
  for (size_t gi = 0; gi < groups.size(); ++gi) {
    const auto& grp = groups[gi];
    const Optics m = m_of(grp[0]);
    if (direct[gi]) {
      // A spheroid group (engine.rs:1558-1606 with direct_node, 1896-1961 for one radius): the
      // solved nodes' rows with their declared errors, summed with |w| on the errors.
      std::vector<double> row(len), rowe(len);
      auto node_row = [&](double r) {
        std::fill(row.begin(), row.end(), 0.0);
        std::fill(rowe.begin(), rowe.end(), 0.0);
        fill_direct(sph_node(r, lambda, m), r, m.rtol_t, row.data(), rowe.data(), d_start,
                    ld + 1);
      };
      for (int p : grp) {
        const Part& part = parts[p];
        if (!part.theta.empty() || part.dir_derivatives())
          throw Failure{INVALID_INPUT, "derivatives of spheroids are not on this path"};
        Avg& a = avg[p];
        if (part.support == POINT) {
          node_row(part.s_a);
          a.v = row;
          a.e = rowe;
          continue;
        }
        std::vector<double> S(len, 0.0), E(len, 0.0);
        for (auto& ab : firsts[gi].panels) {
          Node nd[15];
          gk_panel(ab.first, ab.second, nd);
          std::vector<double> K(len, 0.0), G(len, 0.0), NE(len, 0.0);
          for (int i = 0; i < 15; ++i) {
            const double r = std::exp(nd[i].t);
            const double ur = density_eval(part.den, r, nullptr) * r;
            node_row(r);
            for (int64_t j = 0; j < len; ++j) {
              K[j] += nd[i].wk * ur * row[j];
              G[j] += nd[i].wg * ur * row[j];
              NE[j] += std::fabs(nd[i].wk * ur) * rowe[j];
            }
          }
          for (int64_t j = 0; j < len; ++j) {
            S[j] += K[j];
            E[j] += std::fabs(K[j] - G[j]) + NE[j];
          }
        }
        const double trunc = part.support == UNBOUNDED ? 0.2 * o.rtol : 0.0;
        const double z = part.mom.z, ez = part.mom.ez;
        a.v.resize(len);
        a.e.resize(len);
        for (int64_t j = 0; j < len; ++j) {
          a.v[j] = S[j] / z;
          a.e[j] = (E[j] + std::fabs(a.v[j]) * ez) / z + trunc * std::fabs(a.v[j]);
        }
        for (int k = 0; k < 2; ++k) {
          a.v[S_R2 + k] = part.mom.v[k];
          a.e[S_R2 + k] = part.mom.e[k];
        }
      }
      continue;
    }
    bool derivs = false;
    for (int p : grp) derivs = derivs || parts[p].dir_derivatives();
    if (parts[grp[0]].support == POINT) {
      // monodisperse (engine.rs:1838-1890): the particle itself, exact.
      const Part& part = parts[grp[0]];
      const bool radius = !part.theta.empty();  // monodisperse: radius, its one parameter
      if (radius && !m.fr.empty())
        throw Failure{INVALID_INPUT, "the radius derivative of a layered sphere is not here"};
      const double r = part.s_a;
      int64_t n;
      solve(r, lambda, m, o.allow_unvalidated, st, &n, derivs || radius);
      std::fill(g.begin(), g.end(), 0.0);
      std::fill(dmv.begin(), dmv.end(), 0.0);
      std::vector<double> drv(radius ? len : 0, 0.0);
      const int band = order >= 0 ? L.band_of(n) : -1;
      quantities2(st, n, r, lambda, L, mu, band, n, g.data(), derivs ? dmv.data() : nullptr,
                  radius ? drv.data() : nullptr);
      Avg& a = avg[grp[0]];
      a.v = g;
      a.e.assign(len, 0.0);
      if (radius) {
        a.d.push_back({part.theta[0].first, drv});
        a.de.push_back({part.theta[0].first, std::vector<double>(len, 0.0)});
      }
      for (int dir = 0; dir < 2; ++dir)
        if (part.dir_col[dir] >= 0) {
          a.d.push_back({part.dir_col[dir],
                         std::vector<double>(dmv.begin() + dir * len,
                                             dmv.begin() + (dir + 1) * len)});
          a.de.push_back({part.dir_col[dir], std::vector<double>(len, 0.0)});
        }
      continue;
    }
    const size_t np = grp.size();
    // s[p][blk * len + i], e[p][blk * len + i].
    std::vector<int> nblk(np);
    std::vector<std::vector<double>> s(np), e(np);
    for (size_t p = 0; p < np; ++p) {
      const Part& part = parts[grp[p]];
      nblk[p] = 1 + (int)part.theta.size() + (part.dir_derivatives() ? 2 : 0);
      s[p].assign(nblk[p] * len, 0.0);
      e[p].assign(nblk[p] * len, 0.0);
    }
    for (auto& ab : firsts[gi].panels) {
      const int64_t bt = order >= 0 ? panel_terms(ab.first, ab.second, lambda, m,
                                                  o.allow_unvalidated)
                                    : 0;
      const int band = order >= 0 ? L.band_of(bt) : -1;
      Node nd[15];
      gk_panel(ab.first, ab.second, nd);
      std::vector<std::vector<double>> vals(15, std::vector<double>(len, 0.0));
      std::vector<std::vector<double>> dvals(derivs ? 15 : 0, std::vector<double>(2 * len, 0.0));
      for (int i = 0; i < 15; ++i) {
        const double r = std::exp(nd[i].t);
        int64_t n;
        solve(r, lambda, m, o.allow_unvalidated, st, &n, derivs);
        quantities2(st, n, r, lambda, L, mu, band, bt, vals[i].data(),
                    derivs ? dvals[i].data() : nullptr);
      }
      // The ranges the panel touches: the common part and its band's tables.
      const int64_t common = SCALARS + 4 * n_mu;
      const int64_t b_lo = band >= 0 ? L.start[band] : 0;
      const int64_t b_hi = band >= 0 ? b_lo + 4 * L.bands[band].n_q : 0;
      for (size_t p = 0; p < np; ++p) {
        const Part& part = parts[grp[p]];
        const int nt = (int)part.theta.size();
        // Kronrod and Gauss weights of each block's rows at the panel's nodes.
        std::vector<double> wk((1 + nt) * 15), wg((1 + nt) * 15);
        for (int i = 0; i < 15; ++i) {
          const double r = std::exp(nd[i].t);
          const double u = density_eval(part.den, r, grad);
          wk[i] = nd[i].wk * (u * r);
          wg[i] = nd[i].wg * (u * r);
          for (int b = 0; b < nt; ++b) {
            const double dw = grad[part.theta[b].second] * r;
            wk[(1 + b) * 15 + i] = nd[i].wk * dw;
            wg[(1 + b) * 15 + i] = nd[i].wg * dw;
          }
        }
        auto add = [&](int64_t a, int64_t b) {
          for (int blk = 0; blk < nblk[p]; ++blk) {
            const int row = blk <= nt ? blk : 0;  // the m blocks take the values' weights
            const int dir = blk - 1 - nt;
            for (int64_t idx = a; idx < b; ++idx) {
              double K = 0.0, G = 0.0;
              for (int i = 0; i < 15; ++i) {
                const double q = blk <= nt ? vals[i][idx] : dvals[i][dir * len + idx];
                K += wk[row * 15 + i] * q;
                G += wg[row * 15 + i] * q;
              }
              s[p][blk * len + idx] += K;
              e[p][blk * len + idx] += std::fabs(K - G);
            }
          }
        };
        add(0, common);
        add(b_lo, b_hi);
      }
    }
    for (size_t p = 0; p < np; ++p) {
      const Part& part = parts[grp[p]];
      const int nt = (int)part.theta.size();
      const double trunc = part.support == UNBOUNDED ? 0.2 * o.rtol : 0.0;
      const double z = part.mom.z, ez = part.mom.ez;
      Avg& a = avg[grp[p]];
      a.v.resize(len);
      a.e.resize(len);
      for (int64_t i = 0; i < len; ++i) {
        a.v[i] = s[p][i] / z;
        a.e[i] = (e[p][i] + std::fabs(a.v[i]) * ez) / z + trunc * std::fabs(a.v[i]);
      }
      for (int b = 0; b < nt; ++b) {
        const double dz = part.mom.dz[b], edz = part.mom.dez[b];
        std::vector<double> dv(len), de(len);
        for (int64_t i = 0; i < len; ++i) {
          const double sb = s[p][(1 + b) * len + i], eb = e[p][(1 + b) * len + i];
          dv[i] = (sb - a.v[i] * dz) / z;
          de[i] = (eb + std::fabs(a.v[i]) * edz + std::fabs(dv[i]) * ez + a.e[i] * std::fabs(dz)) /
                      z +
                  trunc * std::fabs(dv[i]);
        }
        a.d.push_back({part.theta[b].first, std::move(dv)});
        a.de.push_back({part.theta[b].first, std::move(de)});
      }
      for (int dir = 0; dir < 2; ++dir) {
        if (part.dir_col[dir] < 0) continue;
        const int blk = 1 + nt + dir;
        std::vector<double> dv(len), de(len);
        for (int64_t i = 0; i < len; ++i) {
          dv[i] = s[p][blk * len + i] / z;
          de[i] = (e[p][blk * len + i] + std::fabs(dv[i]) * ez) / z + trunc * std::fabs(dv[i]);
        }
        a.d.push_back({part.dir_col[dir], std::move(dv)});
        a.de.push_back({part.dir_col[dir], std::move(de)});
      }
      // <r^2>, <r^3> and their derivatives from the moments (0 along m).
      for (int k = 0; k < 2; ++k) {
        a.v[S_R2 + k] = part.mom.v[k];
        a.e[S_R2 + k] = part.mom.e[k];
        for (size_t c = 0; c < a.d.size(); ++c) {
          int b = -1;
          for (int t = 0; t < nt; ++t)
            if (part.theta[t].first == a.d[c].first) b = t;
          a.d[c].second[S_R2 + k] = b >= 0 ? part.mom.d[b][k] : 0.0;
          a.de[c].second[S_R2 + k] = b >= 0 ? part.mom.de[b][k] : 0.0;
        }
      }
    }
  }
  // Units: the mixture of their parts with their number fractions and the weight derivatives
  // (engine.rs:2121-2176).
  std::vector<UnitOut> out;
  for (auto& un : units) {
    double w_total = 0.0;
    {
      std::set<int> comps;
      for (int p : un)
        if (comps.insert(parts[p].component).second) w_total += parts[p].w;
    }
    std::vector<double> v(len, 0.0), e(len, 0.0);
    std::vector<std::vector<double>> d(n_cols, std::vector<double>(len, 0.0)),
        de(n_cols, std::vector<double>(len, 0.0));
    for (int p : un) {
      const double f = parts[p].f;
      for (int64_t i = 0; i < len; ++i) {
        v[i] += f * avg[p].v[i];
        e[i] += f * avg[p].e[i];
      }
      for (size_t c = 0; c < avg[p].d.size(); ++c) {
        const int col = avg[p].d[c].first;
        for (int64_t i = 0; i < len; ++i) {
          d[col][i] += f * avg[p].d[c].second[i];
          de[col][i] += f * avg[p].de[c].second[i];
        }
      }
    }
    for (size_t col = 0; col < n_cols; ++col) {
      const Param& pr = params[col];
      if (pr.kind != PK_WEIGHT) continue;
      for (int q : un) {
        const Part& part = parts[q];
        const double f = part.w / w_total * part.v / part.v_total;
        double df;
        if (pr.mode < 0) {
          const double own = part.component == pr.component ? part.v / part.v_total : 0.0;
          df = (own - f) / w_total;
        } else if (part.component != pr.component) {
          df = 0.0;
        } else {
          const double own = part.mode == pr.mode ? 1.0 : 0.0;
          df = part.w / w_total * (own - part.v / part.v_total) / part.v_total;
        }
        for (int64_t i = 0; i < len; ++i) {
          d[col][i] += df * avg[q].v[i];
          de[col][i] += std::fabs(df) * avg[q].e[i];
        }
      }
    }
    UnitOut u;
    auto lin = [&](int64_t i) {
      LinD x;
      x.v = v[i];
      x.e = e[i];
      x.d.resize(n_cols);
      x.de.resize(n_cols);
      for (size_t c = 0; c < n_cols; ++c) {
        x.d[c] = d[c][i];
        x.de[c] = de[c][i];
      }
      return x;
    };
    const LinD ext = lin(S_EXT), sca = lin(S_SCA), scag = lin(S_SCAG), ab = lin(S_ABS),
               back = lin(S_BACK), r2 = lin(S_R2), r3 = lin(S_R3);
    for (const LinD* l : {&ext, &sca, &back})
      if (!(std::isfinite(l->v) && l->v != 0.0))
        throw Failure{INVALID_INPUT,
                      "a ratio's denominator (<C_ext>, <C_sca> or <C_back>) is 0 or not finite"};
    // (F11 - F22)/(F11 + F22) at 180 degrees for units with spheroids: the numerator over
    // 2 C_back minus it (engine.rs:2432-2438).
    bool has_direct = false;
    for (int p : un) has_direct = has_direct || parts[p].eps > 0.0;
    LinD depol = LinD::constant(0.0, n_cols);
    if (has_direct) {
      const LinD num = lin(SCALARS - 1);
      LinD den = num;
      den.v = 2.0 * back.v - num.v;
      den.e = 2.0 * back.e + num.e;
      for (size_t c = 0; c < n_cols; ++c) {
        den.d[c] = 2.0 * back.d[c] - num.d[c];
        den.de[c] = 2.0 * back.de[c] + num.de[c];
      }
      depol = num.div(den);
    }
    const LinD sc[11] = {ext,
                         sca,
                         ab,
                         back,
                         sca.div(ext),
                         scag.div(sca),
                         ext.div(back).scale(4.0 * PI),
                         depol,
                         r3.div(r2),
                         r2.scale(PI),
                         r3.scale(4.0 * PI / 3.0)};
    // Adds c x to t as Lin::combine does (errors as bounds).
    auto add_to = [&](LinD& t, double c, const LinD& x) {
      t.v += c * x.v;
      t.e += std::fabs(c) * x.e;
      for (size_t k = 0; k < n_cols; ++k) {
        t.d[k] += c * x.d[k];
        t.de[k] += std::fabs(c) * x.de[k];
      }
    };
    auto direct_g = [&](int f, int64_t l) { return lin(d_start + f * (ld + 1) + l); };
    u.d_values.assign(n_cols * 11, 0.0);
    u.d_errors.assign(n_cols * 11, 0.0);
    for (int k = 0; k < 11; ++k) {
      u.values[k] = sc[k].v;
      u.errors[k] = sc[k].e;
      for (size_t c = 0; c < n_cols; ++c) {
        u.d_values[c * 11 + k] = sc[k].d[c];
        u.d_errors[c * 11 + k] = sc[k].de[c];
      }
    }
    if (n_mu > 0) {
      u.phase.assign(6 * n_mu, 0.0);
      u.phase_err.assign(6 * n_mu, 0.0);
      u.d_phase.assign(n_cols * 6 * n_mu, 0.0);
      u.d_phase_err.assign(n_cols * 6 * n_mu, 0.0);
      const int src[6] = {0, 1, 0, 2, 3, 2};
      // greek_phase (engine.rs:2363-2390) of the spheroids' averaged direct coefficients.
      std::vector<std::vector<LinD>> fd(n_mu);
      if (has_direct && ld >= 0) {
        std::vector<double> d00(ld + 1), d22(ld + 1), d2m2(ld + 1), d02(ld + 1);
        for (int64_t j = 0; j < n_mu; ++j) {
          wigner_d(0, 0, mu[j], d00.data(), ld + 1);
          wigner_d(2, 2, mu[j], d22.data(), ld + 1);
          wigner_d(2, -2, mu[j], d2m2.data(), ld + 1);
          wigner_d(0, 2, mu[j], d02.data(), ld + 1);
          fd[j].assign(6, LinD::constant(0.0, n_cols));
          for (int64_t l = 0; l <= ld; ++l) {
            const double pl = 0.5 * (d22[l] + d2m2[l]), mn = 0.5 * (d22[l] - d2m2[l]);
            add_to(fd[j][0], d00[l], direct_g(0, l));
            add_to(fd[j][1], d02[l], direct_g(4, l));
            add_to(fd[j][2], pl, direct_g(1, l));
            add_to(fd[j][2], mn, direct_g(2, l));
            add_to(fd[j][3], mn, direct_g(1, l));
            add_to(fd[j][3], pl, direct_g(2, l));
            add_to(fd[j][4], d02[l], direct_g(5, l));
            add_to(fd[j][5], d00[l], direct_g(3, l));
          }
        }
      }
      for (int el = 0; el < 6; ++el)
        for (int64_t j = 0; j < n_mu; ++j) {
          LinD f = lin(SCALARS + src[el] * n_mu + j);
          if (!fd[j].empty()) add_to(f, 1.0, fd[j][el]);
          if (normalized) f = f.div(sca);
          u.phase[el * n_mu + j] = f.v;
          u.phase_err[el * n_mu + j] = f.e;
          for (size_t c = 0; c < n_cols; ++c) {
            u.d_phase[(c * 6 + el) * n_mu + j] = f.d[c];
            u.d_phase_err[(c * 6 + el) * n_mu + j] = f.de[c];
          }
        }
    }
    if (order >= 0) {
      int64_t top = 0;
      for (auto& B : L.bands) top = std::max(top, std::min(order, 2 * B.upper));
      std::vector<LinD> gk(6 * (top + 1), LinD::constant(0.0, n_cols));
      // project (engine.rs:2310-2355): values and derivatives projected, errors as bounds.
      auto project = [&](const double* f, const double* fe, const BandData& B, int64_t qn,
                         int64_t l, double c[6], double cerr[6]) {
        const int64_t blen = B.order + 1;
        double pp = 0, mi = 0, ce[4] = {0, 0, 0, 0}, bp = 0, bm = 0;
        for (int t = 0; t < 6; ++t) c[t] = 0.0;
        for (int64_t k = 0; k < qn; ++k) {
          const double d00 = B.dmat[0][k * blen + l], d22 = B.dmat[1][k * blen + l];
          const double d2m2 = B.dmat[2][k * blen + l], d02 = B.dmat[3][k * blen + l];
          c[0] += f[k] * d00;
          c[3] += f[2 * qn + k] * d00;
          pp += (f[k] + f[2 * qn + k]) * d22;
          mi += (f[k] - f[2 * qn + k]) * d2m2;
          c[4] += f[qn + k] * d02;
          c[5] += f[3 * qn + k] * d02;
          const double es = fe[k] + fe[2 * qn + k];
          ce[0] += fe[k] * std::fabs(d00);
          ce[1] += fe[2 * qn + k] * std::fabs(d00);
          ce[2] += fe[qn + k] * std::fabs(d02);
          ce[3] += fe[3 * qn + k] * std::fabs(d02);
          bp += es * std::fabs(d22);
          bm += es * std::fabs(d2m2);
        }
        c[1] = (pp + mi) * 0.5;
        c[2] = (pp - mi) * 0.5;
        const double both = (bp + bm) * 0.5;
        const double cr[6] = {ce[0], both, both, ce[1], ce[2], ce[3]};
        for (int t = 0; t < 6; ++t) cerr[t] = cr[t];
      };
      for (size_t b = 0; b < L.bands.size(); ++b) {
        const BandData& B = L.bands[b];
        const int64_t qn = B.n_q, blen = B.order + 1;
        for (int64_t l = 0; l < blen; ++l) {
          double c[6], cerr[6];
          project(v.data() + L.start[b], e.data() + L.start[b], B, qn, l, c, cerr);
          for (int el = 0; el < 6; ++el) {
            gk[el * (top + 1) + l].v += c[el];
            gk[el * (top + 1) + l].e += cerr[el];
          }
          for (size_t col = 0; col < n_cols; ++col) {
            project(d[col].data() + L.start[b], de[col].data() + L.start[b], B, qn, l, c, cerr);
            for (int el = 0; el < 6; ++el) {
              gk[el * (top + 1) + l].d[col] += c[el];
              gk[el * (top + 1) + l].de[col] += cerr[el];
            }
          }
        }
      }
      if (has_direct && ld >= 0) {
        // The spheroids' coefficients added to the spheres' (engine.rs:2196-2216).
        const int64_t top_d = std::min<int64_t>(ld, order);
        if (top_d > top) {
          std::vector<LinD> wider(6 * (top_d + 1), LinD::constant(0.0, n_cols));
          for (int el = 0; el < 6; ++el)
            for (int64_t l = 0; l <= top; ++l) wider[el * (top_d + 1) + l] = gk[el * (top + 1) + l];
          gk.swap(wider);
          top = top_d;
        }
        for (int el = 0; el < 6; ++el)
          for (int64_t l = 0; l <= top_d; ++l) add_to(gk[el * (top + 1) + l], 1.0, direct_g(el, l));
      }
      if (normalized) {
        const LinD a0 = gk[0];
        for (auto& x : gk) x = x.div(a0);
        gk[0] = LinD::constant(1.0, n_cols);
      }
      const int64_t glen = order + 1;
      u.greek.assign(6 * glen, 0.0);
      u.greek_err.assign(6 * glen, 0.0);
      u.d_greek.assign(n_cols * 6 * glen, 0.0);
      u.d_greek_err.assign(n_cols * 6 * glen, 0.0);
      for (int el = 0; el < 6; ++el)
        for (int64_t l = 0; l <= std::min(top, order); ++l) {
          const LinD& x = gk[el * (top + 1) + l];
          u.greek[el * glen + l] = x.v;
          u.greek_err[el * glen + l] = x.e;
          for (size_t c = 0; c < n_cols; ++c) {
            u.d_greek[(c * 6 + el) * glen + l] = x.d[c];
            u.d_greek_err[(c * 6 + el) * glen + l] = x.de[c];
          }
        }
    }
    std::set<int> ug;
    for (int p : un) {
      u.converged = u.converged && firsts[group_of[p]].converged[place[p]];
      ug.insert(group_of[p]);
    }
    for (int gi : ug) u.panels += (int64_t)firsts[gi].panels.size();
    out.push_back(std::move(u));
  }
  return out;
}

}  // namespace

extern "C" {

// The adaptive ensemble of spheres with m per wavelength (complex, n_wl). batch = 0: every
// distribution on its own (`compute` per distribution); batch = 1: one `compute_batch` over
// all (shared panels per wavelength). Outputs distribution-major (unit = d * n_wl + i): values
// and errors (11, n), phase and phase_err (6, n, n_mu), greek and greek_err (6, n, L + 1),
// converged (n) as bytes, panels (n). Returns a status, the first error in wavelength order.
static int adaptive_impl(const FixedDist* dists, int64_t n_dist, int batch, const double* wl,
                         int64_t n_wl, const double* m, int n_layers, const double* fractions,
                         const double* m_layers, const double* mu, int64_t n_mu,
                         int64_t greek_order, int normalized, double rtol, int64_t max_panels,
                         int allow_unvalidated, int refine_backscatter, int n_threads,
                         double* values, double* errors, double* phase, double* phase_err,
                         double* greek, double* greek_err, int8_t* converged, int64_t* panels,
                         char* err, int64_t err_len, double eps = 0.0) {
  const int64_t n_units = n_dist * n_wl;
  Options o{rtol, (size_t)max_panels, allow_unvalidated != 0, refine_backscatter != 0};
  auto fail = [&](const Failure& f) {
    if (err && err_len > 0) snprintf(err, err_len, "%s", f.msg.c_str());
    return f.status;
  };
  if (!(rtol >= 1e-13 && rtol <= 0.1)) return fail({INVALID_INPUT, "rtol must be in [1e-13, 0.1]"});
  if (max_panels < 1) return fail({INVALID_INPUT, "max_panels must be at least 1"});
  std::vector<Part> parts;
  try {
    for (int64_t d = 0; d < n_dist; ++d) {
      parts.push_back(make_part(dists[d], rtol));
      parts.back().m = m;
      parts.back().n_wl = n_wl;
      parts.back().eps = eps;
      if (n_layers > 1) {
        parts.back().n_layers = n_layers;
        parts.back().fractions = fractions + d * (n_layers - 1);
        parts.back().m_layers = m_layers + 2 * d * n_layers * n_wl;
      }
    }
  } catch (const Failure& f) {
    return fail(f);
  }
  // Groups and units: a batch shares one group (point parts alone); single calls are one
  // part per group and unit.
  std::vector<std::vector<std::vector<int>>> groups_of, units_of;  // per call
  if (batch) {
    std::vector<std::vector<int>> groups, units;
    std::vector<int> shared;
    for (int64_t d = 0; d < n_dist; ++d) {
      if (parts[d].support == POINT)
        groups.push_back({(int)d});
      else
        shared.push_back((int)d);
      units.push_back({(int)d});
    }
    if (!shared.empty()) groups.push_back(shared);
    groups_of.push_back(groups);
    units_of.push_back(units);
  } else {
    for (int64_t d = 0; d < n_dist; ++d) {
      groups_of.push_back({{(int)d}});
      units_of.push_back({{(int)d}});
    }
  }
  const int64_t n_calls = (int64_t)groups_of.size();
  const int64_t glen = greek_order >= 0 ? greek_order + 1 : 0;
  const bool all = greek_order == GREEK_ALL;
  std::vector<std::vector<double>> all_g(all ? n_units : 0), all_ge(all_g.size()), none;
  std::vector<Failure> fails(n_calls * n_wl, Failure{OK, ""});
  if (n_threads > 0) omp_set_num_threads(n_threads);
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t job = 0; job < n_calls * n_wl; ++job) {
    const int64_t c = job / n_wl, i = job % n_wl;
    try {
      auto res = wavelength(parts, groups_of[c], units_of[c], wl[i], i, mu, n_mu, greek_order,
                            normalized != 0, o);
      for (size_t k = 0; k < units_of[c].size(); ++k) {
        const int64_t d = units_of[c][k][0];
        const int64_t unit = d * n_wl + i;
        const UnitOut& u = res[k];
        for (int q = 0; q < 11; ++q) {
          values[q * n_units + unit] = u.values[q];
          errors[q * n_units + unit] = u.errors[q];
        }
        if (phase && n_mu > 0)
          for (int el = 0; el < 6; ++el)
            for (int64_t j = 0; j < n_mu; ++j) {
              phase[(el * n_units + unit) * n_mu + j] = u.phase[el * n_mu + j];
              phase_err[(el * n_units + unit) * n_mu + j] = u.phase_err[el * n_mu + j];
            }
        if (greek && glen > 0)
          for (int el = 0; el < 6; ++el)
            for (int64_t l = 0; l < glen; ++l) {
              greek[(el * n_units + unit) * glen + l] = u.greek[el * glen + l];
              greek_err[(el * n_units + unit) * glen + l] = u.greek_err[el * glen + l];
            }
        if (all) {
          all_g[unit] = u.greek;
          all_ge[unit] = u.greek_err;
        }
        converged[unit] = u.converged ? 1 : 0;
        panels[unit] = u.panels;
      }
    } catch (const Failure& f) {
      fails[job] = f;
    }
  }
  if (all) keep_all_orders(all_g, all_ge, none, none, 0);
  // The first error in (wavelength, call) order, as the reference reports the first in order.
  for (int64_t i = 0; i < n_wl; ++i)
    for (int64_t c = 0; c < n_calls; ++c)
      if (fails[c * n_wl + i].status != OK) return fail(fails[c * n_wl + i]);
  return OK;
}

// The last GREEK_ALL call's Greek coefficients: the width (the longest order plus one), and the
// arrays (6, n, width) and (P, 6, n, width), zero above each unit's order.
int64_t orc_greek_all_width() {
  size_t w = 1;
  for (auto& g : g_all_orders.g) w = std::max(w, g.size() / 6);
  return (int64_t)w;
}

void orc_greek_all_take(double* greek, double* greek_err, double* d_greek, double* d_greek_err) {
  const AllOrders& a = g_all_orders;
  const int64_t n = (int64_t)a.g.size(), w = orc_greek_all_width(), P = (int64_t)a.P;
  for (int64_t u = 0; u < n; ++u) {
    const int64_t len = (int64_t)a.g[u].size() / 6;
    for (int el = 0; el < 6; ++el)
      for (int64_t l = 0; l < w; ++l) {
        const bool in = l < len;
        greek[(el * n + u) * w + l] = in ? a.g[u][el * len + l] : 0.0;
        greek_err[(el * n + u) * w + l] = in ? a.ge[u][el * len + l] : 0.0;
        for (int64_t c = 0; c < P && d_greek; ++c) {
          d_greek[((c * 6 + el) * n + u) * w + l] = in ? a.dg[u][(c * 6 + el) * len + l] : 0.0;
          d_greek_err[((c * 6 + el) * n + u) * w + l] = in ? a.dge[u][(c * 6 + el) * len + l] : 0.0;
        }
      }
  }
}

int orc_ensemble_adaptive(const FixedDist* dists, int64_t n_dist, int batch, const double* wl,
                          int64_t n_wl, const double* m, const double* mu, int64_t n_mu,
                          int64_t greek_order, int normalized, double rtol, int64_t max_panels,
                          int allow_unvalidated, int refine_backscatter, int n_threads,
                          double* values, double* errors, double* phase, double* phase_err,
                          double* greek, double* greek_err, int8_t* converged, int64_t* panels,
                          char* err, int64_t err_len) {
  return adaptive_impl(dists, n_dist, batch, wl, n_wl, m, 1, nullptr, nullptr, mu, n_mu,
                       greek_order, normalized, rtol, max_panels, allow_unvalidated,
                       refine_backscatter, n_threads, values, errors, phase, phase_err, greek,
                       greek_err, converged, panels, err, err_len);
}

// orc_ensemble_adaptive for layered spheres: n_layers layers, fractions [n_dist][n_layers - 1],
// m_layers complex [n_dist][n_layers][n_wl] (layered/kernel.rs per node; particle.rs:186-195).
int orc_ensemble_adaptive_layered(const FixedDist* dists, int64_t n_dist, int batch,
                                  const double* wl, int64_t n_wl, int n_layers,
                                  const double* fractions, const double* m_layers,
                                  const double* mu, int64_t n_mu, int64_t greek_order,
                                  int normalized, double rtol, int64_t max_panels,
                                  int allow_unvalidated, int refine_backscatter, int n_threads,
                                  double* values, double* errors, double* phase,
                                  double* phase_err, double* greek, double* greek_err,
                                  int8_t* converged, int64_t* panels, char* err,
                                  int64_t err_len) {
  return adaptive_impl(dists, n_dist, batch, wl, n_wl, m_layers, n_layers, fractions, m_layers,
                       mu, n_mu, greek_order, normalized, rtol, max_panels, allow_unvalidated,
                       refine_backscatter, n_threads, values, errors, phase, phase_err, greek,
                       greek_err, converged, panels, err, err_len);
}

// orc_ensemble_adaptive for randomly oriented spheroids of aspect ratio eps (m per wavelength):
// every node solved by the oracle's EBCM and orientation average, pass 2 on the direct path.
int orc_ensemble_adaptive_spheroid(const FixedDist* dists, int64_t n_dist, int batch,
                                   const double* wl, int64_t n_wl, double eps, const double* m,
                                   const double* mu, int64_t n_mu, int64_t greek_order,
                                   int normalized, double rtol, int64_t max_panels,
                                   int allow_unvalidated, int refine_backscatter, int n_threads,
                                   double* values, double* errors, double* phase,
                                   double* phase_err, double* greek, double* greek_err,
                                   int8_t* converged, int64_t* panels, char* err,
                                   int64_t err_len) {
  return adaptive_impl(dists, n_dist, batch, wl, n_wl, m, 1, nullptr, nullptr, mu, n_mu,
                       greek_order, normalized, rtol, max_panels, allow_unvalidated,
                       refine_backscatter, n_threads, values, errors, phase, phase_err, greek,
                       greek_err, converged, panels, err, err_len, eps);
}

// The adaptive ensemble of a mixture with the derivatives along `params` (n_params of them,
// each {component, mode (-1 none), kind (0 distribution parameter by gradient index, 1 Re m,
// 2 Im m, 3 weight), index}): compute_mixture (ensemble/mod.rs:609-625) with
// EnsembleOptions::derivatives. Components as orc_ensemble_mixture, multimodal[c] != 0 when
// component c is a multimodal distribution (its parameters then carry a mode). Outputs per
// wavelength as orc_ensemble_mixture, and d_values, d_errors (P, 11, n_wl), d_phase,
// d_phase_err (P, 6, n_wl, n_mu), d_greek, d_greek_err (P, 6, n_wl, L + 1).
int orc_ensemble_mixture_d(const FixedDist* modes, const double* mode_w, const int32_t* n_modes,
                           const int32_t* multimodal, const int32_t* n_layers,
                           const double* fractions, const double* eps, const double* w,
                           const double* m,
                           int64_t n_comp, const double* wl, int64_t n_wl, const double* mu,
                           int64_t n_mu, int64_t greek_order, int normalized, double rtol,
                           int64_t max_panels, int allow_unvalidated, int refine_backscatter,
                           const Param* params, int64_t n_params, double* values,
                           double* errors, double* phase, double* phase_err, double* greek,
                           double* greek_err, double* d_values, double* d_errors,
                           double* d_phase, double* d_phase_err, double* d_greek,
                           double* d_greek_err, int8_t* converged, int64_t* panels, char* err,
                           int64_t err_len) {
  Options o{rtol, (size_t)max_panels, allow_unvalidated != 0, refine_backscatter != 0};
  auto fail = [&](const Failure& f) {
    if (err && err_len > 0) snprintf(err, err_len, "%s", f.msg.c_str());
    return f.status;
  };
  if (!(rtol >= 1e-13 && rtol <= 0.1)) return fail({INVALID_INPUT, "rtol must be in [1e-13, 0.1]"});
  std::vector<Param> ps(params, params + n_params);
  for (int64_t k = 0; k < n_params; ++k)
    for (int64_t j = 0; j < k; ++j)
      if (ps[j].component == ps[k].component && ps[j].mode == ps[k].mode &&
          ps[j].kind == ps[k].kind && ps[j].index == ps[k].index)
        return fail({INVALID_INPUT, "a parameter is requested twice"});
  double w_total = 0.0;
  for (int64_t c = 0; c < n_comp; ++c) w_total += w[c];
  std::vector<Part> parts;
  std::vector<int> unit;
  try {
    int64_t k = 0, m_off = 0, fr_off = 0;
    for (int64_t c = 0; c < n_comp; ++c) {
      // The component's particle (engine.rs:95-115; particle.rs): a sphere, a layered sphere
      // (its fractions, indices [n_layers][n_wl]) or a spheroid of aspect ratio eps.
      const int nl = n_layers ? std::max(1, n_layers[c]) : 1;
      const double* mc = m + 2 * m_off;
      const double* fc = nl > 1 ? fractions + fr_off : nullptr;
      m_off += (int64_t)nl * n_wl;
      fr_off += nl - 1;
      double v_total = 0.0;
      for (int j = 0; j < n_modes[c]; ++j) v_total += multimodal[c] ? mode_w[k + j] : 1.0;
      for (int j = 0; j < n_modes[c]; ++j) {
        const int mode = multimodal[c] ? j : -1;
        // engine.rs:153-176: the part's parameters.
        std::vector<std::pair<int, int>> theta;
        int dir_col[2] = {-1, -1};
        std::vector<int> grads;
        for (int64_t col = 0; col < n_params; ++col) {
          const Param& pr = ps[col];
          if (pr.component != c) continue;
          if (pr.kind == PK_DIST && pr.mode == mode) {
            theta.push_back({(int)col, pr.index});
            grads.push_back(pr.index);
          } else if (pr.kind == PK_REFR_REAL) {
            dir_col[0] = (int)col;
          } else if (pr.kind == PK_REFR_IMAG) {
            dir_col[1] = (int)col;
          }
        }
        const double v = multimodal[c] ? mode_w[k + j] : 1.0;
        parts.push_back(make_part(modes[k + j], rtol, grads));
        Part& pt = parts.back();
        pt.m = mc;
        pt.n_wl = n_wl;
        if (nl > 1) {
          pt.n_layers = nl;
          pt.fractions = fc;
          pt.m_layers = mc;
        }
        if (eps && eps[c] > 0.0) pt.eps = eps[c];
        if ((nl > 1 || pt.eps > 0.0) && (!theta.empty() || dir_col[0] >= 0 || dir_col[1] >= 0))
          throw Failure{INVALID_INPUT,
                        "derivatives of layered spheres and spheroids are not on this path"};
        pt.f = w[c] / w_total * v / v_total;
        pt.component = (int)c;
        pt.mode = mode;
        pt.w = w[c];
        pt.v = v;
        pt.v_total = v_total;
        pt.theta = theta;
        pt.dir_col[0] = dir_col[0];
        pt.dir_col[1] = dir_col[1];
        unit.push_back((int)parts.size() - 1);
      }
      k += n_modes[c];
    }
  } catch (const Failure& f) {
    return fail(f);
  }
  std::vector<std::vector<int>> groups;
  for (size_t p = 0; p < parts.size(); ++p) groups.push_back({(int)p});
  std::vector<std::vector<int>> units{unit};
  const int64_t glen = greek_order >= 0 ? greek_order + 1 : 0;
  const int64_t P = n_params;
  const bool all = greek_order == GREEK_ALL;
  std::vector<std::vector<double>> all_g(all ? n_wl : 0), all_ge(all_g.size()),
      all_dg(all_g.size()), all_dge(all_g.size());
  std::vector<Failure> fails(n_wl, Failure{OK, ""});
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t i = 0; i < n_wl; ++i) {
    try {
      auto res = wavelength(parts, groups, units, wl[i], i, mu, n_mu, greek_order,
                            normalized != 0, o, ps);
      const UnitOut& u = res[0];
      for (int q = 0; q < 11; ++q) {
        values[q * n_wl + i] = u.values[q];
        errors[q * n_wl + i] = u.errors[q];
        for (int64_t c = 0; c < P; ++c) {
          d_values[(c * 11 + q) * n_wl + i] = u.d_values[c * 11 + q];
          d_errors[(c * 11 + q) * n_wl + i] = u.d_errors[c * 11 + q];
        }
      }
      if (phase && n_mu > 0)
        for (int el = 0; el < 6; ++el)
          for (int64_t j = 0; j < n_mu; ++j) {
            phase[(el * n_wl + i) * n_mu + j] = u.phase[el * n_mu + j];
            phase_err[(el * n_wl + i) * n_mu + j] = u.phase_err[el * n_mu + j];
            for (int64_t c = 0; c < P; ++c) {
              d_phase[((c * 6 + el) * n_wl + i) * n_mu + j] = u.d_phase[(c * 6 + el) * n_mu + j];
              d_phase_err[((c * 6 + el) * n_wl + i) * n_mu + j] =
                  u.d_phase_err[(c * 6 + el) * n_mu + j];
            }
          }
      if (greek && glen > 0)
        for (int el = 0; el < 6; ++el)
          for (int64_t l = 0; l < glen; ++l) {
            greek[(el * n_wl + i) * glen + l] = u.greek[el * glen + l];
            greek_err[(el * n_wl + i) * glen + l] = u.greek_err[el * glen + l];
            for (int64_t c = 0; c < P; ++c) {
              d_greek[((c * 6 + el) * n_wl + i) * glen + l] = u.d_greek[(c * 6 + el) * glen + l];
              d_greek_err[((c * 6 + el) * n_wl + i) * glen + l] =
                  u.d_greek_err[(c * 6 + el) * glen + l];
            }
          }
      if (all) {
        all_g[i] = u.greek;
        all_ge[i] = u.greek_err;
        all_dg[i] = u.d_greek;
        all_dge[i] = u.d_greek_err;
      }
      converged[i] = u.converged ? 1 : 0;
      panels[i] = u.panels;
    } catch (const Failure& f) {
      fails[i] = f;
    }
  }
  if (all) keep_all_orders(all_g, all_ge, all_dg, all_dge, (size_t)P);
  for (int64_t i = 0; i < n_wl; ++i)
    if (fails[i].status != OK) return fail(fails[i]);
  return OK;
}

// The adaptive ensemble of a mixture (compute_mixture, ensemble/mod.rs:609-625): n_comp
// components, component c with n_modes[c] modes (its distributions, consecutive in `modes`,
// with weights mode_w, ignored for one mode), weight w[c] and m of its own (complex per
// wavelength, consecutive n_wl per component). Each mode is a part on its own panels; the
// outputs per wavelength as orc_ensemble_adaptive with n_units = n_wl.
int orc_ensemble_mixture(const FixedDist* modes, const double* mode_w, const int32_t* n_modes,
                         const double* w, const double* m, int64_t n_comp, const double* wl,
                         int64_t n_wl, const double* mu, int64_t n_mu, int64_t greek_order,
                         int normalized, double rtol, int64_t max_panels, int allow_unvalidated,
                         int refine_backscatter, double* values, double* errors, double* phase,
                         double* phase_err, double* greek, double* greek_err, int8_t* converged,
                         int64_t* panels, char* err, int64_t err_len) {
  Options o{rtol, (size_t)max_panels, allow_unvalidated != 0, refine_backscatter != 0};
  auto fail = [&](const Failure& f) {
    if (err && err_len > 0) snprintf(err, err_len, "%s", f.msg.c_str());
    return f.status;
  };
  if (!(rtol >= 1e-13 && rtol <= 0.1)) return fail({INVALID_INPUT, "rtol must be in [1e-13, 0.1]"});
  double w_total = 0.0;
  for (int64_t c = 0; c < n_comp; ++c) w_total += w[c];
  std::vector<Part> parts;
  std::vector<int> unit;
  try {
    int64_t k = 0;
    for (int64_t c = 0; c < n_comp; ++c) {
      double v_total = 0.0;
      for (int j = 0; j < n_modes[c]; ++j) v_total += n_modes[c] > 1 ? mode_w[k + j] : 1.0;
      for (int j = 0; j < n_modes[c]; ++j) {
        const double v = n_modes[c] > 1 ? mode_w[k + j] : 1.0;
        parts.push_back(make_part(modes[k + j], rtol));
        parts.back().m = m + 2 * n_wl * c;
        parts.back().n_wl = n_wl;
        parts.back().f = w[c] / w_total * v / v_total;
        unit.push_back((int)parts.size() - 1);
      }
      k += n_modes[c];
    }
  } catch (const Failure& f) {
    return fail(f);
  }
  std::vector<std::vector<int>> groups;
  for (size_t p = 0; p < parts.size(); ++p) groups.push_back({(int)p});
  std::vector<std::vector<int>> units{unit};
  const int64_t glen = greek_order >= 0 ? greek_order + 1 : 0;
  std::vector<Failure> fails(n_wl, Failure{OK, ""});
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t i = 0; i < n_wl; ++i) {
    try {
      auto res = wavelength(parts, groups, units, wl[i], i, mu, n_mu, greek_order,
                            normalized != 0, o);
      const UnitOut& u = res[0];
      for (int q = 0; q < 11; ++q) {
        values[q * n_wl + i] = u.values[q];
        errors[q * n_wl + i] = u.errors[q];
      }
      if (phase && n_mu > 0)
        for (int el = 0; el < 6; ++el)
          for (int64_t j = 0; j < n_mu; ++j) {
            phase[(el * n_wl + i) * n_mu + j] = u.phase[el * n_mu + j];
            phase_err[(el * n_wl + i) * n_mu + j] = u.phase_err[el * n_mu + j];
          }
      if (greek && glen > 0)
        for (int el = 0; el < 6; ++el)
          for (int64_t l = 0; l < glen; ++l) {
            greek[(el * n_wl + i) * glen + l] = u.greek[el * glen + l];
            greek_err[(el * n_wl + i) * glen + l] = u.greek_err[el * glen + l];
          }
      converged[i] = u.converged ? 1 : 0;
      panels[i] = u.panels;
    } catch (const Failure& f) {
      fails[i] = f;
    }
  }
  for (auto& f : fails)
    if (f.status != OK) return fail(f);
  return OK;
}

}  // extern "C"
