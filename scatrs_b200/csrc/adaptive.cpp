// The adaptive ensemble's host logic: see adaptive.h. Each function cites the reference code
// whose decisions it makes; the numbers it decides on (the pass-1 sums) come from the device.
#include "adaptive.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <limits>

#include "tables.h"

namespace sb {
namespace adaptive {

namespace {

constexpr double kStep = 0.5;          // range.rs:8
constexpr int kMaxSteps = 400;         // range.rs:11
constexpr int kMaxExtensions = 100;    // engine.rs:60
constexpr double kMinWidth = 1e-10;    // engine.rs:63
constexpr double kMaxDx = 20.0;        // engine.rs:67
constexpr size_t kMomentPanels = 100000;  // moments.rs:10
constexpr double kInf = std::numeric_limits<double>::infinity();
constexpr double kPi = 3.14159265358979323846264338327950288;
constexpr double kMaxSizeParameter = 1e6;  // mie/mod.rs MAX_SIZE_PARAMETER

// Pass-1 indices (engine.rs:43-54).
constexpr int ONE = 0, EXT = 1, SCA = 2, SCAG = 3, BACK = 4, ABS = 5;

double max_step(const Part& p, double step) { return std::min(step, 0.5 * p.log_width); }

std::string at(double lambda, double r) {
  char buf[128];
  snprintf(buf, sizeof buf, "at wavelength %e, radius %e: ", lambda, r);
  return buf;
}

// The masses of r^k u over [t0, t1] for k in {0, 2, 3} as selected (range.rs:25-36).
void masses(const Part& p, double t0, double t1, const std::vector<int>& pw, double* out) {
  Node nd[15];
  gk15(t0, t1, nd);
  for (size_t k = 0; k < pw.size(); ++k) out[k] = 0.0;
  for (const Node& n : nd) {
    const double r = std::exp(n.t);
    const double wu = n.wk * r * p.u(r);
    for (size_t k = 0; k < pw.size(); ++k)
      out[k] += wu * (pw[k] == 0 ? 1.0 : pw[k] == 2 ? r * r : r * r * r);
  }
}

// range.rs:48-93: march outward in steps of ln r until each side's tail, bounded
// geometrically, holds at most eps of every moment.
std::pair<double, double> cutoffs(const Part& p, double center, double eps,
                                  const std::vector<int>& pw) {
  const double t0 = std::log(center), step = max_step(p, kStep);
  const size_t np = pw.size();
  std::vector<double> total(np, 0.0), mass(np);
  std::vector<double> last[2] = {std::vector<double>(np, kInf), std::vector<double>(np, kInf)};
  double ends[2] = {t0, t0};
  bool done[2] = {false, false};
  for (int i = 0; i < kMaxSteps; ++i) {
    for (int side = 0; side < 2; ++side) {
      if (done[side]) continue;
      const double a = ends[side], b = a + (side == 0 ? -1.0 : 1.0) * step;
      masses(p, std::min(a, b), std::max(a, b), pw, mass.data());
      for (double m : mass)
        if (!std::isfinite(m)) {
          char buf[128];
          snprintf(buf, sizeof buf, "the size distribution's density is not finite near r = %e",
                   std::exp(b));
          throw Error{1, buf};
        }
      ends[side] = b;
      bool small = i >= 1;
      for (size_t k = 0; k < np; ++k) {
        total[k] += mass[k];
        const double q = mass[k] / last[side][k];
        last[side][k] = mass[k];
        small = small && (mass[k] == 0.0 || (q < 1.0 && mass[k] / (1.0 - q) <= eps * total[k]));
      }
      done[side] = small;
    }
    if (done[0] && done[1]) return {std::exp(ends[0]), std::exp(ends[1])};
  }
  char buf[160];
  snprintf(buf, sizeof buf,
           "the size distribution is too broad: its tails do not decay within e^%g of r = %e",
           kMaxSteps * step, center);
  throw Error{1, buf};
}

// moments.rs:62-167: GK15 panels of at most max_step (the breaks inside the range as edges),
// split where a sum's |Kronrod - Gauss| is above its share, until Z, <r^2 u>, <r^3 u> and,
// along each requested parameter, their derivatives meet rtol (the derivatives of their
// absolute integrands' Kronrod sums); then the quotient rule with first-order error
// propagation (moments.rs:171-212).
Moments moments(const Part& p, double lo, double hi, double rtol, double truncation,
                const std::vector<double>& breaks = {}) {
  const double step = max_step(p, kStep);
  const double t_lo = std::log(lo), t_hi = std::log(hi);
  const int nt = (int)p.grads.size(), nq = 3 * (1 + nt);
  std::vector<std::pair<double, double>> panels;
  {
    // The breaks inside the range are panel edges; each interval in equal panels of at most
    // the step (moments.rs:72-86).
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
  auto result = [&](const std::vector<double>& s, const std::vector<double>& e) {
    if (!(std::isfinite(s[0]) && s[0] > 0.0)) {
      char buf[128];
      snprintf(buf, sizeof buf,
               "the size distribution has no finite positive mass on its range (got %e)", s[0]);
      throw Error{1, buf};
    }
    Moments m;
    m.z = s[0];
    m.ez = e[0];
    for (int k = 0; k < 2; ++k) {
      m.v[k] = s[1 + k] / m.z;
      m.e[k] = (e[1 + k] + std::fabs(m.v[k]) * m.ez) / m.z + truncation * std::fabs(m.v[k]);
    }
    for (int b = 0; b < nt; ++b) {
      const int o = 3 * (1 + b);
      const double dz = s[o];
      std::array<double, 2> dv, dev;
      for (int k = 0; k < 2; ++k) dv[k] = (s[o + 1 + k] - m.v[k] * dz) / m.z;
      for (int k = 0; k < 2; ++k)
        dev[k] = (e[o + 1 + k] + std::fabs(m.v[k]) * e[o] + std::fabs(dv[k]) * m.ez +
                  m.e[k] * std::fabs(dz)) / m.z +
                 truncation * std::fabs(dv[k]);
      m.d.push_back(dv);
      m.de.push_back(dev);
      m.dz.push_back(dz);
      m.dez.push_back(e[o]);
    }
    return m;
  };
  double grad[3];
  for (;;) {
    // Per panel (moments.rs:31-53): Kronrod sums, |K - G| and the Kronrod sums of the
    // absolute derivative integrands.
    const size_t n = panels.size();
    std::vector<double> K(n * nq, 0.0), E(n * nq, 0.0), A(n * nq, 0.0), g(nq);
    for (size_t i = 0; i < n; ++i) {
      Node nd[15];
      gk15(panels[i].first, panels[i].second, nd);
      std::fill(g.begin(), g.end(), 0.0);
      for (const Node& x : nd) {
        const double r = std::exp(x.t), u = nt > 0 ? p.u(r, grad) : p.u(r);
        const double q[3] = {1.0, r * r, r * r * r};
        for (int j = 0; j < 3; ++j) {
          K[i * nq + j] += x.wk * u * r * q[j];
          g[j] += x.wg * u * r * q[j];
          for (int b = 0; b < nt; ++b) {
            const int o = 3 * (1 + b) + j;
            const double y = grad[p.grads[b]] * r * q[j];
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
    if (met || n >= kMomentPanels) return result(total, terr);
    std::vector<std::pair<double, double>> next;
    for (size_t i = 0; i < n; ++i) {
      bool bad = false;
      for (int j = 0; j < nq; ++j)
        bad = bad || (E[i * nq + j] * (double)n > target[j] && terr[j] > target[j]);
      if (bad && panels[i].second - panels[i].first > 1e-10) {
        const double mid = 0.5 * (panels[i].first + panels[i].second);
        next.push_back({panels[i].first, mid});
        next.push_back({mid, panels[i].second});
      } else {
        next.push_back(panels[i]);
      }
    }
    if (next.size() == n) return result(total, terr);
    panels.swap(next);
  }
}

double size_param(double r, double lambda) { return 2.0 * kPi * r / lambda; }

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
      const double step = std::min(step_of(a), std::log(1.0 + kMaxDx / x));
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

// One panel's pass-1 sums for one part (engine.rs:358-373, 482-549): the Kronrod sums of each
// refined quantity, then of each theta-weighted one (a block of n_refined per requested
// parameter), |Kronrod - Gauss| of the same, the Kronrod sums of |du/dtheta| r |q| and of
// u r |q| (the scales of the parameter blocks and of the derivatives along m), and the
// integrands per unit ln r at the first and last nodes.
// One panel's pass-1 sums for one part, in one buffer (a panel of a job of many parts holds one
// per part): the Kronrod sums k[nb] and their |Kronrod - Gauss| errors err[nb], the parameter
// blocks' absolute integrals abs[nt nr], the absolute value integrals absv[nr], and the
// integrands at the panel's two ends edge(0)[nb], edge(1)[nb].
struct Sums1 {
  std::vector<double> buf;
  int nb = 0, nab = 0, nr = 0;
  void init(int nb_, int nab_, int nr_) {
    nb = nb_, nab = nab_, nr = nr_;
    buf.assign((size_t)4 * nb + nab + nr, 0.0);
  }
  double* k() { return buf.data(); }
  double* err() { return buf.data() + nb; }
  double* abs() { return buf.data() + 2 * nb; }
  double* absv() { return buf.data() + 2 * nb + nab; }
  double* edge(int e) { return buf.data() + 2 * nb + nab + nr + e * nb; }
  const double* k() const { return buf.data(); }
  const double* err() const { return buf.data() + nb; }
  const double* abs() const { return buf.data() + 2 * nb; }
  const double* absv() const { return buf.data() + 2 * nb + nab; }
  const double* edge(int e) const { return buf.data() + 2 * nb + nab + nr + e * nb; }
};

// The targets, errors and ends of a part (engine.rs:620-720, no Greek refinement).
struct Status {
  std::vector<double> target, errors;
  bool met, small[2];
};

Status status_of(const Part& part, const std::vector<const Sums1*>& s, const Options& o,
                 double ext) {
  const int nr = part.n_refined(), nt = (int)part.grads.size(), nb = (1 + nt) * nr;
  const int n_greek = kPass1;
  Status st;
  st.target.assign(nb, 0.0);
  auto total = [&](int j) {
    double t = 0.0;
    for (auto* x : s) t += x->k()[j];
    return t;
  };
  auto abs_of = [&](int k) {
    double t = 0.0;
    for (auto* x : s) t += x->abs()[k];
    return t;
  };
  // C_abs and each direction's derivative of it are refined to rtol of C_ext's.
  auto scale_of = [&](int j) {
    if (j == ABS) return EXT;
    if (j >= n_greek && (j - n_greek) % kGroup == kGroup - 1) return j + 1 - kGroup;
    return j;
  };
  const double c_sca = std::fabs(total(SCA));
  for (int j = 0; j < nr; ++j) {
    double scale;
    if (j == SCAG) {
      scale = c_sca;
    } else if (j == BACK) {
      scale = std::max(std::fabs(total(BACK)), c_sca);
    } else if (j >= n_greek) {
      // The derivatives along m can cancel: their absolute integrands.
      scale = 0.0;
      for (auto* x : s) scale += x->absv()[scale_of(j)];
    } else {
      scale = std::fabs(total(scale_of(j)));
    }
    st.target[j] = o.rtol * scale;
    for (int b = 0; b < nt; ++b) st.target[(1 + b) * nr + j] = o.rtol * abs_of(b * nr + scale_of(j));
  }
  // Z comes from the moments; the theta blocks of the derivatives along m are no outputs.
  for (int b = 0; b <= nt; ++b) st.target[b * nr + ONE] = kInf;
  for (int b = 1; b <= nt; ++b)
    for (int j = n_greek; j < nr; ++j) st.target[b * nr + j] = kInf;
  if (!o.refine_backscatter)
    for (int b = 0; b <= nt; ++b) {
      st.target[b * nr + BACK] = kInf;
      for (int j = n_greek + 3; j < nr; j += kGroup) st.target[b * nr + j] = kInf;
    }
  st.errors.assign(nb, 0.0);
  st.met = true;
  for (int j = 0; j < nb; ++j) {
    double e = 0.0;
    for (auto* x : s) e += x->err()[j];
    st.errors[j] = e;
    st.met = st.met && e <= st.target[j];
  }
  // The ends: a tenth of the target per ext/STEP units of ln r; the parameter blocks against
  // their own size, floored at 1e-3 of the absolute integral.
  std::vector<double> end_target(nb);
  for (int x = 0; x < nb; ++x) {
    if (x < nr || std::isinf(st.target[x])) {
      end_target[x] = st.target[x];
    } else {
      const int b = x / nr - 1, j = x % nr;
      end_target[x] = o.rtol * std::max(std::fabs(total(x)), 1e-3 * abs_of(b * nr + scale_of(j)));
    }
  }
  auto small = [&](const double* d) {
    for (int j = 0; j < nb; ++j)
      if (!(std::fabs(d[j]) * (ext / kStep) <= 0.1 * end_target[j])) return false;
    return true;
  };
  st.small[0] = small(s.front()->edge(0));
  st.small[1] = small(s.back()->edge(1));
  return st;
}

struct Panel {
  double a, b;
  bool done = false;
  int64_t n_terms = 0;
  std::vector<Sums1> sums;  // per part of the job
};

struct State {
  std::vector<Panel> panels;
  double t_lo = 0, t_hi = 0;
  int extensions[2] = {0, 0};
  std::vector<double> exts;                     // per part
  std::vector<std::array<double, 3>> steps;     // per part: ln lo, ln hi, step
  bool finished = false;
};

}  // namespace

double Part::u(double r) const {
  if (support == POINT) return 0.0;
  if (kind == kTabulated) return table_density(table.data(), (int64_t)table.size() / 2, r);
  return density(kind, p, r);
}

double Part::u(double r, double grad[3]) const {
  grad[0] = grad[1] = grad[2] = 0.0;
  if (support == POINT) return 0.0;
  if (kind == kTabulated) return table_density(table.data(), (int64_t)table.size() / 2, r);
  return density_gradient(kind, p, r, grad);
}

std::vector<double> Part::breaks() const {
  std::vector<double> out;
  if (support == FINITE) {
    out.push_back(lo);
    out.push_back(hi);
  }
  if (kind == kTabulated)
    out.insert(out.end(), table.begin(), table.begin() + (int64_t)table.size() / 2);
  return out;
}

void gk15(double a, double b, Node out[15]) {
  // kronrod.rs:5-52 (QUADPACK's qk15 abscissae and weights).
  static const double kn[8] = {0.991455371120812639206854697526329,
                               0.949107912342758524526189684047851,
                               0.864864423359769072789712788640926,
                               0.741531185599394439863864773280788,
                               0.586087235467691130294144845693013,
                               0.405845151377397166906606412076961,
                               0.207784955007898467600689403773245,
                               0.0};
  static const double kw[8] = {0.022935322010529224963732008058970,
                               0.063092092629978553290700663189204,
                               0.104790010322250183839876322541518,
                               0.140653259715525918745189590510238,
                               0.169004726639267902826583426598550,
                               0.190350578064785409913256402421014,
                               0.204432940075298892414161999234649,
                               0.209482141084727828012999174891714};
  static const double gw[4] = {0.129484966168869693270611432679082,
                               0.279705391489276667901467771423780,
                               0.381830050505118944950369775488975,
                               0.417959183673469387755102040816327};
  const double c = 0.5 * (a + b), h = 0.5 * (b - a);
  for (int i = 0; i < 7; ++i) {
    const double g = i % 2 == 1 ? h * gw[i / 2] : 0.0;
    const double k = h * kw[i];
    out[i] = {c - h * kn[i], k, g};
    out[14 - i] = {c + h * kn[i], k, g};
  }
  out[7] = {c, h * kw[7], h * gw[3]};
}

Part make_part(int kind, const double* p, double rtol, const double* table, int64_t table_len,
               const std::vector<int>& grads) {
  Part part;
  part.kind = kind;
  for (int k = 0; k < 3; ++k) part.p[k] = p[k];
  part.grads = grads;
  if (kind == kTabulated) {
    // Finite support between the table's first and last radii (distribution.rs:285-287),
    // reference radius 1, no width limit; the moments with the table's radii as edges.
    std::string msg;
    if (!validate_table(table, table_len, &msg)) throw Error{1, msg};
    part.table.assign(table, table + 2 * table_len);
    part.reference = 1.0;
    part.log_width = kInf;  // the steps are not limited by a width
    part.support = FINITE;
    part.lo = table[0];
    part.hi = table[table_len - 1];
    part.mom = moments(part, part.lo, part.hi, rtol, 0.0, part.breaks());
    return part;
  }
  if (kind == kMonodisperse) {
    if (!(std::isfinite(p[0]) && p[0] > 0.0)) throw Error{1, "radius must be finite and > 0"};
    part.support = POINT;
    part.lo = part.hi = p[0];
    return part;
  }
  std::string msg;
  if (!validate_distribution(kind, p, &msg)) throw Error{1, msg};
  const DensityInfo info = density_info(kind, p);
  part.reference = info.reference;
  part.log_width = info.log_width;
  if (kind == 4) {  // finite support [min_radius, max_radius]
    part.support = FINITE;
    part.lo = p[1];
    part.hi = p[2];
    part.mom = moments(part, p[1], p[2], rtol, 0.0);
    return part;
  }
  // Unbounded (distribution.rs:272-290): about the median, the effective radius or the
  // reference radius; the Mie range bounds the area's tails to rtol/10, the moments' range
  // every tail to 1e-3 rtol (engine.rs:190-205).
  part.support = UNBOUNDED;
  const double center = kind == 3 ? part.reference : p[0];
  auto mie = cutoffs(part, center, rtol / 10.0, {2});
  part.lo = mie.first;
  part.hi = mie.second;
  auto wide = cutoffs(part, center, std::max(1e-3 * rtol, 1e-16), {0, 2, 3});
  part.mom = moments(part, wide.first, wide.second, rtol, 0.2 * rtol);
  return part;
}

// engine.rs:724-924, every job at once: a round evaluates the unevaluated panels of every
// unfinished job, then each job refines (splits worst first), extends its range or finishes.
void pass1(std::vector<Job>& jobs, const std::vector<Part>& parts, const double* wavelengths,
           const Options& o, const Evaluate& eval) {
  const size_t budget_max = (size_t)o.max_panels;
  std::vector<State> states(jobs.size());
  for (size_t ji = 0; ji < jobs.size(); ++ji) {
    Job& job = jobs[ji];
    State& st = states[ji];
    const double lambda = wavelengths[job.wl];
    std::vector<double> breaks;
    double lo = kInf, hi = 0.0;
    for (int pi : job.parts) {
      const Part& p = parts[pi];
      const std::vector<double> pb = p.breaks();
      breaks.insert(breaks.end(), pb.begin(), pb.end());
      lo = std::min(lo, p.lo);
      hi = std::max(hi, p.hi);
      st.exts.push_back(std::min(kStep, p.log_width));
      st.steps.push_back({std::log(p.lo), std::log(p.hi), max_step(p, kStep)});
    }
    std::sort(breaks.begin(), breaks.end());
    breaks.erase(std::unique(breaks.begin(), breaks.end()), breaks.end());
    const double x_hi = size_param(hi, lambda);
    if (x_hi > kMaxSizeParameter) {
      char buf[200];
      snprintf(buf, sizeof buf,
               "the integration range reaches size parameter %e, above the accepted %e", x_hi,
               kMaxSizeParameter);
      job.status = 1;
      job.msg = at(lambda, hi) + buf;
      st.finished = true;
      continue;
    }
    st.t_lo = std::log(lo);
    st.t_hi = std::log(hi);
    auto step_of = [&st](double t) {
      double s = kStep;
      for (auto& x : st.steps)
        if (x[0] <= t && t < x[1]) s = std::min(s, x[2]);
      return s;
    };
    for (auto& ab : initial_panels(st.t_lo, st.t_hi, lambda, breaks, step_of, budget_max))
      st.panels.push_back({ab.first, ab.second});
  }
  // The rounds' node lists and results, kept across rounds (their memory touched once).
  std::vector<Query> qs;
  std::vector<NodeResult> res;
  for (;;) {
    // Gather this round's nodes: the open panels in (job, panel) order, then their 15 nodes each
    // (filled on the host's threads; the order, and so every sum, does not depend on them).
    std::vector<std::pair<size_t, size_t>> owner;  // (job, panel) per 15 nodes
    for (size_t ji = 0; ji < jobs.size(); ++ji) {
      if (states[ji].finished) continue;
      for (size_t pi = 0; pi < states[ji].panels.size(); ++pi)
        if (!states[ji].panels[pi].done) owner.push_back({ji, pi});
    }
    if (owner.empty()) break;
    qs.resize(15 * owner.size());
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < (int64_t)owner.size(); ++k) {
      const Panel& pn = states[owner[k].first].panels[owner[k].second];
      Node nd[15];
      gk15(pn.a, pn.b, nd);
      for (int i = 0; i < 15; ++i) qs[15 * k + i] = {std::exp(nd[i].t), jobs[owner[k].first].wl};
    }
    res.resize(qs.size());
    eval(qs, res);
    // Each job's first failing node in panel order (in order, on one thread), then the panel
    // sums of the panels whose nodes all succeeded (each panel on its own, on the host's threads).
    std::vector<int> first_fail(jobs.size(), -1);
    std::vector<char> node_ok(owner.size(), 1);
    for (size_t k = 0; k < owner.size(); ++k) {
      const size_t ji = owner[k].first, pi = owner[k].second;
      bool ok = true;
      for (int i = 0; i < 15 && ok; ++i)
        if (res[15 * k + i].status != 0) {
          ok = false;
          if (first_fail[ji] < 0 || (int)pi < first_fail[ji]) {
            first_fail[ji] = (int)pi;
            jobs[ji].status = res[15 * k + i].status;
            jobs[ji].msg = at(wavelengths[jobs[ji].wl], qs[15 * k + i].r) +
                           (res[15 * k + i].msg ? std::string(res[15 * k + i].msg)
                            : jobs[ji].status == 3
                                ? "the size parameter and refractive index are outside the "
                                  "validated domain x in [1e-06, 2e4], 0 < Re m <= 10, "
                                  "0 <= Im m <= 10, |m| >= 0.1"
                                : "the size parameter x must be in [1e-30, 1e6] and the "
                                  "refractive index finite with Re m >= 0, Im m >= 0 and |m| in "
                                  "[1e-6, 1e3]");
          }
        }
      node_ok[k] = ok ? 1 : 0;
    }
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t k = 0; k < (int64_t)owner.size(); ++k) {
      if (!node_ok[k]) continue;
      const size_t ji = owner[k].first, pi = owner[k].second;
      Panel& pn = states[ji].panels[pi];
      Node nd[15];
      gk15(pn.a, pn.b, nd);
      pn.done = true;
      pn.n_terms = 0;
      for (int i = 0; i < 15; ++i) pn.n_terms = std::max(pn.n_terms, res[15 * k + i].n);
      pn.sums.assign(jobs[ji].parts.size(), Sums1{});
      // The quantities of the group's first part's directions (engine.rs:491-506).
      const Part& first = parts[jobs[ji].parts[0]];
      const int nr = first.n_refined();
      int qi[kPass1 + kGroup * kMaxAllDirs];  // make_part's callers keep nr within it
      for (int j = 0; j < kPass1; ++j) qi[j] = j;
      {
        int at = kPass1;
        for (int dir = 0; dir < (int)first.dirs.size(); ++dir)
          if (first.dirs[dir])
            for (int j = 0; j < kGroup; ++j) qi[at++] = kPass1 + kGroup * dir + j;
      }
      double grad[3];
      for (size_t p = 0; p < jobs[ji].parts.size(); ++p) {
        const Part& part = parts[jobs[ji].parts[p]];
        const int nt = (int)part.grads.size(), nb = (1 + nt) * nr;
        Sums1& s = pn.sums[p];
        s.init(nb, nt * nr, nr);
        double *sk = s.k(), *serr = s.err(), *sabs = s.abs(), *sabsv = s.absv();
        double *e0 = s.edge(0), *e1 = s.edge(1);
        std::vector<double> g(nb, 0.0);
        for (int i = 0; i < 15; ++i) {
          const double r = qs[15 * k + i].r;
          const double base = (nt > 0 ? part.u(r, grad) : part.u(r)) * r;
          const double* q = res[15 * k + i].q;
          const double* dq = res[15 * k + i].dq;
          for (int j = 0; j < nr; ++j) {
            const double qj = dq && qi[j] >= kPass1 ? dq[qi[j] - kPass1] : q[qi[j]];
            sk[j] += nd[i].wk * base * qj;
            g[j] += nd[i].wg * base * qj;
            sabsv[j] += nd[i].wk * std::fabs(base * qj);
            if (i == 0) e0[j] = base * qj;
            if (i == 14) e1[j] = base * qj;
            for (int b = 0; b < nt; ++b) {
              const double dw = grad[part.grads[b]] * r;
              const int x = (1 + b) * nr + j;
              sk[x] += nd[i].wk * dw * qj;
              g[x] += nd[i].wg * dw * qj;
              sabs[b * nr + j] += nd[i].wk * std::fabs(dw * qj);
              if (i == 0) e0[x] = dw * qj;
              if (i == 14) e1[x] = dw * qj;
            }
          }
        }
        for (int j = 0; j < nb; ++j) serr[j] = std::fabs(sk[j] - g[j]);
      }
    }
    // Each job's targets, extensions and splits (jobs are independent of one another).
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t ji = 0; ji < (int64_t)jobs.size(); ++ji) {
      State& st = states[ji];
      Job& job = jobs[ji];
      if (st.finished) continue;
      if (first_fail[ji] >= 0) {
        st.finished = true;
        continue;
      }
      const double lambda = wavelengths[job.wl];
      const size_t np = job.parts.size();
      std::vector<Status> stat;
      for (size_t p = 0; p < np; ++p) {
        std::vector<const Sums1*> s;
        for (auto& pn : st.panels) s.push_back(&pn.sums[p]);
        stat.push_back(status_of(parts[job.parts[p]], s, o, st.exts[p]));
      }
      auto finish = [&]() {
        job.panels.clear();
        job.panel_terms.clear();
        job.n_terms = 0;
        for (auto& pn : st.panels) {
          job.panels.push_back({pn.a, pn.b});
          job.panel_terms.push_back(pn.n_terms);
          job.n_terms = std::max(job.n_terms, pn.n_terms);
        }
        job.converged.assign(np, false);
        for (size_t p = 0; p < np; ++p) {
          const bool ext = parts[job.parts[p]].support == UNBOUNDED;
          job.converged[p] = stat[p].met && (!ext || (stat[p].small[0] && stat[p].small[1]));
        }
        st.finished = true;
      };
      bool all_met = true;
      for (auto& s : stat) all_met = all_met && s.met;
      const size_t n = st.panels.size();
      if (all_met) {
        // Extend at an end where an unbounded part's integrand is not negligible.
        auto wanting = [&](int end, double* ext, double* step) {
          if (st.extensions[end] >= kMaxExtensions) return false;
          bool any = false;
          for (size_t p = 0; p < np; ++p)
            if (parts[job.parts[p]].support == UNBOUNDED && !stat[p].small[end]) {
              *ext = any ? std::min(*ext, st.exts[p]) : st.exts[p];
              *step = any ? std::min(*step, st.steps[p][2]) : st.steps[p][2];
              any = true;
            }
          return any;
        };
        double e0 = 0, s0 = 0, e1 = 0, s1 = 0;
        const bool w0 = wanting(0, &e0, &s0), w1 = wanting(1, &e1, &s1);
        bool extended = false, stop = false;
        if (w0) {
          auto fresh = initial_panels(st.t_lo - e0, st.t_lo, lambda, {},
                                      [s0](double) { return s0; }, budget_max);
          if (st.panels.size() + fresh.size() > budget_max) {
            stop = true;
          } else {
            st.t_lo -= e0;
            st.extensions[0] += 1;
            std::vector<Panel> nw;
            for (auto& ab : fresh) nw.push_back({ab.first, ab.second});
            for (auto& pn : st.panels) nw.push_back(std::move(pn));
            st.panels.swap(nw);
            extended = true;
          }
        }
        if (!stop && w1) {
          auto fresh = initial_panels(st.t_hi, st.t_hi + e1, lambda, {},
                                      [s1](double) { return s1; }, budget_max);
          if (st.panels.size() + fresh.size() > budget_max) {
            stop = true;
          } else {
            st.t_hi += e1;
            st.extensions[1] += 1;
            for (auto& ab : fresh) st.panels.push_back({ab.first, ab.second});
            extended = true;
          }
        }
        if (stop || !extended) finish();
        continue;
      }
      // Split every panel above its share of a target still missed, worst first.
      std::vector<std::pair<double, size_t>> cand;
      for (size_t i = 0; i < n; ++i) {
        if (!(st.panels[i].b - st.panels[i].a > kMinWidth)) continue;
        double bad = 0.0;
        for (size_t p = 0; p < np; ++p)
          for (size_t j = 0; j < stat[p].target.size(); ++j) {
            if (!(stat[p].errors[j] > stat[p].target[j])) continue;
            const double t = std::max(stat[p].target[j], std::numeric_limits<double>::min());
            bad = std::max(bad, st.panels[i].sums[p].err()[j] * (double)n / t);
          }
        if (bad > 1.0) cand.push_back({bad, i});
      }
      const size_t budget = budget_max > n ? budget_max - n : 0;
      if (cand.empty() || budget == 0) {
        finish();
        continue;
      }
      std::sort(cand.begin(), cand.end(), [](const auto& x, const auto& y) {
        return x.first != y.first ? x.first > y.first : x.second < y.second;
      });
      if (cand.size() > budget) cand.resize(budget);
      std::vector<char> split(n, 0);
      for (auto& c : cand) split[c.second] = 1;
      std::vector<Panel> next;
      next.reserve(n + cand.size());
      for (size_t i = 0; i < n; ++i) {
        if (split[i]) {
          const double a = st.panels[i].a, b = st.panels[i].b, mid = 0.5 * (a + b);
          next.push_back({a, mid});
          next.push_back({mid, b});
        } else {
          next.push_back(std::move(st.panels[i]));
        }
      }
      st.panels.swap(next);
    }
  }
}

}  // namespace adaptive
}  // namespace sb
