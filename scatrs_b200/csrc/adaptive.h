// Host side of the adaptive ensemble (the reference's default integration,
// scatrs/src/ensemble/engine.rs pass 1 with range.rs, moments.rs and kronrod.rs): the parts of
// a call, their cut-offs and moments, and pass 1's panels, refined round by round. The node
// evaluations of every round of every (group, wavelength) job go to the device in one batch
// through the `Evaluate` callback; pass 2 then runs on the final panels' nodes.
#pragma once

#include <array>
#include <cstdint>
#include <functional>
#include <string>
#include <utility>
#include <vector>

namespace sb {
namespace adaptive {

constexpr int kMonodisperse = 5;  // a single radius (param[0])
constexpr int kPass1 = 6;         // 1, C_ext, C_sca, C_sca g, C_back, C_abs (engine.rs:43-54)
constexpr int kGroup = 5;         // per direction: d of C_ext, C_sca, C_sca g, C_back, C_abs
// The particle's directions (particle.rs:119-145): Re m and Im m, and a spheroid's aspect ratio.
constexpr int kMaxDirs = 3;
constexpr int kSphereQ = kPass1 + 2 * kGroup;       // a sphere node's quantities with Re m, Im m
constexpr int kNodeQ = kPass1 + kMaxDirs * kGroup;  // a node's quantities with every direction
constexpr int kMaxAllDirs = 3 * 16 - 1;             // the most directions: a 16-layer sphere's

struct Error {
  int status;
  std::string msg;
};

enum Support { UNBOUNDED, FINITE, POINT };

struct Moments {
  double v[2] = {0, 0}, e[2] = {0, 0};  // <r^2>, <r^3> and their error estimates
  double z = 1.0, ez = 0.0;             // the normalization Z = integral of u dr
  // Along each requested distribution parameter (moments.rs:15-26): d<r^2>, d<r^3> and their
  // error estimates, dZ and its error estimate.
  std::vector<std::array<double, 2>> d, de;
  std::vector<double> dz, dez;
};

// One distribution of a call (engine.rs:95-115 Part; the mixing weights live with the caller).
struct Part {
  int kind = 0;
  double p[3] = {0, 0, 0};
  // The requested distribution parameters (indices into the density's gradient, in the order
  // of their result columns) and the requested derivatives along Re m, Im m and (a spheroid)
  // the aspect ratio.
  std::vector<int> grads;
  // A layered sphere has 3 L - 1 directions (each layer's Re m and Im m, then each radius
  // fraction, particle.rs:119-145).
  std::vector<char> dirs = std::vector<char>(kMaxDirs, 0);
  bool dir_derivatives() const {
    for (char d : dirs)
      if (d) return true;
    return false;
  }
  // The pass-1 quantities (engine.rs:464-471): the base ones, then kGroup per requested
  // direction.
  int n_refined() const {
    int k = 0;
    for (char d : dirs) k += d ? 1 : 0;
    return kPass1 + kGroup * k;
  }
  double reference = 1.0, log_width = 0.0;  // distribution.rs:292-336
  Support support = UNBOUNDED;
  double lo = 0.0, hi = 0.0;  // the Mie range before extensions (a point: r, r)
  Moments mom;
  std::vector<double> table;  // a tabulated distribution's [radii..., densities...]
  double u(double r) const;  // the unnormalized density
  double u(double r, double grad[3]) const;  // and its gradient along the parameters
  // The radii that are panel edges (engine.rs:181-184, 738-751): a finite support's ends and a
  // table's points.
  std::vector<double> breaks() const;
};

// Parses and prepares a part: validation, support, cut-offs (range.rs) and moments
// (moments.rs), the moments with their derivatives along `grads` (indices into the density's
// gradient). A tabulated distribution (kind 6) brings its table. Throws Error.
Part make_part(int kind, const double* p, double rtol, const double* table = nullptr,
               int64_t table_len = 0, const std::vector<int>& grads = {});

struct Options {
  double rtol = 1e-6;
  int64_t max_panels = 4096;
  bool allow_unvalidated = false;
  bool refine_backscatter = false;
};

// A node to evaluate: radius and wavelength index; the result: the pass-1 quantities, the
// number of terms, and a status (0 or the node's error).
struct Query {
  double r;
  int wl;
};
struct NodeResult {
  double q[kNodeQ];  // the kPass1 quantities, then kGroup derivatives along each direction
  // If set, the kGroup derivatives of every direction of the particle, in order, in place of
  // q's (a layered sphere's, more than kMaxDirs); owned by the evaluator until its next call.
  const double* dq = nullptr;
  int64_t n;
  int status;
  const char* msg = nullptr;  // with a status: the reason, if not the node's domain
};
using Evaluate = std::function<void(const std::vector<Query>&, std::vector<NodeResult>&)>;

// Pass 1 of one group of parts sharing panels at one wavelength.
struct Job {
  std::vector<int> parts;  // indices into the call's parts (none a point)
  int wl = 0;
  // results
  std::vector<std::pair<double, double>> panels;  // final panels in t = ln r
  std::vector<int64_t> panel_terms;               // each panel's largest number of terms
  std::vector<bool> converged;                    // per part
  int64_t n_terms = 0;
  int status = 0;  // the first node error in panel order, if any
  std::string msg;
};

// Runs pass 1 of every job in rounds; each round evaluates all jobs' new panels (15 GK nodes
// each) with one eval call.
void pass1(std::vector<Job>& jobs, const std::vector<Part>& parts, const double* wavelengths,
           const Options& o, const Evaluate& eval);

// The GK15 rule on [a, b] in t: nodes ascending with Kronrod and Gauss weights (kronrod.rs).
struct Node {
  double t, wk, wg;
};
void gk15(double a, double b, Node out[15]);

}  // namespace adaptive
}  // namespace sb
