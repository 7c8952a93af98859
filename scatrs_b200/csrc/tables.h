// Host-side tables shared by every launch: Gauss-Legendre rules, the generalized spherical
// functions of the projection, the pi/tau tables of the angle GEMMs, and the size
// distributions' densities. Compiled with -ffp-contract=off so that the tables hold the
// reference's doubles.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace sb {

// n-point Gauss-Legendre rule on [-1, 1], nodes ascending, exactly symmetric
// (scatrs/src/special/gauss_legendre.rs:188-260).
void gauss_legendre(int64_t n, double* nodes, double* weights);

// d^l_{mn}(x) for l = 0..len-1 and |m|, |n| <= 2 (scatrs/src/special/wigner.rs:152-184).
void wigner_d(int m, int n, double x, double* out, int64_t len);

// (w pi_n, w tau_n) at cosine mu for n = 1..n_max into ge/go split by parity: G_E holds w pi_n
// for odd n and w tau_n for even n, G_O the other (scatrs/src/ensemble/fast.rs:31-45 with
// scatrs/src/mie/amplitudes.rs:52-65).
void pi_tau_row(double mu, int64_t n_max, double* ge, double* go);

// The number of terms of the band containing n (engine.rs:951-957) and its index in the
// sequence 1, 2, 3, 4, 5, 7, 9, ...
int64_t bucket(int64_t n);
int band_index(int64_t n);
int64_t band_upper(int index);

// Size distributions (scatrs/src/ensemble/distribution.rs): validation and the unnormalized
// density u(r).
bool validate_distribution(int kind, const double* p, std::string* msg);
double density(int kind, const double* p, double r);
// Tabulated distributions (kind 6): table = [r_0..r_{n-1}, u_0..u_{n-1}], n(r) linear between
// the points and 0 outside them (distribution.rs:406-417); their checks
// (distribution.rs:149-171).
constexpr int kTabulated = 6;
double table_density(const double* table, int64_t n, double r);
bool validate_table(const double* table, int64_t n, std::string* msg);

// The number of a distribution kind's parameters (ensemble/mod.rs:254-337) and the gradient of
// u(r) along them at a fixed reference radius (distribution.rs:370-441); the reference radius'
// own dependence cancels in every average. Returns u(r).
int parameter_count(int kind);

// The reference radius, where the density is about 1, and the width of its peak in ln r
// (infinite for a power law): Density of distribution.rs:292-336.
struct DensityInfo {
  double reference, log_width;
};
DensityInfo density_info(int kind, const double* p);
double density_gradient(int kind, const double* p, double r, double grad[3]);

}  // namespace sb
