/*
 * scatrs_b200: the size-distribution ensemble path of usask-arg/scatrs on NVIDIA B200
 * (sm_100a), behind a C ABI.
 *
 * Every entry point takes plain pointers and sizes, returns a status code, and (on failure)
 * writes a message into a caller-owned buffer. The status codes mirror the reference's error
 * enum (scatrs/src/error.rs:17-32), as its Python binding maps them
 * (scatrs-py/src/errors.rs:14-45):
 *   0 OK, 1 INVALID_INPUT, 2 NOT_CONVERGED, 3 OUTSIDE_VALIDATED_DOMAIN,
 *   4 CUDA (a CUDA runtime error or a device-side wait that gave up), 5 NO_DEVICE.
 *
 * Units are distribution-major, like the reference's batch (scatrs-py/src/ensemble.rs:452-454):
 * unit u = d * n_wavelengths + i for distribution d and wavelength i.
 */
#ifndef SCATRS_B200_H
#define SCATRS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum scatrs_status {
  SCATRS_OK = 0,
  SCATRS_INVALID_INPUT = 1,
  SCATRS_NOT_CONVERGED = 2,
  SCATRS_OUTSIDE_VALIDATED_DOMAIN = 3,
  SCATRS_CUDA = 4,
  SCATRS_NO_DEVICE = 5
};

/* Distribution kinds, with the parameters in the order of the reference's tagged tuples
 * (scatrs-py/src/ensemble.rs:38-57; SizeDistribution, scatrs/src/ensemble/distribution.rs:15-66):
 *   LOGNORMAL (median_radius, width), GAMMA (effective_radius, effective_variance),
 *   MODIFIED_GAMMA (alpha, b, gamma), POWER_LAW (exponent, min_radius, max_radius). */
enum scatrs_distribution_kind {
  SCATRS_LOGNORMAL = 1,
  SCATRS_GAMMA = 2,
  SCATRS_MODIFIED_GAMMA = 3,
  SCATRS_POWER_LAW = 4,
  /* n(r) linear between table_len points (radii increasing and > 0, densities >= 0 and not all
   * 0), 0 outside them: table = [radii..., densities...] (distribution.rs:55-62, 406-417);
   * no parameters. */
  SCATRS_TABULATED = 6
};

/* One size distribution on a fixed grid: n_nodes Gauss-Legendre nodes in t = ln r over
 * [ln r_lo, ln r_hi] (the radius of a sphere). table / table_len: SCATRS_TABULATED only (NULL,
 * 0 otherwise). */
typedef struct scatrs_distribution {
  int32_t kind;
  int32_t reserved;
  double param[3];
  double r_lo;
  double r_hi;
  const double* table;
  int64_t table_len;
} scatrs_distribution;

/* Options of the fixed-grid ensemble. The reference's EnsembleOptions
 * (scatrs/src/ensemble/mod.rs:342-382) minus the adaptive controls (rtol, max_panels,
 * refine_*), which the fixed grid does not have. */
typedef struct scatrs_fixed_options {
  int32_t n_nodes;           /* radius nodes per distribution, >= 1 */
  int32_t greek_order;       /* highest Greek order L, or -1 for none */
  int32_t normalized;        /* 1: normalized phase matrix and Greek coefficients */
  int32_t allow_unvalidated; /* 1: compute outside the Mie validated domain */
} scatrs_fixed_options;

/* Sizes of the outputs of scatrs_ensemble_fixed for n_units units: the reference dict's arrays
 * (scatrs-py/src/ensemble.rs:289-294): values (11, n_units), phase (6, n_units, n_mu) and
 * greek (6, n_units, L + 1), in doubles. */
void scatrs_ensemble_fixed_sizes(int64_t n_units, int64_t n_mu, int32_t greek_order,
                                 int64_t* values_len, int64_t* phase_len, int64_t* greek_len);

/*
 * The fixed-grid ensemble of every (distribution, wavelength) unit, from HOST buffers into HOST
 * buffers (host-device copies included).
 *
 * Replaces compute_batch_with_particle (scatrs/src/ensemble/mod.rs:654-686), reached from Python
 * as _scatrs.ensemble_compute_batch (scatrs-py/src/ensemble.rs:455-504), for spheres, extended
 * to a refractive index per (distribution, wavelength) and to a fixed size grid: the pass-2
 * sums of scatrs/src/ensemble/engine.rs:1423-1766 on fixed nodes, the averages (1782-1836), the
 * band projection (2310-2355) and the assembly (2396-2497).
 *
 *   dists[n_dist], wavelengths[n_wl], m[2 * n_dist * n_wl] (complex128: re, im, unit-major),
 *   mu[n_mu] (cosines for the phase matrix; may be NULL with n_mu = 0),
 *   values[11 * n_units] (c_ext, c_sca, c_abs, c_back, ssa, g, lidar_ratio, depolarization,
 *   effective_radius, mean_area, mean_volume per unit), phase[6 * n_units * n_mu] (F11, F12,
 *   F22, F33, F34, F44) or NULL, greek[6 * n_units * (L + 1)] (alpha1..4, beta1, beta2) or NULL.
 */
int scatrs_ensemble_fixed(const scatrs_distribution* dists, int64_t n_dist,
                          const double* wavelengths, int64_t n_wl, const double* m,
                          const double* mu, int64_t n_mu, const scatrs_fixed_options* options,
                          double* values, double* phase, double* greek, char* err,
                          size_t err_len);

/*
 * scatrs_ensemble_fixed with the derivatives of every output (the reference's
 * `derivatives=True` of Ensemble.compute: compute_with_particle with derivative parameters,
 * scatrs/src/ensemble/mod.rs:254-337 for their order, engine.rs:1047-1200 per node,
 * 1782-1836 for the averages, ensemble/lin.rs for the ratios), for homogeneous spheres with
 * every distribution of one kind. The P = n_theta + 2 directions are the distribution's
 * parameters in ensemble_parameters order (lognormal: median_radius, width; gamma:
 * effective_radius, effective_variance; modified gamma: alpha, b, gamma; power law: exponent),
 * then Re m and Im m of the unit's own index. The size grid [r_lo, r_hi] is held fixed.
 *
 *   d_values[P * 11 * n_units], d_phase[P * 6 * n_units * n_mu] or NULL,
 *   d_greek[P * 6 * n_units * (L + 1)] or NULL: direction-major, each block laid out as the
 *   value arrays.
 */
int scatrs_ensemble_fixed_d(const scatrs_distribution* dists, int64_t n_dist,
                            const double* wavelengths, int64_t n_wl, const double* m,
                            const double* mu, int64_t n_mu, const scatrs_fixed_options* options,
                            double* values, double* phase, double* greek, double* d_values,
                            double* d_phase, double* d_greek, char* err, size_t err_len);

/* A single radius (SizeDistribution::Monodisperse, distribution.rs:50-53): param[0] the
 * radius. Adaptive calls only. */
#define SCATRS_MONODISPERSE 5

/* Options of the adaptive ensemble: the reference's EnsembleOptions (scatrs/src/ensemble/
 * mod.rs:342-382; defaults rtol 1e-6, max_panels 4096). */
typedef struct scatrs_adaptive_options {
  double rtol;                /* relative tolerance of the size integration, in [1e-13, 0.1] */
  int64_t max_panels;         /* panels per part and wavelength, >= 1 */
  int32_t greek_order;        /* highest Greek order L, -1 for none, or SCATRS_GREEK_ALL */
  int32_t normalized;         /* 1: normalized phase matrix and Greek coefficients */
  int32_t allow_unvalidated;  /* 1: compute outside the Mie validated domain */
  int32_t refine_backscatter; /* 1: also refine on <C_back> */
} scatrs_adaptive_options;

/* greek_order = SCATRS_GREEK_ALL (GreekOrder::All, ensemble/mod.rs:163-170): every order up to
 * 2 N_max at each wavelength (N_max the largest number of terms there, over every part of the
 * call: spheres, layered spheres and spheroids, alone or mixed). The call then leaves its greek
 * arrays unwritten; the coefficients of the calling
 * thread's last such call come from scatrs_greek_all_take, (6, n, W) and with derivatives
 * (P, 6, n, W) as the call's other outputs, W = scatrs_greek_all_width() the longest plus one,
 * zero above each wavelength's order (scatrs-py/src/ensemble.rs:419-429). */
#define SCATRS_GREEK_ALL (-2)
int64_t scatrs_greek_all_width(void);
int scatrs_greek_all_take(double* greek, double* greek_err, double* d_greek, double* d_greek_err);

/*
 * The adaptive ensemble of spheres, the reference's default integration: per distribution
 * (batch = 0: `compute`, scatrs/src/ensemble/mod.rs:548-606) or as one batch sharing panels per
 * wavelength (batch = 1: `compute_batch`, mod.rs:613-686), with the reference's tail cut-offs
 * (range.rs), moments (moments.rs), GK15 pass 1 refined on C_ext, C_sca, C_sca g, C_abs (and
 * C_back if asked) with range extensions, and pass 2 on the final panels with Kronrod sums and
 * |Kronrod - Gauss| error estimates (engine.rs:724-1836, 2310-2497). m is complex128 per
 * wavelength (one particle, as the reference's). Distributions as scatrs_distribution (r_lo,
 * r_hi unused) or SCATRS_MONODISPERSE. Outputs as scatrs_ensemble_fixed, each with its error
 * estimate in the *_err / errors array of the same layout; converged[n_units] (0/1) and
 * panels[n_units] (the shared panels of a batch; 0 for a single radius).
 */
int scatrs_ensemble_adaptive(const scatrs_distribution* dists, int64_t n_dist, int32_t batch,
                             const double* wavelengths, int64_t n_wl, const double* m,
                             const double* mu, int64_t n_mu,
                             const scatrs_adaptive_options* options, double* values,
                             double* errors, double* phase, double* phase_err, double* greek,
                             double* greek_err, int8_t* converged, int64_t* panels, char* err,
                             size_t err_len);

/* One component of a mixture (scatrs::ensemble::Component, ensemble/mod.rs:136-160): its
 * distribution, or the modes of a multimodal one (SizeDistribution::MultiModal,
 * distribution.rs:60-66) with their weights, its weight w in the mixture, and its particle
 * (Particle, ensemble/particle.rs): a homogeneous sphere (n_layers 0 or 1, aspect_ratio 0), a
 * layered sphere (n_layers > 1, its radius fractions) or a randomly oriented spheroid
 * (aspect_ratio > 0). */
typedef struct scatrs_component {
  const scatrs_distribution* modes; /* n_modes distributions (one for a plain distribution) */
  const double* mode_weights;       /* n_modes weights v_j of a multimodal one, or NULL */
  int32_t n_modes;
  int32_t n_layers;                 /* > 1: a layered sphere of n_layers layers */
  double weight;                    /* w */
  const double* m;                  /* complex128 per wavelength; layered: [n_layers][n_wl] */
  const double* fractions;          /* layered: the n_layers - 1 radius fractions, else NULL */
  double aspect_ratio;              /* > 0: a spheroid of this aspect ratio, else 0 */
} scatrs_component;

/*
 * The adaptive ensemble of an external mixture of sphere components (`compute_mixture`,
 * scatrs/src/ensemble/mod.rs:609-625; a multimodal distribution alone is a mixture of one
 * component): every mode of every component integrated on its own panels, the averages mixed
 * with the number fractions (w / sum w) (v_j / sum v) (engine.rs:2121-2176) before the ratios,
 * normalizations and the Greek projection. Outputs per wavelength as scatrs_ensemble_adaptive
 * with n_units = n_wl; converged when every part converged, panels summed over the parts.
 * Components of different particles (spheres, layered spheres, spheroids) are integrated by
 * their own engines and mixed on one layout (engine.rs:1964-2250): the spheres' tables and
 * projected Greek coefficients, the spheroids' direct Greek segment (to the largest 2 N of the
 * mixture's spheroids at each wavelength), the depolarization ratio from the spheroids, and the
 * phase matrix from the spheres' tables plus the spheroids' averaged expansion. Such mixtures
 * take their derivatives through scatrs_ensemble_mixture_d; with SCATRS_GREEK_ALL each
 * wavelength's order is 2 N_max over every part.
 */
int scatrs_ensemble_mixture(const scatrs_component* components, int64_t n_comp,
                            const double* wavelengths, int64_t n_wl, const double* mu,
                            int64_t n_mu, const scatrs_adaptive_options* options, double* values,
                            double* errors, double* phase, double* phase_err, double* greek,
                            double* greek_err, int8_t* converged, int64_t* panels, char* err,
                            size_t err_len);

/* A parameter to differentiate the outputs with respect to (scatrs::ensemble::EnsembleParam,
 * ensemble/mod.rs:180-215): the mixture component (0 for a single distribution), the mode of a
 * multimodal distribution (-1 when the component's distribution is not multimodal, or for its
 * refractive index and its weight), the kind, and for a distribution parameter its index in the
 * distribution's parameter list (SizeDistribution::parameter_names: lognormal median_radius,
 * width; gamma effective_radius, effective_variance; modified gamma alpha, b, gamma; power law
 * exponent). */
enum {
  SCATRS_PARAM_DISTRIBUTION = 0, /* ParamKind::Distribution(name) */
  SCATRS_PARAM_REFR_REAL = 1,    /* ParamKind::RefrReal */
  SCATRS_PARAM_REFR_IMAG = 2,    /* ParamKind::RefrImag */
  SCATRS_PARAM_WEIGHT = 3,       /* ParamKind::Weight: a component's (mode -1) or a mode's */
  SCATRS_PARAM_ASPECT_RATIO = 4,     /* ParamKind::AspectRatio: a spheroid component's */
  SCATRS_PARAM_LAYER_REFR_REAL = 5,  /* ParamKind::LayerRefrReal(index): layer index's Re m */
  SCATRS_PARAM_LAYER_REFR_IMAG = 6,  /* ParamKind::LayerRefrImag(index) */
  SCATRS_PARAM_RADIUS_FRACTION = 7   /* ParamKind::RadiusFraction(index), index < n_layers - 1 */
};
typedef struct scatrs_param {
  int32_t component;
  int32_t mode;
  int32_t kind;
  int32_t index;
} scatrs_param;

/*
 * scatrs_ensemble_mixture with the derivatives of every output along `params`
 * (EnsembleOptions::derivatives; the adaptive engine's derivative blocks, engine.rs:1370-1380,
 * 1782-1836, 2121-2176): each pass refines and integrates the requested distribution parameters'
 * blocks (weights du/dtheta r) and the derivatives along Re m and Im m, the averages follow
 * the quotient rule against the moments' dZ, the mixing adds the weight derivatives, and the
 * ratios carry the derivatives with first-order error estimates (ensemble/lin.rs). A component
 * is multimodal when its mode_weights are given. Spheres; or one spheroid component of one
 * distribution, along its distribution's parameters, Re m, Im m and the aspect ratio
 * (SCATRS_PARAM_ASPECT_RATIO), each node's derivatives those of its solution at its converged N
 * and n_theta (engine.rs:379-471, 1281-1340 direct path); or one layered component, along its
 * distribution's parameters, each layer's Re m and Im m and each radius fraction
 * (SCATRS_PARAM_LAYER_REFR_REAL/_IMAG, SCATRS_PARAM_RADIUS_FRACTION; validated up to
 * x_L = 1000, layered/domain.rs:39-70); or a mixture of different particles along any of
 * its components' parameters and weights (each part on its own engine, mixed and assembled on
 * the host). A single sphere radius's radius is
 * exact (engine.rs:1158-1170), with zero error estimates; a single spheroid's follows
 * monodisperse_direct (engine.rs:1896-1961). d_values, d_errors (P, 11, n_wl); d_phase, d_phase_err (P, 6, n_wl, n_mu); d_greek,
 * d_greek_err (P, 6, n_wl, L + 1), P = n_params, in the order of `params`. Invalid or
 * repeated parameters: SCATRS_INVALID_INPUT naming the parameter.
 * Replaces: the derivative path of Mixture::compute / Ensemble.compute(derivatives=...)
 * (scatrs/src/ensemble/mod.rs:548-625; scatrs-py/src/ensemble.rs:295-349 deriv_idx).
 */
int scatrs_ensemble_mixture_d(const scatrs_component* components, int64_t n_comp,
                              const double* wavelengths, int64_t n_wl, const double* mu,
                              int64_t n_mu, const scatrs_adaptive_options* options,
                              const scatrs_param* params, int64_t n_params, double* values,
                              double* errors, double* d_values, double* d_errors, double* phase,
                              double* phase_err, double* d_phase, double* d_phase_err,
                              double* greek, double* greek_err, double* d_greek,
                              double* d_greek_err, int8_t* converged, int64_t* panels, char* err,
                              size_t err_len);

/*
 * The Greek coefficients of phase matrices tabulated at the n_q Gauss-Legendre cosines
 * (ascending, the rule of scatrs_gauss_legendre), projected with the reference's projector
 * (2l+1)/2 w_k d_l(mu_k) (scatrs/src/mie/greek.rs:131-335; the band projection of
 * scatrs/src/ensemble/fast.rs:210-271 on one rule): exact for tables of polynomial degree up to
 * 2 n_q - 1 - order. phase_dev [6][n_units][n_q] as scatrs_ensemble_fixed_device writes it
 * (F11, F12, F22, F33, F34, F44), greek_dev [6][n_units][order + 1]; DEVICE pointers, enqueued
 * on `stream`. precision 0: FP64; 1: 3xTF32 on the tensor cores (each operand a TF32 head and
 * tail, FP32 accumulation over the cosines: about 1e-5 of the largest coefficient at order
 * 1000 and 4096 cosines, less at lower orders). Returns after the FP64 form
 * is enqueued, or after the tensor-core form completed (it checks its pipeline).
 */
int scatrs_project_greek_device(const double* phase_dev, int64_t n_units, int64_t n_q,
                                int32_t order, int32_t precision, double* greek_dev,
                                void* stream, char* err, size_t err_len);

/*
 * Spheroids by the extended boundary condition method (scatrs/src/tmatrix; Shape::Spheroid,
 * aspect ratio eps = a/c > 1 oblate; x the equal-volume sphere's size parameter; m complex128).
 *
 * scatrs_spheroid_tmatrix: the T-matrix of azimuthal mode `mode` at truncation n_terms and
 * n_theta Gauss nodes in 0 < theta < pi/2 (TMatrix::compute with fixed N and n_theta,
 * tmatrix/mod.rs:221-362, kernel.rs:516-563): t[2 (2K)^2], row-major complex (2K)^2 with
 * K = n_terms - max(mode, 1) + 1 and blocks [T11 T12; T21 T22].
 *
 * scatrs_spheroid_efficiencies: the orientation-averaged Q_ext, Q_sca, Q_abs of n spheroids
 * (q[3 n]), converged in N and n_theta to rtol as driver.rs:343-420 converges them on mode 0,
 * then every mode at the final N (n_terms[n], n_theta[n] the values used; either may be NULL).
 * Status 2 when N reaches its cap, or n_theta its cap 4 theta(start) + 40 (mod.rs:293-300).
 * The surface integrals are the classical ones from the definition, assembled in double-double
 * (about 106 bits) against their cancellation, then solved in FP64 with double-double residual
 * refinement (the last sweep's relative correction is below 2^-54 on return): T agrees with a
 * quadruple-precision EBCM to about 1e-26 of its largest element on the reference's records.
 * Where the cancellation exceeds double-double's reach (about 1e28: aspect ratios near 0.4 or 3
 * at size parameters above about 17), the N loop does not settle and status 2 is returned.
 */
int scatrs_spheroid_tmatrix(double x, double aspect_ratio, const double* m, int32_t mode,
                            int32_t n_terms, int32_t n_theta, double* t, char* err,
                            size_t err_len);
int scatrs_spheroid_efficiencies(int64_t n, const double* x, const double* aspect_ratio,
                                 const double* m, double rtol, double* q, int32_t* n_terms,
                                 int32_t* n_theta, char* err, size_t err_len);

/*
 * Randomly oriented spheroids (TMatrix::compute and its solution's efficiencies() and greek(),
 * tmatrix/mod.rs:221-362, 437-491; the orientation average random.rs:85-335): n spheroids in one
 * batch. n_terms / n_theta > 0 fix N / n_theta (TMatrixOptions::n_terms, n_theta), 0 converges
 * them to rtol. eff[5 n]: Q_ext, Q_sca, Q_abs, Q_back, g (Q_back and g from the averaged Greek
 * expansion, exact to 2N). greek[6 n (greek_order + 1)] (alpha1..alpha4, beta1, beta2, each
 * zero above 2N), normalized (alpha1_0 = 1) or unnormalized (times Q_sca); greek_order -1 for
 * none. n_terms, n_theta, error_estimate (the largest relative correction of the last refinement
 * sweep over the modes) may be NULL. N is limited to 120 here.
 */
/*
 * scatrs_ensemble_adaptive for randomly oriented spheroids (Particle::Spheroid on the default
 * adaptive engine, its direct path): one aspect ratio, m per wavelength, the outputs and batch
 * semantics of scatrs_ensemble_adaptive. Pass 1 solves every node's T-matrix (to rtol / 100
 * clamped to [1e-12, 1e-8]) and its orientation average on the GPU in batches; pass 2
 * integrates those values with their declared errors (4 or 16 times max(rtol_T, the solution's
 * estimate), tmatrix/domain.rs) without solving again. The phase matrix comes from the averaged
 * Greek expansion (every order to 2N).
 */
int scatrs_ensemble_adaptive_spheroid(const scatrs_distribution* dists, int64_t n_dist,
                                      int32_t batch, const double* wavelengths, int64_t n_wl,
                                      double aspect_ratio, const double* m, const double* mu,
                                      int64_t n_mu, const scatrs_adaptive_options* options,
                                      double* values, double* errors, double* phase,
                                      double* phase_err, double* greek, double* greek_err,
                                      int8_t* converged, int64_t* panels, char* err,
                                      size_t err_len);

typedef struct scatrs_spheroid_options {
  double rtol;
  int32_t n_terms;
  int32_t n_theta;
  int32_t greek_order;
  int32_t normalized;
  /* 1: compute outside the spheroids' validated domain (tmatrix/domain.rs:45-79: aspect ratio
   * 0.2-5, x >= 1e-6, |m| x_max <= 60, 1.3 <= Re m <= 3, Im m <= 0.5, rtol >= 1e-12); else such
   * a spheroid returns SCATRS_OUTSIDE_VALIDATED_DOMAIN (TMatrix::compute, tmatrix/mod.rs:280-292) */
  int32_t allow_unvalidated;
} scatrs_spheroid_options;

int scatrs_spheroid_compute(int64_t n, const double* x, const double* aspect_ratio,
                            const double* m, const scatrs_spheroid_options* options, double* eff,
                            double* greek, int32_t* n_terms, int32_t* n_theta,
                            double* error_estimate, char* err, size_t err_len);

/*
 * scatrs_spheroid_compute with the derivatives of every output along x, the aspect ratio, Re m
 * and Im m (TMatrix::compute_with_derivatives, tmatrix/mod.rs:231-245, with the efficiencies'
 * Jacobian and greek_with_derivatives, mod.rs:695-760): the derivatives of the solution at each
 * spheroid's converged N and n_theta, as the reference takes them. They come from the outputs
 * solved at perturbed parameters at the same (N, n_theta), in one batch with the values: central
 * differences at steps h and h/2 (h = 1e-4 of the parameter, of |m| for m), Richardson-
 * extrapolated, and a one-sided fourth-order stencil along Im m when Im m < 4h (Im m cannot go
 * below zero); accurate to about 1e-9 of each output's scale (the reference's dual numbers are
 * exact to rounding). eff, greek as scatrs_spheroid_compute's (their values at that N and
 * n_theta); d_eff[4][n][5] and d_greek[4][n][6 (greek_order + 1)], direction-major in the order
 * x, aspect ratio, Re m, Im m. Seventeen solutions of every mode per spheroid.
 */
int scatrs_spheroid_compute_d(int64_t n, const double* x, const double* aspect_ratio,
                              const double* m, const scatrs_spheroid_options* options,
                              double* eff, double* greek, double* d_eff, double* d_greek,
                              int32_t* n_terms, int32_t* n_theta, double* error_estimate,
                              char* err, size_t err_len);

/*
 * The fixed-grid ensemble of randomly oriented spheroids (Particle::Spheroid; the engine's
 * direct path, engine.rs:1207-1339, 2192-2216, 2359-2497): each distribution's nodes as
 * scatrs_ensemble_fixed's, one aspect ratio per distribution (aspect_ratio[n_dist]) and m per
 * (distribution, wavelength) unit (complex128, distribution-major). Every node's spheroid is
 * converged to tmatrix_rtol (the reference uses its ensemble rtol / 100 clamped to
 * [1e-12, 1e-8], engine.rs:87) in one batch of GPU work with its orientation average; the
 * unit's averages, ratios (the depolarization ratio from Q_back - Q_sca F22(180 deg)) and Greek
 * coefficients follow, and the phase matrix at mu from the averaged Greek expansion (every order
 * to 2N). Outputs as scatrs_ensemble_fixed's (values [11][n_units], phase [6][n_units][n_mu],
 * greek [6][n_units][L+1]); node_terms[n_units][n_nodes][2] (N, n_theta per node) may be NULL.
 */
int scatrs_ensemble_fixed_spheroid(const scatrs_distribution* dists, int64_t n_dist,
                                   const double* wavelengths, int64_t n_wl,
                                   const double* aspect_ratio, const double* m, const double* mu,
                                   int64_t n_mu, const scatrs_fixed_options* options,
                                   double tmatrix_rtol, double* values, double* phase,
                                   double* greek, int32_t* node_terms, char* err,
                                   size_t err_len);

/*
 * scatrs_ensemble_fixed_spheroid with the derivatives of every output (the directions of a
 * spheroid's solution, ensemble/particle.rs:142-237 with tmatrix/mod.rs:231-245, through the
 * averages and the ratios of engine.rs:1782-1836, 2396-2497): P = n_theta + 3 directions, the
 * distribution's parameters (every distribution of one kind; the size grid held fixed), then the
 * aspect ratio of the unit's distribution, Re m and Im m of the unit's index. Each node's
 * derivatives along the aspect ratio and m are those of its solution at its converged N and
 * n_theta (scatrs_spheroid_compute_d), the weights' along the parameters are exact, and the
 * averages, the ratios, the Greek coefficients and the phase matrix carry them in forward mode.
 * The values equal scatrs_ensemble_fixed_spheroid's. d_values[P][11][n_units], d_phase
 * [P][6][n_units][n_mu] and d_greek[P][6][n_units][L + 1], required beside their value arrays.
 */
int scatrs_ensemble_fixed_spheroid_d(const scatrs_distribution* dists, int64_t n_dist,
                                     const double* wavelengths, int64_t n_wl,
                                     const double* aspect_ratio, const double* m,
                                     const double* mu, int64_t n_mu,
                                     const scatrs_fixed_options* options, double tmatrix_rtol,
                                     double* values, double* phase, double* greek,
                                     double* d_values, double* d_phase, double* d_greek,
                                     int32_t* node_terms, char* err, size_t err_len);

/* Layered spheres (scatrs/src/layered/mod.rs; Particle::LayeredSphere,
 * scatrs/src/ensemble/mod.rs:58-65): n_layers layers, the core first; per distribution the
 * n_layers - 1 outer radii of layers 0..L-2 as fractions of the particle's radius (nondecreasing
 * in (0, 1]), and each layer's index per distribution and wavelength. One layer is a
 * homogeneous sphere (m then as in scatrs_ensemble_fixed). */
typedef struct scatrs_layers {
  int32_t n_layers;
  int32_t reserved;
  const double* fractions; /* [n_dist][n_layers - 1] */
  const double* m;         /* complex128 [n_dist][n_layers][n_wl] */
} scatrs_layers;

/*
 * scatrs_ensemble_fixed for layered spheres (at most 16 layers): the per-node solve is
 * Layered::compute (scatrs/src/layered/mod.rs:137-160, kernel.rs:308-465) at x_l = f_l x
 * (scatrs/src/ensemble/particle.rs:186-195); everything after the coefficients is the sphere's.
 */
int scatrs_ensemble_fixed_layered(const scatrs_distribution* dists, int64_t n_dist,
                                  const double* wavelengths, int64_t n_wl,
                                  const scatrs_layers* layers, const double* mu, int64_t n_mu,
                                  const scatrs_fixed_options* options, double* values,
                                  double* phase, double* greek, char* err, size_t err_len);

/*
 * scatrs_ensemble_fixed_layered with the derivatives (forward mode, as scatrs_ensemble_fixed_d)
 * along the distribution's parameters, then Re m_l and Im m_l of every layer l (each unit's
 * own index at its wavelength), then the radius fractions f_1..f_{L-1} (n_layers >= 2; every
 * distribution of one kind): P = n_theta + 3 L - 1 blocks, d_values [P][11][n], d_phase
 * [P][6][n][n_mu], d_greek [P][6][n][L+1]. The layered recursion carries its derivatives
 * (layered/kernel.rs's solve and its derivatives); one pass of the derivative pipeline per
 * layer index and per fraction.
 */
int scatrs_ensemble_fixed_layered_d(const scatrs_distribution* dists, int64_t n_dist,
                                    const double* wavelengths, int64_t n_wl,
                                    const scatrs_layers* layers, const double* mu, int64_t n_mu,
                                    const scatrs_fixed_options* options, double* values,
                                    double* phase, double* greek, double* d_values,
                                    double* d_phase, double* d_greek, char* err,
                                    size_t err_len);

/*
 * scatrs_ensemble_adaptive for layered spheres (Particle::LayeredSphere on the default adaptive
 * engine): the layers as scatrs_ensemble_fixed_layered takes them (per distribution), the
 * outputs and batch semantics of scatrs_ensemble_adaptive.
 */
int scatrs_ensemble_adaptive_layered(const scatrs_distribution* dists, int64_t n_dist,
                                     int32_t batch, const double* wavelengths, int64_t n_wl,
                                     const scatrs_layers* layers, const double* mu, int64_t n_mu,
                                     const scatrs_adaptive_options* options, double* values,
                                     double* errors, double* phase, double* phase_err,
                                     double* greek, double* greek_err, int8_t* converged,
                                     int64_t* panels, char* err, size_t err_len);


/*
 * As scatrs_ensemble_fixed, with every array in DEVICE memory of the current device, launched
 * on `stream` (a cudaStream_t, or NULL for the default stream). Returns after the work is
 * enqueued and the launch checks passed; input errors found on the device (a size node outside
 * the accepted or validated range) are reported by the NEXT call of scatrs_check_errors, which
 * synchronizes the stream.
 */
int scatrs_ensemble_fixed_device(const scatrs_distribution* dists_host, int64_t n_dist,
                                 const double* wavelengths_dev, int64_t n_wl,
                                 const double* m_dev, const double* mu_host, int64_t n_mu,
                                 const scatrs_fixed_options* options, double* values_dev,
                                 double* phase_dev, double* greek_dev, void* stream, char* err,
                                 size_t err_len);

/* Options of the mixed form: chunks with i8_above < N_c <= 4096 take the int8 path (i8_above
 * <= 0: none); levels, the product levels kept (i + j < levels): 5 (15 digit products), 6 (19),
 * or 0 for 5. */
typedef struct scatrs_mixed_options {
  int32_t i8_above;
  int32_t levels;
} scatrs_mixed_options;

/*
 * The mixed form of scatrs_ensemble_fixed / scatrs_ensemble_fixed_device (values; homogeneous
 * spheres): the angle GEMMs that replace the reference's FP64 band products
 * (PanelProducts::multiply, scatrs/src/ensemble/fast.rs:141-145) run, for every chunk of 32
 * nodes whose largest number of terms N_c satisfies i8_above < N_c <= 4096, as exact integer
 * products on the tensor cores: each table row and each coefficient column is a 40-bit
 * fixed-point integer with its own power-of-two scale, split into five balanced signed bytes,
 * and the digit products of the leading levels (i + j < levels) are summed exactly in INT32
 * (tcgen05.mma kind::i8); every product term keeps about 2^-38 (5 levels) of its row's largest
 * |table| value times its column's largest |coefficient|, the dropped terms centred on zero.
 * The Mie coefficients, the elements, the weighted sums, the projection and the outputs are
 * FP64 as in the plain form; chunks at or below i8_above run the plain FP64 path. mixed NULL or
 * i8_above <= 0 is the plain form exactly. This form has no counterpart in the reference, whose
 * band products are FP64 GEMMs.
 */
int scatrs_ensemble_fixed_mixed(const scatrs_distribution* dists, int64_t n_dist,
                                const double* wavelengths, int64_t n_wl, const double* m,
                                const double* mu, int64_t n_mu,
                                const scatrs_fixed_options* options,
                                const scatrs_mixed_options* mixed, double* values,
                                double* phase, double* greek, char* err, size_t err_len);
int scatrs_ensemble_fixed_mixed_device(const scatrs_distribution* dists_host, int64_t n_dist,
                                       const double* wavelengths_dev, int64_t n_wl,
                                       const double* m_dev, const double* mu_host, int64_t n_mu,
                                       const scatrs_fixed_options* options,
                                       const scatrs_mixed_options* mixed, double* values_dev,
                                       double* phase_dev, double* greek_dev, void* stream,
                                       char* err, size_t err_len);

/*
 * scatrs_ensemble_fixed_d and scatrs_ensemble_fixed_layered_d with DEVICE arrays for the index
 * (m_dev: complex [n_dist][n_wl]; layers->m: complex [n_dist][L][n_wl] in device memory, the
 * fractions on the host), the wavelengths and every output (laid out as the host entries';
 * phase and greek arrays required when n_mu > 0 and L >= 0), run on `stream` (a cudaStream_t or
 * NULL), which they synchronize before returning, device-side input errors included. For
 * callers whose inputs and outputs live on the GPU (the torch autograd layer): only the
 * distributions, the cosines and the fractions cross from the host.
 */
int scatrs_ensemble_fixed_d_device(const scatrs_distribution* dists_host, int64_t n_dist,
                                   const double* wavelengths_dev, int64_t n_wl,
                                   const double* m_dev, const double* mu_host, int64_t n_mu,
                                   const scatrs_fixed_options* options, double* values_dev,
                                   double* phase_dev, double* greek_dev, double* d_values_dev,
                                   double* d_phase_dev, double* d_greek_dev, void* stream,
                                   char* err, size_t err_len);
int scatrs_ensemble_fixed_layered_d_device(const scatrs_distribution* dists_host,
                                           int64_t n_dist, const double* wavelengths_dev,
                                           int64_t n_wl, const scatrs_layers* layers,
                                           const double* mu_host, int64_t n_mu,
                                           const scatrs_fixed_options* options,
                                           double* values_dev, double* phase_dev,
                                           double* greek_dev, double* d_values_dev,
                                           double* d_phase_dev, double* d_greek_dev,
                                           void* stream, char* err, size_t err_len);

/* Refractive-index models m(lambda) (python/scatrs/refractive.py:168-354), evaluated on the
 * device:
 *   SCATRS_M_CONSTANT      m = p[0] + i p[1]; parameters n, k
 *   SCATRS_M_TABLE         n points: table = wavelengths[n] then m as (re, im) pairs[n],
 *                          interpolated linearly in lambda (np.interp); no parameters
 *   SCATRS_M_TABLE_LOG_K   the same with ln Im m interpolated (Im m > 0 at every point)
 *   SCATRS_M_CAUCHY        n = p[0] + p[1] / lambda^2 + p[2] / lambda^4, Im m = p[3];
 *                          parameters A, B, C, k
 *   SCATRS_M_SELLMEIER     n^2 = 1 + sum_i B_i lambda^2 / (lambda^2 - C_i), Im m = p[3], n terms:
 *                          table = B[n] then C[n]; parameters B_0.., C_0.., k
 * A model given as a Python function (refractive.py:357-368) is evaluated by the caller. */
enum scatrs_refractive_kind {
  SCATRS_M_CONSTANT = 0,
  SCATRS_M_TABLE = 1,
  SCATRS_M_TABLE_LOG_K = 2,
  SCATRS_M_CAUCHY = 3,
  SCATRS_M_SELLMEIER = 4
};
typedef struct scatrs_refractive_model {
  int32_t kind;
  int32_t n;
  double p[4];
  const double* table; /* host memory, as above */
} scatrs_refractive_model;

/* The number of parameters of a model (-1 for an unknown kind). */
int scatrs_refractive_parameter_count(const scatrs_refractive_model* model);

/* m of every model at every wavelength into m_dev (complex [n_models][n_wl], device) and, when
 * dm_dev is not NULL, dm/dtheta into dm_dev (complex [n_models][p_max][n_wl], zero past each
 * model's own parameters), with the checks and messages of refractive.py (a wavelength outside a
 * table's range, Sellmeier's n^2 not positive, the first failure in (model, wavelength) order).
 * Runs on `stream` and synchronizes it. */
int scatrs_refractive_index_device(const scatrs_refractive_model* models, int64_t n_models,
                                   const double* wavelengths_dev, int64_t n_wl, double* m_dev,
                                   double* dm_dev, int32_t p_max, void* stream, char* err,
                                   size_t err_len);

/* Synchronizes `stream` and returns the first device-side input error of the last
 * scatrs_ensemble_fixed_device call on it (in wavelength, distribution, radius order). */
int scatrs_check_errors(void* stream, char* err, size_t err_len);

/*
 * Mie coefficients of independent spheres, from HOST buffers: the batched Mie::compute
 * (scatrs/src/mie/mod.rs:227-271; State::prepare and State::finish,
 * scatrs/src/mie/kernel.rs:249-559) and MieSolution::efficiencies
 * (scatrs/src/mie/efficiencies.rs:164-187).
 *
 *   x[n], m[2 * n]; n_terms[n] receives the number of terms N of each sphere (the default
 *   truncation ceil(x + 6 x^(1/3) + 3)); coeffs (may be NULL) receives, for sphere s, a_1..a_N
 *   then b_1..b_N as complex pairs from offset 4 * coeff_offset[s] doubles, where coeff_offset is
 *   the caller's exclusive prefix sum of the n_terms of the first call (call once with
 *   coeffs = NULL to size it); eff[5 * n] (may be NULL) receives Q_ext, Q_sca, Q_abs, Q_back, g.
 */
int scatrs_mie(const double* x, const double* m, int64_t n, int32_t allow_unvalidated,
               int64_t* n_terms, const int64_t* coeff_offset, double* coeffs, double* eff,
               char* err, size_t err_len);

/*
 * The batched Mie solve of scatrs_mie without any allocation, for callers that cannot call
 * cudaMalloc (a plugin inside a host process whose pool owns every device allocation, or a
 * loop that must not risk an allocation failure or the implicit synchronization of
 * cudaMalloc/cudaFree). This entry point has no counterpart in the reference.
 *
 * Every array is in DEVICE memory of the current device and is the caller's: x[n], m[2 * n],
 * coeff_offset[n] (the exclusive prefix sum of the terms N_s = ceil(x_s + 6 x_s^(1/3) + 3)),
 * n_terms[n], coeffs[4 * total_terms] (laid out as in scatrs_mie), eff[5 * n] or NULL;
 * total_terms is the sum of the N_s. The recurrences' scratch is a fixed 12 MiB array compiled
 * into the library (every GPU that loads it holds the array until exit): calls needing more than
 * its 524288 rows (total_terms + 2 n) are rejected with SCATRS_INVALID_INPUT. A sphere whose N_s
 * terms (the device's own count) start below 0, reach the next sphere's offset or pass
 * total_terms is rejected with SCATRS_INVALID_INPUT before it writes anything; on any error the
 * outputs' contents are unspecified, but nothing is written outside [0, total_terms) terms. The
 * first call on a device (and the first after its current CUDA context changed) resolves the
 * array's address with that device current, so make it before any stream capture. All calls
 * on a device share the array: calls that overlap on the GPU race on it.
 * Runs on `stream` (a cudaStream_t, or NULL) and synchronizes it before returning.
 */
int scatrs_mie_static(const double* x, const double* m, int64_t n, int32_t allow_unvalidated,
                      int64_t total_terms, int64_t* n_terms, const int64_t* coeff_offset,
                      double* coeffs, double* eff, void* stream, char* err, size_t err_len);

/* The accuracy reached and the accuracy requested of the last call on this thread that failed
 * with SCATRS_NOT_CONVERGED (scatrs::Error::NotConverged { achieved, requested },
 * scatrs/src/error.rs:22-28, which the reference's binding passes to NotConvergedError,
 * scatrs-py/src/errors.rs:24-31): returns 1 and writes both when the last call on this thread
 * returned SCATRS_NOT_CONVERGED, else returns 0 and writes NaN. */
int scatrs_not_converged_detail(double* achieved, double* requested);

/* Test hooks, not part of the API (the reference's scatrs._scatrs._testing,
 * scatrs-py/src/testing.rs:29-57):
 * scatrs_testing_raise fails with `status` (1-5), `message` and, for SCATRS_NOT_CONVERGED,
 *   `achieved`/`requested`, through the same error path as every entry point (the status, the
 *   message buffer and scatrs_not_converged_detail); status 0 returns SCATRS_OK.
 * scatrs_testing_fail_allocation(k): the k-th device buffer growth from now fails as an
 *   out-of-memory cudaMalloc would (SCATRS_CUDA); 0 disarms it.
 * scatrs_testing_force_node_error(key, status): the next fixed-grid call's device error word
 *   also holds a node error `status` (1 invalid input, 3 outside the validated domain) at
 *   key = (wavelength * n_dist + distribution) * n_nodes + node, merged as the kernels merge
 *   theirs (the first in order wins); a negative key disarms it. */
int scatrs_testing_raise(int32_t status, const char* message, double achieved, double requested,
                         char* err, size_t err_len);
void scatrs_testing_fail_allocation(int64_t k);
void scatrs_testing_force_node_error(int64_t key, int32_t status);

/* The library's limits, which it enforces, as the reference module exports them
 * (scatrs-py/src/lib.rs:17-50); -1 for an unknown `which`. */
enum scatrs_limit_kind {
  SCATRS_LIMIT_MIE_ORDER = 0,             /* terms of one sphere (mie/mod.rs:101) */
  SCATRS_LIMIT_MIE_VALUES = 1,            /* real values of one output array / 2 */
  SCATRS_LIMIT_GREEK_ORDER = 2,           /* Greek order (mie/greek.rs:344) */
  SCATRS_LIMIT_LAYERS = 3,                /* layers of a layered sphere on the GPU (16) */
  SCATRS_LIMIT_TMATRIX_ORDER = 4,         /* spheroid truncation N (tmatrix/mod.rs:180) */
  SCATRS_LIMIT_GAUSS_LEGENDRE_POINTS = 5, /* points of a Gauss-Legendre rule */
  SCATRS_LIMIT_WIGNER_D_VALUES = 6        /* Wigner values of one projection table */
};
int64_t scatrs_limit(int32_t which);

/*
 * Work-division settings of the fixed-grid entries, process-wide; they change how the work is cut
 * and scheduled, never a result (every output sum runs over its chunks in the same order whatever
 * the settings). split: a unit's table-row tiles are cut into work items of about
 * (work per slab) / (split x resident CTAs) each, 1..64 (0: the default, 4); arena_rows: the
 * coefficient rows (1 KiB each) a slab's arena holds, 2^16..2^24 (0: the default, 2^22). The
 * reference has no counterpart (its batch runs on host threads); the tuner in
 * scatrs_b200.tune picks them, and the mixed form's i8_above, by timing a sample of a workload.
 */
typedef struct scatrs_tuning {
  int32_t split;
  int32_t reserved; /* 0 */
  int64_t arena_rows;
} scatrs_tuning;
int scatrs_set_tuning(const scatrs_tuning* tuning, char* err, size_t err_len);
int scatrs_get_tuning(scatrs_tuning* tuning);

/* The CUDA device count, or -1 when the runtime is unusable. */
int scatrs_device_count(void);

/* Kernel launches made by this library since load (for the benchmark's launch count). */
int64_t scatrs_launch_count(void);

/* Per-kernel timing for profiling runs: with on = 1, every launch is bracketed by CUDA events on
 * its stream; scatrs_kernel_times synchronizes and returns, for the kernels 0 plan_chunks,
 * 1 mie_fixed (K-a), 2 unit (K-b/c), 3 mie_nodes, 4 final (the outputs), 5 proj (K-d), the total
 * milliseconds and launch counts since the last scatrs_set_profiling call, and the number of
 * kernels. */
void scatrs_set_profiling(int32_t on);
int scatrs_kernel_times(double* ms, int64_t* launches, int32_t n);
/* While profiling: the work of each tm_surface_kernel launch (the sum over its modes of K^2
 * pairs times 2 n_theta nodes) into per_launch[cap]; returns the number of launches. Kernel ids
 * 6-9 of scatrs_kernel_times are the T-matrix tables, surface integrals, solve and the
 * orientation average. */
int64_t scatrs_spheroid_work(int64_t* per_launch, int64_t cap);

/* Gauss-Legendre rule of n points on [-1, 1] (ascending nodes), as the host tables use it
 * (scatrs/src/special/gauss_legendre.rs:188-260); writes nothing unless
 * 1 <= n <= SCATRS_LIMIT_GAUSS_LEGENDRE_POINTS. */
void scatrs_gauss_legendre(int64_t n, double* nodes, double* weights);

/* Frees the cached tables and buffers of the current device. */
void scatrs_release(void);

#ifdef __cplusplus
}
#endif

#endif /* SCATRS_B200_H */
