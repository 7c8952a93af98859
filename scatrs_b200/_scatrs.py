"""The reference's binding surface for the ensemble path (scatrs-py/src/ensemble.rs), backed by
the GPU library.

* ``ensemble_parameters(items, mixture)``: the parameter names of ensemble.rs:172-188.
* ``ensemble_compute_fixed(specs, particle_spec, wavelengths, greek, all_orders, mu,
  normalized, n_nodes, spread, allow_unvalidated, ranges, derivatives)``: the batch call of
  ensemble.rs:455-504 on a fixed size grid, returning the same dict (values/errors (11, n),
  d/d_errors (k, 11, n), greek* (6, n, L + 1) and (k, 6, n, L + 1), phase* (6, n, n_mu) and
  (k, 6, n, n_mu), converged (n), panels (n)), rows distribution-major. The particle spec is
  ("sphere", m) with m of shape (n_wl,) as in the reference, or (n_dist, n_wl) for a
  refractive index per distribution and wavelength; or ("layered", fractions, m) with
  fractions (L - 1,) and m (L, n_wl) as in the reference, or per distribution (n_dist, L - 1)
  and (n_dist, L, n_wl). ``derivatives`` are indices into ensemble_parameters (the
  reference's deriv_idx, ensemble.rs:295-311), computed in forward mode like the reference's.

* ``ensemble_compute(items, wavelengths, mixture, greek, all_orders, mu, normalized,
  derivatives, rtol, max_panels, allow_unvalidated, refine_backscatter)`` and
  ``ensemble_compute_batch(specs, particle_spec, wavelengths, greek, all_orders, mu,
  normalized, rtol, max_panels, allow_unvalidated, refine_backscatter)``: the reference's
  calls (ensemble.rs:295-349, 455-504) on the adaptive GPU engine: sphere components (a
  mixture), each a lognormal, gamma, modified gamma, power law, monodisperse or multimodal
  distribution; values and error estimates.

Errors are those of the reference's Python package: the classes of ``scatrs.errors`` when this
module serves that package as its extension (``scatrs._scatrs``), else the same hierarchy from
``scatrs_b200.errors``; NotConvergedError carries ``achieved`` and ``requested``.

Module attributes read by the reference package at import (scatrs-py/src/lib.rs:17-50):
``__version__`` (the reference workspace version this module stands in for) and the ``MAX_*``
limits, read from the library, which enforces them.
"""

from __future__ import annotations

import numpy as np

from . import _native
from .errors import InvalidInputError

# The reference's workspace version (Cargo.toml:6) that this binding surface follows.
__version__ = "0.3.0"

MAX_MIE_ORDER: int = _native.limit("MIE_ORDER")
MAX_MIE_VALUES: int = _native.limit("MIE_VALUES")
MAX_GREEK_ORDER: int = _native.limit("GREEK_ORDER")
MAX_LAYERS: int = _native.limit("LAYERS")
MAX_TMATRIX_ORDER: int = _native.limit("TMATRIX_ORDER")
MAX_GAUSS_LEGENDRE_POINTS: int = _native.limit("GAUSS_LEGENDRE_POINTS")
MAX_WIGNER_D_VALUES: int = _native.limit("WIGNER_D_VALUES")

_PARAMS = {
    "lognormal": ("median_radius", "width"),
    "gamma": ("effective_radius", "effective_variance"),
    "modified_gamma": ("alpha", "b", "gamma"),
    "power_law": ("exponent",),
    "monodisperse": ("radius",),
    "tabulated": (),
}


def ensemble_parameters(items, mixture: bool) -> list[str]:
    """Parameter names in the order ensemble_compute indexes them (scatrs/src/ensemble/mod.rs:
    254-337): the distribution's, then the particle's, then the weight in a mixture."""
    if not items:
        return []
    if not mixture and len(items) != 1:
        raise InvalidInputError(
            f"a single distribution needs exactly one component, got {len(items)}")
    out = []
    for ci, (spec, particle, _w) in enumerate(items):
        prefix = f"c{ci}." if mixture else ""
        kind = spec[0]
        if kind == "multimodal":
            for j, (_v, mode) in enumerate(spec[1]):
                out += [f"{prefix}mode{j}.{n}" for n in _PARAMS[mode[0]]]
                out.append(f"{prefix}mode{j}.weight")
        elif kind in _PARAMS:
            out += [prefix + n for n in _PARAMS[kind]]
        else:
            raise TypeError(f"unknown distribution kind {kind!r}")
        pk = particle[0]
        if pk == "sphere":
            out += [prefix + "m_real", prefix + "m_imag"]
        elif pk == "spheroid":
            out += [prefix + "m_real", prefix + "m_imag", prefix + "aspect_ratio"]
        elif pk == "layered":
            layers = np.asarray(particle[2]).shape[0]
            for layer in range(layers):
                out += [f"{prefix}layer{layer}.m_real", f"{prefix}layer{layer}.m_imag"]
            for layer in range(np.asarray(particle[1]).size):
                out.append(f"{prefix}layer{layer}.radius_fraction")
        else:
            raise TypeError(f"unknown particle kind {pk!r}")
        if mixture:
            out.append(prefix + "weight")
    return out


def _parameter_records(items, mixture: bool) -> list:
    """The (component, mode, kind, index) of every name of ensemble_parameters, in its order
    (scatrs/src/ensemble/mod.rs:254-337); a layered sphere's are LayerRefrReal(l),
    LayerRefrImag(l) per layer, then RadiusFraction(l) (the record's index the layer)."""
    out = []
    for ci, (spec, particle, _w) in enumerate(items):
        kind = spec[0]
        if kind == "multimodal":
            for j, (_v, mode) in enumerate(spec[1]):
                out += [(ci, j, _native.PARAM_DISTRIBUTION, k) for k in range(len(_PARAMS[mode[0]]))]
                out.append((ci, j, _native.PARAM_WEIGHT, 0))
        else:
            out += [(ci, -1, _native.PARAM_DISTRIBUTION, k) for k in range(len(_PARAMS[kind]))]
        pk = particle[0]
        if pk == "sphere":
            out += [(ci, -1, _native.PARAM_REFR_REAL, 0), (ci, -1, _native.PARAM_REFR_IMAG, 0)]
        elif pk == "spheroid":
            out += [(ci, -1, _native.PARAM_REFR_REAL, 0), (ci, -1, _native.PARAM_REFR_IMAG, 0),
                    (ci, -1, _native.PARAM_ASPECT_RATIO, 0)]
        else:
            layers = np.asarray(particle[2]).shape[0]
            for layer in range(layers):
                out += [(ci, -1, _native.PARAM_LAYER_REFR_REAL, layer),
                        (ci, -1, _native.PARAM_LAYER_REFR_IMAG, layer)]
            out += [(ci, -1, _native.PARAM_RADIUS_FRACTION, layer)
                    for layer in range(layers - 1)]
        if mixture:
            out.append((ci, -1, _native.PARAM_WEIGHT, 0))
    return out


def _dist_array(specs, spread: float, ranges=None) -> np.ndarray:
    d = _native.dist_records(len(specs))
    for k, spec in enumerate(specs):
        if not isinstance(spec, tuple):
            raise TypeError("a distribution spec must be a tuple")
        kind = spec[0]
        if kind == "tabulated":
            # The grid spans the table unless a range is given.
            _native.set_table(d, k, spec[1], spec[2])
            if ranges is not None:
                d[k]["r_lo"], d[k]["r_hi"] = ranges[k]
            continue
        if kind not in _native.KINDS:
            raise TypeError(f"unknown distribution kind {kind!r}")
        p = [float(v) for v in spec[1:]]
        d[k]["kind"] = _native.KINDS[kind]
        d[k]["param"][: len(p)] = p
        if ranges is not None:
            d[k]["r_lo"], d[k]["r_hi"] = ranges[k]
        elif kind == "lognormal":
            d[k]["r_lo"] = p[0] * p[1] ** (-spread)
            d[k]["r_hi"] = p[0] * p[1] ** spread
        elif kind == "power_law":
            d[k]["r_lo"], d[k]["r_hi"] = p[1], p[2]
        else:
            raise InvalidInputError(f"a {kind} distribution needs an explicit grid range")
    return d


def _adaptive_dists(specs) -> np.ndarray:
    d = _native.dist_records(len(specs))
    for k, spec in enumerate(specs):
        if not isinstance(spec, tuple):
            raise TypeError("a distribution spec must be a tuple")
        kind = spec[0]
        if kind == "tabulated":
            # ("tabulated", radii, densities) (scatrs-py/src/ensemble.rs:58-61).
            _native.set_table(d, k, spec[1], spec[2])
            continue
        p = [float(v) for v in spec[1:]]
        if kind == "monodisperse":
            d[k]["kind"] = _native.MONODISPERSE
        elif kind in _native.KINDS:
            d[k]["kind"] = _native.KINDS[kind]
        elif kind == "multimodal":
            raise InvalidInputError("a multimodal distribution is not one distribution here")
        else:
            raise TypeError(f"unknown distribution kind {kind!r}")
        d[k]["param"][: len(p)] = p
    return d


def _adaptive_dict(out: dict, mu_size: int, k: int) -> dict:
    n = out["values"].shape[1]
    raw = {"values": out["values"], "errors": out["errors"], "d": np.zeros((k, 11, n)),
           "d_errors": np.zeros((k, 11, n))}
    for prefix in ("greek", "phase"):
        if prefix in out:
            arr = out[prefix]
            raw[prefix] = arr
            raw[f"{prefix}_errors"] = out[f"{prefix}_err"]
            raw[f"{prefix}_d"] = np.zeros((k,) + arr.shape)
            raw[f"{prefix}_d_errors"] = np.zeros((k,) + arr.shape)
    raw["converged"] = out["converged"]
    raw["panels"] = out["panels"].astype(np.uint64)
    return raw


def _layers(particle_spec, n_wl: int):
    """(fractions (L - 1), m (L, n_wl)) of a ('layered', fractions, m) spec
    (scatrs-py/src/ensemble.rs:80-135)."""
    fr = np.ascontiguousarray(np.asarray(particle_spec[1], dtype=np.float64).reshape(-1))
    ml = np.ascontiguousarray(np.asarray(particle_spec[2], dtype=np.complex128))
    if ml.ndim != 2 or ml.shape[1] != n_wl or ml.shape[0] != fr.size + 1:
        raise InvalidInputError(f"layered m must be ({fr.size + 1}, {n_wl}), got {ml.shape}")
    return fr, ml


def _spheroid(particle_spec, n_wl: int):
    """(aspect ratio, m (n_wl)) of a ('spheroid', aspect_ratio, m) spec."""
    m = np.ascontiguousarray(np.asarray(particle_spec[2], dtype=np.complex128).reshape(-1))
    if m.size != n_wl:
        raise InvalidInputError(f"{m.size} refractive indices for {n_wl} wavelengths")
    return float(particle_spec[1]), m


def _sphere_m(particle_spec, n_wl: int) -> np.ndarray:
    if not isinstance(particle_spec, tuple):
        raise TypeError("a particle spec must be a tuple")
    if particle_spec[0] != "sphere":
        if particle_spec[0] in ("layered", "spheroid"):
            raise InvalidInputError(
                f"{particle_spec[0]} particles are not on this GPU path here (mixtures)")
        raise TypeError(f"unknown particle kind {particle_spec[0]!r}")
    m = np.asarray(particle_spec[1], dtype=np.complex128).reshape(-1)
    if m.size != n_wl:
        raise InvalidInputError(f"{m.size} refractive indices for {n_wl} wavelengths")
    return m


def _particle(particle_spec, n_wl: int):
    """A mixture component's particle for _native: m (a sphere) or the checked layered or
    spheroid spec."""
    if not isinstance(particle_spec, tuple) or not particle_spec:
        raise TypeError("a particle spec must be a tuple")
    if particle_spec[0] == "layered":
        fr, ml = _layers(particle_spec, n_wl)
        return ("layered", fr, ml)
    if particle_spec[0] == "spheroid":
        eps, m = _spheroid(particle_spec, n_wl)
        return ("spheroid", eps, m)
    return _sphere_m(particle_spec, n_wl)


def _modes(spec):
    """(DIST_DTYPE modes, mode weights or None) of a spec; multimodal specs list (v, spec)."""
    if isinstance(spec, tuple) and spec and spec[0] == "multimodal":
        modes = list(spec[1])
        if not modes:
            raise InvalidInputError("a multimodal distribution needs a mode")
        for _v, mode in modes:
            if isinstance(mode, tuple) and mode and mode[0] == "multimodal":
                raise InvalidInputError(
                    "the modes of a multimodal distribution cannot be multimodal")
        return _adaptive_dists([mode for _v, mode in modes]), [float(v) for v, _m in modes]
    return _adaptive_dists([spec]), None


def _greek_order(greek, all_orders) -> int:
    """The C ABI's Greek order: -1 none, GREEK_ALL for greek='all' (every order up to 2 N_max
    per wavelength, GreekOrder::All), else the order."""
    if all_orders:
        return _native.GREEK_ALL
    return -1 if greek is None else int(greek)


def ensemble_compute(items, wavelengths, mixture, greek, all_orders, mu, normalized, derivatives,
                     rtol, max_panels, allow_unvalidated, refine_backscatter) -> dict:
    """The reference's ``_scatrs.ensemble_compute`` on the GPU: one or more components (a
    mixture) of spheres, layered spheres or spheroids, each a distribution or a multimodal
    one, one output per wavelength."""
    if not items:
        raise InvalidInputError("a mixture needs a component")
    derivatives = [int(i) for i in derivatives]
    if derivatives:
        return _compute_with_derivatives(items, wavelengths, mixture, greek, all_orders, mu,
                                         normalized, derivatives, rtol, max_panels,
                                         allow_unvalidated, refine_backscatter)
    wl = np.ascontiguousarray(wavelengths, dtype=np.float64).reshape(-1)
    mu = np.zeros(0) if mu is None else np.ascontiguousarray(mu, dtype=np.float64).reshape(-1)
    L = _greek_order(greek, all_orders)
    kinds = {p[0] if isinstance(p, tuple) and p else None for _, p, _ in items}
    single = len(items) == 1 and not (isinstance(items[0][0], tuple)
                                      and items[0][0][0] == "multimodal")
    if kinds - {"sphere"} and not single:
        # Components of different particles, or multimodal ones: the mixture path.
        comps = []
        for spec, particle, weight in items:
            dists, mode_w = _modes(spec)
            comps.append((dists, mode_w, float(weight), _particle(particle, wl.size)))
        out = _native.ensemble_mixture(comps, wl, mu, L, bool(normalized), float(rtol),
                                       int(max_panels), bool(allow_unvalidated),
                                       bool(refine_backscatter))
        return _adaptive_dict(out, mu.size, 0)
    if "spheroid" in kinds:
        spec, particle, _ = items[0]
        eps, m = _spheroid(particle, wl.size)
        out = _native.ensemble_adaptive_spheroid(
            _adaptive_dists([spec]), wl, eps, m, mu, L, bool(normalized), float(rtol),
            int(max_panels), bool(allow_unvalidated), bool(refine_backscatter))
        return _adaptive_dict(out, mu.size, 0)
    if "layered" in kinds:
        spec, particle, _ = items[0]
        fr, ml = _layers(particle, wl.size)
        out = _native.ensemble_adaptive_layered(
            _adaptive_dists([spec]), wl, fr[None], ml[None], mu, L, bool(normalized),
            float(rtol), int(max_panels), bool(allow_unvalidated), bool(refine_backscatter))
        return _adaptive_dict(out, mu.size, 0)
    comps = []
    for spec, particle, weight in items:
        dists, mode_w = _modes(spec)
        comps.append((dists, mode_w, float(weight), _sphere_m(particle, wl.size)))
    out = _native.ensemble_mixture(comps, wl, mu, L,
                                   bool(normalized), float(rtol), int(max_panels),
                                   bool(allow_unvalidated), bool(refine_backscatter))
    return _adaptive_dict(out, mu.size, 0)


def _compute_with_derivatives(items, wavelengths, mixture, greek, all_orders, mu, normalized,
                              derivatives, rtol, max_panels, allow_unvalidated,
                              refine_backscatter) -> dict:
    """ensemble_compute with derivatives (scatrs-py/src/ensemble.rs:318-349): the parameters by
    their index in ensemble_parameters, every one once, through scatrs_ensemble_mixture_d
    (compute_mixture with EnsembleOptions::derivatives): spheres, or one spheroid or layered
    sphere component."""
    names = ensemble_parameters(items, mixture)
    records = _parameter_records(items, mixture)
    chosen = []
    for i in derivatives:
        if not 0 <= i < len(records):
            raise InvalidInputError(f"no parameter {i}")
        if i in chosen:
            raise InvalidInputError(f"parameter {names[i]} requested twice")
        chosen.append(i)
    wl = np.ascontiguousarray(wavelengths, dtype=np.float64).reshape(-1)
    mu = np.zeros(0) if mu is None else np.ascontiguousarray(mu, dtype=np.float64).reshape(-1)
    L = _greek_order(greek, all_orders)
    comps = []
    for spec, particle, weight in items:
        dists, mode_w = _modes(spec)
        # A spheroid or a layered sphere (one component) goes as its checked spec.
        part = (_particle(particle, wl.size) if isinstance(particle, tuple) and particle
                and particle[0] in ("spheroid", "layered") else _sphere_m(particle, wl.size))
        comps.append((dists, mode_w, float(weight), part))
    params = np.array([records[i] for i in chosen], dtype=_native.PARAM_DTYPE)
    out = _native.ensemble_mixture_d(comps, wl, params, mu, L, bool(normalized), float(rtol),
                                     int(max_panels), bool(allow_unvalidated),
                                     bool(refine_backscatter))
    raw = {"values": out["values"], "errors": out["errors"], "d": out["d"],
           "d_errors": out["d_err"]}
    for prefix in ("greek", "phase"):
        if prefix in out:
            raw[prefix] = out[prefix]
            raw[f"{prefix}_errors"] = out[f"{prefix}_err"]
            raw[f"{prefix}_d"] = out[f"{prefix}_d"]
            raw[f"{prefix}_d_errors"] = out[f"{prefix}_d_err"]
    raw["converged"] = out["converged"]
    raw["panels"] = out["panels"].astype(np.uint64)
    return raw


def ensemble_compute_batch(specs, particle_spec, wavelengths, greek, all_orders, mu, normalized,
                           rtol, max_panels, allow_unvalidated, refine_backscatter) -> dict:
    """The reference's ``_scatrs.ensemble_compute_batch`` on the GPU: every distribution of
    one sphere material on shared panels per wavelength, rows distribution-major."""
    if not specs:
        raise InvalidInputError("a batch needs a distribution")
    wl = np.ascontiguousarray(wavelengths, dtype=np.float64).reshape(-1)
    greek = _greek_order(greek, all_orders)
    greek = None if greek == -1 else greek
    mu = np.zeros(0) if mu is None else np.ascontiguousarray(mu, dtype=np.float64).reshape(-1)
    if isinstance(particle_spec, tuple) and particle_spec and particle_spec[0] == "spheroid":
        eps, m = _spheroid(particle_spec, wl.size)
        out = _native.ensemble_adaptive_spheroid(
            _adaptive_dists(list(specs)), wl, eps, m, mu, -1 if greek is None else int(greek),
            bool(normalized), float(rtol), int(max_panels), bool(allow_unvalidated),
            bool(refine_backscatter), batch=True)
        return _adaptive_dict(out, mu.size, 0)
    if isinstance(particle_spec, tuple) and particle_spec and particle_spec[0] == "layered":
        fr, ml = _layers(particle_spec, wl.size)
        n = len(specs)
        out = _native.ensemble_adaptive_layered(
            _adaptive_dists(list(specs)), wl, np.broadcast_to(fr, (n,) + fr.shape),
            np.broadcast_to(ml, (n,) + ml.shape), mu, -1 if greek is None else int(greek),
            bool(normalized), float(rtol), int(max_panels), bool(allow_unvalidated),
            bool(refine_backscatter), batch=True)
        return _adaptive_dict(out, mu.size, 0)
    m = _sphere_m(particle_spec, wl.size)
    out = _native.ensemble_adaptive(_adaptive_dists(list(specs)), wl, m, mu,
                                    -1 if greek is None else int(greek), bool(normalized),
                                    float(rtol), int(max_panels), bool(allow_unvalidated),
                                    bool(refine_backscatter), batch=True)
    return _adaptive_dict(out, mu.size, 0)


def ensemble_compute_fixed(specs, particle_spec, wavelengths, greek, all_orders, mu, normalized,
                           n_nodes: int = 256, spread: float = 5.0, allow_unvalidated=False,
                           ranges=None, derivatives=(), tmatrix_rtol: float = 1e-8) -> dict:
    """The batch dict on a fixed grid. ``derivatives`` selects parameters by their index in
    ``ensemble_parameters([(specs[0], particle_spec, 1.0)], False)`` (the reference's
    ``deriv_idx``): homogeneous or layered spheres or spheroids, every distribution of one kind.
    Spheroids (``('spheroid', aspect_ratio, m)``) converge every node's T-matrix to
    ``tmatrix_rtol``."""
    if not isinstance(particle_spec, tuple) or particle_spec[0] not in ("sphere", "layered",
                                                                         "spheroid"):
        raise TypeError("the fixed-grid ensemble takes ('sphere', m), ('layered', fractions, m) "
                        "or ('spheroid', aspect_ratio, m)")
    if all_orders:
        raise InvalidInputError("the fixed-grid ensemble needs a finite Greek order")
    wl = np.ascontiguousarray(wavelengths, dtype=np.float64).reshape(-1)
    dists = _dist_array(specs, spread, ranges)
    mu = np.zeros(0) if mu is None else np.ascontiguousarray(mu, dtype=np.float64).reshape(-1)
    L = -1 if greek is None else int(greek)
    derivatives = [int(k) for k in derivatives]
    d = dp = dg = None
    if particle_spec[0] == "spheroid":
        m = np.asarray(particle_spec[2], dtype=np.complex128)
        if m.ndim == 1:
            m = np.broadcast_to(m, (dists.size, wl.size))
        if derivatives:
            names = ensemble_parameters([(specs[0], particle_spec, 1.0)], False)
            for k in derivatives:
                if not 0 <= k < len(names):
                    raise InvalidInputError(f"derivative index {k} out of range of {names}")
            values, phase, g, d, dp, dg, _ = _native.ensemble_fixed_spheroid_d(
                dists, wl, float(particle_spec[1]), m, mu, n_nodes, L, bool(normalized),
                tmatrix_rtol=tmatrix_rtol, allow_unvalidated=bool(allow_unvalidated))
            # The library's blocks: the distribution's parameters, the aspect ratio, Re m, Im m;
            # the names': the distribution's, m_real, m_imag, aspect_ratio.
            pt = len(names) - 3
            col = [k if k < pt else {pt: pt + 1, pt + 1: pt + 2, pt + 2: pt}[k]
                   for k in derivatives]
            d, dp, dg = (None if a is None else np.ascontiguousarray(a[col])
                         for a in (d, dp, dg))
        else:
            values, phase, g, _ = _native.ensemble_fixed_spheroid(
                dists, wl, float(particle_spec[1]), m, mu, n_nodes, L, bool(normalized),
                tmatrix_rtol=tmatrix_rtol, allow_unvalidated=bool(allow_unvalidated))
    elif particle_spec[0] == "layered":
        ml = np.asarray(particle_spec[2], dtype=np.complex128)
        fr = np.asarray(particle_spec[1], dtype=np.float64)
        if ml.ndim == 2:  # (L, n_wl): the same particle for every distribution
            fr = fr.reshape(-1)
            ml = np.broadcast_to(ml, (dists.size,) + ml.shape)
            fr = np.broadcast_to(fr, (dists.size, fr.size))
        else:
            fr = fr.reshape(dists.size, -1)
        if derivatives:
            # The derivative blocks come in ensemble_parameters' order: the distribution's
            # parameters, each layer's Re m and Im m, each radius fraction.
            names = ensemble_parameters([(specs[0], ("layered", fr[0], ml[0]), 1.0)], False)
            for k in derivatives:
                if not 0 <= k < len(names):
                    raise InvalidInputError(f"derivative index {k} out of range of {names}")
            values, phase, g, d, dp, dg = _native.ensemble_fixed_layered_d(
                dists, wl, fr, ml, mu, n_nodes, L, bool(normalized), bool(allow_unvalidated))
            d, dp, dg = (None if a is None else np.ascontiguousarray(a[derivatives])
                         for a in (d, dp, dg))
        else:
            values, phase, g = _native.ensemble_fixed_layered(dists, wl, fr, ml, mu, n_nodes, L,
                                                              bool(normalized),
                                                              bool(allow_unvalidated))
    else:
        m = np.asarray(particle_spec[1], dtype=np.complex128)
        if m.ndim == 1:
            m = np.broadcast_to(m, (dists.size, wl.size))
        if derivatives:
            names = ensemble_parameters([(specs[0], particle_spec, 1.0)], False)
            for k in derivatives:
                if not 0 <= k < len(names):
                    raise InvalidInputError(f"derivative index {k} out of range of {names}")
            values, phase, g, d, dp, dg = _native.ensemble_fixed_d(
                dists, wl, m, mu, n_nodes, L, bool(normalized), bool(allow_unvalidated))
            d, dp, dg = (None if a is None else np.ascontiguousarray(a[derivatives])
                         for a in (d, dp, dg))
        else:
            values, phase, g = _native.ensemble_fixed(dists, wl, m, mu, n_nodes, L,
                                                      bool(normalized), bool(allow_unvalidated))
    n = values.shape[1]
    k = len(derivatives)
    out = {"values": values, "errors": np.zeros_like(values),
           "d": d if d is not None else np.zeros((0, 11, n)), "d_errors": np.zeros((k, 11, n))}
    for prefix, arr, darr in (("greek", g, dg), ("phase", phase, dp)):
        if arr is not None:
            out[prefix] = arr
            out[f"{prefix}_errors"] = np.zeros_like(arr)
            out[f"{prefix}_d"] = darr if darr is not None else np.zeros((0,) + arr.shape)
            out[f"{prefix}_d_errors"] = np.zeros((k,) + arr.shape)
    out["converged"] = np.ones(n, dtype=bool)
    out["panels"] = np.zeros(n, dtype=np.uint64)
    return out


class _Testing:
    """Hooks for tests, not part of the API (the reference's ``scatrs._scatrs._testing``,
    scatrs-py/src/testing.rs:29-57): ``raise_core_error`` raises what a failed library call with
    that error raises, through the library's own error path."""

    _STATUS = {"InvalidInput": 1, "NotConverged": 2, "OutsideValidatedDomain": 3}

    @staticmethod
    def raise_core_error(variant: str, message: str = "", achieved: float = 0.0,
                         requested: float = 0.0) -> None:
        import ctypes

        if variant not in _Testing._STATUS:
            raise ValueError(f"unknown scatrs::Error variant {variant!r}")
        # The reference's Display texts (scatrs/src/error.rs:18-31).
        text = {"InvalidInput": f"invalid input: {message}",
                "NotConverged": f"not converged: achieved {achieved:e}, requested {requested:e}",
                "OutsideValidatedDomain": f"outside validated domain: {message}"}[variant]
        err = ctypes.create_string_buffer(1024)
        st = _native.load().scatrs_testing_raise(_Testing._STATUS[variant], text.encode(),
                                                 achieved, requested, err, 1024)
        _native._check(st, err)


_testing = _Testing()
