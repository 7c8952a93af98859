"""ctypes binding of libscatrs_b200.so (the C ABI of include/scatrs_b200.h).

The library is the only compute path: if it is missing, or no CUDA device is usable, the calls
raise instead of falling back to anything else.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

from .errors import DeviceError, InvalidInputError, classes, raise_for

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libscatrs_b200.so")

_D = ctypes.c_double
_I32 = ctypes.c_int32
_I64 = ctypes.c_int64
_PD = ctypes.POINTER(ctypes.c_double)
_PI64 = ctypes.POINTER(ctypes.c_int64)
_VP = ctypes.c_void_p
_CP = ctypes.c_char_p
_SZ = ctypes.c_size_t

DIST_DTYPE = np.dtype([("kind", np.int32), ("reserved", np.int32), ("param", np.float64, 3),
                       ("r_lo", np.float64), ("r_hi", np.float64), ("table", np.uint64),
                       ("table_len", np.int64)])
TABULATED = 6  # table = address of [radii..., densities...], table_len points


class DistArray(np.ndarray):
    """A DIST_DTYPE array that owns the tables its tabulated records point at."""

    def __array_finalize__(self, obj):
        self.tables = getattr(obj, "tables", [])


def dist_records(n: int) -> DistArray:
    """n zeroed distribution records."""
    d = np.zeros(n, dtype=DIST_DTYPE).view(DistArray)
    d.tables = []
    return d


def set_table(d: DistArray, k: int, radii, densities) -> None:
    """Make record k the tabulated n(r) through (radii, densities), linear between the points
    and 0 outside them (scatrs/src/ensemble/distribution.rs:55-62); d keeps the table alive."""
    r = np.asarray(radii, dtype=np.float64).reshape(-1)
    n = np.asarray(densities, dtype=np.float64).reshape(-1)
    if r.size < 2 or r.size != n.size:
        raise InvalidInputError(
            "a tabulated distribution needs at least 2 points and as many densities as radii, "
            f"got {r.size} radii and {n.size} densities")
    tab = np.ascontiguousarray(np.concatenate([r, n]))
    d.tables.append(tab)
    d[k]["kind"] = TABULATED
    d[k]["table"] = tab.ctypes.data
    d[k]["table_len"] = r.size
    d[k]["r_lo"], d[k]["r_hi"] = r[0], r[-1]
KINDS = {"lognormal": 1, "gamma": 2, "modified_gamma": 3, "power_law": 4}
MONODISPERSE = 5  # adaptive calls only: param[0] the radius


class Layers(ctypes.Structure):
    _fields_ = [("n_layers", _I32), ("reserved", _I32), ("fractions", _PD), ("m", _PD)]


class AdaptiveOptions(ctypes.Structure):
    _fields_ = [("rtol", _D), ("max_panels", _I64), ("greek_order", _I32), ("normalized", _I32),
                ("allow_unvalidated", _I32), ("refine_backscatter", _I32)]


class Component(ctypes.Structure):
    _fields_ = [("modes", _VP), ("mode_weights", _PD), ("n_modes", _I32), ("n_layers", _I32),
                ("weight", _D), ("m", _PD), ("fractions", _PD), ("aspect_ratio", _D)]


class SpheroidOptions(ctypes.Structure):
    _fields_ = [("rtol", _D), ("n_terms", _I32), ("n_theta", _I32), ("greek_order", _I32),
                ("normalized", _I32), ("allow_unvalidated", _I32)]


class FixedOptions(ctypes.Structure):
    _fields_ = [("n_nodes", _I32), ("greek_order", _I32), ("normalized", _I32),
                ("allow_unvalidated", _I32)]


class MixedOptions(ctypes.Structure):
    _fields_ = [("i8_above", _I32), ("levels", _I32)]


class Tuning(ctypes.Structure):
    _fields_ = [("split", _I32), ("reserved", _I32), ("arena_rows", _I64)]


class RefractiveModel(ctypes.Structure):
    _fields_ = [("kind", _I32), ("n", _I32), ("p", _D * 4), ("table", _PD)]


REFRACTIVE_KINDS = {"constant": 0, "table": 1, "table_log_k": 2, "cauchy": 3, "sellmeier": 4}


# Every symbol the header declares, with (restype, argtypes).
SYMBOLS = {
    "scatrs_ensemble_fixed_sizes": (None, [_I64, _I64, _I32, _PI64, _PI64, _PI64]),
    "scatrs_ensemble_fixed": (ctypes.c_int, [_VP, _I64, _PD, _I64, _PD, _PD, _I64,
                                             ctypes.POINTER(FixedOptions), _PD, _PD, _PD, _CP,
                                             _SZ]),
    "scatrs_ensemble_fixed_spheroid": (ctypes.c_int, [_VP, _I64, _PD, _I64, _PD, _PD, _PD, _I64,
                                                      ctypes.POINTER(FixedOptions), _D, _PD, _PD,
                                                      _PD, _VP, _CP, _SZ]),
    "scatrs_ensemble_fixed_spheroid_d": (ctypes.c_int, [_VP, _I64, _PD, _I64, _PD, _PD, _PD,
                                                        _I64, ctypes.POINTER(FixedOptions), _D,
                                                        _PD, _PD, _PD, _PD, _PD, _PD, _VP, _CP,
                                                        _SZ]),
    "scatrs_ensemble_fixed_d": (ctypes.c_int, [_VP, _I64, _PD, _I64, _PD, _PD, _I64,
                                               ctypes.POINTER(FixedOptions), _PD, _PD, _PD, _PD,
                                               _PD, _PD, _CP, _SZ]),
    "scatrs_ensemble_fixed_layered": (ctypes.c_int, [_VP, _I64, _PD, _I64, ctypes.POINTER(Layers),
                                                     _PD, _I64, ctypes.POINTER(FixedOptions), _PD,
                                                     _PD, _PD, _CP, _SZ]),
    "scatrs_ensemble_fixed_device": (ctypes.c_int, [_VP, _I64, _VP, _I64, _VP, _PD, _I64,
                                                    ctypes.POINTER(FixedOptions), _VP, _VP, _VP,
                                                    _VP, _CP, _SZ]),
    "scatrs_ensemble_fixed_mixed": (ctypes.c_int, [_VP, _I64, _PD, _I64, _PD, _PD, _I64,
                                                   ctypes.POINTER(FixedOptions),
                                                   ctypes.POINTER(MixedOptions), _PD, _PD, _PD,
                                                   _CP, _SZ]),
    "scatrs_ensemble_fixed_mixed_device": (ctypes.c_int, [_VP, _I64, _VP, _I64, _VP, _PD, _I64,
                                                          ctypes.POINTER(FixedOptions),
                                                          ctypes.POINTER(MixedOptions), _VP, _VP,
                                                          _VP, _VP, _CP, _SZ]),
    "scatrs_ensemble_adaptive": (ctypes.c_int, [_VP, _I64, _I32, _PD, _I64, _PD, _PD, _I64,
                                                ctypes.POINTER(AdaptiveOptions), _PD, _PD, _PD,
                                                _PD, _PD, _PD, _VP, _VP, _CP, _SZ]),
    "scatrs_ensemble_fixed_layered_d": (ctypes.c_int, [_VP, _I64, _PD, _I64, ctypes.POINTER(Layers),
                                                       _PD, _I64, ctypes.POINTER(FixedOptions),
                                                       _PD, _PD, _PD, _PD, _PD, _PD, _CP, _SZ]),
    "scatrs_ensemble_adaptive_layered": (ctypes.c_int, [_VP, _I64, _I32, _PD, _I64,
                                                        ctypes.POINTER(Layers), _PD, _I64,
                                                        ctypes.POINTER(AdaptiveOptions), _PD, _PD,
                                                        _PD, _PD, _PD, _PD, _VP, _VP, _CP, _SZ]),
    "scatrs_ensemble_adaptive_spheroid": (ctypes.c_int, [_VP, _I64, _I32, _PD, _I64, _D, _PD,
                                                         _PD, _I64,
                                                         ctypes.POINTER(AdaptiveOptions), _PD,
                                                         _PD, _PD, _PD, _PD, _PD, _VP, _VP, _CP,
                                                         _SZ]),
    "scatrs_ensemble_mixture": (ctypes.c_int, [ctypes.POINTER(Component), _I64, _PD, _I64, _PD,
                                               _I64, ctypes.POINTER(AdaptiveOptions), _PD, _PD,
                                               _PD, _PD, _PD, _PD, _VP, _VP, _CP, _SZ]),
    "scatrs_greek_all_width": (_I64, []),
    "scatrs_greek_all_take": (ctypes.c_int, [_PD, _PD, _PD, _PD]),
    "scatrs_ensemble_mixture_d": (ctypes.c_int, [ctypes.POINTER(Component), _I64, _PD, _I64, _PD,
                                                 _I64, ctypes.POINTER(AdaptiveOptions), _VP, _I64]
                                  + [_PD] * 12 + [_VP, _VP, _CP, _SZ]),
    "scatrs_project_greek_device": (ctypes.c_int, [_VP, _I64, _I64, _I32, _I32, _VP, _VP, _CP,
                                                   _SZ]),
    "scatrs_spheroid_tmatrix": (ctypes.c_int, [_D, _D, _PD, _I32, _I32, _I32, _PD, _CP, _SZ]),
    "scatrs_spheroid_efficiencies": (ctypes.c_int, [_I64, _PD, _PD, _PD, _D, _PD, _VP, _VP, _CP,
                                                    _SZ]),
    "scatrs_spheroid_compute": (ctypes.c_int, [_I64, _PD, _PD, _PD, ctypes.POINTER(SpheroidOptions),
                                               _PD, _PD, _VP, _VP, _PD, _CP, _SZ]),
    "scatrs_spheroid_compute_d": (ctypes.c_int, [_I64, _PD, _PD, _PD,
                                                 ctypes.POINTER(SpheroidOptions), _PD, _PD, _PD,
                                                 _PD, _VP, _VP, _PD, _CP, _SZ]),
    "scatrs_spheroid_work": (ctypes.c_int64, [_VP, _I64]),
    "scatrs_check_errors": (ctypes.c_int, [_VP, _CP, _SZ]),
    "scatrs_mie": (ctypes.c_int, [_PD, _PD, _I64, _I32, _PI64, _PI64, _PD, _PD, _CP, _SZ]),
    "scatrs_mie_static": (ctypes.c_int, [_VP, _VP, _I64, _I32, _I64, _VP, _VP, _VP, _VP, _VP,
                                         _CP, _SZ]),
    "scatrs_not_converged_detail": (ctypes.c_int, [_PD, _PD]),
    "scatrs_ensemble_fixed_d_device": (ctypes.c_int, [_VP, _I64, _VP, _I64, _VP, _PD, _I64,
                                                      ctypes.POINTER(FixedOptions), _VP, _VP,
                                                      _VP, _VP, _VP, _VP, _VP, _CP, _SZ]),
    "scatrs_ensemble_fixed_layered_d_device": (ctypes.c_int, [_VP, _I64, _VP, _I64,
                                                              ctypes.POINTER(Layers), _PD, _I64,
                                                              ctypes.POINTER(FixedOptions), _VP,
                                                              _VP, _VP, _VP, _VP, _VP, _VP, _CP,
                                                              _SZ]),
    "scatrs_refractive_parameter_count": (ctypes.c_int, [ctypes.POINTER(RefractiveModel)]),
    "scatrs_refractive_index_device": (ctypes.c_int, [ctypes.POINTER(RefractiveModel), _I64,
                                                      _VP, _I64, _VP, _VP, _I32, _VP, _CP,
                                                      _SZ]),
    "scatrs_testing_raise": (ctypes.c_int, [_I32, _CP, _D, _D, _CP, _SZ]),
    "scatrs_testing_fail_allocation": (None, [_I64]),
    "scatrs_testing_force_node_error": (None, [_I64, _I32]),
    "scatrs_limit": (_I64, [_I32]),
    "scatrs_set_tuning": (ctypes.c_int, [ctypes.POINTER(Tuning), _CP, _SZ]),
    "scatrs_get_tuning": (ctypes.c_int, [ctypes.POINTER(Tuning)]),
    "scatrs_device_count": (ctypes.c_int, []),
    "scatrs_launch_count": (_I64, []),
    "scatrs_gauss_legendre": (None, [_I64, _PD, _PD]),
    "scatrs_release": (None, []),
    "scatrs_set_profiling": (None, [_I32]),
    "scatrs_kernel_times": (ctypes.c_int, [_PD, _PI64, _I32]),
}

KERNEL_NAMES = ("plan_chunks_kernel", "mie_fixed_kernel", "unit_kernel", "mie_nodes_kernel",
                "final_kernel", "proj_kernel", "tm_tables_kernels", "tm_surface_kernel",
                "tm_solve_kernel", "ro_kernels", "unit_i8_kernel", "x_split_kernel")
# The kernels each id covers: K-a also as mie_layered_kernel / mie_deriv_kernel, the unit kernel
# as unit_deriv_kernel, the final kernel as final_deriv_kernel.

_lib = None


def load() -> ctypes.CDLL:
    """The library (loaded once); raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise DeviceError(f"{LIB_PATH} is missing: build it with python -m scatrs_b200.build")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SYMBOLS.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
    return _lib


def require_device() -> None:
    n = load().scatrs_device_count()
    if n <= 0:
        raise classes()[3]("no usable CUDA device: the ensemble path runs on the GPU only")


def _p(a):
    return None if a is None else a.ctypes.data_as(_PD)


def _check(status: int, buf) -> None:
    achieved = requested = None
    if status == 2:
        a, r = _D(), _D()
        if load().scatrs_not_converged_detail(ctypes.byref(a), ctypes.byref(r)):
            achieved, requested = a.value, r.value
    raise_for(status, buf.value.decode(errors="replace"), achieved, requested)


_LIMITS = {"MIE_ORDER": 0, "MIE_VALUES": 1, "GREEK_ORDER": 2, "LAYERS": 3, "TMATRIX_ORDER": 4,
           "GAUSS_LEGENDRE_POINTS": 5, "WIGNER_D_VALUES": 6}


def limit(name: str) -> int:
    """One of the library's limits (scatrs_limit), by its SCATRS_LIMIT_ name."""
    return int(load().scatrs_limit(_LIMITS[name]))


def set_tuning(split: int = 0, arena_rows: int = 0) -> None:
    """The fixed-grid entries' work division (scatrs_set_tuning; 0 = the default)."""
    t = Tuning(int(split), 0, int(arena_rows))
    buf = ctypes.create_string_buffer(512)
    st = load().scatrs_set_tuning(ctypes.byref(t), buf, 512)
    if st != 0:
        _check(st, buf)


def get_tuning() -> dict:
    t = Tuning()
    load().scatrs_get_tuning(ctypes.byref(t))
    return {"split": int(t.split), "arena_rows": int(t.arena_rows)}


def gauss_legendre(n: int):
    if not 1 <= n <= limit("GAUSS_LEGENDRE_POINTS"):
        raise InvalidInputError(
            f"a Gauss-Legendre rule needs 1 <= n <= MAX_GAUSS_LEGENDRE_POINTS, got {n}")
    x = np.zeros(n)
    w = np.zeros(n)
    load().scatrs_gauss_legendre(n, _p(x), _p(w))
    return x, w


def launch_count() -> int:
    return int(load().scatrs_launch_count())


def set_profiling(on: bool) -> None:
    load().scatrs_set_profiling(int(on))


def kernel_times() -> dict:
    """{kernel: (total ms, launches)} since set_profiling (synchronizes)."""
    ms = np.zeros(len(KERNEL_NAMES))
    n = np.zeros(len(KERNEL_NAMES), dtype=np.int64)
    k = load().scatrs_kernel_times(_p(ms), n.ctypes.data_as(_PI64), len(KERNEL_NAMES))
    return {KERNEL_NAMES[i]: (float(ms[i]), int(n[i])) for i in range(k)}


def spheroid_work() -> np.ndarray:
    """While profiling: each tm_surface_kernel launch's (pair, node) count."""
    n = int(load().scatrs_spheroid_work(None, 0))
    out = np.zeros(n, dtype=np.int64)
    load().scatrs_spheroid_work(out.ctypes.data, n)
    return out


def mie(x, m, allow_unvalidated: bool = False):
    """Coefficients and efficiencies of independent spheres on the GPU (batched Mie::compute):
    a list of (a, b) complex arrays and an (n, 5) array of Q_ext, Q_sca, Q_abs, Q_back, g."""
    require_device()
    x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
    m = np.ascontiguousarray(np.broadcast_to(np.asarray(m, dtype=np.complex128), x.shape))
    n = x.size
    nt = np.zeros(n, dtype=np.int64)
    err = ctypes.create_string_buffer(512)
    mv = m.view(np.float64)
    st = load().scatrs_mie(_p(x), _p(mv), n, int(allow_unvalidated), nt.ctypes.data_as(_PI64),
                           None, None, None, err, 512)
    _check(st, err)
    off = np.zeros(n, dtype=np.int64)
    off[1:] = np.cumsum(nt)[:-1]
    coeffs = np.zeros(4 * int(nt.sum()))
    eff = np.zeros(5 * n)
    st = load().scatrs_mie(_p(x), _p(mv), n, int(allow_unvalidated), nt.ctypes.data_as(_PI64),
                           off.ctypes.data_as(_PI64), _p(coeffs), _p(eff), err, 512)
    _check(st, err)
    c = coeffs.view(np.complex128)
    out = []
    for i in range(n):
        o, k = 2 * off[i], nt[i]
        out.append((c[o:o + k], c[o + k:o + 2 * k]))
    return out, eff.reshape(n, 5)


def ensemble_fixed(dists: np.ndarray, wavelengths, m, mu, n_nodes: int, greek_order: int = -1,
                   normalized: bool = True, allow_unvalidated: bool = False, i8_above: int = 0,
                   levels: int = 0):
    """The fixed-grid ensemble from host arrays; returns (values, phase or None, greek or None)
    shaped (11, n), (6, n, n_mu), (6, n, L + 1) with n = n_dist * n_wl, distribution-major.
    i8_above > 0: the mixed form (scatrs_ensemble_fixed_mixed), the angle GEMMs of the chunks
    with more terms than i8_above as exact int8 digit products on the tensor cores, keeping
    `levels` product levels (0: the library's default)."""
    require_device()
    dists = np.ascontiguousarray(dists, dtype=DIST_DTYPE)
    wl = np.ascontiguousarray(wavelengths, dtype=np.float64).reshape(-1)
    m = np.ascontiguousarray(np.broadcast_to(np.asarray(m, dtype=np.complex128),
                                             (dists.size, wl.size)))
    mu = np.zeros(0) if mu is None else np.ascontiguousarray(mu, dtype=np.float64).reshape(-1)
    n = dists.size * wl.size
    opts = FixedOptions(int(n_nodes), int(greek_order), int(normalized), int(allow_unvalidated))
    values = np.zeros((11, n))
    phase = np.zeros((6, n, mu.size)) if mu.size else None
    greek = np.zeros((6, n, greek_order + 1)) if greek_order >= 0 else None
    err = ctypes.create_string_buffer(1024)
    if i8_above > 0:
        st = load().scatrs_ensemble_fixed_mixed(dists.ctypes.data, dists.size, _p(wl), wl.size,
                                                _p(m.view(np.float64)), _p(mu), mu.size,
                                                ctypes.byref(opts),
                                                ctypes.byref(MixedOptions(int(i8_above),
                                                                          int(levels))),
                                                _p(values), _p(phase), _p(greek), err, 1024)
    else:
        st = load().scatrs_ensemble_fixed(dists.ctypes.data, dists.size, _p(wl), wl.size,
                                          _p(m.view(np.float64)), _p(mu), mu.size,
                                          ctypes.byref(opts), _p(values), _p(phase), _p(greek),
                                          err, 1024)
    _check(st, err)
    return values, phase, greek


def ensemble_fixed_spheroid(dists: np.ndarray, wavelengths, aspect_ratio, m, mu, n_nodes: int,
                            greek_order: int = -1, normalized: bool = True,
                            tmatrix_rtol: float = 1e-8, allow_unvalidated: bool = False):
    """The fixed-grid ensemble of randomly oriented spheroids (one aspect ratio per
    distribution); returns (values, phase or None, greek or None, node_terms) with node_terms
    (n, n_nodes, 2) the N and n_theta of each node."""
    require_device()
    dists = np.ascontiguousarray(dists, dtype=DIST_DTYPE)
    wl = np.ascontiguousarray(wavelengths, dtype=np.float64).reshape(-1)
    eps = np.ascontiguousarray(np.broadcast_to(np.asarray(aspect_ratio, dtype=np.float64),
                                               (dists.size,)))
    m = np.ascontiguousarray(np.broadcast_to(np.asarray(m, dtype=np.complex128),
                                             (dists.size, wl.size)))
    mu = np.zeros(0) if mu is None else np.ascontiguousarray(mu, dtype=np.float64).reshape(-1)
    n = dists.size * wl.size
    opts = FixedOptions(int(n_nodes), int(greek_order), int(normalized), int(allow_unvalidated))
    values = np.zeros((11, n))
    phase = np.zeros((6, n, mu.size)) if mu.size else None
    greek = np.zeros((6, n, greek_order + 1)) if greek_order >= 0 else None
    terms = np.zeros((n, int(n_nodes), 2), dtype=np.int32)
    err = ctypes.create_string_buffer(1024)
    st = load().scatrs_ensemble_fixed_spheroid(dists.ctypes.data, dists.size, _p(wl), wl.size,
                                               _p(eps), _p(m.view(np.float64)), _p(mu), mu.size,
                                               ctypes.byref(opts), float(tmatrix_rtol),
                                               _p(values), _p(phase), _p(greek),
                                               terms.ctypes.data, err, 1024)
    _check(st, err)
    return values, phase, greek, terms


def ensemble_fixed_spheroid_d(dists: np.ndarray, wavelengths, aspect_ratio, m, mu,
                              n_nodes: int, greek_order: int = -1, normalized: bool = True,
                              tmatrix_rtol: float = 1e-8, allow_unvalidated: bool = False):
    """ensemble_fixed_spheroid with the derivatives along the distribution's parameters, the
    aspect ratio, Re m and Im m (P of them): returns (values, phase, greek, d_values, d_phase,
    d_greek, node_terms), the derivative arrays shaped (P,) + the value array's shape."""
    require_device()
    dists = np.ascontiguousarray(dists, dtype=DIST_DTYPE)
    wl = np.ascontiguousarray(wavelengths, dtype=np.float64).reshape(-1)
    eps = np.ascontiguousarray(np.broadcast_to(np.asarray(aspect_ratio, dtype=np.float64),
                                               (dists.size,)))
    m = np.ascontiguousarray(np.broadcast_to(np.asarray(m, dtype=np.complex128),
                                             (dists.size, wl.size)))
    mu = np.zeros(0) if mu is None else np.ascontiguousarray(mu, dtype=np.float64).reshape(-1)
    n = dists.size * wl.size
    kind = int(dists["kind"][0]) if dists.size else 1
    P = {3: 3, 4: 1, TABULATED: 0}.get(kind, 2) + 3
    opts = FixedOptions(int(n_nodes), int(greek_order), int(normalized), int(allow_unvalidated))
    values = np.zeros((11, n))
    d_values = np.zeros((P, 11, n))
    phase = np.zeros((6, n, mu.size)) if mu.size else None
    d_phase = np.zeros((P, 6, n, mu.size)) if mu.size else None
    greek = np.zeros((6, n, greek_order + 1)) if greek_order >= 0 else None
    d_greek = np.zeros((P, 6, n, greek_order + 1)) if greek_order >= 0 else None
    terms = np.zeros((n, int(n_nodes), 2), dtype=np.int32)
    err = ctypes.create_string_buffer(1024)
    st = load().scatrs_ensemble_fixed_spheroid_d(
        dists.ctypes.data, dists.size, _p(wl), wl.size, _p(eps), _p(m.view(np.float64)), _p(mu),
        mu.size, ctypes.byref(opts), float(tmatrix_rtol), _p(values), _p(phase), _p(greek),
        _p(d_values), _p(d_phase), _p(d_greek), terms.ctypes.data, err, 1024)
    _check(st, err)
    return values, phase, greek, d_values, d_phase, d_greek, terms


def ensemble_fixed_d(dists: np.ndarray, wavelengths, m, mu, n_nodes: int, greek_order: int = -1,
                     normalized: bool = True, allow_unvalidated: bool = False):
    """ensemble_fixed with the derivatives along the distribution's parameters, then Re m and
    Im m (P of them; every distribution of one kind): returns (values, phase, greek, d_values,
    d_phase, d_greek), the derivative arrays shaped (P,) + the value array's shape."""
    require_device()
    dists = np.ascontiguousarray(dists, dtype=DIST_DTYPE)
    wl = np.ascontiguousarray(wavelengths, dtype=np.float64).reshape(-1)
    m = np.ascontiguousarray(np.broadcast_to(np.asarray(m, dtype=np.complex128),
                                             (dists.size, wl.size)))
    mu = np.zeros(0) if mu is None else np.ascontiguousarray(mu, dtype=np.float64).reshape(-1)
    n = dists.size * wl.size
    kind = int(dists["kind"][0]) if dists.size else KINDS["lognormal"]
    P = {3: 3, 4: 1, TABULATED: 0}.get(kind, 2) + 2
    opts = FixedOptions(int(n_nodes), int(greek_order), int(normalized), int(allow_unvalidated))
    values, d_values = np.zeros((11, n)), np.zeros((P, 11, n))
    phase = np.zeros((6, n, mu.size)) if mu.size else None
    d_phase = np.zeros((P, 6, n, mu.size)) if mu.size else None
    greek = np.zeros((6, n, greek_order + 1)) if greek_order >= 0 else None
    d_greek = np.zeros((P, 6, n, greek_order + 1)) if greek_order >= 0 else None
    err = ctypes.create_string_buffer(1024)
    st = load().scatrs_ensemble_fixed_d(dists.ctypes.data, dists.size, _p(wl), wl.size,
                                        _p(m.view(np.float64)), _p(mu), mu.size,
                                        ctypes.byref(opts), _p(values), _p(phase), _p(greek),
                                        _p(d_values), _p(d_phase), _p(d_greek), err, 1024)
    _check(st, err)
    return values, phase, greek, d_values, d_phase, d_greek


def ensemble_adaptive(dists: np.ndarray, wavelengths, m, mu=None, greek_order: int = -1,
                      normalized: bool = True, rtol: float = 1e-6, max_panels: int = 4096,
                      allow_unvalidated: bool = False, refine_backscatter: bool = False,
                      batch: bool = False) -> dict:
    """The adaptive ensemble of spheres (the reference's default integration) with m per
    wavelength: each distribution on its own, or one batch sharing panels. Returns values,
    errors (11, n), phase/phase_err (6, n, n_mu), greek/greek_err (6, n, L + 1), converged,
    panels (n), units distribution-major."""
    require_device()
    dists = np.ascontiguousarray(dists, dtype=DIST_DTYPE)
    wl = np.ascontiguousarray(wavelengths, dtype=np.float64).reshape(-1)
    m = np.ascontiguousarray(np.broadcast_to(np.asarray(m, dtype=np.complex128), wl.shape))
    mu = np.zeros(0) if mu is None else np.ascontiguousarray(mu, dtype=np.float64).reshape(-1)
    n = dists.size * wl.size
    L = int(greek_order)
    opts = AdaptiveOptions(float(rtol), int(max_panels), L, int(normalized),
                           int(allow_unvalidated), int(refine_backscatter))
    out = {"values": np.zeros((11, n)), "errors": np.zeros((11, n)),
           "converged": np.zeros(n, dtype=np.int8), "panels": np.zeros(n, dtype=np.int64)}
    ph = pe = g = ge = None
    if mu.size:
        ph, pe = np.zeros((6, n, mu.size)), np.zeros((6, n, mu.size))
    if L >= 0:
        g, ge = np.zeros((6, n, L + 1)), np.zeros((6, n, L + 1))
    err = ctypes.create_string_buffer(1024)
    st = load().scatrs_ensemble_adaptive(dists.ctypes.data, dists.size, int(batch), _p(wl),
                                         wl.size, _p(m.view(np.float64)), _p(mu), mu.size,
                                         ctypes.byref(opts), _p(out["values"]),
                                         _p(out["errors"]), _p(ph), _p(pe), _p(g), _p(ge),
                                         out["converged"].ctypes.data, out["panels"].ctypes.data,
                                         err, 1024)
    _check(st, err)
    out["converged"] = out["converged"].astype(bool)
    if ph is not None:
        out["phase"], out["phase_err"] = ph, pe
    if g is not None:
        out["greek"], out["greek_err"] = g, ge
    if L == GREEK_ALL:
        _take_all_orders(out, n)
    return out


def ensemble_adaptive_layered(dists: np.ndarray, wavelengths, fractions, m_layers, mu=None,
                               greek_order: int = -1, normalized: bool = True,
                               rtol: float = 1e-6, max_panels: int = 4096,
                               allow_unvalidated: bool = False, refine_backscatter: bool = False,
                               batch: bool = False) -> dict:
    """ensemble_adaptive for layered spheres: fractions (n_dist, L - 1), m_layers complex
    (n_dist, L, n_wl); the same outputs."""
    require_device()
    dists = np.ascontiguousarray(dists, dtype=DIST_DTYPE)
    wl = np.ascontiguousarray(wavelengths, dtype=np.float64).reshape(-1)
    ml = np.ascontiguousarray(np.asarray(m_layers, dtype=np.complex128))
    nl = ml.shape[1]
    fr = np.ascontiguousarray(np.asarray(fractions, dtype=np.float64).reshape(dists.size,
                                                                              max(nl - 1, 0)))
    mu = np.zeros(0) if mu is None else np.ascontiguousarray(mu, dtype=np.float64).reshape(-1)
    n = dists.size * wl.size
    L = int(greek_order)
    opts = AdaptiveOptions(float(rtol), int(max_panels), L, int(normalized),
                           int(allow_unvalidated), int(refine_backscatter))
    lay = Layers(nl, 0, _p(fr), _p(ml.view(np.float64)))
    out = {"values": np.zeros((11, n)), "errors": np.zeros((11, n)),
           "converged": np.zeros(n, dtype=np.int8), "panels": np.zeros(n, dtype=np.int64)}
    ph = pe = g = ge = None
    if mu.size:
        ph, pe = np.zeros((6, n, mu.size)), np.zeros((6, n, mu.size))
    if L >= 0:
        g, ge = np.zeros((6, n, L + 1)), np.zeros((6, n, L + 1))
    err = ctypes.create_string_buffer(1024)
    st = load().scatrs_ensemble_adaptive_layered(
        dists.ctypes.data, dists.size, int(batch), _p(wl), wl.size, ctypes.byref(lay), _p(mu),
        mu.size, ctypes.byref(opts), _p(out["values"]), _p(out["errors"]), _p(ph), _p(pe),
        _p(g), _p(ge), out["converged"].ctypes.data, out["panels"].ctypes.data, err, 1024)
    _check(st, err)
    out["converged"] = out["converged"].astype(bool)
    if ph is not None:
        out["phase"], out["phase_err"] = ph, pe
    if g is not None:
        out["greek"], out["greek_err"] = g, ge
    if L == GREEK_ALL:
        _take_all_orders(out, n)
    return out


def ensemble_adaptive_spheroid(dists: np.ndarray, wavelengths, aspect_ratio: float, m, mu=None,
                                greek_order: int = -1, normalized: bool = True,
                                rtol: float = 1e-6, max_panels: int = 4096,
                                allow_unvalidated: bool = False,
                                refine_backscatter: bool = False, batch: bool = False) -> dict:
    """ensemble_adaptive for randomly oriented spheroids (one aspect ratio, m per wavelength);
    the same outputs."""
    require_device()
    dists = np.ascontiguousarray(dists, dtype=DIST_DTYPE)
    wl = np.ascontiguousarray(wavelengths, dtype=np.float64).reshape(-1)
    m = np.ascontiguousarray(np.broadcast_to(np.asarray(m, dtype=np.complex128), wl.shape))
    mu = np.zeros(0) if mu is None else np.ascontiguousarray(mu, dtype=np.float64).reshape(-1)
    n = dists.size * wl.size
    L = int(greek_order)
    opts = AdaptiveOptions(float(rtol), int(max_panels), L, int(normalized),
                           int(allow_unvalidated), int(refine_backscatter))
    out = {"values": np.zeros((11, n)), "errors": np.zeros((11, n)),
           "converged": np.zeros(n, dtype=np.int8), "panels": np.zeros(n, dtype=np.int64)}
    ph = pe = g = ge = None
    if mu.size:
        ph, pe = np.zeros((6, n, mu.size)), np.zeros((6, n, mu.size))
    if L >= 0:
        g, ge = np.zeros((6, n, L + 1)), np.zeros((6, n, L + 1))
    err = ctypes.create_string_buffer(1024)
    st = load().scatrs_ensemble_adaptive_spheroid(
        dists.ctypes.data, dists.size, int(batch), _p(wl), wl.size, float(aspect_ratio),
        _p(m.view(np.float64)), _p(mu), mu.size, ctypes.byref(opts), _p(out["values"]),
        _p(out["errors"]), _p(ph), _p(pe), _p(g), _p(ge), out["converged"].ctypes.data,
        out["panels"].ctypes.data, err, 1024)
    _check(st, err)
    out["converged"] = out["converged"].astype(bool)
    if ph is not None:
        out["phase"], out["phase_err"] = ph, pe
    if g is not None:
        out["greek"], out["greek_err"] = g, ge
    if L == GREEK_ALL:
        _take_all_orders(out, n)
    return out


def ensemble_mixture(components, wavelengths, mu=None, greek_order: int = -1,
                     normalized: bool = True, rtol: float = 1e-6, max_panels: int = 4096,
                     allow_unvalidated: bool = False, refine_backscatter: bool = False) -> dict:
    """The adaptive ensemble of a mixture of sphere components [(dists, mode_weights or None,
    weight, m)], dists a DIST_DTYPE array (one distribution, or a multimodal one's modes), m per
    wavelength. Outputs per wavelength, as ensemble_adaptive."""
    require_device()
    wl = np.ascontiguousarray(wavelengths, dtype=np.float64).reshape(-1)
    keep = []
    comps = (Component * max(len(components), 1))()
    for k, (dists, mode_w, weight, m) in enumerate(components):
        comps[k] = _component(dists, mode_w, weight, m, wl.size, keep)
    mu = np.zeros(0) if mu is None else np.ascontiguousarray(mu, dtype=np.float64).reshape(-1)
    n = wl.size
    L = int(greek_order)
    opts = AdaptiveOptions(float(rtol), int(max_panels), L, int(normalized),
                           int(allow_unvalidated), int(refine_backscatter))
    out = {"values": np.zeros((11, n)), "errors": np.zeros((11, n)),
           "converged": np.zeros(n, dtype=np.int8), "panels": np.zeros(n, dtype=np.int64)}
    ph = pe = g = ge = None
    if mu.size:
        ph, pe = np.zeros((6, n, mu.size)), np.zeros((6, n, mu.size))
    if L >= 0:
        g, ge = np.zeros((6, n, L + 1)), np.zeros((6, n, L + 1))
    err = ctypes.create_string_buffer(1024)
    st = load().scatrs_ensemble_mixture(comps, len(components), _p(wl), wl.size, _p(mu), mu.size,
                                        ctypes.byref(opts), _p(out["values"]), _p(out["errors"]),
                                        _p(ph), _p(pe), _p(g), _p(ge),
                                        out["converged"].ctypes.data, out["panels"].ctypes.data,
                                        err, 1024)
    _check(st, err)
    out["converged"] = out["converged"].astype(bool)
    if ph is not None:
        out["phase"], out["phase_err"] = ph, pe
    if g is not None:
        out["greek"], out["greek_err"] = g, ge
    if L == GREEK_ALL:
        _take_all_orders(out, n)
    return out


GREEK_ALL = -2  # every order up to 2 N_max per wavelength (adaptive calls)


def _take_all_orders(out: dict, n: int, P: int = 0) -> None:
    """The Greek coefficients of this thread's last GREEK_ALL call into out, (6, n, W) and
    with derivatives (P, 6, n, W)."""
    w = int(load().scatrs_greek_all_width())
    g, ge = np.zeros((6, n, w)), np.zeros((6, n, w))
    dg, dge = np.zeros((P, 6, n, w)), np.zeros((P, 6, n, w))
    load().scatrs_greek_all_take(_p(g), _p(ge), _p(dg) if P else None, _p(dge) if P else None)
    out["greek"], out["greek_err"] = g, ge
    if P:
        out["greek_d"], out["greek_d_err"] = dg, dge


def _component(dists, mode_w, weight, m, n_wl: int, keep: list) -> Component:
    """A mixture component: its distribution records, mode weights (or None) and weight, and
    its particle: m per wavelength (a sphere), or ("sphere", m), ("layered", fractions,
    m (L, n_wl)), ("spheroid", aspect_ratio, m). The arrays go to keep."""
    d = np.ascontiguousarray(np.atleast_1d(dists), dtype=DIST_DTYPE)
    mw = None if mode_w is None else np.ascontiguousarray(mode_w, dtype=np.float64)
    n_layers, fr, eps = 0, None, 0.0
    if isinstance(m, tuple) and m[0] == "layered":
        fr = np.ascontiguousarray(np.asarray(m[1], dtype=np.float64).reshape(-1))
        mm = np.ascontiguousarray(np.asarray(m[2], dtype=np.complex128).reshape(-1, n_wl))
        n_layers = mm.shape[0]
    else:
        if isinstance(m, tuple):
            eps = float(m[1]) if m[0] == "spheroid" else 0.0
            m = m[-1]
        mm = np.ascontiguousarray(np.broadcast_to(np.asarray(m, dtype=np.complex128), (n_wl,)))
    keep += [d, mw, mm, fr]
    return Component(d.ctypes.data, _p(mw), d.size, n_layers, float(weight),
                     _p(mm.view(np.float64).reshape(-1)), _p(fr), eps)


# scatrs_param: (component, mode or -1, kind, index); kinds as SCATRS_PARAM_*.
PARAM_DTYPE = np.dtype([("component", np.int32), ("mode", np.int32), ("kind", np.int32),
                        ("index", np.int32)])
PARAM_DISTRIBUTION, PARAM_REFR_REAL, PARAM_REFR_IMAG, PARAM_WEIGHT = 0, 1, 2, 3
PARAM_ASPECT_RATIO, PARAM_LAYER_REFR_REAL, PARAM_LAYER_REFR_IMAG, PARAM_RADIUS_FRACTION = 4, 5, 6, 7


def ensemble_mixture_d(components, wavelengths, params, mu=None, greek_order: int = -1,
                       normalized: bool = True, rtol: float = 1e-6, max_panels: int = 4096,
                       allow_unvalidated: bool = False, refine_backscatter: bool = False) -> dict:
    """ensemble_mixture with the derivatives along `params` (PARAM_DTYPE records); a component
    whose mode weights are given is multimodal. Adds d, d_err (P, 11, n), and with phase or
    Greek coefficients phase_d, phase_d_err (P, 6, n, n_mu), greek_d, greek_d_err
    (P, 6, n, L + 1)."""
    require_device()
    wl = np.ascontiguousarray(wavelengths, dtype=np.float64).reshape(-1)
    keep = []
    comps = (Component * max(len(components), 1))()
    for k, (dists, mode_w, weight, m) in enumerate(components):
        comps[k] = _component(dists, mode_w, weight, m, wl.size, keep)
    pr = np.ascontiguousarray(np.atleast_1d(np.asarray(params, dtype=PARAM_DTYPE)))
    P = pr.size
    mu = np.zeros(0) if mu is None else np.ascontiguousarray(mu, dtype=np.float64).reshape(-1)
    n = wl.size
    L = int(greek_order)
    opts = AdaptiveOptions(float(rtol), int(max_panels), L, int(normalized),
                           int(allow_unvalidated), int(refine_backscatter))
    out = {"values": np.zeros((11, n)), "errors": np.zeros((11, n)),
           "d": np.zeros((P, 11, n)), "d_err": np.zeros((P, 11, n)),
           "converged": np.zeros(n, dtype=np.int8), "panels": np.zeros(n, dtype=np.int64)}
    ph = pe = g = ge = dph = dpe = dg = dge = None
    if mu.size:
        ph, pe = np.zeros((6, n, mu.size)), np.zeros((6, n, mu.size))
        dph, dpe = np.zeros((P, 6, n, mu.size)), np.zeros((P, 6, n, mu.size))
    if L >= 0:
        g, ge = np.zeros((6, n, L + 1)), np.zeros((6, n, L + 1))
        dg, dge = np.zeros((P, 6, n, L + 1)), np.zeros((P, 6, n, L + 1))
    err = ctypes.create_string_buffer(1024)
    st = load().scatrs_ensemble_mixture_d(
        comps, len(components), _p(wl), wl.size, _p(mu), mu.size, ctypes.byref(opts),
        pr.ctypes.data if P else None, P, _p(out["values"]), _p(out["errors"]), _p(out["d"]),
        _p(out["d_err"]), _p(ph), _p(pe), _p(dph), _p(dpe), _p(g), _p(ge), _p(dg), _p(dge),
        out["converged"].ctypes.data, out["panels"].ctypes.data, err, 1024)
    _check(st, err)
    out["converged"] = out["converged"].astype(bool)
    if ph is not None:
        out["phase"], out["phase_err"], out["phase_d"], out["phase_d_err"] = ph, pe, dph, dpe
    if g is not None:
        out["greek"], out["greek_err"], out["greek_d"], out["greek_d_err"] = g, ge, dg, dge
    if L == GREEK_ALL:
        _take_all_orders(out, n, P)
    return out


def ensemble_fixed_layered(dists: np.ndarray, wavelengths, fractions, m_layers, mu,
                           n_nodes: int, greek_order: int = -1, normalized: bool = True,
                           allow_unvalidated: bool = False):
    """The fixed-grid ensemble of layered spheres: fractions (n_dist, L - 1), m_layers complex
    (n_dist, L, n_wl); outputs as ensemble_fixed."""
    require_device()
    dists = np.ascontiguousarray(dists, dtype=DIST_DTYPE)
    wl = np.ascontiguousarray(wavelengths, dtype=np.float64).reshape(-1)
    ml = np.ascontiguousarray(m_layers, dtype=np.complex128)
    n_layers = ml.shape[1]
    fr = np.ascontiguousarray(fractions, dtype=np.float64).reshape(dists.size, n_layers - 1)
    mu = np.zeros(0) if mu is None else np.ascontiguousarray(mu, dtype=np.float64).reshape(-1)
    n = dists.size * wl.size
    lay = Layers(n_layers, 0, _p(fr), _p(ml.view(np.float64).reshape(-1)))
    opts = FixedOptions(int(n_nodes), int(greek_order), int(normalized), int(allow_unvalidated))
    values = np.zeros((11, n))
    phase = np.zeros((6, n, mu.size)) if mu.size else None
    greek = np.zeros((6, n, greek_order + 1)) if greek_order >= 0 else None
    err = ctypes.create_string_buffer(1024)
    st = load().scatrs_ensemble_fixed_layered(dists.ctypes.data, dists.size, _p(wl), wl.size,
                                              ctypes.byref(lay), _p(mu), mu.size,
                                              ctypes.byref(opts), _p(values), _p(phase),
                                              _p(greek), err, 1024)
    _check(st, err)
    return values, phase, greek


def ensemble_fixed_layered_d(dists: np.ndarray, wavelengths, fractions, m_layers, mu,
                             n_nodes: int, greek_order: int = -1, normalized: bool = True,
                             allow_unvalidated: bool = False):
    """ensemble_fixed_layered with the derivatives along the distribution's parameters, then
    Re m_l and Im m_l of every layer, then the fractions (P blocks); returns (values, phase,
    greek, d_values, d_phase, d_greek), the derivative arrays shaped (P,) + the value array's
    shape."""
    require_device()
    dists = np.ascontiguousarray(dists, dtype=DIST_DTYPE)
    wl = np.ascontiguousarray(wavelengths, dtype=np.float64).reshape(-1)
    ml = np.ascontiguousarray(m_layers, dtype=np.complex128)
    nl = ml.shape[1]
    fr = np.ascontiguousarray(fractions, dtype=np.float64).reshape(dists.size, nl - 1)
    mu = np.zeros(0) if mu is None else np.ascontiguousarray(mu, dtype=np.float64).reshape(-1)
    n = dists.size * wl.size
    kind = int(dists["kind"][0]) if dists.size else KINDS["lognormal"]
    P = {3: 3, 4: 1, TABULATED: 0}.get(kind, 2) + 3 * nl - 1
    lay = Layers(nl, 0, _p(fr), _p(ml.view(np.float64).reshape(-1)))
    opts = FixedOptions(int(n_nodes), int(greek_order), int(normalized), int(allow_unvalidated))
    values, d_values = np.zeros((11, n)), np.zeros((P, 11, n))
    phase = np.zeros((6, n, mu.size)) if mu.size else None
    d_phase = np.zeros((P, 6, n, mu.size)) if mu.size else None
    greek = np.zeros((6, n, greek_order + 1)) if greek_order >= 0 else None
    d_greek = np.zeros((P, 6, n, greek_order + 1)) if greek_order >= 0 else None
    err = ctypes.create_string_buffer(1024)
    st = load().scatrs_ensemble_fixed_layered_d(dists.ctypes.data, dists.size, _p(wl), wl.size,
                                                ctypes.byref(lay), _p(mu), mu.size,
                                                ctypes.byref(opts), _p(values), _p(phase),
                                                _p(greek), _p(d_values), _p(d_phase),
                                                _p(d_greek), err, 1024)
    _check(st, err)
    return values, phase, greek, d_values, d_phase, d_greek


def ensemble_fixed_device(dists: np.ndarray, wl_ptr: int, n_wl: int, m_ptr: int, mu, n_nodes: int,
                          greek_order: int, normalized: bool, values_ptr: int, phase_ptr: int,
                          greek_ptr: int, stream: int = 0, allow_unvalidated: bool = False,
                          i8_above: int = 0, levels: int = 0):
    """The fixed-grid ensemble on device arrays (raw pointers, e.g. torch's data_ptr()),
    enqueued on `stream`; device-side input errors surface in check_errors(stream).
    i8_above > 0: the mixed form (scatrs_ensemble_fixed_mixed_device)."""
    dists = np.ascontiguousarray(dists, dtype=DIST_DTYPE)
    mu = np.zeros(0) if mu is None else np.ascontiguousarray(mu, dtype=np.float64).reshape(-1)
    opts = FixedOptions(int(n_nodes), int(greek_order), int(normalized), int(allow_unvalidated))
    err = ctypes.create_string_buffer(1024)
    if i8_above > 0:
        st = load().scatrs_ensemble_fixed_mixed_device(
            dists.ctypes.data, dists.size, wl_ptr, n_wl, m_ptr, _p(mu), mu.size,
            ctypes.byref(opts), ctypes.byref(MixedOptions(int(i8_above), int(levels))),
            values_ptr, phase_ptr or None, greek_ptr or None, stream or None, err, 1024)
    else:
        st = load().scatrs_ensemble_fixed_device(dists.ctypes.data, dists.size, wl_ptr, n_wl,
                                                 m_ptr, _p(mu), mu.size, ctypes.byref(opts),
                                                 values_ptr, phase_ptr or None,
                                                 greek_ptr or None, stream or None, err, 1024)
    _check(st, err)


def project_greek_device(phase_ptr: int, n_units: int, n_q: int, order: int, precision: int,
                         greek_ptr: int, stream: int = 0) -> None:
    """Greek coefficients of device tables at the n_q Gauss cosines (raw device pointers):
    precision 0 FP64, 1 3xTF32 on the tensor cores."""
    err = ctypes.create_string_buffer(1024)
    _check(load().scatrs_project_greek_device(phase_ptr, int(n_units), int(n_q), int(order),
                                              int(precision), greek_ptr, stream or None, err,
                                              1024), err)


def spheroid_tmatrix(x: float, aspect_ratio: float, m: complex, mode: int, n_terms: int,
                     n_theta: int) -> np.ndarray:
    """The T-matrix of one azimuthal mode of a spheroid: (2K, 2K) complex."""
    require_device()
    k = n_terms - max(mode, 1) + 1
    t = np.zeros(2 * (2 * k) ** 2)
    mm = np.array([complex(m).real, complex(m).imag])
    err = ctypes.create_string_buffer(1024)
    _check(load().scatrs_spheroid_tmatrix(float(x), float(aspect_ratio), _p(mm), int(mode),
                                          int(n_terms), int(n_theta), _p(t), err, 1024), err)
    return t.view(np.complex128).reshape(2 * k, 2 * k)


def spheroid_efficiencies(x, aspect_ratio, m, rtol: float = 1e-8):
    """Orientation-averaged (Q_ext, Q_sca, Q_abs) of spheroids ((n, 3)), with the N and n_theta
    each converged at."""
    require_device()
    x = np.ascontiguousarray(np.atleast_1d(x), dtype=np.float64)
    eps = np.ascontiguousarray(np.broadcast_to(np.asarray(aspect_ratio, dtype=np.float64), x.shape))
    mm = np.ascontiguousarray(np.broadcast_to(np.asarray(m, dtype=np.complex128), x.shape))
    q = np.zeros((x.size, 3))
    n_terms = np.zeros(x.size, dtype=np.int32)
    n_theta = np.zeros(x.size, dtype=np.int32)
    err = ctypes.create_string_buffer(1024)
    _check(load().scatrs_spheroid_efficiencies(x.size, _p(x), _p(eps), _p(mm.view(np.float64)),
                                               float(rtol), _p(q), n_terms.ctypes.data,
                                               n_theta.ctypes.data, err, 1024), err)
    return q, n_terms, n_theta


def spheroid_compute(x, aspect_ratio, m, rtol: float = 1e-8, n_terms: int = 0, n_theta: int = 0,
                     greek_order: int = -1, normalized: bool = True,
                     allow_unvalidated: bool = False) -> dict:
    """Randomly oriented spheroids: efficiencies (n, 5) = Q_ext, Q_sca, Q_abs, Q_back, g; Greek
    coefficients (n, 6, order + 1) if greek_order >= 0; the N and n_theta used and the
    refinement's error estimate."""
    require_device()
    x = np.ascontiguousarray(np.atleast_1d(x), dtype=np.float64)
    eps = np.ascontiguousarray(np.broadcast_to(np.asarray(aspect_ratio, dtype=np.float64), x.shape))
    mm = np.ascontiguousarray(np.broadcast_to(np.asarray(m, dtype=np.complex128), x.shape))
    eff = np.zeros((x.size, 5))
    greek = np.zeros((x.size, 6, greek_order + 1)) if greek_order >= 0 else None
    nt = np.zeros(x.size, dtype=np.int32)
    nth = np.zeros(x.size, dtype=np.int32)
    est = np.zeros(x.size)
    o = SpheroidOptions(rtol, n_terms, n_theta, greek_order, int(normalized),
                        int(allow_unvalidated))
    err = ctypes.create_string_buffer(1024)
    _check(load().scatrs_spheroid_compute(x.size, _p(x), _p(eps), _p(mm.view(np.float64)),
                                          ctypes.byref(o), _p(eff), _p(greek), nt.ctypes.data,
                                          nth.ctypes.data, _p(est), err, 1024), err)
    return {"efficiencies": eff, "greek": greek, "n_terms": nt, "n_theta": nth,
            "error_estimate": est}


SPHEROID_DIRECTIONS = ("x", "aspect_ratio", "m_re", "m_im")


def spheroid_compute_d(x, aspect_ratio, m, rtol: float = 1e-8, n_terms: int = 0,
                       n_theta: int = 0, greek_order: int = -1, normalized: bool = True,
                       allow_unvalidated: bool = False) -> dict:
    """spheroid_compute with the derivatives of the efficiencies and Greek coefficients along
    x, the aspect ratio, Re m and Im m (scatrs_spheroid_compute_d): d_efficiencies (4, n, 5),
    d_greek (4, n, 6, order + 1), in the order of SPHEROID_DIRECTIONS."""
    require_device()
    x = np.ascontiguousarray(np.atleast_1d(x), dtype=np.float64)
    eps = np.ascontiguousarray(np.broadcast_to(np.asarray(aspect_ratio, dtype=np.float64), x.shape))
    mm = np.ascontiguousarray(np.broadcast_to(np.asarray(m, dtype=np.complex128), x.shape))
    n = x.size
    eff = np.zeros((n, 5))
    d_eff = np.zeros((4, n, 5))
    greek = np.zeros((n, 6, greek_order + 1)) if greek_order >= 0 else None
    d_greek = np.zeros((4, n, 6, greek_order + 1)) if greek_order >= 0 else None
    nt = np.zeros(n, dtype=np.int32)
    nth = np.zeros(n, dtype=np.int32)
    est = np.zeros(n)
    o = SpheroidOptions(rtol, n_terms, n_theta, greek_order, int(normalized),
                        int(allow_unvalidated))
    err = ctypes.create_string_buffer(1024)
    _check(load().scatrs_spheroid_compute_d(n, _p(x), _p(eps), _p(mm.view(np.float64)),
                                            ctypes.byref(o), _p(eff), _p(greek), _p(d_eff),
                                            _p(d_greek), nt.ctypes.data, nth.ctypes.data,
                                            _p(est), err, 1024), err)
    return {"efficiencies": eff, "greek": greek, "d_efficiencies": d_eff, "d_greek": d_greek,
            "n_terms": nt, "n_theta": nth, "error_estimate": est}


def check_errors(stream: int = 0) -> None:
    err = ctypes.create_string_buffer(1024)
    _check(load().scatrs_check_errors(stream or None, err, 1024), err)


def ensemble_fixed_d_device(dists: np.ndarray, wl_ptr: int, n_wl: int, m_ptr: int, mu,
                            n_nodes: int, greek_order: int, normalized: bool, out_ptrs,
                            stream: int = 0, allow_unvalidated: bool = False) -> None:
    """scatrs_ensemble_fixed_d_device: device arrays (raw pointers) for the wavelengths, m and the
    six outputs out_ptrs = (values, phase, greek, d_values, d_phase, d_greek); synchronizes."""
    dists = np.ascontiguousarray(dists, dtype=DIST_DTYPE)
    mu = np.zeros(0) if mu is None else np.ascontiguousarray(mu, dtype=np.float64).reshape(-1)
    opts = FixedOptions(int(n_nodes), int(greek_order), int(normalized), int(allow_unvalidated))
    err = ctypes.create_string_buffer(1024)
    st = load().scatrs_ensemble_fixed_d_device(dists.ctypes.data, dists.size, wl_ptr, n_wl, m_ptr,
                                               _p(mu), mu.size, ctypes.byref(opts),
                                               *[p or None for p in out_ptrs], stream or None,
                                               err, 1024)
    _check(st, err)


def ensemble_fixed_layered_d_device(dists: np.ndarray, wl_ptr: int, n_wl: int, fractions,
                                    n_layers: int, m_ptr: int, mu, n_nodes: int,
                                    greek_order: int, normalized: bool, out_ptrs,
                                    stream: int = 0, allow_unvalidated: bool = False) -> None:
    """scatrs_ensemble_fixed_layered_d_device: the layers' m (complex [n_dist][L][n_wl]) and the
    outputs on the device, the fractions (n_dist, L - 1) on the host; synchronizes."""
    dists = np.ascontiguousarray(dists, dtype=DIST_DTYPE)
    fr = np.ascontiguousarray(fractions, dtype=np.float64).reshape(dists.size, n_layers - 1)
    mu = np.zeros(0) if mu is None else np.ascontiguousarray(mu, dtype=np.float64).reshape(-1)
    lay = Layers(int(n_layers), 0, _p(fr), ctypes.cast(m_ptr, _PD))
    opts = FixedOptions(int(n_nodes), int(greek_order), int(normalized), int(allow_unvalidated))
    err = ctypes.create_string_buffer(1024)
    st = load().scatrs_ensemble_fixed_layered_d_device(
        dists.ctypes.data, dists.size, wl_ptr, n_wl, ctypes.byref(lay), _p(mu), mu.size,
        ctypes.byref(opts), *[p or None for p in out_ptrs], stream or None, err, 1024)
    _check(st, err)


def refractive_models(specs):
    """scatrs_refractive_model records (and the arrays they point at) from specs: ("constant", m),
    ("cauchy", A, B, C, k), ("sellmeier", B, C, k), ("table", wavelengths, m) or
    ("table_log_k", wavelengths, m)."""
    recs = (RefractiveModel * max(len(specs), 1))()
    keep = []
    for i, spec in enumerate(specs):
        kind = spec[0]
        if kind not in REFRACTIVE_KINDS:
            raise TypeError(f"unknown refractive-index model {kind!r}")
        r = recs[i]
        r.kind = REFRACTIVE_KINDS[kind]
        if kind == "constant":
            m = complex(spec[1])
            r.p[0], r.p[1] = m.real, m.imag
        elif kind == "cauchy":
            for j in range(4):
                r.p[j] = float(spec[1 + j])
        elif kind == "sellmeier":
            b = np.asarray(spec[1], dtype=np.float64).reshape(-1)
            c = np.asarray(spec[2], dtype=np.float64).reshape(-1)
            if b.size != c.size:
                raise InvalidInputError("invalid input: Sellmeier: B and C must have the same "
                                        f"length, got {b.size} and {c.size}")
            tab = np.ascontiguousarray(np.concatenate([b, c]))
            keep.append(tab)
            r.n, r.p[3], r.table = b.size, float(spec[3]), _p(tab)
        else:
            wl = np.asarray(spec[1], dtype=np.float64).reshape(-1)
            m = np.asarray(spec[2], dtype=np.complex128).reshape(-1)
            if m.size != wl.size:
                raise InvalidInputError("invalid input: a Table needs as many m as wavelengths")
            tab = np.ascontiguousarray(np.concatenate([wl, m.view(np.float64)]))
            keep.append(tab)
            r.n, r.table = wl.size, _p(tab)
    return recs, keep


def refractive_parameter_count(spec) -> int:
    recs, _keep = refractive_models([spec])
    return int(load().scatrs_refractive_parameter_count(ctypes.byref(recs[0])))


def refractive_index_device(specs, wl_ptr: int, n_wl: int, m_ptr: int, dm_ptr: int = 0,
                            p_max: int = 0, stream: int = 0) -> None:
    """m (complex [n_models][n_wl]) of every model at every wavelength into device memory, and
    dm/dtheta (complex [n_models][p_max][n_wl]) when dm_ptr is given; synchronizes."""
    recs, _keep = refractive_models(specs)
    err = ctypes.create_string_buffer(1024)
    st = load().scatrs_refractive_index_device(recs, len(specs), wl_ptr, n_wl, m_ptr,
                                               dm_ptr or None, int(p_max), stream or None, err,
                                               1024)
    _check(st, err)
