"""ctypes binding of the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY. The oracle is a plain double-precision restatement of the reference
(usask-arg/scatrs) algorithms on the size-distribution ensemble path; the parity tests, the
smoke check and the CPU-baseline leg of the benchmark use it as the checker. Nothing in the
product package imports this module.
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")
_lib = None

_D = ctypes.c_double
_I64 = ctypes.c_int64
_PD = ctypes.POINTER(ctypes.c_double)


def build() -> str:
    """Compiles liboracle.so if it is missing or older than its sources."""
    srcs = [os.path.join(_HERE, f) for f in ("oracle_capi.cpp", "oracle_core.hpp", "Makefile")]
    if not os.path.exists(_LIB) or any(os.path.getmtime(s) > os.path.getmtime(_LIB) for s in srcs):
        subprocess.run(["make", "-C", _HERE, "CXX=g++"], check=True, capture_output=True)
    return _LIB


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = ctypes.CDLL(_LIB)
        _lib.orc_mie.argtypes = [_D, _D, _D, _I64, ctypes.c_int, ctypes.c_int,
                                 ctypes.POINTER(_I64), _PD, _PD, _PD, _PD, _PD, _PD, _PD, _PD,
                                 _PD]
        _lib.orc_amplitudes.argtypes = [_D, _D, _D, _I64, _PD, _I64, _PD, _PD]
        _lib.orc_gauss_legendre.argtypes = [_I64, _PD, _PD]
        _lib.orc_gauss_legendre.restype = None
        _lib.orc_wigner_d.argtypes = [ctypes.c_int, ctypes.c_int, _D, _I64, _PD]
        _lib.orc_wigner_d.restype = None
        _lib.orc_mie_greek.argtypes = [_D, _D, _D, _I64, ctypes.c_int, _PD]
        _lib.orc_density.argtypes = [ctypes.c_int, _D, _D, _D, _D, _PD]
        _lib.orc_density.restype = _D
        _lib.orc_bucket.argtypes = [_I64]
        _lib.orc_bucket.restype = _I64
        _lib.orc_default_n_max.argtypes = [_D]
        _lib.orc_ensemble_fixed.argtypes = [ctypes.c_void_p, _I64, _PD, _I64, _PD, _I64, _PD,
                                            _I64, _I64, ctypes.c_int, ctypes.c_int,
                                            ctypes.c_int, _PD, _PD, _PD, ctypes.c_char_p, _I64]
    return _lib


def _p(a: np.ndarray | None):
    if a is None:
        return None
    return a.ctypes.data_as(_PD)


class OracleError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"status {status}: {message}")
        self.status = status


def mie(x: float, m: complex, n_max: int = 0, allow_unvalidated: bool = True,
        derivatives: bool = False) -> dict:
    """a_n, b_n (n = 1..N), efficiencies and the absorption sum of one sphere."""
    L = lib()
    n = _I64(0)
    st = L.orc_mie(x, m.real, m.imag, n_max, int(allow_unvalidated), 0, ctypes.byref(n), None,
                   None, None, None, None, None, None, None, None)
    if st != 0:
        raise OracleError(st, f"mie({x}, {m})")
    N = n.value
    a = np.zeros(2 * N)
    b = np.zeros(2 * N)
    eff = np.zeros(5)
    asum = np.zeros(1)
    d = [np.zeros(2 * N) for _ in range(4)] if derivatives else [None] * 4
    jac = np.zeros(3)
    L.orc_mie(x, m.real, m.imag, n_max, int(allow_unvalidated), int(derivatives),
              ctypes.byref(n), _p(a), _p(b), _p(eff), _p(asum), _p(d[0]), _p(d[1]), _p(d[2]),
              _p(d[3]), _p(jac))
    out = {
        "a": a.view(np.complex128), "b": b.view(np.complex128),
        "q_ext": eff[0], "q_sca": eff[1], "q_abs": eff[2], "q_back": eff[3], "g": eff[4],
        "abs_sum": asum[0], "n": N,
    }
    if derivatives:
        out.update(da_dx=d[0].view(np.complex128), da_dm=d[1].view(np.complex128),
                   db_dx=d[2].view(np.complex128), db_dm=d[3].view(np.complex128),
                   abs_jac=jac)
    return out


def amplitudes(x: float, m: complex, mu, n_max: int = 0):
    mu = np.ascontiguousarray(mu, dtype=np.float64)
    s1 = np.zeros(2 * mu.size)
    s2 = np.zeros(2 * mu.size)
    st = lib().orc_amplitudes(x, m.real, m.imag, n_max, _p(mu), mu.size, _p(s1), _p(s2))
    if st != 0:
        raise OracleError(st, "amplitudes")
    return s1.view(np.complex128), s2.view(np.complex128)


def gauss_legendre(n: int):
    x = np.zeros(n)
    w = np.zeros(n)
    lib().orc_gauss_legendre(n, _p(x), _p(w))
    return x, w


def wigner_d(m: int, n: int, x: float, l_max: int):
    out = np.zeros(l_max + 1)
    lib().orc_wigner_d(m, n, x, l_max + 1, _p(out))
    return out


def mie_greek(x: float, m: complex, order: int, normalized: bool = True):
    out = np.zeros(6 * (order + 1))
    st = lib().orc_mie_greek(x, m.real, m.imag, order, int(normalized), _p(out))
    if st != 0:
        raise OracleError(st, "greek")
    return out.reshape(6, order + 1)


def density(kind: int, params, r: float):
    p = list(params) + [0.0] * (3 - len(params))
    g = np.zeros(3)
    u = lib().orc_density(kind, p[0], p[1], p[2], r, _p(g))
    return u, g


def bucket(n: int) -> int:
    return lib().orc_bucket(n)


def default_n_max(x: float) -> int:
    return lib().orc_default_n_max(x)


DIST_DTYPE = np.dtype([("kind", np.int32), ("pad", np.int32), ("p", np.float64, 3),
                       ("r_lo", np.float64), ("r_hi", np.float64), ("table", np.uint64),
                       ("table_len", np.int64)])
TABULATED = 6


def ensemble_fixed(dists: np.ndarray, wavelengths, m, n_nodes: int, mu=None,
                   greek_order: int | None = None, normalized: bool = True,
                   allow_unvalidated: bool = False, threads: int = 0) -> dict:
    """The fixed-grid ensemble of every (distribution, wavelength) unit, distribution-major.

    ``dists`` is a structured array of ``DIST_DTYPE``; ``m`` has shape (n_dist, n_wl)."""
    dists = np.ascontiguousarray(dists, dtype=DIST_DTYPE)
    wl = np.ascontiguousarray(wavelengths, dtype=np.float64).reshape(-1)
    m = np.ascontiguousarray(np.broadcast_to(np.asarray(m, dtype=np.complex128),
                                             (dists.size, wl.size)))
    mu = np.zeros(0) if mu is None else np.ascontiguousarray(mu, dtype=np.float64).reshape(-1)
    n_units = dists.size * wl.size
    values = np.zeros((11, n_units))
    phase = np.zeros((6, n_units, mu.size)) if mu.size else None
    L = -1 if greek_order is None else int(greek_order)
    greek = np.zeros((6, n_units, L + 1)) if L >= 0 else None
    err = ctypes.create_string_buffer(512)
    mv = m.view(np.float64).reshape(-1)
    st = lib().orc_ensemble_fixed(dists.ctypes.data, dists.size, _p(wl), wl.size, _p(mv),
                                  n_nodes, _p(mu), mu.size, L, int(normalized),
                                  int(allow_unvalidated), threads, _p(values), _p(phase),
                                  _p(greek), err, 512)
    if st != 0:
        raise OracleError(st, err.value.decode())
    out = {"values": values}
    if phase is not None:
        out["phase"] = phase
    if greek is not None:
        out["greek"] = greek
    return out


def layered(x, m):
    """A layered sphere: x the interface size parameters (outer last), m the layers' indices."""
    L = lib()
    x = np.ascontiguousarray(x, dtype=np.float64)
    mv = np.ascontiguousarray(np.asarray(m, dtype=np.complex128)).view(np.float64)
    f = L.orc_layered
    f.argtypes = [_PD, _PD, _I64, ctypes.POINTER(_I64), _PD, _PD, _PD]
    n = _I64(0)
    f(_p(x), _p(mv), x.size, ctypes.byref(n), None, None, None)
    N = n.value
    a, b, eff = np.zeros(2 * N), np.zeros(2 * N), np.zeros(5)
    f(_p(x), _p(mv), x.size, ctypes.byref(n), _p(a), _p(b), _p(eff))
    return {"a": a.view(np.complex128), "b": b.view(np.complex128), "q_ext": eff[0],
            "q_sca": eff[1], "q_abs": eff[2], "q_back": eff[3], "g": eff[4], "n": N}


def ensemble_fixed_layered(dists: np.ndarray, wavelengths, fractions, m_layers, n_nodes: int,
                           mu=None, greek_order: int | None = None, normalized: bool = True,
                           allow_unvalidated: bool = False, threads: int = 0) -> dict:
    """As ensemble_fixed for layered spheres: fractions (n_dist, L - 1), m_layers complex
    (n_dist, L, n_wl)."""
    dists = np.ascontiguousarray(dists, dtype=DIST_DTYPE)
    wl = np.ascontiguousarray(wavelengths, dtype=np.float64).reshape(-1)
    ml = np.ascontiguousarray(m_layers, dtype=np.complex128)
    L = ml.shape[1]
    fr = np.ascontiguousarray(fractions, dtype=np.float64).reshape(dists.size, L - 1)
    mu = np.zeros(0) if mu is None else np.ascontiguousarray(mu, dtype=np.float64).reshape(-1)
    n_units = dists.size * wl.size
    values = np.zeros((11, n_units))
    phase = np.zeros((6, n_units, mu.size)) if mu.size else None
    G = -1 if greek_order is None else int(greek_order)
    greek = np.zeros((6, n_units, G + 1)) if G >= 0 else None
    err = ctypes.create_string_buffer(512)
    f = lib().orc_ensemble_fixed_layered
    f.argtypes = [ctypes.c_void_p, _I64, _PD, _I64, ctypes.c_int, _PD, _PD, _I64, _PD, _I64,
                  _I64, ctypes.c_int, ctypes.c_int, ctypes.c_int, _PD, _PD, _PD,
                  ctypes.c_char_p, _I64]
    st = f(dists.ctypes.data, dists.size, _p(wl), wl.size, L, _p(fr),
           _p(ml.view(np.float64).reshape(-1)), n_nodes, _p(mu), mu.size, G, int(normalized),
           int(allow_unvalidated), threads, _p(values), _p(phase), _p(greek), err, 512)
    if st != 0:
        raise OracleError(st, err.value.decode())
    out = {"values": values}
    if phase is not None:
        out["phase"] = phase
    if greek is not None:
        out["greek"] = greek
    return out


def ensemble_fixed_d(dists: np.ndarray, wavelengths, m, n_nodes: int, mu=None,
                     greek_order: int | None = None, normalized: bool = True,
                     allow_unvalidated: bool = False, threads: int = 0) -> dict:
    """ensemble_fixed with the derivatives of every output along the distribution's parameters
    and then Re m and Im m (P directions, every distribution of one kind): d_values (P, 11, n),
    d_phase (P, 6, n, n_mu), d_greek (P, 6, n, L + 1)."""
    dists = np.ascontiguousarray(dists, dtype=DIST_DTYPE)
    wl = np.ascontiguousarray(wavelengths, dtype=np.float64).reshape(-1)
    m = np.ascontiguousarray(np.broadcast_to(np.asarray(m, dtype=np.complex128),
                                             (dists.size, wl.size)))
    mu = np.zeros(0) if mu is None else np.ascontiguousarray(mu, dtype=np.float64).reshape(-1)
    kinds = set(int(k) for k in dists["kind"])
    P = 2 + ({3: 3, 4: 1, TABULATED: 0}.get(kinds.pop(), 2) if len(kinds) == 1 else 2)
    n_units = dists.size * wl.size
    L = -1 if greek_order is None else int(greek_order)
    values = np.zeros((11, n_units))
    d_values = np.zeros((P, 11, n_units))
    phase = np.zeros((6, n_units, mu.size)) if mu.size else None
    d_phase = np.zeros((P, 6, n_units, mu.size)) if mu.size else None
    greek = np.zeros((6, n_units, L + 1)) if L >= 0 else None
    d_greek = np.zeros((P, 6, n_units, L + 1)) if L >= 0 else None
    err = ctypes.create_string_buffer(512)
    f = lib().orc_ensemble_fixed_d
    f.argtypes = [ctypes.c_void_p, _I64, _PD, _I64, _PD, _I64, _PD, _I64, _I64, ctypes.c_int,
                  ctypes.c_int, ctypes.c_int, _PD, _PD, _PD, _PD, _PD, _PD, ctypes.c_char_p,
                  _I64]
    st = f(dists.ctypes.data, dists.size, _p(wl), wl.size, _p(m.view(np.float64).reshape(-1)),
           n_nodes, _p(mu), mu.size, L, int(normalized), int(allow_unvalidated), threads,
           _p(values), _p(phase), _p(greek), _p(d_values), _p(d_phase), _p(d_greek), err, 512)
    if st != 0:
        raise OracleError(st, err.value.decode())
    out = {"values": values, "d_values": d_values}
    if phase is not None:
        out["phase"], out["d_phase"] = phase, d_phase
    if greek is not None:
        out["greek"], out["d_greek"] = greek, d_greek
    return out


MONODISPERSE = 5


def _take_all_orders(out: dict, n: int, P: int = 0) -> None:
    """The Greek coefficients of the last greek_order="all" call, zero-padded to the longest."""
    f = lib().orc_greek_all_width
    f.restype = _I64
    w = int(f())
    g, ge = np.zeros((6, n, w)), np.zeros((6, n, w))
    dg, dge = np.zeros((P, 6, n, w)), np.zeros((P, 6, n, w))
    t = lib().orc_greek_all_take
    t.argtypes = [_PD, _PD, _PD, _PD]
    t(_p(g), _p(ge), _p(dg) if P else None, _p(dge) if P else None)
    out["greek"], out["greek_err"] = g, ge
    if P:
        out["greek_d"], out["greek_d_err"] = dg, dge


def ensemble_adaptive(dists: np.ndarray, wavelengths, m, mu=None, greek_order=None,
                      normalized: bool = True, rtol: float = 1e-6, max_panels: int = 4096,
                      allow_unvalidated: bool = False, refine_backscatter: bool = False,
                      batch: bool = False, threads: int = 0) -> dict:
    """The reference's adaptive ensemble of spheres (m per wavelength): every distribution on
    its own (batch=False) or as one batch sharing panels (batch=True). Distribution kinds as
    DIST_DTYPE, plus MONODISPERSE (p[0] the radius); r_lo, r_hi unused. Returns values,
    errors, phase(_err), greek(_err), converged, panels; units distribution-major."""
    dists = np.ascontiguousarray(dists, dtype=DIST_DTYPE)
    wl = np.ascontiguousarray(wavelengths, dtype=np.float64).reshape(-1)
    m = np.ascontiguousarray(np.broadcast_to(np.asarray(m, dtype=np.complex128), wl.shape))
    mu = np.zeros(0) if mu is None else np.ascontiguousarray(mu, dtype=np.float64).reshape(-1)
    n = dists.size * wl.size
    L = -1 if greek_order is None else (-2 if greek_order == "all" else int(greek_order))
    out = {"values": np.zeros((11, n)), "errors": np.zeros((11, n)),
           "converged": np.zeros(n, dtype=np.int8), "panels": np.zeros(n, dtype=np.int64)}
    ph = pe = g = ge = None
    if mu.size:
        ph, pe = np.zeros((6, n, mu.size)), np.zeros((6, n, mu.size))
    if L >= 0:
        g, ge = np.zeros((6, n, L + 1)), np.zeros((6, n, L + 1))
    err = ctypes.create_string_buffer(512)
    f = lib().orc_ensemble_adaptive
    f.argtypes = [ctypes.c_void_p, _I64, ctypes.c_int, _PD, _I64, _PD, _PD, _I64, _I64,
                  ctypes.c_int, _D, _I64, ctypes.c_int, ctypes.c_int, ctypes.c_int, _PD, _PD,
                  _PD, _PD, _PD, _PD, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_char_p, _I64]
    st = f(dists.ctypes.data, dists.size, int(batch), _p(wl), wl.size,
           _p(m.view(np.float64).reshape(-1)), _p(mu), mu.size, L, int(normalized), rtol,
           max_panels, int(allow_unvalidated), int(refine_backscatter), threads,
           _p(out["values"]), _p(out["errors"]), _p(ph), _p(pe), _p(g), _p(ge),
           out["converged"].ctypes.data, out["panels"].ctypes.data, err, 512)
    if st != 0:
        raise OracleError(st, err.value.decode())
    out["converged"] = out["converged"].astype(bool)
    if ph is not None:
        out["phase"], out["phase_err"] = ph, pe
    if g is not None:
        out["greek"], out["greek_err"] = g, ge
    if L == -2:
        _take_all_orders(out, n)
    return out


def ensemble_adaptive_layered(dists: np.ndarray, wavelengths, fractions, m_layers, mu=None,
                               greek_order=None, normalized: bool = True, rtol: float = 1e-6,
                               max_panels: int = 4096, allow_unvalidated: bool = False,
                               refine_backscatter: bool = False, batch: bool = False,
                               threads: int = 0) -> dict:
    """ensemble_adaptive for layered spheres: fractions (n_dist, L - 1), m_layers complex
    (n_dist, L, n_wl)."""
    dists = np.ascontiguousarray(dists, dtype=DIST_DTYPE)
    wl = np.ascontiguousarray(wavelengths, dtype=np.float64).reshape(-1)
    ml = np.ascontiguousarray(np.asarray(m_layers, dtype=np.complex128))
    nl = ml.shape[1]
    fr = np.ascontiguousarray(np.asarray(fractions, dtype=np.float64).reshape(dists.size,
                                                                              max(nl - 1, 0)))
    mu = np.zeros(0) if mu is None else np.ascontiguousarray(mu, dtype=np.float64).reshape(-1)
    n = dists.size * wl.size
    L = -1 if greek_order is None else (-2 if greek_order == "all" else int(greek_order))
    out = {"values": np.zeros((11, n)), "errors": np.zeros((11, n)),
           "converged": np.zeros(n, dtype=np.int8), "panels": np.zeros(n, dtype=np.int64)}
    ph = pe = g = ge = None
    if mu.size:
        ph, pe = np.zeros((6, n, mu.size)), np.zeros((6, n, mu.size))
    if L >= 0:
        g, ge = np.zeros((6, n, L + 1)), np.zeros((6, n, L + 1))
    err = ctypes.create_string_buffer(512)
    f = lib().orc_ensemble_adaptive_layered
    f.argtypes = [ctypes.c_void_p, _I64, ctypes.c_int, _PD, _I64, ctypes.c_int, _PD, _PD, _PD,
                  _I64, _I64, ctypes.c_int, _D, _I64, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                  _PD, _PD, _PD, _PD, _PD, _PD, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_char_p, _I64]
    st = f(dists.ctypes.data, dists.size, int(batch), _p(wl), wl.size, nl, _p(fr),
           _p(ml.view(np.float64).reshape(-1)), _p(mu), mu.size, L, int(normalized), rtol,
           max_panels, int(allow_unvalidated), int(refine_backscatter), threads,
           _p(out["values"]), _p(out["errors"]), _p(ph), _p(pe), _p(g), _p(ge),
           out["converged"].ctypes.data, out["panels"].ctypes.data, err, 512)
    if st != 0:
        raise OracleError(st, err.value.decode())
    out["converged"] = out["converged"].astype(bool)
    if ph is not None:
        out["phase"], out["phase_err"] = ph, pe
    if g is not None:
        out["greek"], out["greek_err"] = g, ge
    if L == -2:
        _take_all_orders(out, n)
    return out


def ensemble_adaptive_spheroid(dists: np.ndarray, wavelengths, eps: float, m, mu=None,
                                greek_order=None, normalized: bool = True, rtol: float = 1e-6,
                                max_panels: int = 4096, allow_unvalidated: bool = False,
                                refine_backscatter: bool = False, batch: bool = False,
                                threads: int = 0) -> dict:
    """ensemble_adaptive for randomly oriented spheroids of aspect ratio eps (m per
    wavelength), on the engine's direct path."""
    dists = np.ascontiguousarray(dists, dtype=DIST_DTYPE)
    wl = np.ascontiguousarray(wavelengths, dtype=np.float64).reshape(-1)
    m = np.ascontiguousarray(np.broadcast_to(np.asarray(m, dtype=np.complex128), wl.shape))
    mu = np.zeros(0) if mu is None else np.ascontiguousarray(mu, dtype=np.float64).reshape(-1)
    n = dists.size * wl.size
    L = -1 if greek_order is None else (-2 if greek_order == "all" else int(greek_order))
    out = {"values": np.zeros((11, n)), "errors": np.zeros((11, n)),
           "converged": np.zeros(n, dtype=np.int8), "panels": np.zeros(n, dtype=np.int64)}
    ph = pe = g = ge = None
    if mu.size:
        ph, pe = np.zeros((6, n, mu.size)), np.zeros((6, n, mu.size))
    if L >= 0:
        g, ge = np.zeros((6, n, L + 1)), np.zeros((6, n, L + 1))
    err = ctypes.create_string_buffer(512)
    f = lib().orc_ensemble_adaptive_spheroid
    f.argtypes = [ctypes.c_void_p, _I64, ctypes.c_int, _PD, _I64, _D, _PD, _PD, _I64, _I64,
                  ctypes.c_int, _D, _I64, ctypes.c_int, ctypes.c_int, ctypes.c_int, _PD, _PD,
                  _PD, _PD, _PD, _PD, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_char_p, _I64]
    st = f(dists.ctypes.data, dists.size, int(batch), _p(wl), wl.size, float(eps),
           _p(m.view(np.float64).reshape(-1)), _p(mu), mu.size, L, int(normalized), rtol,
           max_panels, int(allow_unvalidated), int(refine_backscatter), threads,
           _p(out["values"]), _p(out["errors"]), _p(ph), _p(pe), _p(g), _p(ge),
           out["converged"].ctypes.data, out["panels"].ctypes.data, err, 512)
    if st != 0:
        raise OracleError(st, err.value.decode())
    out["converged"] = out["converged"].astype(bool)
    if ph is not None:
        out["phase"], out["phase_err"] = ph, pe
    if g is not None:
        out["greek"], out["greek_err"] = g, ge
    if L == -2:
        _take_all_orders(out, n)
    return out


def dist(kind: int, *params) -> np.ndarray:
    """One distribution record (kind as DIST_DTYPE's, or MONODISPERSE)."""
    d = np.zeros(1, dtype=DIST_DTYPE)
    d["kind"] = kind
    d["p"][0, :len(params)] = params
    return d


class TableRecords(np.ndarray):
    """DIST_DTYPE records that own the tables their TABULATED entries point at."""

    def __array_finalize__(self, obj):
        self.tables = getattr(obj, "tables", [])


def table_dist(radii, densities) -> np.ndarray:
    """One TABULATED record: n(r) linear through (radii, densities), 0 outside them
    (scatrs/src/ensemble/distribution.rs:55-62); the record owns the table. Concatenate such
    records with ``join`` to keep the tables alive."""
    r = np.asarray(radii, dtype=np.float64).reshape(-1)
    n = np.asarray(densities, dtype=np.float64).reshape(-1)
    if r.size != n.size:
        raise ValueError("as many densities as radii")
    tab = np.ascontiguousarray(np.concatenate([r, n]))
    d = np.zeros(1, dtype=DIST_DTYPE).view(TableRecords)
    d.tables = [tab]
    d["kind"] = TABULATED
    d["table"] = tab.ctypes.data
    d["table_len"] = r.size
    if r.size:
        d["r_lo"], d["r_hi"] = r[0], r[-1]
    return d


def join(*records) -> np.ndarray:
    """Concatenate distribution records, keeping every table alive."""
    d = np.concatenate([np.asarray(r) for r in records]).view(TableRecords)
    d.tables = [t for r in records for t in getattr(r, "tables", [])]
    return d


def _mixture_arrays(components, n_wl):
    """(modes, mode weights, n_modes, w, m) arrays from [(dists, mode_weights or None, w, m)]."""
    modes, mw, nm, w, ms = [], [], [], [], []
    for dists, mode_w, weight, m in components:
        dists = np.atleast_1d(np.asarray(dists, dtype=DIST_DTYPE))
        modes.append(dists)
        mw.extend(list(mode_w) if mode_w is not None else [1.0] * dists.size)
        nm.append(dists.size)
        w.append(float(weight))
        ms.append(np.broadcast_to(np.asarray(m, dtype=np.complex128), (n_wl,)))
    return (np.ascontiguousarray(np.concatenate(modes)), np.ascontiguousarray(mw, dtype=np.float64),
            np.ascontiguousarray(nm, dtype=np.int32), np.ascontiguousarray(w, dtype=np.float64),
            np.ascontiguousarray(np.concatenate(ms)))


def ensemble_mixture(components, wavelengths, mu=None, greek_order=None, normalized=True,
                     rtol=1e-6, max_panels=4096, allow_unvalidated=False,
                     refine_backscatter=False) -> dict:
    """The adaptive ensemble of a mixture: components [(dists, mode_weights or None, w, m)],
    a component's dists one distribution or the modes of a multimodal one; m per wavelength.
    Outputs per wavelength (n = n_wl)."""
    wl = np.ascontiguousarray(wavelengths, dtype=np.float64).reshape(-1)
    modes, mw, nm, w, ms = _mixture_arrays(components, wl.size)
    mu = np.zeros(0) if mu is None else np.ascontiguousarray(mu, dtype=np.float64).reshape(-1)
    n = wl.size
    L = -1 if greek_order is None else int(greek_order)
    out = {"values": np.zeros((11, n)), "errors": np.zeros((11, n)),
           "converged": np.zeros(n, dtype=np.int8), "panels": np.zeros(n, dtype=np.int64)}
    ph = pe = g = ge = None
    if mu.size:
        ph, pe = np.zeros((6, n, mu.size)), np.zeros((6, n, mu.size))
    if L >= 0:
        g, ge = np.zeros((6, n, L + 1)), np.zeros((6, n, L + 1))
    err = ctypes.create_string_buffer(512)
    f = lib().orc_ensemble_mixture
    f.argtypes = [ctypes.c_void_p, _PD, ctypes.c_void_p, _PD, _PD, _I64, _PD, _I64, _PD, _I64,
                  _I64, ctypes.c_int, _D, _I64, ctypes.c_int, ctypes.c_int, _PD, _PD, _PD, _PD,
                  _PD, _PD, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_char_p, _I64]
    st = f(modes.ctypes.data, _p(mw), nm.ctypes.data, _p(w), _p(ms.view(np.float64)), nm.size,
           _p(wl), wl.size, _p(mu), mu.size, L, int(normalized), rtol, max_panels,
           int(allow_unvalidated), int(refine_backscatter), _p(out["values"]),
           _p(out["errors"]), _p(ph), _p(pe), _p(g), _p(ge), out["converged"].ctypes.data,
           out["panels"].ctypes.data, err, 512)
    if st != 0:
        raise OracleError(st, err.value.decode())
    out["converged"] = out["converged"].astype(bool)
    if ph is not None:
        out["phase"], out["phase_err"] = ph, pe
    if g is not None:
        out["greek"], out["greek_err"] = g, ge
    return out


PARAM_DTYPE = np.dtype([("component", np.int32), ("mode", np.int32), ("kind", np.int32),
                        ("index", np.int32)])
PK_DIST, PK_REFR_REAL, PK_REFR_IMAG, PK_WEIGHT = 0, 1, 2, 3


def params(*specs) -> np.ndarray:
    """Parameter records from (component, mode or -1, kind, index) tuples."""
    return np.array([tuple(p) for p in specs], dtype=PARAM_DTYPE)


def ensemble_mixture_d(components, wavelengths, derivs, mu=None, greek_order=None,
                       normalized=True, rtol=1e-6, max_panels=4096, allow_unvalidated=False,
                       refine_backscatter=False) -> dict:
    """ensemble_mixture with the derivatives along `derivs` (PARAM_DTYPE records): adds d, d_err
    (P, 11, n), phase_d, phase_d_err (P, 6, n, n_mu), greek_d, greek_d_err (P, 6, n, L + 1).
    A component whose mode weights are given is multimodal (its parameters carry a mode)."""
    wl = np.ascontiguousarray(wavelengths, dtype=np.float64).reshape(-1)
    # A component's m may be a particle: ("sphere", m), ("layered", fractions, m [L][n_wl]) or
    # ("spheroid", aspect_ratio, m).
    nls, frs, eps, mlist, plain = [], [], [], [], []
    for dists, mode_w, weight, m in components:
        if isinstance(m, tuple) and m[0] == "layered":
            ml = np.asarray(m[2], dtype=np.complex128).reshape(-1, wl.size)
            nls.append(ml.shape[0])
            frs += [float(f) for f in np.asarray(m[1]).reshape(-1)]
            eps.append(0.0)
            mlist.append(ml.reshape(-1))
        elif isinstance(m, tuple):
            nls.append(1)
            eps.append(float(m[1]) if m[0] == "spheroid" else 0.0)
            mlist.append(np.broadcast_to(np.asarray(m[-1], dtype=np.complex128), wl.shape))
        else:
            nls.append(1)
            eps.append(0.0)
            mlist.append(np.broadcast_to(np.asarray(m, dtype=np.complex128), wl.shape))
        plain.append((dists, mode_w, weight, np.zeros(wl.size, dtype=np.complex128)))
    modes, mw, nm, w, _ = _mixture_arrays(plain, wl.size)
    ms = np.ascontiguousarray(np.concatenate(mlist))
    nls = np.array(nls, dtype=np.int32)
    frs = np.array(frs + [0.0], dtype=np.float64)
    eps = np.array(eps, dtype=np.float64)
    mm = np.array([1 if mwc is not None else 0 for _d, mwc, _w, _m in components], dtype=np.int32)
    pr = np.ascontiguousarray(np.atleast_1d(np.asarray(derivs, dtype=PARAM_DTYPE)))
    P = pr.size
    mu = np.zeros(0) if mu is None else np.ascontiguousarray(mu, dtype=np.float64).reshape(-1)
    n = wl.size
    L = -1 if greek_order is None else (-2 if greek_order == "all" else int(greek_order))
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
    err = ctypes.create_string_buffer(512)
    f = lib().orc_ensemble_mixture_d
    f.argtypes = [ctypes.c_void_p, _PD, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, _PD,
                  _PD, _PD, _PD, _I64, _PD,
                  _I64, _PD, _I64, _I64, ctypes.c_int, _D, _I64, ctypes.c_int, ctypes.c_int,
                  ctypes.c_void_p, _I64] + [_PD] * 12 + [ctypes.c_void_p, ctypes.c_void_p,
                                                         ctypes.c_char_p, _I64]
    st = f(modes.ctypes.data, _p(mw), nm.ctypes.data, mm.ctypes.data, nls.ctypes.data, _p(frs),
           _p(eps), _p(w), _p(ms.view(np.float64)), nm.size, _p(wl), wl.size, _p(mu), mu.size, L,
           int(normalized), rtol, max_panels, int(allow_unvalidated), int(refine_backscatter),
           pr.ctypes.data if P else None, P, _p(out["values"]), _p(out["errors"]), _p(ph),
           _p(pe), _p(g), _p(ge), _p(out["d"]), _p(out["d_err"]), _p(dph), _p(dpe), _p(dg),
           _p(dge), out["converged"].ctypes.data, out["panels"].ctypes.data, err, 512)
    if st != 0:
        raise OracleError(st, err.value.decode())
    out["converged"] = out["converged"].astype(bool)
    if ph is not None:
        out["phase"], out["phase_err"], out["phase_d"], out["phase_d_err"] = ph, pe, dph, dpe
    if g is not None:
        out["greek"], out["greek_err"], out["greek_d"], out["greek_d_err"] = g, ge, dg, dge
    if L == -2:
        _take_all_orders(out, n, P)
    return out


def tmatrix_mode(x: float, eps: float, s: complex, m: int, n: int, n_theta: int,
                 quad: bool = False) -> np.ndarray:
    """One azimuthal mode's T-matrix of a spheroid (2K x 2K complex, K = n - max(m, 1) + 1); in
    quadruple precision with `quad`."""
    k = n - max(m, 1) + 1
    t = np.zeros(2 * (2 * k) ** 2)
    f = lib().orc_tmatrix_mode_q if quad else lib().orc_tmatrix_mode
    f.argtypes = [_D, _D, _D, _D, ctypes.c_int, ctypes.c_int, ctypes.c_int, _PD]
    st = f(x, eps, s.real, s.imag, m, n, n_theta, _p(t))
    if st != 0:
        raise OracleError(st, "tmatrix_mode")
    return t.view(np.complex128).reshape(2 * k, 2 * k)


def spheroid_q(x: float, eps: float, s: complex, n: int, n_theta: int, quad: bool = False):
    """Orientation-averaged (Q_ext, Q_sca) of a spheroid at truncation n and n_theta nodes; in
    quadruple precision with `quad`."""
    q = np.zeros(2)
    f = lib().orc_spheroid_q_q if quad else lib().orc_spheroid_q
    f.argtypes = [_D, _D, _D, _D, ctypes.c_int, ctypes.c_int, _PD]
    st = f(x, eps, s.real, s.imag, n, n_theta, _p(q))
    if st != 0:
        raise OracleError(st, "spheroid_q")
    return q[0], q[1]


def spheroid_converged(x: float, eps: float, s: complex, rtol: float = 1e-8):
    """Converged orientation-averaged (Q_ext, Q_sca, Q_abs), N and n_theta of a spheroid."""
    q = np.zeros(3)
    n, nth = ctypes.c_int(0), ctypes.c_int(0)
    f = lib().orc_spheroid_converged
    f.argtypes = [_D, _D, _D, _D, _D, _PD, ctypes.POINTER(ctypes.c_int),
                  ctypes.POINTER(ctypes.c_int)]
    st = f(x, eps, s.real, s.imag, rtol, _p(q), ctypes.byref(n), ctypes.byref(nth))
    if st != 0:
        raise OracleError(st, "spheroid_converged")
    return q, n.value, nth.value


def tmatrix_modes(x: float, eps: float, s: complex, n: int, n_theta: int, quad: bool = False):
    """Every mode's T-matrix (m = 0..n) of a spheroid."""
    return [tmatrix_mode(x, eps, s, m, n, n_theta, quad) for m in range(n + 1)]


def _flat_modes(modes) -> np.ndarray:
    return np.ascontiguousarray(np.concatenate([np.ascontiguousarray(t).reshape(-1)
                                                for t in modes])).view(np.float64)


def random_orientation(modes, mu) -> np.ndarray:
    """The orientation-averaged phase matrix (6, n_mu): F11, F12, F22, F33, F34, F44 in 1/k^2
    per steradian, of the T-matrix modes 0..N."""
    n = len(modes) - 1
    mu = np.ascontiguousarray(mu, dtype=np.float64)
    f = np.zeros(6 * mu.size)
    fn = lib().orc_random_orientation
    fn.argtypes = [ctypes.c_int, _PD, _PD, ctypes.c_int, _PD]
    fn(n, _p(_flat_modes(modes)), _p(mu), mu.size, _p(f))
    return f.reshape(6, mu.size)


def random_greek(modes, order: int) -> np.ndarray:
    """The unnormalized Greek coefficients (6, L + 1), L = min(order, 2N): alpha1..alpha4,
    beta1, beta2 of the average."""
    n = len(modes) - 1
    L = min(order, 2 * n)
    out = np.zeros(6 * (L + 1))
    fn = lib().orc_random_greek
    fn.argtypes = [ctypes.c_int, _PD, ctypes.c_int, _PD]
    fn(n, _p(_flat_modes(modes)), order, _p(out))
    return out.reshape(6, L + 1)


def ensemble_fixed_spheroid(dists: np.ndarray, wavelengths, eps, m, n_nodes: int, node_terms,
                            mu=None, greek_order: int | None = None, normalized: bool = True,
                            quad: bool = False) -> dict:
    """The fixed-grid spheroid ensemble, restated over the oracle's per-node solutions: each
    node's T-matrix at the given (N, n_theta) (node_terms (n_units, n_nodes, 2)), its orientation
    average (random_greek), the per-particle quantities and direct segment of
    scatrs/src/ensemble/engine.rs:1207-1339 and particle.rs:276-285, the averages on the grid's
    weights w u(r) r, and the outputs of engine.rs:2359-2497 (the phase matrix from the averaged
    Greek expansion). Units distribution-major."""
    dists = np.ascontiguousarray(dists, dtype=DIST_DTYPE)
    wl = np.ascontiguousarray(wavelengths, dtype=np.float64).reshape(-1)
    eps = np.broadcast_to(np.asarray(eps, dtype=np.float64), (dists.size,))
    m = np.broadcast_to(np.asarray(m, dtype=np.complex128), (dists.size, wl.size))
    mu = np.zeros(0) if mu is None else np.asarray(mu, dtype=np.float64).reshape(-1)
    xi, om = gauss_legendre(n_nodes)
    n_units = dists.size * wl.size
    L = -1 if greek_order is None else int(greek_order)
    values = np.zeros((11, n_units))
    phase = np.zeros((6, n_units, mu.size))
    greek = np.zeros((6, n_units, max(L, 0) + 1))
    for d in range(dists.size):
        a, b = np.log(dists["r_lo"][d]), np.log(dists["r_hi"][d])
        c, h = 0.5 * (a + b), 0.5 * (b - a)
        r = np.exp(c + h * xi)
        params = list(dists["p"][d])
        W = np.array([h * om[j] * (density(int(dists["kind"][d]), params, r[j])[0] * r[j])
                      for j in range(n_nodes)])
        for w in range(wl.size):
            u = d * wl.size + w
            rows = []
            for j in range(n_nodes):
                x = 2 * np.pi * r[j] / wl[w]
                N, nth = (int(v) for v in node_terms[u, j])
                modes = tmatrix_modes(x, eps[d], complex(m[d, w]), N, nth, quad)
                ext = sum((1 if k == 0 else 2) * -np.trace(t).real for k, t in enumerate(modes))
                sca = sum((1 if k == 0 else 2) * (abs(t) ** 2).sum() for k, t in enumerate(modes))
                raw = random_greek(modes, 2 * N)
                area_x = np.pi * x * x
                q_ext, q_sca = 2 * np.pi * ext / area_x, 2 * np.pi * sca / area_x
                g = raw[0, 1] / (3 * raw[0, 0])
                sgn = (-1.0) ** np.arange(2 * N + 1)
                q_back = 4 * np.pi * np.dot(sgn, raw[0]) / area_x
                un = raw * 4 / (x * x)
                depol = np.dot(sgn, un[0] - 0.5 * (un[1] - un[2]))
                area = np.pi * r[j] ** 2
                rows.append((W[j], area, r[j], q_ext, q_sca, g, q_back, depol, un))
            Z = sum(row[0] for row in rows)
            top = max(row[8].shape[1] for row in rows)
            G = np.zeros((6, max(top, L + 1)))
            acc = np.zeros(9)
            for (Wj, area, rj, qe, qs, g, qb, dep, un) in rows:
                acc += Wj * np.array([area * qe, area * qs, area * qs * g, area * (qe - qs),
                                      area * qb, rj * rj, rj ** 3, area * dep, 0.0])
                G[:, : un.shape[1]] += Wj * area * un
            ext, sca, scag, ab, back, r2, r3, dep, _ = acc / Z
            G /= Z
            values[:, u] = [ext, sca, ab, back, sca / ext, scag / sca, 4 * np.pi * ext / back,
                            dep / (2 * back - dep), r3 / r2, np.pi * r2, 4 * np.pi / 3 * r3]
            if L >= 0:
                gg = G[:, : L + 1] / (G[0, 0] if normalized else 1.0)
                if normalized:
                    gg[0, 0] = 1.0
                greek[:, u, :] = gg
            for j, c0 in enumerate(mu):
                dd = [wigner_d(p, q, c0, top - 1) for p, q in ((0, 0), (2, 2), (2, -2), (0, 2))]
                plus, minus = 0.5 * (dd[1] + dd[2]), 0.5 * (dd[1] - dd[2])
                Gt = G[:, :top]
                f = [np.dot(Gt[0], dd[0]), np.dot(Gt[4], dd[3]),
                     np.dot(Gt[1], plus) + np.dot(Gt[2], minus),
                     np.dot(Gt[1], minus) + np.dot(Gt[2], plus), np.dot(Gt[5], dd[3]),
                     np.dot(Gt[3], dd[0])]
                phase[:, u, j] = np.array(f) / (sca if normalized else 1.0)
    out = {"values": values}
    if mu.size:
        out["phase"] = phase
    if L >= 0:
        out["greek"] = greek
    return out


def spheroid_node(x: float, eps: float, s: complex, rtol: float = 1e-8):
    """One spheroid node of the ensemble's direct path in double precision: (Q_ext, Q_sca,
    Q_abs, Q_back, g), N, n_theta."""
    q = np.zeros(5)
    n = np.zeros(2, dtype=np.int32)
    f = lib().orc_spheroid_node
    f.argtypes = [_D, _D, _D, _D, _D, _PD, ctypes.c_void_p]
    st = f(x, eps, s.real, s.imag, rtol, _p(q), n.ctypes.data)
    if st != 0:
        raise OracleError(st, "spheroid_node")
    return q, int(n[0]), int(n[1])


# ---------------------------------------------------------------------------------------------
# Refractive-index models (python/scatrs/refractive.py:168-354), restated with numpy in the
# reference's order of operations: m at the wavelengths and dm/dtheta for each parameter.
# ---------------------------------------------------------------------------------------------
def refractive_index(spec, wavelength):
    """m of a model spec at `wavelength` (1-D), and dm (P, n): ("constant", m) (refractive.py:
    190-197), ("table", wl, m) / ("table_log_k", wl, m) (246-262, np.interp), ("cauchy", A, B,
    C, k) (283-294), ("sellmeier", B, C, k) (326-354). Raises ValueError where the reference
    raises InvalidInputError (a wavelength outside a table, Sellmeier's n^2 <= 0)."""
    lam = np.asarray(wavelength, dtype=np.float64).reshape(-1)
    kind = spec[0]
    if kind == "constant":
        m = complex(spec[1])
        dm = np.empty((2, lam.size), dtype=complex)
        dm[0], dm[1] = 1.0, 1j
        return np.full(lam.shape, m), dm
    if kind in ("table", "table_log_k"):
        wl = np.asarray(spec[1], dtype=np.float64)
        nodes = np.asarray(spec[2], dtype=np.complex128)
        if np.any(~((lam >= wl[0]) & (lam <= wl[-1]))):
            raise ValueError("a wavelength is outside the Table's range")
        n = np.interp(lam, wl, nodes.real)
        if kind == "table":
            k = np.interp(lam, wl, nodes.imag)
        else:
            k = np.exp(np.interp(lam, wl, np.log(nodes.imag)))
        return n + 1j * k, np.zeros((0, lam.size), dtype=complex)
    if kind == "cauchy":
        A, B, C, k = (float(v) for v in spec[1:5])
        s = lam ** -2.0
        dm = np.empty((4, lam.size), dtype=complex)
        dm[0], dm[1], dm[2], dm[3] = 1.0, s, s * s, 1j
        return A + B * s + C * s * s + 1j * k, dm
    if kind == "sellmeier":
        b = np.asarray(spec[1], dtype=np.float64).reshape(-1)
        c = np.asarray(spec[2], dtype=np.float64).reshape(-1)
        k = float(spec[3])
        l2 = lam * lam
        n2 = np.ones_like(l2)
        for bi, ci in zip(b, c):
            n2 += bi * l2 / (l2 - ci)
        if np.any(~(n2 > 0) | ~np.isfinite(n2)):
            raise ValueError("Sellmeier gives n^2 <= 0")
        n = np.sqrt(n2)
        t = b.size
        dm = np.empty((2 * t + 1, lam.size), dtype=complex)
        for i, (bi, ci) in enumerate(zip(b, c)):
            dm[i] = l2 / (l2 - ci) / (2 * n)
            dm[t + i] = bi * l2 / (l2 - ci) ** 2 / (2 * n)
        dm[-1] = 1j
        return n + 1j * k, dm
    raise TypeError(f"unknown refractive-index model {kind!r}")
