"""The C ABI library without a GPU: it loads, exports every function include/scatrs_b200.h
declares (and the binding declares each), and its host-only entry points work."""

import ctypes
import os
import re

import numpy as np

from scatrs_b200 import _native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    src = open(os.path.join(ROOT, "include", "scatrs_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(scatrs_[a-z_0-9]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = _native.load()
    names = declared()
    assert len(names) >= 12
    for name in names:
        assert hasattr(lib, name), name
        assert name in _native.SYMBOLS, name


def test_gauss_legendre_matches_oracle():
    from oracle import oracle as O

    for n in (1, 2, 7, 64, 180, 360, 1201, 4096):
        x, w = _native.gauss_legendre(n)
        xo, wo = O.gauss_legendre(n)
        assert np.abs(x - xo).max() <= 2.3e-16
        assert (np.abs(w - wo) / wo).max() <= 4.5e-16
        assert abs(w.sum() - 2.0) <= 1e-13


def test_output_sizes():
    v, p, g = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
    _native.load().scatrs_ensemble_fixed_sizes(10, 7, 4, ctypes.byref(v), ctypes.byref(p),
                                               ctypes.byref(g))
    assert (v.value, p.value, g.value) == (110, 420, 300)
    _native.load().scatrs_ensemble_fixed_sizes(10, 0, -1, ctypes.byref(v), ctypes.byref(p),
                                               ctypes.byref(g))
    assert (p.value, g.value) == (0, 0)


def test_device_count_is_an_integer():
    assert isinstance(_native.load().scatrs_device_count(), int)


def test_parameter_kinds_match_the_header():
    """The binding's parameter kinds are the header's SCATRS_PARAM_* values
    (ParamKind, scatrs/src/ensemble/mod.rs:180-215)."""
    src = open(os.path.join(ROOT, "include", "scatrs_b200.h")).read()
    values = {m.group(1): int(m.group(2))
              for m in re.finditer(r"SCATRS_PARAM_([A-Z_]+)\s*=\s*(\d+)", src)}
    assert values == {"DISTRIBUTION": _native.PARAM_DISTRIBUTION,
                      "REFR_REAL": _native.PARAM_REFR_REAL,
                      "REFR_IMAG": _native.PARAM_REFR_IMAG,
                      "WEIGHT": _native.PARAM_WEIGHT,
                      "ASPECT_RATIO": _native.PARAM_ASPECT_RATIO,
                      "LAYER_REFR_REAL": _native.PARAM_LAYER_REFR_REAL,
                      "LAYER_REFR_IMAG": _native.PARAM_LAYER_REFR_IMAG,
                      "RADIUS_FRACTION": _native.PARAM_RADIUS_FRACTION}
