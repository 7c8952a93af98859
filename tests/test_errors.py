"""The library's error path on the host (no GPU): statuses, messages and NotConverged's
achieved/requested reach Python as the reference's exception classes
(scatrs-py/src/errors.rs:14-45, python/scatrs/errors.py:36-70), through the test hook that fails
a call the way every entry point fails (scatrs_testing_raise)."""

import ctypes
import math
import pickle

import pytest

from scatrs_b200 import _native, _scatrs
from scatrs_b200.errors import (DeviceError, InvalidInputError, NotConvergedError,
                                OutsideValidatedDomainError, ScatrsError)


def test_hierarchy():
    for cls, std in ((InvalidInputError, ValueError), (NotConvergedError, ArithmeticError),
                     (OutsideValidatedDomainError, ValueError), (DeviceError, RuntimeError)):
        assert issubclass(cls, ScatrsError) and issubclass(cls, std)


@pytest.mark.parametrize("variant,cls", [("InvalidInput", InvalidInputError),
                                         ("OutsideValidatedDomain", OutsideValidatedDomainError)])
def test_status_reaches_python_as_its_class(variant, cls):
    with pytest.raises(cls, match="x > 2e4"):
        _scatrs._testing.raise_core_error(variant, "x > 2e4")


def test_not_converged_carries_achieved_and_requested():
    with pytest.raises(NotConvergedError) as info:
        _scatrs._testing.raise_core_error("NotConverged", achieved=3e-7, requested=1e-9)
    e = info.value
    assert (e.achieved, e.requested) == (3e-7, 1e-9)
    assert "achieved 3.000000e-07, requested 1.000000e-09" in str(e)
    back = pickle.loads(pickle.dumps(e))
    assert type(back) is NotConvergedError and (back.achieved, back.requested) == (3e-7, 1e-9)
    with pytest.raises(NotConvergedError) as info:
        _scatrs._testing.raise_core_error("NotConverged", achieved=math.inf, requested=1e-6)
    assert info.value.achieved == math.inf


def test_detail_belongs_to_the_last_call():
    lib = _native.load()
    err = ctypes.create_string_buffer(256)
    assert lib.scatrs_testing_raise(2, b"nc", 1e-3, 1e-6, err, 256) == 2
    a, r = ctypes.c_double(), ctypes.c_double()
    assert lib.scatrs_not_converged_detail(ctypes.byref(a), ctypes.byref(r)) == 1
    assert (a.value, r.value) == (1e-3, 1e-6)
    assert lib.scatrs_testing_raise(0, b"", 0.0, 0.0, err, 256) == 0  # a call that succeeds
    assert lib.scatrs_not_converged_detail(ctypes.byref(a), ctypes.byref(r)) == 0
    assert math.isnan(a.value) and math.isnan(r.value)
    assert lib.scatrs_testing_raise(4, b"cudaMalloc: out of memory", 0.0, 0.0, err, 256) == 4
    with pytest.raises(DeviceError, match="out of memory"):
        _native._check(4, err)
    with pytest.raises(ValueError):
        _scatrs._testing.raise_core_error("Bogus")


def test_limits_are_enforced_by_the_library():
    assert _scatrs.MAX_GAUSS_LEGENDRE_POINTS == 1 << 17
    with pytest.raises(InvalidInputError):
        _native.gauss_legendre(0)
    with pytest.raises(InvalidInputError):
        _native.gauss_legendre(_scatrs.MAX_GAUSS_LEGENDRE_POINTS + 1)
    assert _native.load().scatrs_limit(99) == -1
