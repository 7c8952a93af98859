"""The exception classes of the reference's Python package (python/scatrs/errors.py:36-70),
which the C ABI's status codes map onto as the reference's binding maps scatrs::Error
(scatrs-py/src/errors.rs:14-45).

When this package serves the reference's Python package as its extension module
(``scatrs._scatrs``), ``scatrs.errors`` is loaded and its own classes are raised, so that the
package's callers catch exactly the classes they expect; otherwise the same hierarchy below is
raised. A CUDA failure has no class of its own in the reference and maps to its ScatrsError
(errors.rs:33), or to DeviceError (a ScatrsError) here.
"""

from __future__ import annotations

import sys

__all__ = ["InvalidInputError", "NotConvergedError", "OutsideValidatedDomainError", "ScatrsError",
           "DeviceError"]


class ScatrsError(Exception):
    """Base class for every error raised by scatrs."""


class InvalidInputError(ScatrsError, ValueError):
    """An input is outside its valid range (its mathematical domain or a documented limit)."""


class NotConvergedError(ScatrsError, ArithmeticError):
    """A computation did not reach the requested accuracy."""

    def __init__(self, message: str, achieved: float | None = None,
                 requested: float | None = None) -> None:
        super().__init__(message)
        self.achieved = achieved
        self.requested = requested

    def __reduce__(self):
        return (type(self), (str(self), self.achieved, self.requested))


class OutsideValidatedDomainError(ScatrsError, ValueError):
    """Inputs are valid but outside the domain where accuracy has been validated."""


class DeviceError(ScatrsError, RuntimeError):
    """The GPU failed: a CUDA runtime error, or no usable device."""


def classes():
    """The classes raised for the status codes 1, 2, 3 and 4: those of ``scatrs.errors`` when
    the reference package has loaded it, else this module's."""
    ref = sys.modules.get("scatrs.errors")
    if ref is not None and all(hasattr(ref, n) for n in (
            "InvalidInputError", "NotConvergedError", "OutsideValidatedDomainError",
            "ScatrsError")):
        return (ref.InvalidInputError, ref.NotConvergedError, ref.OutsideValidatedDomainError,
                ref.ScatrsError)
    return InvalidInputError, NotConvergedError, OutsideValidatedDomainError, DeviceError


def raise_for(status: int, message: str, achieved: float | None = None,
              requested: float | None = None) -> None:
    """Raises the class of a C-ABI status (nothing for 0); NotConvergedError with the accuracy
    reached and requested when the library reported them."""
    if status == 0:
        return
    invalid, not_converged, outside, other = classes()
    if status == 1:
        raise invalid(message)
    if status == 2:
        raise not_converged(message, achieved, requested)
    if status == 3:
        raise outside(message)
    raise other(message)
