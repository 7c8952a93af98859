"""The exception classes of the reference's Python package (python/scatrs/errors.py:36-70),
which the C ABI's status codes map onto (scatrs-py/src/errors.rs:14-45)."""

from __future__ import annotations

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


class OutsideValidatedDomainError(ScatrsError, ValueError):
    """Inputs are valid but outside the domain where accuracy has been validated."""


class DeviceError(ScatrsError, RuntimeError):
    """The GPU failed: a CUDA runtime error, or no usable device."""


def raise_for(status: int, message: str) -> None:
    """Raises the class of a C-ABI status (nothing for 0)."""
    if status == 0:
        return
    cls = {1: InvalidInputError, 2: NotConvergedError, 3: OutsideValidatedDomainError}.get(
        status, DeviceError)
    raise cls(message)
