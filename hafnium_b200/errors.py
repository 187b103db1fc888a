"""Exceptions with the reference's names and meanings (hafnium/errors.py:13-43).

When the reference package is importable its classes are used, so a caller
catching ``hafnium.errors.InputError`` catches errors raised here too.
"""

from __future__ import annotations

try:  # pragma: no cover - depends on the caller's environment
    from hafnium.errors import BackendError, ConvergenceError, HafniumError, InputError
except Exception:  # noqa: BLE001 - the reference is optional at run time

    class HafniumError(Exception):
        """Base class of every error this package raises."""

    class InputError(HafniumError, ValueError):
        """Invalid input: shapes, sizes, values outside the supported range."""

    class BackendError(HafniumError, RuntimeError):
        """A device, driver or kernel failure (CUDA error, out of memory, timeout)."""

    class ConvergenceError(HafniumError, RuntimeError):
        """The SCF did not converge; ``last`` holds the final state."""

        def __init__(self, message: str, last=None) -> None:
            super().__init__(message)
            self.last = last


__all__ = ["BackendError", "ConvergenceError", "HafniumError", "InputError"]
