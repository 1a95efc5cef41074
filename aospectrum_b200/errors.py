"""Exception hierarchy of the Band path.

Mirrors ``src/aospectrum/errors.py:4-13`` of the reference: every user-facing
failure is an ``AOSpectrumError``; malformed inputs raise ``InputError`` and
numerical or device failures raise ``SolverError``.  The CLI maps both to exit
code 2 (reference ``cli.py:608-610``).
"""

from __future__ import annotations


class AOSpectrumError(RuntimeError):
    """Base class of all errors the engine reports to a user."""


class InputError(AOSpectrumError):
    """A configuration, bundle, k-path or request is invalid."""


class SolverError(AOSpectrumError):
    """The numerical engine or the GPU could not produce a result."""
