"""Exception hierarchy of the scorer.

Mirrors ``src/gpusw/errors.py:5-31`` of the reference package: one base class and four
leaf classes, so callers that catch the reference's exceptions keep working. Every
non-zero status returned by the native C-ABI is mapped onto one of these classes by
:mod:`gpusw_b200._native`.
"""
from __future__ import annotations

__all__ = ["GpuSWError", "NoGpuError", "SchemeError", "OverflowRiskError", "EncodeError"]


class GpuSWError(Exception):
    """Base class of every error raised by this package."""


class NoGpuError(GpuSWError):
    """The native CUDA library or a usable NVIDIA GPU is not available.

    Importing the package, building schemes and encoding sequences never need a GPU;
    only the scoring entry points raise this.
    """


class SchemeError(GpuSWError):
    """A :class:`~gpusw_b200.Scheme` or :class:`~gpusw_b200.Matrix` is invalid."""


class OverflowRiskError(GpuSWError):
    """``dtype="int16"`` was forced but the worst-case score range does not fit int16.

    ``dtype="auto"`` never raises this: it scores in int16 and rescores in int32 exactly
    the pairs whose int16 run could have overflowed.
    """


class EncodeError(GpuSWError):
    """Input sequences could not be turned into the encoded (codes, offsets) form."""
