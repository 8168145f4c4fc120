"""The :class:`Scheme`: every parameter of one scoring problem in a frozen, hashable form.

Field names, defaults, validation and the int16/int32 envelope follow
``src/gpusw/scheme.py:26-185`` of the reference package:

* defaults: local mode, match 2 / mismatch -3, gap open -5 / extend -2, both
  free-end-gap flags True, unknown symbols score as the worst mismatch, case folded,
  dtype "auto" (``scheme.py:57-68``);
* validation (``scheme.py:74-92``) raises :class:`SchemeError`;
* ``resolve_dtype`` (``scheme.py:116-141``) is the reference's *static* envelope:
  upper = min(maxq, maxr) * max(max_pos, 1), lower = min(go, ge, min_sub, 0) *
  max(maxq, maxr) for non-local modes, int16 iff both are within +/-30000;
* ``substitution_table`` (``scheme.py:149-162``) is the (NS, NS) int32 table with
  ``table[a, b]`` = reference code ``a`` against query code ``b``.

The native engine does not need the static envelope to be exact: with ``dtype="auto"`` it
scores every pair in int16 and rescores in int32 only the pairs whose int16 run could have
overflowed, which returns the same integers as scoring everything in int32.
"""
from __future__ import annotations

import hashlib
from dataclasses import dataclass, field, replace

import numpy as np

from .errors import OverflowRiskError, SchemeError
from .matrix import Matrix

__all__ = ["Scheme", "MODES", "MODE_CODES"]

MODES = ("local", "global", "semiglobal")
MODE_CODES = {"local": 0, "global": 1, "semiglobal": 2}
UNKNOWN_POLICIES = ("mismatch", "zero", "error")
DTYPES = ("auto", "int16", "int32")
INT16_SAFE = 30000


@dataclass(frozen=True)
class Scheme:
    """A complete specification of an alignment-scoring problem.

    ``gap_open`` is the cost of the first residue of a gap and ``gap_extend`` the cost of
    each later residue. ``free_end_gaps_query`` / ``free_end_gaps_ref`` only matter in
    ``"semiglobal"`` mode. ``dtype`` picks the DP integer width: ``"auto"``, ``"int16"``
    or ``"int32"``.
    """

    mode: str = "local"
    match: int = 2
    mismatch: int = -3
    gap_open: int = -5
    gap_extend: int = -2
    matrix: Matrix | None = None
    alphabet: str | None = None
    free_end_gaps_query: bool = True
    free_end_gaps_ref: bool = True
    unknown: str = "mismatch"
    case_insensitive: bool = True
    dtype: str = "auto"
    eff_alphabet: str = field(default="ACGT", repr=False)

    def __post_init__(self) -> None:
        if self.mode not in MODES:
            raise SchemeError(f"mode must be one of {MODES}, got {self.mode!r}")
        if self.unknown not in UNKNOWN_POLICIES:
            raise SchemeError(f"unknown must be one of {UNKNOWN_POLICIES}")
        if self.dtype not in DTYPES:
            raise SchemeError(f"dtype must be one of {DTYPES}")
        for name in ("match", "mismatch", "gap_open", "gap_extend"):
            value = getattr(self, name)
            if int(value) != value:
                raise SchemeError(f"{name} must be an integer, got {value!r}")
            object.__setattr__(self, name, int(value))
        if self.gap_open > 0 or self.gap_extend > 0:
            raise SchemeError("gap_open and gap_extend must be <= 0")
        alpha = self.matrix.alphabet if self.matrix is not None else (self.alphabet or "ACGT")
        if self.case_insensitive:
            alpha = alpha.upper()
        if len(set(alpha)) != len(alpha):
            raise SchemeError(f"alphabet {alpha!r} has duplicate symbols")
        object.__setattr__(self, "eff_alphabet", alpha)

    @classmethod
    def preset(cls, name: str) -> Scheme:
        from . import schemes

        preset = getattr(schemes, name.upper(), None)
        if not isinstance(preset, Scheme):
            raise SchemeError(f"unknown preset {name!r}; available: {', '.join(schemes.__all__)}")
        return preset

    def replace(self, **kw) -> Scheme:
        """Copy with the given fields overridden."""
        return replace(self, **kw)

    def _score_extremes(self) -> tuple[int, int]:
        """(largest positive substitution score or 0, smallest substitution score)."""
        if self.matrix is not None:
            return max(self.matrix.max_score, 0), self.matrix.min_score
        return max(self.match, 0), min(self.mismatch, self.match)

    def resolve_dtype(self, max_q_len: int, max_r_len: int) -> str:
        """The reference's static int16/int32 choice for the longest query/reference."""
        if self.dtype == "int32":
            return "int32"
        max_pos, min_sub = self._score_extremes()
        upper = min(max_q_len, max_r_len) * max(max_pos, 1)
        if self.mode == "local":
            lower = 0
        else:
            lower = min(self.gap_open, self.gap_extend, min_sub, 0) * max(max_q_len, max_r_len)
        fits = upper <= INT16_SAFE and lower >= -INT16_SAFE
        if self.dtype == "int16":
            if not fits:
                raise OverflowRiskError(
                    f"dtype='int16' unsafe: worst-case score range [{lower}, {upper}] "
                    f"exceeds +/-{INT16_SAFE}. Use dtype='auto' or 'int32'."
                )
            return "int16"
        return "int16" if fits else "int32"

    @property
    def ns(self) -> int:
        """Side of the sentinel-padded substitution table."""
        return len(self.eff_alphabet) + 1

    def substitution_table(self) -> np.ndarray:
        base = self.matrix if self.matrix is not None else Matrix.from_match_mismatch(
            self.match, self.mismatch, self.eff_alphabet)
        return base.packed(self.unknown)[1]

    def table_hash(self) -> str:
        h = hashlib.blake2b(digest_size=12)
        h.update(self.substitution_table().tobytes())
        return h.hexdigest()

    def module_fields(self) -> dict:
        """The kernel-configuration fields (mode, gaps, free-end flags, table side)."""
        return {
            "mode": self.mode,
            "gap_open": self.gap_open,
            "gap_extend": self.gap_extend,
            "free_q": bool(self.free_end_gaps_query),
            "free_r": bool(self.free_end_gaps_ref),
            "ns": self.ns,
        }
