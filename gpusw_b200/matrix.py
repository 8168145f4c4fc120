"""Substitution matrices: an alphabet plus a square integer score table.

Behaviour follows ``src/gpusw/matrix.py`` of the reference package:

* NCBI/BLAST text parsing (``matrix.py:24-52``): ``#`` and ``//`` lines are comments,
  the first data line is the column header, every row starts with its symbol and the
  row order must equal the column order; values are rounded to int.
* ``packed(unknown)`` (``matrix.py:132-151``) appends the out-of-alphabet sentinel row
  and column: the most negative off-diagonal value for ``"mismatch"``/``"error"``, or 0
  for ``"zero"``.
* ``named(name)`` loads a bundled table; ``-`` and ``_`` are ignored and case is folded
  (``matrix.py:115-129``).
"""
from __future__ import annotations

import hashlib
import os
from dataclasses import dataclass
from importlib import resources

import numpy as np

from .errors import SchemeError

__all__ = ["Matrix", "available"]


def _parse_ncbi(text: str) -> tuple[str, np.ndarray]:
    header: list[str] | None = None
    symbols: list[str] = []
    table: list[list[int]] = []
    for line in text.splitlines():
        stripped = line.strip()
        if not stripped or stripped.startswith("#") or stripped.startswith("//"):
            continue
        fields = stripped.split()
        if header is None:
            header = fields
            continue
        sym, values = fields[0], fields[1:]
        if len(values) != len(header):
            raise SchemeError(
                f"matrix row {sym!r} has {len(values)} values but the header has "
                f"{len(header)} symbols"
            )
        symbols.append(sym)
        table.append([int(round(float(v))) for v in values])
    if header is None or not table:
        raise SchemeError("no substitution matrix found in the given text")
    if symbols != header:
        raise SchemeError(
            f"matrix rows {symbols} are not in the column order {header}; only square "
            "matrices with matching row/column order are supported"
        )
    return "".join(header), np.asarray(table, dtype=np.int32)


@dataclass(frozen=True, eq=False)
class Matrix:
    """A ``(K, K)`` int32 score table over ``alphabet``; ``array[a, b]`` scores code
    ``a`` (reference residue) against code ``b`` (query residue)."""

    alphabet: str
    array: np.ndarray
    name: str | None = None

    def __post_init__(self) -> None:
        arr = np.ascontiguousarray(self.array, dtype=np.int32)
        object.__setattr__(self, "array", arr)
        k = len(self.alphabet)
        if arr.shape != (k, k):
            raise SchemeError(f"matrix shape {arr.shape} does not fit an alphabet of {k}")
        if len(set(self.alphabet)) != k:
            raise SchemeError(f"alphabet {self.alphabet!r} repeats a symbol")

    def __eq__(self, other) -> bool:
        return (isinstance(other, Matrix) and self.alphabet == other.alphabet
                and np.array_equal(self.array, other.array))

    def __hash__(self) -> int:
        return hash((self.alphabet, self.array.tobytes()))

    @classmethod
    def from_match_mismatch(cls, match: int, mismatch: int, alphabet: str = "ACGT") -> Matrix:
        k = len(alphabet)
        arr = np.where(np.eye(k, dtype=bool), np.int32(match), np.int32(mismatch))
        return cls(alphabet, arr.astype(np.int32), name=f"match{match}_mismatch{mismatch}")

    @classmethod
    def from_array(cls, alphabet: str, arr) -> Matrix:
        return cls(alphabet, np.asarray(arr, dtype=np.int32))

    @classmethod
    def from_ncbi(cls, text_or_path, name: str | None = None) -> Matrix:
        text = text_or_path
        if isinstance(text_or_path, (str, bytes, os.PathLike)) and os.path.exists(text_or_path):
            with open(text_or_path) as fh:
                text = fh.read()
        alphabet, arr = _parse_ncbi(text)
        return cls(alphabet, arr, name=name)

    @classmethod
    def named(cls, name: str) -> Matrix:
        key = name.upper().replace("-", "").replace("_", "")
        res = resources.files("gpusw_b200.data.matrices").joinpath(f"{key}.txt")
        try:
            text = res.read_text()
        except (FileNotFoundError, OSError) as exc:
            raise SchemeError(
                f"unknown matrix {name!r}; bundled: {', '.join(sorted(available()))}"
            ) from exc
        return cls.from_ncbi(text, name=key)

    def packed(self, unknown: str) -> tuple[str, np.ndarray]:
        """``(alphabet, (K+1, K+1) int32)`` with the sentinel row/column appended."""
        k = len(self.alphabet)
        out = np.zeros((k + 1, k + 1), dtype=np.int32)
        out[:k, :k] = self.array
        if unknown == "zero":
            fill = 0
        else:
            off = self.array[~np.eye(k, dtype=bool)]
            fill = int(off.min()) if off.size else int(self.array.min())
        out[k, :] = fill
        out[:, k] = fill
        return self.alphabet, out

    @property
    def max_score(self) -> int:
        return int(self.array.max())

    @property
    def min_score(self) -> int:
        return int(self.array.min())

    def hash(self) -> str:
        h = hashlib.blake2b(digest_size=12)
        h.update(self.alphabet.encode())
        h.update(np.ascontiguousarray(self.array, dtype=np.int32).tobytes())
        return h.hexdigest()

    def __repr__(self) -> str:  # pragma: no cover - cosmetic
        return f"Matrix({self.name or 'custom'!r}, alphabet={self.alphabet!r}, K={len(self.alphabet)})"


def available() -> list[str]:
    """Names of the bundled matrices."""
    root = resources.files("gpusw_b200.data.matrices")
    return sorted(p.name[:-4] for p in root.iterdir() if p.name.endswith(".txt"))
