"""Persisted encoded sequence sets (an on-disk form for ``Aligner.index``).

The reference re-encodes its references in every process (``src/gpusw/aligner.py:69-77``
through the Python funnel, ``src/gpusw/encode.py:204-215``). ``save_db`` writes an
:class:`~gpusw_b200.encode.Encoded` set once as a directory of raw little-endian arrays;
``load_db`` maps them back without copying (``numpy.memmap``), so a server restart or a new
process can ``Aligner.index(load_db(path))`` straight away. Layout::

    path/meta.json      {"format": 1, "n": N, "residues": R, "alphabet": "...", "scheme": {...}}
    path/codes.u8       R residue codes (uint8, the scheme's LUT codes; sentinel = len(alphabet))
    path/offsets.i32    N + 1 int32 offsets
    path/ids.txt        N identifiers, one per line
"""
from __future__ import annotations

import json
import os

import numpy as np

from .encode import Encoded
from .errors import EncodeError

__all__ = ["save_db", "load_db"]

FORMAT = 1


def _scheme_meta(scheme) -> dict | None:
    if scheme is None:
        return None
    return {"mode": scheme.mode, "alphabet": scheme.eff_alphabet, "table_hash": scheme.table_hash(),
            "case_insensitive": scheme.case_insensitive, "unknown": scheme.unknown}


def save_db(enc: Encoded, path: str, scheme=None) -> str:
    """Write ``enc`` (and, optionally, the scheme it was encoded for) under ``path``."""
    os.makedirs(path, exist_ok=True)
    codes = np.ascontiguousarray(enc.codes, dtype=np.uint8)
    offsets = np.ascontiguousarray(enc.offsets, dtype="<i4")
    for name in ("\n", "\r"):
        if any(name in str(i) for i in enc.ids):
            raise EncodeError("sequence ids must not contain line breaks")
    codes.tofile(os.path.join(path, "codes.u8"))
    offsets.tofile(os.path.join(path, "offsets.i32"))
    with open(os.path.join(path, "ids.txt"), "w") as fh:
        fh.write("\n".join(str(i) for i in enc.ids))
    meta = {"format": FORMAT, "n": enc.n, "residues": int(codes.size), "alphabet": enc.alphabet,
            "scheme": _scheme_meta(scheme)}
    with open(os.path.join(path, "meta.json"), "w") as fh:
        json.dump(meta, fh)
    return path


def load_db(path: str, scheme=None, mmap: bool = True) -> Encoded:
    """Load a set written by :func:`save_db`. With ``scheme``, check that the set was encoded
    with the same alphabet (and, when recorded, the same substitution table)."""
    with open(os.path.join(path, "meta.json")) as fh:
        meta = json.load(fh)
    if meta.get("format") != FORMAT:
        raise EncodeError(f"unsupported database format {meta.get('format')!r}")
    n, r = int(meta["n"]), int(meta["residues"])
    if scheme is not None and meta["alphabet"] != scheme.eff_alphabet:
        raise EncodeError(f"database alphabet {meta['alphabet']!r} != scheme alphabet "
                          f"{scheme.eff_alphabet!r}")
    mode = "r" if mmap else None
    cpath, opath = os.path.join(path, "codes.u8"), os.path.join(path, "offsets.i32")
    if mmap and r > 0:
        codes = np.memmap(cpath, dtype=np.uint8, mode=mode, shape=(r,))
    else:
        codes = np.fromfile(cpath, dtype=np.uint8, count=r)
    offsets = np.fromfile(opath, dtype="<i4", count=n + 1).astype(np.int32)
    if offsets.shape[0] != n + 1 or (n and int(offsets[-1]) > r) or (np.diff(offsets) < 0).any():
        raise EncodeError("corrupt database: offsets do not match the codes")
    with open(os.path.join(path, "ids.txt")) as fh:
        ids = fh.read().split("\n") if n else []
    if len(ids) != n:
        raise EncodeError("corrupt database: id count does not match")
    return Encoded(codes, offsets, ids, np.diff(offsets).astype(np.int32), meta["alphabet"])
