"""Persisted packed sequence sets (an on-disk form for ``Aligner.index``).

The reference re-encodes its references in every process (``src/gpusw/aligner.py:69-77``
through the Python funnel, ``src/gpusw/encode.py:204-215``). ``save_db`` encodes once and
stores the set as the engine packs it for the device -- 2 bits per residue for DNA, 5 for
proteins -- so ``load_db`` maps that image from disk (``numpy.memmap``, no copy) and
``Aligner.index(load_db(path))`` uploads it without packing it again. Layout::

    path/meta.json      {"format": 2, "n": N, "residues": R, "bits": B, "nwords": W,
                         "image_bytes": S, "alphabet": "...", "scheme": {...}}
    path/image.bin      the packed device image (gpusw_pack_image): words | int64 word
                        offsets | int32 lengths, 256-byte aligned parts
    path/offsets.i32    N + 1 int32 residue offsets (lengths without reading the image)
    path/ids.txt        N identifiers, one per line

Sets written by the first format (``codes.u8`` with one byte per residue) still load, as an
:class:`~gpusw_b200.encode.Encoded` set that is packed on upload.
"""
from __future__ import annotations

import json
import os

import numpy as np

from .encode import Encoded
from .errors import EncodeError

__all__ = ["save_db", "load_db", "PackedSet"]

FORMAT = 2


class PackedSet:
    """An encoded set held as the engine's packed image (what :func:`load_db` returns).

    It offers the attributes of :class:`~gpusw_b200.encode.Encoded` that callers read --
    ``n``, ``ids``, ``offsets``, ``lengths``, ``alphabet``, ``max_len`` -- and ``codes``,
    which unpacks the image on first use (only coordinate look-ups need it)."""

    def __init__(self, image, bits: int, nwords: int, offsets, ids, alphabet: str):
        self.image = image
        self.bits = int(bits)
        self.nwords = int(nwords)
        self.offsets = offsets
        self.ids = ids
        self.alphabet = alphabet
        self.lengths = np.diff(offsets).astype(np.int32)
        self._codes = None

    @property
    def n(self) -> int:
        return len(self.ids)

    @property
    def max_len(self) -> int:
        return int(self.lengths.max()) if self.n else 0

    @property
    def codes(self) -> np.ndarray:
        if self._codes is None:
            self._codes = unpack_image(self.image, self.bits, self.nwords, self.lengths)
        return self._codes


def _layout(nwords: int, n: int) -> tuple[int, int, int]:
    """(word offsets start, lengths start, image bytes) of a packed image."""
    words_b = (nwords + 64) * 4
    woff_o = (words_b + 255) & ~255
    len_o = woff_o + ((max(1, n) * 8 + 255) & ~255)
    return woff_o, len_o, len_o + max(1, n) * 4


def unpack_image(image, bits: int, nwords: int, lengths) -> np.ndarray:
    """Residue codes of a packed image (all sequences concatenated), with numpy."""
    n = len(lengths)
    woff_o, _, _ = _layout(nwords, n)
    words = np.frombuffer(np.asarray(image), dtype="<u4", count=nwords)
    woff = np.frombuffer(np.asarray(image), dtype="<i8", count=n, offset=woff_o)
    per = 6 if bits == 5 else 32 // bits
    lens = np.asarray(lengths, dtype=np.int64)
    total = int(lens.sum())
    if total == 0:
        return np.zeros(0, dtype=np.uint8)
    seq = np.repeat(np.arange(n), lens)
    pos = np.arange(total, dtype=np.int64) - np.repeat(np.cumsum(lens) - lens, lens)
    w = words[woff[seq] + pos // per]
    return ((w >> ((pos % per) * bits).astype(np.uint32)) & ((1 << bits) - 1)).astype(np.uint8)


def _scheme_meta(scheme) -> dict | None:
    if scheme is None:
        return None
    return {"mode": scheme.mode, "alphabet": scheme.eff_alphabet, "table_hash": scheme.table_hash(),
            "case_insensitive": scheme.case_insensitive, "unknown": scheme.unknown}


def save_db(enc: Encoded, path: str, scheme=None) -> str:
    """Pack ``enc`` with the engine's packer and write it (and, optionally, the scheme it was
    encoded for) under ``path``. Needs the built engine library, not a GPU."""
    from . import _native

    os.makedirs(path, exist_ok=True)
    for name in ("\n", "\r"):
        if any(name in str(i) for i in enc.ids):
            raise EncodeError("sequence ids must not contain line breaks")
    codes = np.ascontiguousarray(enc.codes, dtype=np.uint8)
    offsets = np.ascontiguousarray(enc.offsets, dtype="<i4")
    image, bits, nwords = _native.pack_image(codes, offsets)
    image.tofile(os.path.join(path, "image.bin"))
    offsets.tofile(os.path.join(path, "offsets.i32"))
    with open(os.path.join(path, "ids.txt"), "w") as fh:
        fh.write("\n".join(str(i) for i in enc.ids))
    meta = {"format": FORMAT, "n": enc.n, "residues": int(codes.size), "bits": bits,
            "nwords": nwords, "image_bytes": int(image.size), "alphabet": enc.alphabet,
            "scheme": _scheme_meta(scheme)}
    with open(os.path.join(path, "meta.json"), "w") as fh:
        json.dump(meta, fh)
    return path


def load_db(path: str, scheme=None, mmap: bool = True):
    """Load a set written by :func:`save_db` (a :class:`PackedSet`; format-1 sets load as
    :class:`~gpusw_b200.encode.Encoded`). With ``scheme``, check that the set was encoded
    with the same alphabet."""
    with open(os.path.join(path, "meta.json")) as fh:
        meta = json.load(fh)
    fmt = meta.get("format")
    if fmt not in (1, FORMAT):
        raise EncodeError(f"unsupported database format {fmt!r}")
    n, r = int(meta["n"]), int(meta["residues"])
    if scheme is not None and meta["alphabet"] != scheme.eff_alphabet:
        raise EncodeError(f"database alphabet {meta['alphabet']!r} != scheme alphabet "
                          f"{scheme.eff_alphabet!r}")
    offsets = np.fromfile(os.path.join(path, "offsets.i32"), dtype="<i4", count=n + 1).astype(np.int32)
    if offsets.shape[0] != n + 1 or (n and int(offsets[-1]) > r) or (np.diff(offsets) < 0).any():
        raise EncodeError("corrupt database: offsets do not match the codes")
    with open(os.path.join(path, "ids.txt")) as fh:
        ids = fh.read().split("\n") if n else []
    if len(ids) != n:
        raise EncodeError("corrupt database: id count does not match")
    if fmt == 1:
        cpath = os.path.join(path, "codes.u8")
        if mmap and r > 0:
            codes = np.memmap(cpath, dtype=np.uint8, mode="r", shape=(r,))
        else:
            codes = np.fromfile(cpath, dtype=np.uint8, count=r)
        return Encoded(codes, offsets, ids, np.diff(offsets).astype(np.int32), meta["alphabet"])
    bits, nwords, size = int(meta["bits"]), int(meta["nwords"]), int(meta["image_bytes"])
    if bits not in (2, 4, 5, 8) or _layout(nwords, n)[2] != size:
        raise EncodeError("corrupt database: image layout")
    ipath = os.path.join(path, "image.bin")
    if os.path.getsize(ipath) != size:
        raise EncodeError("corrupt database: image size")
    image = (np.memmap(ipath, dtype=np.uint8, mode="r", shape=(size,)) if mmap
             else np.fromfile(ipath, dtype=np.uint8, count=size))
    woff_o, len_o, _ = _layout(nwords, n)
    if n and not np.array_equal(np.frombuffer(np.asarray(image), dtype="<i4", count=n, offset=len_o),
                                np.diff(offsets)):
        raise EncodeError("corrupt database: image lengths do not match the offsets")
    return PackedSet(image, bits, nwords, offsets, ids, meta["alphabet"])
