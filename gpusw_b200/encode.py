"""The input funnel: every accepted input form becomes one concatenated ``uint8`` code
buffer plus ``int32`` offsets.

Accepted forms and their meaning follow ``src/gpusw/encode.py:1-220`` of the reference
package: lists/tuples/arrays of strings (ids ``q0, q1, ...``), dicts (ids = keys),
``(id, seq)`` pairs or ``.seq`` records, FASTA paths (``.gz`` too), FASTA text, one raw
``str``/``bytes`` sequence, a pre-encoded ``(codes, offsets[, ids])`` tuple (validated like
``encode.py:174-197``) or an :class:`Encoded` (returned as-is when the alphabet matches).

Encoding semantics (``encode.py:30-44``, ``:204-215``): symbol ``alphabet[k]`` -> code
``k``, anything else -> the sentinel ``K = len(alphabet)``; case is folded when the
scheme says so; text is encoded latin-1 with ``"replace"`` so every character is exactly
one byte. Unlike the reference's per-sequence loop, the table lookup here runs once over
all sequences joined together, which gives the same codes and lengths.
"""
from __future__ import annotations

import gzip
import os
from dataclasses import dataclass

import numpy as np

from .errors import EncodeError, NoGpuError

__all__ = ["Encoded", "funnel", "build_lut", "read_fasta"]

_SEQ_EXTS = (".fasta", ".fa", ".fna", ".faa", ".ffn", ".fastq", ".fq", ".txt", ".gz")


def build_lut(scheme) -> tuple[np.ndarray, int]:
    """``(lut[256] uint8, sentinel)`` for the scheme's effective alphabet."""
    alpha = scheme.eff_alphabet
    sentinel = len(alpha)
    lut = np.full(256, sentinel, dtype=np.uint8)
    for code, sym in enumerate(alpha):
        lut[ord(sym)] = code
        if scheme.case_insensitive:
            lut[ord(sym.lower())] = code
            lut[ord(sym.upper())] = code
    return lut, sentinel


@dataclass
class Encoded:
    """Sequences in kernel form: ``codes[offsets[i]:offsets[i+1]]`` is sequence ``i``."""

    codes: np.ndarray
    offsets: np.ndarray
    ids: list
    lengths: np.ndarray
    alphabet: str

    @property
    def n(self) -> int:
        return len(self.ids)

    @property
    def max_len(self) -> int:
        return int(self.lengths.max()) if self.n else 0


def _looks_like_path(s: str) -> bool:
    return ("/" in s) or (os.sep in s) or s.lower().endswith(_SEQ_EXTS)


def read_fasta(path_or_text) -> list[tuple[str, str]]:
    """Parse FASTA from a path (``.gz`` allowed) or from text into ``[(id, seq), ...]``."""
    if isinstance(path_or_text, (str, os.PathLike)) and os.path.exists(path_or_text):
        opener = gzip.open if str(path_or_text).endswith(".gz") else open
        with opener(path_or_text, "rt") as fh:
            text = fh.read()
    else:
        text = str(path_or_text)
        if not text.lstrip().startswith(">") and _looks_like_path(text):
            raise FileNotFoundError(f"FASTA file not found: {path_or_text}")
    records: list[tuple[str, str]] = []
    ident = None
    chunks: list[str] = []
    for raw in text.splitlines():
        line = raw.strip()
        if not line:
            continue
        if line.startswith(">"):
            if ident is not None:
                records.append((ident, "".join(chunks)))
            ident = line[1:].split()[0] if len(line) > 1 else f"seq{len(records)}"
            chunks = []
        else:
            chunks.append(line)
    if ident is not None:
        records.append((ident, "".join(chunks)))
    return records


def _to_pairs(obj, id_prefix: str) -> list[tuple[str, str]]:
    if isinstance(obj, dict):
        return [(str(k), str(v)) for k, v in obj.items()]
    if isinstance(obj, (bytes, bytearray)):
        return [(f"{id_prefix}0", bytes(obj).decode("latin-1"))]
    if isinstance(obj, str):
        if obj.lstrip().startswith(">") or os.path.exists(obj):
            return read_fasta(obj)
        if _looks_like_path(obj):
            raise EncodeError(f"file not found: {obj!r}")
        return [(f"{id_prefix}0", obj)]
    if isinstance(obj, np.ndarray):
        obj = obj.tolist()
    try:
        items = list(obj)
    except TypeError as exc:
        raise EncodeError(f"cannot funnel an object of type {type(obj).__name__}") from exc
    out: list[tuple[str, str]] = []
    for i, item in enumerate(items):
        if isinstance(item, str):
            out.append((f"{id_prefix}{i}", item))
        elif isinstance(item, (tuple, list)) and len(item) == 2:
            out.append((str(item[0]), str(item[1])))
        elif hasattr(item, "seq"):
            out.append((str(getattr(item, "id", None) or f"{id_prefix}{i}"), str(item.seq)))
        else:
            raise EncodeError(
                f"item {i} of type {type(item).__name__} is not a sequence, an (id, seq) "
                "pair or a record with .seq"
            )
    return out


def _pre_encoded(obj, scheme, id_prefix: str) -> Encoded:
    codes = np.ascontiguousarray(obj[0], dtype=np.uint8)
    offsets = np.ascontiguousarray(obj[1], dtype=np.int32)
    if offsets.size == 0:
        raise EncodeError("pre-encoded offsets must have length n+1 (>= 1)")
    if (offsets < 0).any():
        raise EncodeError("pre-encoded offsets must be non-negative")
    if (np.diff(offsets) < 0).any():
        raise EncodeError("pre-encoded offsets must be non-decreasing")
    if int(offsets[-1]) > codes.size:
        raise EncodeError(
            f"pre-encoded offsets[-1]={int(offsets[-1])} exceeds len(codes)={codes.size}"
        )
    n = offsets.size - 1
    ids = list(obj[2]) if len(obj) == 3 else [f"{id_prefix}{i}" for i in range(n)]
    return Encoded(codes, offsets, ids, np.diff(offsets).astype(np.int32), scheme.eff_alphabet)


def encode_pairs(pairs, scheme) -> Encoded:
    """Encode ``[(id, seq), ...]`` with one LUT pass over the joined text."""
    lut, sentinel = build_lut(scheme)
    ids = [p[0] for p in pairs]
    texts = [p[1].upper() for p in pairs] if scheme.case_insensitive else [p[1] for p in pairs]
    lengths = np.fromiter((len(t) for t in texts), dtype=np.int64, count=len(texts))
    total = int(lengths.sum())
    if total >= 2**31:
        raise EncodeError("more than 2**31 - 1 residues in one sequence set")
    raw = np.frombuffer("".join(texts).encode("latin-1", "replace"), dtype=np.uint8)
    codes = lut[raw]
    offsets = np.zeros(len(texts) + 1, dtype=np.int32)
    np.cumsum(lengths, out=offsets[1:])
    if scheme.unknown == "error" and codes.size:
        bad = np.flatnonzero(codes == sentinel)
        if bad.size:
            pos = int(bad[0])
            seq_idx = int(np.searchsorted(offsets, pos, side="right")) - 1
            sym = bytes(raw[pos:pos + 1]).decode("latin-1")
            raise EncodeError(
                f"sequence {ids[seq_idx]!r} contains out-of-alphabet symbol {sym!r} "
                f"(alphabet={scheme.eff_alphabet!r}); set unknown='mismatch' or 'zero'"
            )
    return Encoded(np.ascontiguousarray(codes, dtype=np.uint8), offsets, ids,
                   lengths.astype(np.int32), scheme.eff_alphabet)


def _fasta_bytes(obj: str):
    """The FASTA bytes behind a str input (a path, ``.gz`` too, or FASTA text), else None."""
    if os.path.exists(obj):
        with open(obj, "rb") as fh:
            data = fh.read()
        return gzip.decompress(data) if obj.endswith(".gz") else data
    if obj.lstrip().startswith(">"):
        try:
            return obj.encode("ascii")
        except UnicodeEncodeError:
            return None
    return None


def _encode_fasta_native(data: bytes, scheme) -> Encoded | None:
    """FASTA bytes -> Encoded in one native pass (the engine library's reader; no GPU
    needed). None when the library is not built or the text needs the Unicode reader; an
    out-of-alphabet symbol is also left to the Python path, which words the error."""
    try:
        from . import _native

        lut, sentinel = build_lut(scheme)
        res = _native.parse_fasta(data, lut, sentinel, scheme.unknown == "error")
    except (ImportError, OSError, NoGpuError):  # the library is not built
        return None
    except ValueError as exc:
        if getattr(exc, "bad_record", -1) >= 0:
            return None
        raise EncodeError(str(exc)) from None
    if res is None:
        return None
    codes, offsets, ids = res
    return Encoded(codes, offsets, ids, np.diff(offsets).astype(np.int32), scheme.eff_alphabet)


def funnel(obj, scheme, *, id_prefix: str = "q") -> Encoded:
    """Turn any accepted input into an :class:`Encoded` for ``scheme``.

    FASTA paths and FASTA text go through the engine library's native reader when it is
    built and the text is plain ASCII (one pass: lines, ids, table lookup); everything else,
    and those when the native reader declines, through the Python reader below. Both give
    the same records, codes and errors."""
    if isinstance(obj, Encoded):
        if obj.alphabet != scheme.eff_alphabet:
            raise EncodeError(
                f"Encoded alphabet {obj.alphabet!r} != scheme alphabet "
                f"{scheme.eff_alphabet!r}; re-encode for this scheme"
            )
        return obj
    if (isinstance(obj, tuple) and len(obj) in (2, 3) and isinstance(obj[0], np.ndarray)
            and isinstance(obj[1], np.ndarray) and obj[0].dtype == np.uint8):
        return _pre_encoded(obj, scheme, id_prefix)
    if isinstance(obj, str):
        data = _fasta_bytes(obj)
        if data is not None:
            enc = _encode_fasta_native(data, scheme)
            if enc is not None:
                return enc
    return encode_pairs(_to_pairs(obj, id_prefix), scheme)
