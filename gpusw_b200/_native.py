"""ctypes binding of the native engine ``libgpusw_sm100.so`` (C ABI in include/gpusw_b200.h).

This is the only module that talks to the GPU. It replaces the reference package's CuPy
boundary (``src/gpusw/_compile.py`` and ``src/gpusw/backends/cuda.py``): there is no
runtime compilation and no CPU fallback -- if the shared library is missing or no device
is visible, the scoring calls raise :class:`~gpusw_b200.errors.NoGpuError`.
"""
from __future__ import annotations

import ctypes
import os
import threading

import numpy as np

from .errors import GpuSWError, NoGpuError, OverflowRiskError, SchemeError

__all__ = ["LIB_PATH", "load", "gpu_available", "Context", "context", "Stats", "ServerStats"]

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libgpusw_sm100.so")

OK, E_INVALID, E_NO_GPU, E_CUDA, E_MEMORY, E_OVERFLOW, E_SCHEME = 0, 1, 2, 3, 4, 5, 6
E_QUEUE_FULL, E_NOT_FOUND, E_CANCELLED, E_TIMEOUT, E_UNSUPPORTED = 7, 8, 9, 10, 11
DTYPE_CODES = {"auto": 0, "int16": 1, "int32": 2}
MODE_CODES = {"local": 0, "global": 1, "semiglobal": 2}

_lib = None
_lib_lock = threading.Lock()


class Stats(ctypes.Structure):
    _fields_ = [
        ("last_kernel_ms", ctypes.c_double),
        ("last_score_ms", ctypes.c_double),
        ("last_topk_ms", ctypes.c_double),
        ("last_total_ms", ctypes.c_double),
        ("last_cells", ctypes.c_double),
        ("last_pairs", ctypes.c_int64),
        ("last_overflow", ctypes.c_int64),
        ("last_launches", ctypes.c_int64),
        ("total_launches", ctypes.c_int64),
        ("total_overflow", ctypes.c_int64),
        ("device_bytes", ctypes.c_int64),
        ("last_inter_items", ctypes.c_int64),
    ]


class ServerStats(ctypes.Structure):
    _fields_ = [
        ("submitted", ctypes.c_int64), ("completed", ctypes.c_int64),
        ("cancelled", ctypes.c_int64), ("rejected", ctypes.c_int64),
        ("pending", ctypes.c_int64), ("running", ctypes.c_int64),
        ("batches", ctypes.c_int64), ("mean_batch_queries", ctypes.c_double),
        ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double),
        ("mean_ms", ctypes.c_double), ("max_ms", ctypes.c_double),
        ("cells", ctypes.c_double), ("wall_s", ctypes.c_double), ("gcups", ctypes.c_double),
        ("device_bytes", ctypes.c_int64),
    ]


_VP, _I32, _I64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64

_SIGNATURES = {
    "gpusw_version": ([], ctypes.c_int),
    "gpusw_device_count": ([ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "gpusw_ctx_create": ([ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
    "gpusw_ctx_destroy": ([ctypes.c_void_p], None),
    "gpusw_last_error": ([ctypes.c_void_p], ctypes.c_char_p),
    "gpusw_set_scheme": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                          ctypes.c_int, ctypes.c_int, ctypes.c_void_p], ctypes.c_int),
    "gpusw_db_upload": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
                         ctypes.POINTER(ctypes.c_int32)], ctypes.c_int),
    "gpusw_db_free": ([ctypes.c_void_p, ctypes.c_int32], ctypes.c_int),
    "gpusw_db_bits": ([ctypes.c_void_p, ctypes.c_int32], ctypes.c_int),
    "gpusw_score_cross": ([ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p,
                           ctypes.c_int32, ctypes.c_int, ctypes.c_void_p], ctypes.c_int),
    "gpusw_topk": ([ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p,
                    ctypes.c_int32, ctypes.c_int32, ctypes.c_int, ctypes.c_void_p,
                    ctypes.c_void_p], ctypes.c_int),
    "gpusw_score_pairs": ([ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p,
                           ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_void_p],
                          ctypes.c_int),
    "gpusw_set_options": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_int], ctypes.c_int),
    "gpusw_autotune": ([ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_int32],
                       ctypes.c_int),
    "gpusw_get_stats": ([ctypes.c_void_p, ctypes.POINTER(Stats)], ctypes.c_int),
    "gpusw_sync": ([ctypes.c_void_p], ctypes.c_int),
    "gpusw_measure_dpx_rate": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)], ctypes.c_int),
    "gpusw_flush_l2": ([ctypes.c_void_p, ctypes.c_int64], ctypes.c_int),
    "gpusw_locate_pairs": ([_VP, _I32, _I32, _VP, _VP, _I64, ctypes.c_int, _VP, _VP, _VP], ctypes.c_int),
    "gpusw_get_tune": ([_VP, ctypes.c_int, ctypes.POINTER(ctypes.c_double), _I32], ctypes.c_int),
    "gpusw_set_tune": ([_VP, ctypes.c_int, ctypes.POINTER(ctypes.c_double), _I32], ctypes.c_int),
    "gpusw_device_name": ([ctypes.c_int, ctypes.c_char_p, _I32], ctypes.c_int),
    "gpusw_pack_image": ([_VP, _VP, _I32, _VP, _I64, ctypes.POINTER(_I64), ctypes.POINTER(_I32),
                          ctypes.POINTER(_I64)], ctypes.c_int),
    "gpusw_db_upload_image": ([_VP, _VP, _I64, _I32, _I32, _I64, ctypes.POINTER(_I32)], ctypes.c_int),
    "gpusw_score_pairs_zip": ([_VP, _VP, _VP, _VP, _VP, _I64, ctypes.c_int, _VP], ctypes.c_int),
    "gpusw_score_pairs_noalloc": ([_VP, _VP, _I32, _VP, _VP, _I32, _VP, _VP, _I32, ctypes.c_int,
                                   ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_int, _VP, _I32, _VP, _VP, ctypes.c_char_p, _I32],
                                  ctypes.c_int),
    "gpusw_server_create": ([_VP, _I32, _I32, ctypes.c_int, _I64, _I32, _I32, _I32,
                             ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
    "gpusw_server_submit": ([_VP, _VP, _VP, _I32, ctypes.POINTER(_I64)], ctypes.c_int),
    "gpusw_server_poll": ([_VP, _I64, _I32, ctypes.POINTER(_I32), _VP, _VP], ctypes.c_int),
    "gpusw_server_cancel": ([_VP, _I64], ctypes.c_int),
    "gpusw_server_get_stats": ([_VP, ctypes.POINTER(ServerStats)], ctypes.c_int),
    "gpusw_server_last_error": ([_VP], ctypes.c_char_p),
    "gpusw_server_destroy": ([_VP], None),
    "gpusw_server_set_batch_cells": ([_VP, ctypes.c_double], ctypes.c_int),
    "gpusw_fasta_parse": ([ctypes.c_char_p, _I64, _VP, _I32, ctypes.c_int, ctypes.POINTER(_VP)], ctypes.c_int),
    "gpusw_fasta_count": ([_VP], _I32),
    "gpusw_fasta_residues": ([_VP], _I64),
    "gpusw_fasta_codes": ([_VP], _VP),
    "gpusw_fasta_offsets": ([_VP], _VP),
    "gpusw_fasta_ids": ([_VP], _VP),
    "gpusw_fasta_id_offsets": ([_VP], _VP),
    "gpusw_fasta_error": ([_VP], ctypes.c_char_p),
    "gpusw_fasta_bad_record": ([_VP], _I64),
    "gpusw_fasta_bad_byte": ([_VP], _I32),
    "gpusw_fasta_free": ([_VP], None),
}


def load():
    """Load the shared library (once); raise NoGpuError if it is not built."""
    global _lib
    with _lib_lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise NoGpuError(
                    f"native engine {LIB_PATH} is not built; run `python -c \"import "
                    "__graft_entry__ as g; g.build()\"` or `python -m gpusw_b200.build`")
            lib = ctypes.CDLL(LIB_PATH)
            for name, (args, res) in _SIGNATURES.items():
                fn = getattr(lib, name)
                fn.argtypes = args
                fn.restype = res
            _lib = lib
    return _lib


def parse_fasta(data: bytes, lut: np.ndarray, sentinel: int, unknown_error: bool):
    """FASTA bytes -> (codes uint8, offsets int32, ids) through the native reader, or None
    when the text needs the Unicode reader (a byte >= 0x80, vertical tab, form feed or a
    byte 0x1c-0x1f).

    Raises ``ValueError`` with attributes ``bad_record`` / ``bad_byte`` for an
    out-of-alphabet symbol (unknown="error") or a set beyond 2**31 - 1 residues.
    Needs no GPU.
    """
    lib = load()
    lut = np.ascontiguousarray(lut, dtype=np.uint8)
    h = ctypes.c_void_p()
    rc = lib.gpusw_fasta_parse(data, len(data), _ptr(lut), int(sentinel), int(bool(unknown_error)),
                               ctypes.byref(h))
    try:
        if rc == E_UNSUPPORTED:
            return None
        if rc != OK:
            err = ValueError(lib.gpusw_fasta_error(h).decode() if h.value else f"status {rc}")
            err.bad_record = int(lib.gpusw_fasta_bad_record(h)) if h.value else -1
            err.bad_byte = int(lib.gpusw_fasta_bad_byte(h)) if h.value else -1
            raise err
        n = int(lib.gpusw_fasta_count(h))
        total = int(lib.gpusw_fasta_residues(h))
        codes = np.empty(total, dtype=np.uint8)
        if total:
            ctypes.memmove(codes.ctypes.data, lib.gpusw_fasta_codes(h), total)
        offsets = np.empty(n + 1, dtype=np.int32)
        ctypes.memmove(offsets.ctypes.data, lib.gpusw_fasta_offsets(h), 4 * (n + 1))
        id_off = np.ctypeslib.as_array(ctypes.cast(lib.gpusw_fasta_id_offsets(h), ctypes.POINTER(ctypes.c_int64)),
                                       shape=(n + 1,))
        nbytes = int(id_off[-1])
        blob = ctypes.string_at(lib.gpusw_fasta_ids(h), nbytes).decode("ascii") if nbytes else ""
        bounds = id_off.tolist()
        ids = [blob[bounds[k]:bounds[k + 1]] for k in range(n)]
        return codes, offsets, ids
    finally:
        if h.value:
            lib.gpusw_fasta_free(h)


def pack_image(codes: np.ndarray, offsets: np.ndarray) -> tuple[np.ndarray, int, int]:
    """The engine's packed device image of an encoded set (host only, no GPU needed):
    ``(image uint8, bits per residue, packed words)``."""
    lib = load()
    codes = np.ascontiguousarray(codes, dtype=np.uint8)
    offsets = np.ascontiguousarray(offsets, dtype=np.int32)
    n = offsets.shape[0] - 1
    need, bits, nwords = ctypes.c_int64(0), ctypes.c_int32(0), ctypes.c_int64(0)
    args = (_ptr(codes), _ptr(offsets), n)
    outs = (ctypes.byref(need), ctypes.byref(bits), ctypes.byref(nwords))
    rc = lib.gpusw_pack_image(*args, None, 0, *outs)
    if rc == OK:
        image = np.empty(need.value, dtype=np.uint8)
        rc = lib.gpusw_pack_image(*args, _ptr(image), image.size, *outs)
    if rc != OK:
        _raise(rc, lib.gpusw_last_error(None).decode())
    return image, bits.value, nwords.value


def gpu_available() -> bool:
    """True iff the native engine loads and at least one CUDA device is visible."""
    try:
        lib = load()
    except (NoGpuError, OSError):
        return False
    n = ctypes.c_int(0)
    return lib.gpusw_device_count(ctypes.byref(n)) == OK and n.value > 0


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _raise(code: int, msg: str):
    if code == E_INVALID or code == E_NOT_FOUND:
        raise ValueError(msg)
    if code == E_NO_GPU:
        raise NoGpuError(msg)
    if code == E_OVERFLOW:
        raise OverflowRiskError(msg)
    if code == E_SCHEME:
        raise SchemeError(msg)
    raise GpuSWError(msg)


class Context:
    """One native context: a CUDA stream on one device plus the resident sequence sets."""

    def __init__(self, device: int = 0):
        self.lib = load()
        self.device = int(device)
        handle = ctypes.c_void_p()
        rc = self.lib.gpusw_ctx_create(self.device, ctypes.byref(handle))
        if rc != OK:
            _raise(rc, self.lib.gpusw_last_error(None).decode() or "context creation failed")
        self.handle = handle
        self._scheme_key = None
        self.lock = threading.RLock()

    def _check(self, rc: int):
        if rc != OK:
            _raise(rc, self.lib.gpusw_last_error(self.handle).decode())

    def close(self):
        if getattr(self, "handle", None):
            self.lib.gpusw_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------------ configuration
    def set_scheme(self, scheme) -> None:
        key = (scheme.mode, scheme.gap_open, scheme.gap_extend, bool(scheme.free_end_gaps_query),
               bool(scheme.free_end_gaps_ref), scheme.table_hash())
        if key == self._scheme_key:
            return
        sub = np.ascontiguousarray(scheme.substitution_table(), dtype=np.int32)
        self._check(self.lib.gpusw_set_scheme(
            self.handle, MODE_CODES[scheme.mode], scheme.gap_open, scheme.gap_extend,
            int(bool(scheme.free_end_gaps_query)), int(bool(scheme.free_end_gaps_ref)),
            int(sub.shape[0]), _ptr(sub)))
        self._scheme_key = key
        if scheme.mode == "local":
            self._load_tune(int(sub.shape[0]))

    # ------------------------------------------------------------------ autotune cache
    def _tune_path(self, ns: int, width: int) -> str | None:
        root = os.environ.get("GPUSW_B200_TUNE_DIR",
                              os.path.join(os.path.expanduser("~"), ".cache", "gpusw_b200"))
        buf = ctypes.create_string_buffer(256)
        if self.lib.gpusw_device_name(self.device, buf, 256) != OK:
            return None
        name = "".join(ch if ch.isalnum() else "_" for ch in buf.value.decode())
        return os.path.join(root, f"tune-{name}-v{self.lib.gpusw_version()}-ns{ns}-w{width}.txt")

    def _load_tune(self, ns: int) -> None:
        """Install autotuner tables cached on disk by an earlier process (if any)."""
        for width in (2, 1):
            path = self._tune_path(ns, width)
            if not path or not os.path.exists(path):
                continue
            have = self.lib.gpusw_get_tune(self.handle, width, None, 0)
            if have > 0:
                continue
            try:
                vals = [float(x) for x in open(path).read().split()]
            except (OSError, ValueError):
                continue
            arr = (ctypes.c_double * len(vals))(*vals)
            self.lib.gpusw_set_tune(self.handle, width, arr, len(vals))

    def save_tune(self, ns: int) -> None:
        """Write the context's autotuner tables for alphabet size `ns` to the disk cache."""
        for width in (2, 1):
            out = (ctypes.c_double * 64)()
            got = self.lib.gpusw_get_tune(self.handle, width, out, 64)
            path = self._tune_path(ns, width)
            if got > 0 and path and not os.path.exists(path):
                try:
                    os.makedirs(os.path.dirname(path), exist_ok=True)
                    with open(path + ".tmp", "w") as fh:
                        fh.write(" ".join(repr(out[i]) for i in range(got)))
                    os.replace(path + ".tmp", path)
                except OSError:
                    pass

    def set_options(self, plain: bool = False, mem_budget: int = 0, autotune: bool = True,
                    graphs: bool = True, one_launch: bool = False, inter: bool = True) -> None:
        flags = ((0 if autotune else 1) | (0 if graphs else 2) | (4 if one_launch else 0)
                 | (0 if inter else 8))
        self._check(self.lib.gpusw_set_options(self.handle, int(bool(plain)), int(mem_budget), flags))

    def autotune(self, width: int = 2) -> list[float]:
        """(Re)tune the streaming kernel shapes for the current scheme; microseconds per
        (reference row, column pass) of every compiled shape."""
        out = (ctypes.c_double * 64)()
        self._check(self.lib.gpusw_autotune(self.handle, int(width), out, 64))
        return [out[i] for i in range(64) if out[i] > 0]

    # ------------------------------------------------------------------ sequence sets
    def upload(self, codes: np.ndarray, offsets: np.ndarray) -> int:
        codes = np.ascontiguousarray(codes, dtype=np.uint8)
        offsets = np.ascontiguousarray(offsets, dtype=np.int32)
        n = offsets.shape[0] - 1
        h = ctypes.c_int32(0)
        self._check(self.lib.gpusw_db_upload(self.handle, _ptr(codes), _ptr(offsets), n,
                                             ctypes.byref(h)))
        return h.value

    def upload_image(self, image: np.ndarray, n: int, bits: int, nwords: int) -> int:
        """Upload a packed image made by :func:`pack_image` (it is checked, not re-packed)."""
        image = np.ascontiguousarray(image, dtype=np.uint8)
        h = ctypes.c_int32(0)
        self._check(self.lib.gpusw_db_upload_image(self.handle, _ptr(image), image.size, int(n),
                                                   int(bits), int(nwords), ctypes.byref(h)))
        return h.value

    def free(self, db: int) -> None:
        if self.handle:
            self.lib.gpusw_db_free(self.handle, int(db))

    def bits(self, db: int) -> int:
        v = self.lib.gpusw_db_bits(self.handle, int(db))
        if v < 0:
            self._check(-v)
        return v

    # ----------------------------------------------------------------------- scoring
    def score_cross(self, qdb: int, rdb: int, qlist: np.ndarray, n_refs: int, dtype: str) -> np.ndarray:
        qlist = np.ascontiguousarray(qlist, dtype=np.int32)
        out = np.empty((qlist.shape[0], n_refs), dtype=np.int32)
        self._check(self.lib.gpusw_score_cross(self.handle, qdb, rdb, _ptr(qlist), qlist.shape[0],
                                               DTYPE_CODES[dtype], _ptr(out)))
        return out

    def topk(self, qdb: int, rdb: int, qlist: np.ndarray, n_refs: int, k: int, dtype: str):
        qlist = np.ascontiguousarray(qlist, dtype=np.int32)
        kk = max(0, min(int(k), n_refs))
        idx = np.empty((qlist.shape[0], kk), dtype=np.int32)
        sc = np.empty((qlist.shape[0], kk), dtype=np.int32)
        self._check(self.lib.gpusw_topk(self.handle, qdb, rdb, _ptr(qlist), qlist.shape[0], int(k),
                                        DTYPE_CODES[dtype], _ptr(idx), _ptr(sc)))
        return idx, sc

    def score_pairs(self, qdb: int, rdb: int, qi: np.ndarray, rj: np.ndarray, dtype: str) -> np.ndarray:
        qi = np.ascontiguousarray(qi, dtype=np.int32)
        rj = np.ascontiguousarray(rj, dtype=np.int32)
        out = np.empty(qi.shape[0], dtype=np.int32)
        self._check(self.lib.gpusw_score_pairs(self.handle, qdb, rdb, _ptr(qi), _ptr(rj),
                                               qi.shape[0], DTYPE_CODES[dtype], _ptr(out)))
        return out

    def score_pairs_zip(self, q_codes: np.ndarray, q_offsets: np.ndarray, r_codes: np.ndarray,
                        r_offsets: np.ndarray, dtype: str) -> np.ndarray:
        """Scores of query i vs reference i from host code bytes and offsets, pipelined
        (nothing stays resident)."""
        q_codes = np.ascontiguousarray(q_codes, dtype=np.uint8)
        r_codes = np.ascontiguousarray(r_codes, dtype=np.uint8)
        q_offsets = np.ascontiguousarray(q_offsets, dtype=np.int32)
        r_offsets = np.ascontiguousarray(r_offsets, dtype=np.int32)
        n = q_offsets.shape[0] - 1
        if r_offsets.shape[0] - 1 != n:
            raise ValueError("zipped pairs need as many references as queries")
        out = np.empty(n, dtype=np.int32)
        self._check(self.lib.gpusw_score_pairs_zip(self.handle, _ptr(q_codes), _ptr(q_offsets),
                                                   _ptr(r_codes), _ptr(r_offsets), n,
                                                   DTYPE_CODES[dtype], _ptr(out)))
        return out

    def locate_pairs(self, qdb: int, rdb: int, qi: np.ndarray, rj: np.ndarray, anchored: bool):
        """(score, reference row, query column) of the first best cell of every pair."""
        qi = np.ascontiguousarray(qi, dtype=np.int32)
        rj = np.ascontiguousarray(rj, dtype=np.int32)
        n = qi.shape[0]
        sc, ri, qj = (np.empty(n, dtype=np.int32) for _ in range(3))
        self._check(self.lib.gpusw_locate_pairs(self.handle, qdb, rdb, _ptr(qi), _ptr(rj), n,
                                                int(bool(anchored)), _ptr(sc), _ptr(ri), _ptr(qj)))
        return sc, ri, qj

    # ------------------------------------------------------------------- measurement
    def stats(self) -> Stats:
        s = Stats()
        self._check(self.lib.gpusw_get_stats(self.handle, ctypes.byref(s)))
        return s

    def sync(self) -> None:
        self._check(self.lib.gpusw_sync(self.handle))

    def dpx_rate(self) -> float:
        v = ctypes.c_double(0.0)
        self._check(self.lib.gpusw_measure_dpx_rate(self.handle, ctypes.byref(v)))
        return v.value

    def flush_l2(self, nbytes: int = 256 << 20) -> None:
        self._check(self.lib.gpusw_flush_l2(self.handle, int(nbytes)))


_contexts: dict[int, Context] = {}
_ctx_lock = threading.Lock()


def context(device: int = 0) -> Context:
    """The process-wide context of ``device`` (created on first use)."""
    with _ctx_lock:
        ctx = _contexts.get(int(device))
        if ctx is None:
            ctx = Context(device)
            _contexts[int(device)] = ctx
        return ctx
