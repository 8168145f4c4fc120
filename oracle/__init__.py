"""CPU oracle for the Gotoh scoring path -- TEST INFRASTRUCTURE, never the product.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``
import this package, and only to check or time against it. It holds:

* ``score_codes_py``: a pure-Python restatement of the reference package's
  ``_score_codes`` (``src/gpusw/reference.py:38-125``), for small cases;
* ``score_pairs`` / ``score_cross``: the same recurrence in plain C
  (``oracle/gotoh_oracle.c``), threaded over pairs, for large parity checks;
* ``locate_pairs``: best-cell coordinates (end of the best local alignment, then its start
  from an anchored pass over the reversed prefixes), the CPU restatement of the engine's
  ``Aligner.locate`` (the reference is score-only);
* ``topk_stable``: the reference's top-k order -- a stable sort of the negated scores,
  so ties go to the lower reference index (``src/gpusw/result.py:30-47``).

The C restatement is pinned against the Python one and both against golden vectors
produced by the reference's own oracle (``tests/golden/``).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
SRC_PATH = os.path.join(HERE, "gotoh_oracle.c")
NEG = -(1 << 30)
MODE_CODES = {"local": 0, "global": 1, "semiglobal": 2}

_lib = None


def build(force: bool = False) -> str:
    """Compile ``gotoh_oracle.c`` into ``liboracle.so`` next to it (gcc -O3, pthreads; no
    host-specific instruction set, so the library built here runs on any x86-64 host)."""
    if force or not os.path.exists(LIB_PATH) or (
            os.path.getmtime(LIB_PATH) < os.path.getmtime(SRC_PATH)):
        subprocess.check_call(["gcc", "-O3", "-shared", "-fPIC", "-o", LIB_PATH, SRC_PATH,
                               "-lpthread"])
    return LIB_PATH


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        lib = ctypes.CDLL(LIB_PATH)
        p = ctypes.c_void_p
        i32, i64 = ctypes.c_int, ctypes.c_int64
        lib.oracle_score_pairs.argtypes = [p, p, p, p, p, p, i64, p, i32, i32, i32, i32, i32,
                                           i32, i32, p]
        lib.oracle_score_pairs.restype = i32
        lib.oracle_score_cross.argtypes = [p, p, p, i64, p, p, i64, p, i32, i32, i32, i32, i32,
                                           i32, i32, p]
        lib.oracle_score_cross.restype = i32
        lib.oracle_locate.argtypes = [p, i64, p, i64, p, i32, i32, i32, i32, p]
        lib.oracle_locate.restype = i32
        _lib = lib
    return _lib


def _scheme_args(scheme):
    sub = np.ascontiguousarray(scheme.substitution_table(), dtype=np.int32)
    return (sub, int(scheme.ns), MODE_CODES[scheme.mode], int(scheme.gap_open),
            int(scheme.gap_extend), int(bool(scheme.free_end_gaps_query)),
            int(bool(scheme.free_end_gaps_ref)))


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def score_pairs(q_enc, r_enc, qi, rj, scheme, threads: int | None = None) -> np.ndarray:
    """int64 scores of the pairs ``(qi[k], rj[k])`` from two ``Encoded`` sets (C oracle)."""
    lib = _load()
    qi = np.ascontiguousarray(qi, dtype=np.int32)
    rj = np.ascontiguousarray(rj, dtype=np.int32)
    out = np.empty(qi.shape[0], dtype=np.int64)
    sub, ns, mode, go, ge, fq, fr = _scheme_args(scheme)
    qc = np.ascontiguousarray(q_enc.codes, dtype=np.uint8)
    rc = np.ascontiguousarray(r_enc.codes, dtype=np.uint8)
    qo = np.ascontiguousarray(q_enc.offsets, dtype=np.int32)
    ro = np.ascontiguousarray(r_enc.offsets, dtype=np.int32)
    rc_ = lib.oracle_score_pairs(_ptr(qc), _ptr(qo), _ptr(rc), _ptr(ro), _ptr(qi), _ptr(rj),
                                 qi.shape[0], _ptr(sub), ns, mode, go, ge, fq, fr,
                                 threads or os.cpu_count() or 1, _ptr(out))
    if rc_ != 0:
        raise MemoryError("oracle ran out of memory")
    return out


def score_cross(q_enc, r_enc, scheme, qlist=None, threads: int | None = None) -> np.ndarray:
    """int64 ``(len(qlist), n_refs)`` scores of queries ``qlist`` against every reference."""
    lib = _load()
    if qlist is None:
        qlist = np.arange(q_enc.n, dtype=np.int32)
    qlist = np.ascontiguousarray(qlist, dtype=np.int32)
    nq, nr = qlist.shape[0], r_enc.n
    out = np.empty((nq, nr), dtype=np.int64)
    sub, ns, mode, go, ge, fq, fr = _scheme_args(scheme)
    qc = np.ascontiguousarray(q_enc.codes, dtype=np.uint8)
    rc = np.ascontiguousarray(r_enc.codes, dtype=np.uint8)
    qo = np.ascontiguousarray(q_enc.offsets, dtype=np.int32)
    ro = np.ascontiguousarray(r_enc.offsets, dtype=np.int32)
    rc_ = lib.oracle_score_cross(_ptr(qc), _ptr(qo), _ptr(qlist), nq, _ptr(rc), _ptr(ro), nr,
                                 _ptr(sub), ns, mode, go, ge, fq, fr,
                                 threads or os.cpu_count() or 1, _ptr(out))
    if rc_ != 0:
        raise MemoryError("oracle ran out of memory")
    return out


def locate_cells(qc, rc, scheme, anchored: bool) -> tuple[int, int, int]:
    """(max H, reference row, query column) of the first best cell (C oracle, one pair)."""
    lib = _load()
    qc = np.ascontiguousarray(qc, dtype=np.uint8)
    rc = np.ascontiguousarray(rc, dtype=np.uint8)
    sub = np.ascontiguousarray(scheme.substitution_table(), dtype=np.int32)
    out = np.zeros(3, dtype=np.int64)
    if lib.oracle_locate(_ptr(qc), qc.shape[0], _ptr(rc), rc.shape[0], _ptr(sub),
                         int(scheme.ns), int(scheme.gap_open), int(scheme.gap_extend),
                         int(bool(anchored)), _ptr(out)) != 0:
        raise MemoryError("oracle ran out of memory")
    return int(out[0]), int(out[1]), int(out[2])


def locate_pairs(q_enc, r_enc, qi, rj, scheme) -> dict:
    """Coordinates of the best local alignment of every pair, half-open, -1 when score 0.

    End: the first cell (row-major: reference row, then query column) holding the local
    maximum. Start: the anchored pass over the reversed prefixes ending at that cell; its
    first best cell, mapped back, is the start (the shortest such alignment).
    """
    qi = np.asarray(qi, dtype=np.int64)
    rj = np.asarray(rj, dtype=np.int64)
    n = qi.shape[0]
    res = {k: np.full(n, -1, dtype=np.int64)
           for k in ("query_start", "query_end", "ref_start", "ref_end")}
    res["score"] = np.zeros(n, dtype=np.int64)
    for k in range(n):
        a, b = int(qi[k]), int(rj[k])
        qc = q_enc.codes[q_enc.offsets[a]:q_enc.offsets[a + 1]]
        rc = r_enc.codes[r_enc.offsets[b]:r_enc.offsets[b + 1]]
        best, ie, je = locate_cells(qc, rc, scheme, anchored=False)
        res["score"][k] = best
        if best <= 0:
            continue
        rb, di, dj = locate_cells(qc[:je + 1][::-1], rc[:ie + 1][::-1], scheme, anchored=True)
        assert rb == best
        res["ref_start"][k], res["query_start"][k] = ie - di, je - dj
        res["ref_end"][k], res["query_end"][k] = ie + 1, je + 1
    return res


def score_codes_py(qc, rc, sub, mode: str, go: int, ge: int, free_q: bool, free_r: bool) -> int:
    """Pure-Python restatement of ``src/gpusw/reference.py:38-125`` (small inputs only)."""
    n, m = len(qc), len(rc)
    local, glob, semi = mode == "local", mode == "global", mode == "semiglobal"
    if n == 0 or m == 0:
        if local or (n == 0 and m == 0):
            return 0
        if n == 0:
            return 0 if (semi and free_q) else go + (m - 1) * ge
        return 0 if (semi and free_r) else go + (n - 1) * ge

    def edge(k: int, free: bool) -> int:
        if local:
            return 0
        if glob:
            return go + (k - 1) * ge
        return 0 if free else go + (k - 1) * ge

    hp = [0] + [edge(j, free_r) for j in range(1, n + 1)]
    f = [NEG] * (n + 1)
    best, corner, endcol, endrow = 0, NEG, NEG, NEG
    for i in range(1, m + 1):
        row = sub[int(rc[i - 1])]
        hleft = edge(i, free_q)
        diag, hp[0], eleft = hp[0], hleft, NEG
        for j in range(1, n + 1):
            fj = max(hp[j] + go, f[j] + ge)
            ej = max(hleft + go, eleft + ge)
            h = max(diag + int(row[int(qc[j - 1])]), ej, fj)
            if local and h < 0:
                h = 0
            best = max(best, h)
            if not local:
                if i == m and j == n:
                    corner = h
                if free_q and j == n:
                    endcol = max(endcol, h)
                if free_r and i == m:
                    endrow = max(endrow, h)
            diag, hp[j], f[j], hleft, eleft = hp[j], h, fj, h, ej
    if local:
        return best
    if glob:
        return corner
    res = corner
    if free_q:
        res = max(res, endcol)
    if free_r:
        res = max(res, endrow)
    if free_q and free_r:
        res = max(res, 0)
    return res


def score_py(query: str, ref: str, scheme) -> int:
    """Oracle score of two strings (encode with the scheme's LUT, then ``score_codes_py``)."""
    from gpusw_b200.encode import funnel

    q = funnel([query], scheme)
    r = funnel([ref], scheme)
    return score_codes_py(q.codes, r.codes, scheme.substitution_table().astype(np.int64),
                          scheme.mode, scheme.gap_open, scheme.gap_extend,
                          scheme.free_end_gaps_query, scheme.free_end_gaps_ref)


def topk_stable(scores: np.ndarray, k: int) -> tuple[np.ndarray, np.ndarray]:
    """Per-row top-k in the reference's order: score descending, then index ascending."""
    kk = min(k, scores.shape[1])
    order = np.argsort(-scores.astype(np.int64), axis=1, kind="stable")[:, :kk]
    return order.astype(np.int32), np.take_along_axis(scores, order, axis=1).astype(np.int32)
