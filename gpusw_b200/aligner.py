"""The reusable engine: encode and upload references once, then score many query sets
against them with ``score_cross`` / ``score_pairs`` / ``top_k``.

Same surface as ``src/gpusw/aligner.py:46-242`` of the reference package
(``Aligner(scheme, *, threads=128, device=0, backend="auto")``, ``index``,
``set_queries``, ``score_cross``, ``score_pairs``, ``top_k``, ``backend``, ``gcups``,
``query_ids``, ``reference_ids``, ``cuda_source``). Behind it the encoded sequences live on
the device as packed sets owned by the native engine, and every scoring call is one call
into the C ABI. ``threads`` is accepted for compatibility; kernel shapes are chosen by the
engine's length binning.
"""
from __future__ import annotations

import os

import numpy as np

from . import _native
from .db import PackedSet
from .encode import Encoded, funnel
from .errors import EncodeError, GpuSWError, NoGpuError, SchemeError
from .result import AlignResult
from .scheme import Scheme

__all__ = ["Aligner", "resolve_backend", "available_backends"]

_CSRC = os.path.join(os.path.dirname(os.path.abspath(__file__)), "csrc")


def resolve_backend(name: str | None) -> str:
    """``"auto"``/``"cuda"`` -> ``"cuda"``; ``"metal"`` -> NoGpuError; else ValueError.

    Mirrors ``src/gpusw/backends/__init__.py:90-121``; this engine has exactly one
    backend (hand-written CUDA for sm_100a), so there is no dispatch.
    """
    n = (name or "auto").lower()
    if n == "metal":
        raise NoGpuError("the Metal backend is not part of this engine; use backend='cuda'")
    if n not in ("auto", "cuda"):
        raise ValueError(f"unknown backend {name!r}; choose 'auto', 'cuda', or 'metal'")
    if not _native.gpu_available():
        raise NoGpuError("no usable CUDA device (or the native engine is not built)")
    return "cuda"


def available_backends() -> list[str]:
    return ["cuda"] if _native.gpu_available() else []


def _as_scheme(scheme) -> Scheme:
    if isinstance(scheme, Scheme):
        return scheme
    if isinstance(scheme, str):
        return Scheme.preset(scheme)
    raise TypeError(f"scheme must be a Scheme or preset name, got {type(scheme).__name__}")


def _reversed_prefixes(enc: Encoded, idx: np.ndarray, plen: np.ndarray):
    """Codes and offsets of ``enc[idx[k]][:plen[k]]`` reversed, for every k."""
    plen = plen.astype(np.int64)
    offs = np.zeros(idx.shape[0] + 1, dtype=np.int64)
    np.cumsum(plen, out=offs[1:])
    last = np.asarray(enc.offsets, dtype=np.int64)[idx] + plen - 1
    t = np.arange(offs[-1], dtype=np.int64) - np.repeat(offs[:-1], plen)
    codes = np.asarray(enc.codes)[np.repeat(last, plen) - t]
    return np.ascontiguousarray(codes, dtype=np.uint8), offs.astype(np.int32)


class _DeviceSet:
    """A sequence set resident on the device; freed with the owning Aligner."""

    def __init__(self, ctx: _native.Context, enc):
        self.ctx = ctx
        self.enc = enc
        if isinstance(enc, PackedSet):  # a stored packed image: uploaded without re-packing
            self.handle = ctx.upload_image(enc.image, enc.n, enc.bits, enc.nwords)
        else:
            self.handle = ctx.upload(enc.codes, enc.offsets)

    def __del__(self):  # pragma: no cover - depends on GC timing
        try:
            self.ctx.free(self.handle)
        except Exception:
            pass


class Aligner:
    """Reusable GPU Smith-Waterman / Needleman-Wunsch / semiglobal scorer for one scheme."""

    def __init__(self, scheme="dna", *, threads: int = 128, device: int = 0,
                 backend: str = "auto"):
        self.scheme = _as_scheme(scheme)
        self.threads = int(threads)
        self.device = int(device)
        self._backend_name = backend
        self._backend = None
        self._refs: Encoded | None = None
        self._queries: Encoded | None = None
        self._dref: _DeviceSet | None = None
        self._dq: _DeviceSet | None = None
        self._last_gcups = 0.0
        self._last_kernel = ""

    @property
    def _b(self) -> str:
        if self._backend is None:
            self._backend = resolve_backend(self._backend_name)
        return self._backend

    def _ctx(self) -> _native.Context:
        self._b  # noqa: B018 - resolves (and validates) the backend first
        return _native.context(self.device)

    # ------------------------------------------------------------------------ inputs
    def index(self, refs) -> Aligner:
        """Encode and upload the reference set once; returns ``self``. A
        :class:`~gpusw_b200.db.PackedSet` (``load_db``) is uploaded as stored."""
        ctx = self._ctx()
        if isinstance(refs, PackedSet):
            if refs.alphabet != self.scheme.eff_alphabet:
                raise EncodeError(f"set alphabet {refs.alphabet!r} != scheme alphabet "
                                  f"{self.scheme.eff_alphabet!r}")
            self._refs = refs
            self._dref = _DeviceSet(ctx, refs)
            return self
        enc = funnel(refs, self.scheme, id_prefix="r")
        self._refs = enc
        self._dref = _DeviceSet(ctx, enc)
        return self

    def set_queries(self, queries) -> Aligner:
        """Encode and upload a query set; returns ``self``."""
        ctx = self._ctx()
        enc = funnel(queries, self.scheme, id_prefix="q")
        self._queries = enc
        self._dq = _DeviceSet(ctx, enc)
        return self

    # --------------------------------------------------------------------- internals
    def _resolved_dtype(self) -> str:
        maxq = self._queries.max_len if self._queries else 0
        maxr = self._refs.max_len if self._refs else 0
        return self.scheme.resolve_dtype(max(maxq, 1), max(maxr, 1))

    def _policy(self) -> str:
        """Native width policy: the static check only matters for a forced int16."""
        if self.scheme.dtype == "int32":
            return "int32"
        if self.scheme.dtype == "int16":
            self._resolved_dtype()  # raises OverflowRiskError when int16 is unsafe
            return "int16"
        return "auto"

    def _record(self, ctx: _native.Context, kernel: str) -> None:
        if self.scheme.mode == "local":
            ctx.save_tune(self.scheme.ns)
        st = ctx.stats()
        self._last_gcups = st.last_cells / (st.last_kernel_ms * 1e6) if st.last_kernel_ms > 0 else 0.0
        self._last_kernel = kernel

    # ----------------------------------------------------------------------- scoring
    def score_cross(self, queries=None, *, return_ids: bool = False,
                    query_batch: int | None = None):
        """All-pairs scores ``(n_queries, n_refs)`` int32 (``AlignResult`` if return_ids)."""
        if self._refs is None:
            raise ValueError("call index(refs) before score_cross()")
        if queries is not None:
            self.set_queries(queries)
        if self._queries is None:
            raise ValueError("no queries: pass queries= or call set_queries()")
        ctx = self._ctx()
        nq, nr = self._queries.n, self._refs.n
        policy = self._policy()
        out = np.empty((nq, nr), dtype=np.int32)
        step = max(1, min(query_batch or nq, nq)) if nq else 1
        with ctx.lock:
            ctx.set_scheme(self.scheme)
            for b0 in range(0, nq, step):
                ql = np.arange(b0, min(b0 + step, nq), dtype=np.int32)
                out[b0:b0 + len(ql)] = ctx.score_cross(self._dq.handle, self._dref.handle, ql, nr,
                                                       policy)
            self._record(ctx, "sw_cross")
        if return_ids:
            return AlignResult(out, self._queries.ids, self._refs.ids, self.scheme)
        return out

    def score_pairs(self, qi, rj, *, return_ids: bool = False):
        """Scores of the explicit pairs ``(qi[k], rj[k])`` -> ``(n_pairs,)`` int32."""
        if self._refs is None or self._queries is None:
            raise ValueError("call index(refs) and set_queries(queries) first")
        qi = np.ascontiguousarray(qi, dtype=np.int32)
        rj = np.ascontiguousarray(rj, dtype=np.int32)
        if qi.shape != rj.shape:
            raise ValueError("qi and rj must have the same length")
        ctx = self._ctx()
        policy = self._policy()
        with ctx.lock:
            ctx.set_scheme(self.scheme)
            host = ctx.score_pairs(self._dq.handle, self._dref.handle, qi, rj, policy)
            self._record(ctx, "sw_pairs")
        if return_ids:
            return AlignResult(host, [self._queries.ids[i] for i in qi],
                               [self._refs.ids[j] for j in rj], self.scheme)
        return host

    def score_zipped(self, queries, refs, *, return_ids: bool = False):
        """Scores of query ``i`` against reference ``i`` -- ``align_pairs`` with
        ``pairs=None`` (``src/gpusw/__init__.py:145-189``). Both sets are encoded, then
        packed, uploaded and scored in one pipelined engine call (chunks packed on the host
        while the GPU scores the previous ones); nothing stays resident, and the aligner's
        own indexed sets are left as they were. ``(n,)`` int32, or an ``AlignResult``."""
        r = funnel(refs, self.scheme, id_prefix="r")
        q = funnel(queries, self.scheme, id_prefix="q")
        if q.n != r.n:
            raise ValueError(
                f"pairs=None requires len(queries)==len(refs) for 1:1 scoring (got {q.n} vs "
                f"{r.n}); pass pairs=[(qi, rj), ...]")
        if self.scheme.dtype == "int16":
            self.scheme.resolve_dtype(max(q.max_len, 1), max(r.max_len, 1))  # may raise
        policy = self.scheme.dtype if self.scheme.dtype in ("int16", "int32") else "auto"
        ctx = self._ctx()
        with ctx.lock:
            ctx.set_scheme(self.scheme)
            host = ctx.score_pairs_zip(q.codes, q.offsets, r.codes, r.offsets, policy)
            self._record(ctx, "sw_pairs")
        if return_ids:
            return AlignResult(host, list(q.ids), list(r.ids), self.scheme)
        return host

    def top_k(self, queries=None, k: int = 5, *, query_batch: int = 512) -> AlignResult:
        """Per-query top-``k`` references (score descending, ties to the lower index).

        Only ``(n_queries, k)`` indices and scores come back to the host; the engine
        scores query blocks sized by its device-memory budget (``query_batch`` is kept
        for signature compatibility).
        """
        if self._refs is None:
            raise ValueError("call index(refs) before top_k()")
        if queries is not None:
            self.set_queries(queries)
        if self._queries is None:
            raise ValueError("no queries: pass queries= or call set_queries()")
        ctx = self._ctx()
        nq, nr = self._queries.n, self._refs.n
        policy = self._policy()
        with ctx.lock:
            ctx.set_scheme(self.scheme)
            idx, sc = ctx.topk(self._dq.handle, self._dref.handle, np.arange(nq, dtype=np.int32),
                               nr, k, policy)
            self._record(ctx, "sw_cross")
        return AlignResult(None, self._queries.ids, self._refs.ids, self.scheme,
                           topk_idx=idx, topk_scores=sc)

    def locate(self, qi, rj) -> dict:
        """Coordinates of the best local alignment of the pairs ``(qi[k], rj[k])``.

        Returns int32 arrays ``score``, ``query_start``, ``query_end``, ``ref_start``,
        ``ref_end`` (0-based, end exclusive, ``-1`` where the score is 0). The end is the
        first cell, in row-major order (reference row, then query column), that holds the
        local maximum; the start comes from a second device pass, anchored at that end, over
        the reversed prefixes -- its first best cell is the shortest optimal alignment. Both
        passes are int32 dynamic programming on the device; no traceback matrix is kept.
        The reference is score-only (its examples re-align hits on the CPU for
        coordinates, ``examples/legacy_16s_gpu_align.py:280-292``); this is the device
        counterpart, for local schemes.
        """
        if self.scheme.mode != "local":
            raise SchemeError("locate() needs a local-mode scheme")
        if self._refs is None or self._queries is None:
            raise ValueError("call index(refs) and set_queries(queries) first")
        qi = np.ascontiguousarray(qi, dtype=np.int32)
        rj = np.ascontiguousarray(rj, dtype=np.int32)
        if qi.shape != rj.shape or qi.ndim != 1:
            raise ValueError("qi and rj must be 1-D and of the same length")
        n = qi.shape[0]
        res = {k: np.full(n, -1, dtype=np.int32)
               for k in ("query_start", "query_end", "ref_start", "ref_end")}
        ctx = self._ctx()
        with ctx.lock:
            ctx.set_scheme(self.scheme)
            sc, rend, qend = ctx.locate_pairs(self._dq.handle, self._dref.handle, qi, rj, False)
            res["score"] = sc
            hit = np.flatnonzero(sc > 0)
            if hit.size:
                qrev = _reversed_prefixes(self._queries, qi[hit], qend[hit] + 1)
                rrev = _reversed_prefixes(self._refs, rj[hit], rend[hit] + 1)
                hq, hr = ctx.upload(*qrev), ctx.upload(*rrev)
                try:
                    ident = np.arange(hit.size, dtype=np.int32)
                    sb, di, dj = ctx.locate_pairs(hq, hr, ident, ident, True)
                finally:
                    ctx.free(hq)
                    ctx.free(hr)
                if not np.array_equal(sb, sc[hit]):
                    raise GpuSWError("anchored pass disagrees with the local score")
                res["ref_start"][hit] = rend[hit] - di
                res["query_start"][hit] = qend[hit] - dj
                res["ref_end"][hit] = rend[hit] + 1
                res["query_end"][hit] = qend[hit] + 1
            self._record(ctx, "sw_locate")
        return res

    def locate_top(self, result: AlignResult) -> dict:
        """Coordinates of every hit of ``result``, a ``top_k`` result for this aligner's
        current queries: the arrays of :meth:`locate`, shaped like ``result.topk_idx``."""
        idx = np.asarray(result.topk_idx)
        if idx.ndim != 2 or self._queries is None or idx.shape[0] != self._queries.n:
            raise ValueError("locate_top() takes a top_k result of this aligner's current queries")
        nq, k = idx.shape
        qi = np.repeat(np.arange(nq, dtype=np.int32), k)
        loc = self.locate(qi, idx.reshape(-1).astype(np.int32))
        return {key: v.reshape(nq, k) for key, v in loc.items()}

    # ----------------------------------------------------------------- introspection
    @property
    def backend(self) -> str:
        return self._b

    @property
    def query_ids(self) -> list:
        return list(self._queries.ids) if self._queries else []

    @property
    def reference_ids(self) -> list:
        return list(self._refs.ids) if self._refs else []

    @property
    def gcups(self) -> float:
        """Giga cell updates per second of the most recent scoring call (kernel time)."""
        return self._last_gcups

    def cuda_source(self) -> str:
        """The hand-written CUDA source of the engine's kernels, headed by this scheme's
        kernel configuration (the reference returned its NVRTC-rendered source)."""
        mf = self.scheme.module_fields()
        mode = {"local": 0, "global": 1, "semiglobal": 2}[mf["mode"]]
        head = [
            "// gpusw_b200 kernel configuration for this scheme",
            f"#define MODE ({mode})           /* 0=local 1=global 2=semiglobal */",
            f"#define NS ({mf['ns']})",
            f"#define GOPEN ({mf['gap_open']})",
            f"#define GEXT ({mf['gap_extend']})",
            f"#define FREE_Q ({int(mf['free_q'])})",
            f"#define FREE_R ({int(mf['free_r'])})",
            "// entry points: sw_cross -> gsw::cross_stream_kernel (local) or gsw::pairs_kernel"
            " in cross mode; sw_pairs -> gsw::pairs_kernel",
            "",
        ]
        body = []
        for name in ("dp_core.cuh", "kernels.cuh"):
            with open(os.path.join(_CSRC, name)) as fh:
                body.append(fh.read())
        return "\n".join(head) + "\n".join(body)

    def kernel_source(self) -> str:
        return self.cuda_source()

    def metal_source(self) -> str:
        raise NoGpuError("the Metal backend is not part of this engine")
