"""Continuous-batching top-k server over a resident reference set.

The reference package has no serving layer; this is the serving pattern of its top-k path
(``Aligner.index(db).top_k(queries, k)``, ``src/gpusw/aligner.py:169-195``) for many
concurrent requests. The scheduler runs natively (``gpusw_server_*`` in the C ABI): it
admits queued requests in arrival order while an execution slot and the device-memory
budget allow, merges them into one batch, overlaps batches of different slots on the GPU,
and records each request's submit-to-done latency. Every request's top-k is identical to
``Aligner.top_k`` on its queries alone.

    srv = Server(aligner, k=10)            # aligner.index(refs) done before
    rid = srv.submit(queries)              # any funnel input form
    idx, scores = srv.result(rid, timeout=60)
    srv.stats()                            # p50/p99 latency, GCUPS, batches, ...
"""
from __future__ import annotations

import ctypes
import time

import numpy as np

from . import _native
from .encode import funnel
from .errors import GpuSWError

__all__ = ["Server", "PENDING", "RUNNING", "DONE", "CANCELLED", "FAILED"]

PENDING, RUNNING, DONE, CANCELLED, FAILED = 0, 1, 2, 3, 4


class Server:
    """Top-k server over the references indexed by ``aligner``.

    The aligner's context is reserved for the server while it runs (the server uses its
    own execution slots on the same device).
    """

    def __init__(self, aligner, k: int = 10, *, mem_budget: int = 0, slots: int = 2,
                 max_batch_queries: int = 1024, max_pending: int = 4096,
                 batch_cells: float = 0.0):
        if aligner._refs is None:
            raise ValueError("call index(refs) on the aligner first")
        self.aligner = aligner
        self.scheme = aligner.scheme
        self.ctx = aligner._ctx()
        self.lib = self.ctx.lib
        self.n_refs = aligner._refs.n
        self.kk = max(0, min(int(k), self.n_refs))
        self._nq: dict[int, int] = {}
        with self.ctx.lock:
            self.ctx.set_scheme(self.scheme)
            h = ctypes.c_void_p()
            self.ctx._check(self.lib.gpusw_server_create(
                self.ctx.handle, aligner._dref.handle, int(k), _native.DTYPE_CODES[aligner._policy()],
                int(mem_budget), int(slots), int(max_batch_queries), int(max_pending),
                ctypes.byref(h)))
        self.handle = h
        if batch_cells:  # work per batch in cells (0: the engine default)
            self._check(self.lib.gpusw_server_set_batch_cells(self.handle, float(batch_cells)))

    def _check(self, rc: int):
        if rc != _native.OK:
            _native._raise(rc, self.lib.gpusw_server_last_error(self.handle).decode())

    def submit(self, queries) -> int:
        """Queue a request (any input form the funnel accepts); returns its id."""
        enc = funnel(queries, self.scheme)
        codes = np.ascontiguousarray(enc.codes, dtype=np.uint8)
        offs = np.ascontiguousarray(enc.offsets, dtype=np.int32)
        rid = ctypes.c_int64(0)
        self._check(self.lib.gpusw_server_submit(self.handle, _native._ptr(codes), _native._ptr(offs),
                                                 enc.n, ctypes.byref(rid)))
        self._nq[rid.value] = enc.n
        return rid.value

    def poll(self, rid: int, timeout: float = 0.0):
        """``(state, idx, scores)``; idx/scores are ``(nq, k)`` int32 once the state is DONE
        (the request is then released), else None."""
        nq = self._nq.get(rid, 0)
        idx = np.empty((nq, self.kk), dtype=np.int32)
        sc = np.empty((nq, self.kk), dtype=np.int32)
        state = ctypes.c_int32(-1)
        rc = self.lib.gpusw_server_poll(self.handle, int(rid), int(timeout * 1000),
                                        ctypes.byref(state), _native._ptr(idx), _native._ptr(sc))
        if rc == _native.E_TIMEOUT:
            return state.value, None, None
        self._check(rc)
        if state.value in (DONE, CANCELLED):
            self._nq.pop(rid, None)
        if state.value == DONE:
            return DONE, idx, sc
        return state.value, None, None

    def result(self, rid: int, timeout: float = 600.0):
        """Block (at most ``timeout`` seconds) until the request is done; ``(idx, scores)``."""
        deadline = time.monotonic() + timeout
        while True:
            left = deadline - time.monotonic()
            if left <= 0:
                raise TimeoutError(f"request {rid} not done after {timeout} s")
            state, idx, sc = self.poll(rid, timeout=min(left, 1.0))
            if state == DONE:
                return idx, sc
            if state == CANCELLED:
                raise GpuSWError(f"request {rid} was cancelled")

    def cancel(self, rid: int) -> None:
        self._check(self.lib.gpusw_server_cancel(self.handle, int(rid)))

    def stats(self) -> dict:
        st = _native.ServerStats()
        self._check(self.lib.gpusw_server_get_stats(self.handle, ctypes.byref(st)))
        return {name: getattr(st, name) for name, _ in st._fields_}

    def close(self) -> None:
        if getattr(self, "handle", None):
            self.lib.gpusw_server_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):  # pragma: no cover - GC order
        try:
            self.close()
        except Exception:
            pass
