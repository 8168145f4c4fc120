"""gpusw_b200 -- Gotoh alignment *scoring* on NVIDIA B200 (sm_100a).

A from-scratch engine for the scoring path of the ``gpusw`` package (freiburgermsu/gpuSW):
affine-gap Smith-Waterman (local), Needleman-Wunsch (global) and semiglobal scores of
query/reference pairs. The public names and signatures follow the reference's
``src/gpusw/__init__.py:43-189`` so that ``align_score``, ``align_pairs``, ``Aligner``,
``Scheme``, ``Matrix`` and ``AlignResult`` are drop-in replacements; every score equals
the reference's NumPy oracle to the integer.

Host code is Python; the scoring runs in hand-written CUDA kernels for sm_100a behind a
C ABI (``include/gpusw_b200.h``), loaded with ctypes. There is no CPU fallback: without
the built library or a GPU the scoring calls raise :class:`NoGpuError`.
"""
from __future__ import annotations

import numpy as np

from . import schemes
from ._native import gpu_available
from ._version import __version__
from .aligner import Aligner, available_backends
from .errors import EncodeError, GpuSWError, NoGpuError, OverflowRiskError, SchemeError
from .matrix import Matrix
from .matrix import available as available_matrices
from .result import AlignResult
from .scheme import Scheme

__all__ = [
    "align_score",
    "align_pairs",
    "Aligner",
    "Scheme",
    "Matrix",
    "AlignResult",
    "schemes",
    "available_matrices",
    "gpu_available",
    "metal_available",
    "available_backends",
    "GpuSWError",
    "NoGpuError",
    "SchemeError",
    "OverflowRiskError",
    "EncodeError",
    "__version__",
]


def metal_available() -> bool:
    """Always False: this engine has no Metal backend."""
    return False


def _build_scheme(scheme, *, mode=None, match=None, mismatch=None, gap_open=None,
                  gap_extend=None, matrix=None, alphabet=None, unknown=None,
                  case_insensitive=None, dtype=None, free_end_gaps_query=None,
                  free_end_gaps_ref=None) -> Scheme:
    """A preset (or Scheme) with every non-None override applied
    (``src/gpusw/__init__.py:66-104``)."""
    base = scheme if isinstance(scheme, Scheme) else Scheme.preset(scheme)
    if isinstance(matrix, str):
        matrix = Matrix.named(matrix)
    overrides = {
        k: v for k, v in dict(
            mode=mode, match=match, mismatch=mismatch, gap_open=gap_open,
            gap_extend=gap_extend, matrix=matrix, alphabet=alphabet, unknown=unknown,
            case_insensitive=case_insensitive, dtype=dtype,
            free_end_gaps_query=free_end_gaps_query, free_end_gaps_ref=free_end_gaps_ref,
        ).items() if v is not None
    }
    return base.replace(**overrides) if overrides else base


def align_score(queries, refs, *, scheme="dna", mode=None, match=None, mismatch=None,
                gap_open=None, gap_extend=None, matrix=None, alphabet=None, unknown=None,
                dtype=None, threads=128, backend="auto", return_ids=True, query_batch=None):
    """Scores of every query against every reference (``src/gpusw/__init__.py:107-142``).

    Returns an :class:`AlignResult` whose ``scores`` is ``(n_queries, n_refs)`` int32, or
    the bare array when ``return_ids=False``.
    """
    sch = _build_scheme(scheme, mode=mode, match=match, mismatch=mismatch, gap_open=gap_open,
                        gap_extend=gap_extend, matrix=matrix, alphabet=alphabet,
                        unknown=unknown, dtype=dtype)
    al = Aligner(sch, threads=threads, backend=backend).index(refs).set_queries(queries)
    return al.score_cross(return_ids=return_ids, query_batch=query_batch)


def align_pairs(queries, refs, *, pairs=None, scheme="dna", mode=None, match=None,
                mismatch=None, gap_open=None, gap_extend=None, matrix=None, alphabet=None,
                unknown=None, dtype=None, threads=128, backend="auto", return_ids=True):
    """Scores of specific query/reference pairs (``src/gpusw/__init__.py:145-189``).

    ``pairs=None`` zips the two sets 1:1 (they must have the same length); otherwise
    ``pairs`` lists ``(query_index, reference_index)`` tuples.
    """
    sch = _build_scheme(scheme, mode=mode, match=match, mismatch=mismatch, gap_open=gap_open,
                        gap_extend=gap_extend, matrix=matrix, alphabet=alphabet,
                        unknown=unknown, dtype=dtype)
    al = Aligner(sch, threads=threads, backend=backend)
    if pairs is None:  # 1:1 -- one pipelined upload + score call, nothing kept resident
        return al.score_zipped(queries, refs, return_ids=return_ids)
    al.index(refs).set_queries(queries)
    arr = np.asarray(pairs, dtype=np.int64).reshape(-1, 2) if len(pairs) else \
        np.zeros((0, 2), dtype=np.int64)
    qi = arr[:, 0].astype(np.int32)
    rj = arr[:, 1].astype(np.int32)
    return al.score_pairs(qi, rj, return_ids=return_ids)
