""":class:`AlignResult`: scores with their query/reference ids.

Same fields and methods as ``src/gpusw/result.py:14-85`` of the reference package. In
``top_k`` a dense matrix is ranked by a stable sort of the negated scores, so ties go to
the lower reference index; stored ``topk_idx``/``topk_scores`` produced on the GPU follow
the same (score descending, reference index ascending) order.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

__all__ = ["AlignResult"]


@dataclass
class AlignResult:
    """``scores`` is ``(n_queries, n_refs)`` for a cross product, ``(n_pairs,)`` for pairs,
    or ``None`` when only the per-query ``topk_idx``/``topk_scores`` were kept."""

    scores: np.ndarray | None
    query_ids: list
    reference_ids: list
    scheme: object
    topk_idx: np.ndarray | None = None
    topk_scores: np.ndarray | None = None

    def top_k(self, k: int = 5) -> list[tuple[str, list[tuple[str, int]]]]:
        """Per query, the ``k`` best ``(reference_id, score)``, best first."""
        if self.topk_idx is not None:
            idx, sc = self.topk_idx[:, :k], self.topk_scores[:, :k]
        else:
            if self.scores is None or self.scores.ndim != 2:
                raise ValueError("top_k needs a 2-D cross-product result")
            idx = np.argsort(-self.scores, axis=1, kind="stable")[:, :k]
            sc = np.take_along_axis(self.scores, idx, axis=1)
        return [
            (qid, [(self.reference_ids[int(idx[qi, r])], int(sc[qi, r]))
                   for r in range(idx.shape[1])])
            for qi, qid in enumerate(self.query_ids)
        ]

    def best(self) -> list[tuple[str, str, int]]:
        """The best ``(query_id, reference_id, score)`` of every query."""
        return [(q, hits[0][0], hits[0][1]) for q, hits in self.top_k(1)]

    def to_dataframe(self):
        """Long-format ``pandas.DataFrame`` of the scores or of the stored top-k."""
        import pandas as pd

        if self.topk_idx is not None:
            rows = [(qid, self.reference_ids[int(self.topk_idx[qi, r])], r + 1,
                     int(self.topk_scores[qi, r]))
                    for qi, qid in enumerate(self.query_ids)
                    for r in range(self.topk_idx.shape[1])]
            return pd.DataFrame(rows, columns=["query", "reference", "rank", "score"])
        s = self.scores
        if s is None:
            raise ValueError("no scores to tabulate")
        if s.ndim == 1:
            rows = [(self.query_ids[i] if i < len(self.query_ids) else f"q{i}",
                     self.reference_ids[i] if i < len(self.reference_ids) else f"r{i}",
                     int(v)) for i, v in enumerate(s)]
        else:
            rows = [(qid, rid, int(s[qi, rj])) for qi, qid in enumerate(self.query_ids)
                    for rj, rid in enumerate(self.reference_ids)]
        return pd.DataFrame(rows, columns=["query", "reference", "score"])

    def __repr__(self) -> str:  # pragma: no cover - cosmetic
        shape = None if self.scores is None else self.scores.shape
        return (f"AlignResult(n_queries={len(self.query_ids)}, "
                f"n_refs={len(self.reference_ids)}, scores_shape={shape})")
