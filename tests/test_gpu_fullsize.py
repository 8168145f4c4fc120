"""Parity at the benchmark configurations' full sizes, through properties that do not need
the oracle to score everything: top-k order (score descending, index ascending), whole top-k
rows recomputed by the C oracle for a few seeded queries, top-1 hits rescored through the
independent pairs path, and, for the million read/window pairs, a seeded subsample against the
oracle plus score bounds. Seconds of GPU time each; the exact top-k rows (64 of the 16S
queries, 32 of the protein queries, each against every reference) take one to two minutes
of oracle time on 16 host cores."""
import numpy as np
import pytest

import oracle
from gpusw_b200 import Aligner, workloads
from gpusw_b200.encode import Encoded

pytestmark = pytest.mark.gpu


def _enc(pair, scheme):
    codes, offs = pair
    return Encoded(codes, offs, list(range(offs.shape[0] - 1)), np.diff(offs).astype(np.int32),
                   scheme.eff_alphabet)


def _check_topk_full(wl, sample_rows):
    q, r = _enc(wl.queries, wl.scheme), _enc(wl.refs, wl.scheme)
    al = Aligner(wl.scheme).index(r).set_queries(q)
    tk = al.top_k(k=wl.k)
    idx, sc = tk.topk_idx, tk.topk_scores
    assert idx.shape == (wl.nq, wl.k) and sc.shape == (wl.nq, wl.k)
    # order: score descending, ties by ascending reference index; indices distinct, in range
    d = np.diff(sc.astype(np.int64), axis=1)
    assert (d <= 0).all()
    tie = d == 0
    assert (np.diff(idx.astype(np.int64), axis=1)[tie] > 0).all()
    assert idx.min() >= 0 and idx.max() < wl.nr
    # whole rows of seeded queries against the oracle: exact top-k
    rng = np.random.default_rng(123)
    rows = np.sort(rng.choice(wl.nq, size=sample_rows, replace=False)).astype(np.int32)
    want = oracle.score_cross(q, r, wl.scheme, qlist=rows)
    oi, osc = oracle.topk_stable(want, wl.k)
    assert np.array_equal(idx[rows], oi) and np.array_equal(sc[rows], osc)
    # top-1 of every query rescored through the pairs path
    qi = np.arange(wl.nq, dtype=np.int32)
    assert np.array_equal(al.score_pairs(qi, idx[:, 0]), sc[:, 0])


def test_16s_full_topk():
    _check_topk_full(workloads.sixteen_s(), sample_rows=64)


def test_protein_full_topk():
    _check_topk_full(workloads.protein(), sample_rows=32)


def test_pairs_full_million():
    wl = workloads.pairs()
    q, r = _enc(wl.queries, wl.scheme), _enc(wl.refs, wl.scheme)
    al = Aligner(wl.scheme).index(r).set_queries(q)
    got = al.score_pairs(*wl.pairs)
    assert got.shape == (1_000_000,)
    ql = np.diff(wl.queries[1])
    assert (got >= 0).all()                            # both ends free: empty alignment
    assert (got <= wl.scheme.match * np.minimum(ql, 200)).all()
    rng = np.random.default_rng(7)
    sel = np.sort(rng.choice(1_000_000, size=20_000, replace=False)).astype(np.int32)
    want = oracle.score_pairs(q, r, wl.pairs[0][sel], wl.pairs[1][sel], wl.scheme)
    assert np.array_equal(got[sel].astype(np.int64), want)
