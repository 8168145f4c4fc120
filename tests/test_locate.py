"""Best-cell coordinates (``Aligner.locate``) on the CPU side: the oracle's two-pass
definition checked against properties that need nothing but scores.

For every pair with a positive local score S and coordinates ``[qs, qe) x [rs, re)``:

* the local score of the prefixes ``q[:qe], r[:re]`` is S, of ``q, r[:re-1]`` and of
  ``q[:qe-1], r[:re]`` below S: the end is the first best cell, row-major;
* the global score of the segments ``q[qs:qe], r[rs:re]`` is S: the coordinates bound an
  optimal alignment;
* no segment ending at the same cell with a later reference start reaches S, and with the same
  reference start no later query start does: the start is the first best cell of the
  reversed, anchored pass.

Scores come from the C oracle; the engine is checked against these coordinates on the GPU.
"""
import numpy as np

import oracle
from gpusw_b200 import schemes
from gpusw_b200.encode import Encoded, funnel
from tests._util import rand_seqs


def _set(seqs, alpha):
    codes = np.concatenate([np.asarray(s, dtype=np.uint8) for s in seqs]) if seqs else \
        np.zeros(0, dtype=np.uint8)
    lens = np.array([len(s) for s in seqs], dtype=np.int32)
    offs = np.zeros(len(seqs) + 1, dtype=np.int32)
    np.cumsum(lens, out=offs[1:])
    return Encoded(codes, offs, list(range(len(seqs))), lens, alpha)


def _scores(qsegs, rsegs, scheme):
    q, r = _set(qsegs, "x"), _set(rsegs, "x")
    k = np.arange(len(qsegs), dtype=np.int32)
    return oracle.score_pairs(q, r, k, k, scheme)


def _check(scheme, qs_, rs_, seed):
    q, r = funnel(qs_, scheme), funnel(rs_, scheme)
    rng = np.random.default_rng(seed)
    qi = rng.integers(0, q.n, size=q.n).astype(np.int32)
    rj = rng.integers(0, r.n, size=q.n).astype(np.int32)
    loc = oracle.locate_pairs(q, r, qi, rj, scheme)
    assert np.array_equal(loc["score"], oracle.score_pairs(q, r, qi, rj, scheme))
    glob = scheme.replace(mode="global")
    pre_q, pre_r, seg_q, seg_r, later_q, later_r, later_s = [], [], [], [], [], [], []
    for k in range(qi.shape[0]):
        qc = q.codes[q.offsets[qi[k]]:q.offsets[qi[k] + 1]]
        rc = r.codes[r.offsets[rj[k]]:r.offsets[rj[k] + 1]]
        s = loc["score"][k]
        if s <= 0:
            assert loc["query_end"][k] == -1 and loc["ref_start"][k] == -1
            continue
        a, b = loc["query_start"][k], loc["query_end"][k]
        c, d = loc["ref_start"][k], loc["ref_end"][k]
        assert 0 <= a < b <= qc.shape[0] and 0 <= c < d <= rc.shape[0]
        pre_q += [qc[:b], qc, qc[:b - 1]]
        pre_r += [rc[:d], rc[:d - 1], rc[:d]]
        seg_q.append(qc[a:b])
        seg_r.append(rc[c:d])
        for c2 in range(c + 1, d):
            for a2 in range(0, b):
                later_q.append(qc[a2:b]); later_r.append(rc[c2:d]); later_s.append(s)
        for a2 in range(a + 1, b):
            later_q.append(qc[a2:b]); later_r.append(rc[c:d]); later_s.append(s)
    if not seg_q:
        return 0
    pre = _scores(pre_q, pre_r, scheme).reshape(-1, 3)
    hits = loc["score"][loc["score"] > 0]
    assert np.array_equal(pre[:, 0], hits)
    assert (pre[:, 1] < hits).all() and (pre[:, 2] < hits).all()
    assert np.array_equal(_scores(seg_q, seg_r, glob), hits)
    if later_q:
        assert (_scores(later_q, later_r, glob) < np.array(later_s)).all()
    return len(seg_q)


def test_oracle_locate_dna_properties():
    rng = np.random.default_rng(5)
    qs_ = rand_seqs(rng, 40, 0, 24, "ACGT")
    rs_ = rand_seqs(rng, 40, 0, 30, "ACGT")
    assert _check(schemes.DNA, qs_, rs_, 1) > 20


def test_oracle_locate_protein_properties():
    rng = np.random.default_rng(6)
    alpha = "ARNDCQEGHILKMFPSTWYV"
    qs_ = rand_seqs(rng, 30, 1, 18, alpha)
    rs_ = rand_seqs(rng, 30, 1, 22, alpha)
    assert _check(schemes.BLOSUM62, qs_, rs_, 2) > 15


def test_oracle_locate_ties_take_first_cell():
    sch = schemes.DNA
    q, r = funnel(["ACGT", "AAAA", ""], sch), funnel(["TTACGTTTACGTTT", "CCCC", "ACGT"], sch)
    loc = oracle.locate_pairs(q, r, [0, 1, 2], [0, 1, 2], sch)
    # two exact copies of the query: the first reference copy (rows 2..5) wins
    assert [loc[k][0] for k in ("score", "query_start", "query_end", "ref_start", "ref_end")] \
        == [8, 0, 4, 2, 6]
    assert loc["score"][1] == 0 and loc["ref_end"][1] == -1     # nothing scores above 0
    assert loc["score"][2] == 0 and loc["query_start"][2] == -1  # empty query
