"""Aligner.locate on the device against the oracle's coordinates, bit-exact: DNA and
protein local schemes, queries past one 512-column pass (multi-pass strips), empty
sequences, pairs that score 0, exact-repeat ties, and the anchored pass's self-check."""
import numpy as np
import pytest

import oracle
from gpusw_b200 import Aligner, Scheme, schemes
from gpusw_b200.errors import SchemeError
from tests._util import rand_seqs

pytestmark = pytest.mark.gpu

KEYS = ("score", "query_start", "query_end", "ref_start", "ref_end")


def _mutate(rng, s, alpha, rate):
    out = []
    for ch in s:
        u = rng.random()
        if u < rate / 3:
            continue                                   # deletion
        if u < 2 * rate / 3:
            out.append(alpha[rng.integers(len(alpha))])  # substitution
        else:
            out.append(ch)
        if rng.random() < rate / 3:
            out.append(alpha[rng.integers(len(alpha))])  # insertion
    return "".join(out)


def _compare(sch, qs_, rs_, qi, rj):
    al = Aligner(sch).index(rs_).set_queries(qs_)
    got = al.locate(qi, rj)
    want = oracle.locate_pairs(al._queries, al._refs, qi, rj, sch)
    for k in KEYS:
        assert got[k].dtype == np.int32
        assert np.array_equal(got[k].astype(np.int64), want[k]), k
    return got


def test_locate_dna_related_and_random():
    rng = np.random.default_rng(21)
    alpha = "ACGT"
    base = rand_seqs(rng, 60, 20, 700, alpha)
    refs = [rand_seqs(rng, 1, 0, 200, alpha)[0] + _mutate(rng, b, alpha, 0.1)
            + rand_seqs(rng, 1, 0, 200, alpha)[0] for b in base]
    qs_ = base + rand_seqs(rng, 20, 0, 40, alpha) + [""]
    rs_ = refs + ["", "AC"]
    n = len(qs_)
    qi = np.arange(n, dtype=np.int32)
    rj = np.concatenate([np.arange(60), rng.integers(0, len(rs_), size=n - 60)]).astype(np.int32)
    got = _compare(schemes.DNA, qs_, rs_, qi, rj)
    assert (got["score"][:60] > 0).all()


def test_locate_protein_multipass():
    rng = np.random.default_rng(22)
    alpha = "ARNDCQEGHILKMFPSTWYV"
    base = rand_seqs(rng, 24, 400, 1400, alpha)   # most queries need 2-3 column passes
    refs = [_mutate(rng, b, alpha, 0.2) for b in base]
    qi = np.arange(24, dtype=np.int32)
    _compare(schemes.BLOSUM62, base, refs, qi, qi.copy())


def test_locate_ties_zero_scores_and_modes():
    sch = schemes.DNA
    qs_ = ["ACGT", "AAAA", "", "ACGTACGT"]
    rs_ = ["TTACGTTTACGTTT", "CCCC", "ACGT", "ACGTACGTACGTACGT"]
    idx = np.arange(4, dtype=np.int32)
    got = _compare(sch, qs_, rs_, idx, idx)
    assert [got[k][0] for k in KEYS] == [8, 0, 4, 2, 6]
    assert got["score"][1] == 0 and got["ref_end"][1] == -1
    assert got["score"][2] == 0 and got["query_start"][2] == -1
    assert [got[k][3] for k in KEYS] == [16, 0, 8, 0, 8]
    empty = Aligner(sch).index(rs_).set_queries(qs_).locate(np.zeros(0, np.int32),
                                                              np.zeros(0, np.int32))
    assert all(empty[k].shape == (0,) for k in KEYS)
    with pytest.raises(SchemeError):
        Aligner(schemes.DNA_GLOBAL).index(rs_).set_queries(qs_).locate(idx, idx)
    with pytest.raises(ValueError):
        Aligner(sch).index(rs_).set_queries(qs_).locate(idx, idx[:2])
    with pytest.raises(ValueError):
        Aligner(sch).index(rs_).set_queries(qs_).locate(idx, idx + 1)


def test_locate_scores_equal_score_pairs():
    rng = np.random.default_rng(23)
    sch = Scheme(mode="local", match=3, mismatch=-2, gap_open=-4, gap_extend=-1)
    qs_ = rand_seqs(rng, 200, 1, 300, "ACGTN")
    rs_ = rand_seqs(rng, 200, 1, 300, "ACGTN")
    al = Aligner(sch).index(rs_).set_queries(qs_)
    qi = rng.integers(0, 200, size=500).astype(np.int32)
    rj = rng.integers(0, 200, size=500).astype(np.int32)
    assert np.array_equal(al.locate(qi, rj)["score"], al.score_pairs(qi, rj))


def test_locate_top_hits_match_oracle():
    rng = np.random.default_rng(24)
    alpha = "ARNDCQEGHILKMFPSTWYV"
    refs = rand_seqs(rng, 120, 40, 400, alpha)
    qs_ = [_mutate(rng, refs[int(rng.integers(0, 120))][10:200], alpha, 0.15) for _ in range(9)]
    sch = schemes.BLOSUM62
    al = Aligner(sch).index(refs)
    res = al.top_k(qs_, k=3)
    loc = al.locate_top(res)
    assert np.array_equal(loc["score"], res.topk_scores)
    qi = np.repeat(np.arange(9, dtype=np.int32), 3)
    want = oracle.locate_pairs(al._queries, al._refs, qi, res.topk_idx.reshape(-1), sch)
    for k in KEYS:
        assert np.array_equal(loc[k].reshape(-1).astype(np.int64), want[k]), k
