"""High-level API behaviour on the GPU (the reference's tests/test_api.py cases) plus
top-k order, errors and introspection."""
import numpy as np
import pytest

import oracle
from gpusw_b200 import Aligner, Scheme, align_pairs, align_score
from gpusw_b200.encode import funnel
from gpusw_b200.errors import OverflowRiskError
from tests._util import rand_seqs

pytestmark = pytest.mark.gpu

QUERIES = {"q_a": "ACGTACGTACGT", "q_b": "TTTTGGGG", "q_c": "ACGGACGT"}
REFS = {"r1": "ACGTACGTACGT", "r2": "ACGTAAAA", "r3": "GGGGTTTT", "r4": "TACGGACGTA"}


def test_align_score_shapes_and_ids():
    res = align_score(QUERIES, REFS, scheme="dna")
    assert res.scores.shape == (3, 4) and res.scores.dtype == np.int32
    assert res.query_ids == ["q_a", "q_b", "q_c"]
    assert res.reference_ids == ["r1", "r2", "r3", "r4"]
    arr = align_score(QUERIES, REFS, scheme="dna", return_ids=False)
    assert isinstance(arr, np.ndarray) and arr.shape == (3, 4)


def test_top_k_matches_full_sort():
    al = Aligner("dna").index(REFS).set_queries(QUERIES)
    full = al.score_cross(return_ids=True)
    tk = al.top_k(k=2)
    assert tk.top_k(2) == full.top_k(2)
    assert tk.scores is None and tk.topk_idx.shape == (3, 2)


@pytest.mark.parametrize("k", [1, 5, 8, 9, 16, 17, 31, 32, 33, 70, 400])
@pytest.mark.parametrize("nr", [300, 301, 2003])
def test_top_k_tie_order_any_k(k, nr):
    """Many ties (short, low-entropy sequences): order must be (score desc, index asc), for
    every list depth of the one-pass kernel (k <= 8, 16, 32), the multi-round kernel beyond,
    and rows whose length is not a multiple of four (the scalar tail of the 128-bit loads)."""
    rng = np.random.default_rng(k * 7 + nr)
    qs = rand_seqs(rng, 7, 1, 12, "AC")
    rs = rand_seqs(rng, nr, 0, 12, "AC")
    al = Aligner("dna").index(rs).set_queries(qs)
    tk = al.top_k(k=k)
    full = al.score_cross()
    idx, sc = oracle.topk_stable(full, k)
    assert np.array_equal(tk.topk_idx, idx) and np.array_equal(tk.topk_scores, sc)
    want = oracle.score_cross(funnel(qs, Scheme()), funnel(rs, Scheme()), Scheme())
    assert np.array_equal(full.astype(np.int64), want)


def test_top_k_protein_vs_oracle():
    from gpusw_b200 import schemes
    rng = np.random.default_rng(4)
    alpha = "ARNDCQEGHILKMFPSTWYV"
    qs = rand_seqs(rng, 9, 20, 400, alpha)
    rs = rand_seqs(rng, 500, 20, 500, alpha)
    tk = Aligner(schemes.BLOSUM62).index(rs).top_k(qs, k=10)
    want = oracle.score_cross(funnel(qs, schemes.BLOSUM62), funnel(rs, schemes.BLOSUM62), schemes.BLOSUM62)
    idx, sc = oracle.topk_stable(want, 10)
    assert np.array_equal(tk.topk_idx, idx) and np.array_equal(tk.topk_scores, sc)


def test_align_pairs_known_answers():
    assert align_pairs(["ACGT", "TTTT"], ["ACGT", "TTTA"], scheme="dna").scores.tolist() == [8, 6]
    res = align_pairs(list(QUERIES.values()), list(REFS.values()), pairs=[(0, 0), (0, 3), (2, 3)],
                      scheme="dna", return_ids=False)
    assert res.tolist() == [24, 13, 16]
    with pytest.raises(ValueError):
        align_pairs(["ACGT", "TT"], ["ACGT"], scheme="dna")


def test_pair_index_out_of_range_rejected_before_launch():
    al = Aligner("dna").index(["ACGT", "GG"]).set_queries(["ACGT"])
    with pytest.raises(ValueError):
        al.score_pairs([0, 1], [0, 0])
    with pytest.raises(ValueError):
        al.score_pairs([0], [5])
    with pytest.raises(ValueError):
        al.score_pairs([-1], [0])
    assert al.score_pairs([0], [0]).tolist() == [8]  # context still usable


def test_gcups_and_source():
    al = Aligner("dna").index(REFS).set_queries(QUERIES)
    al.score_cross()
    assert al.gcups > 0
    src = al.cuda_source()
    assert "sw_cross" in src and "#define MODE" in src
    assert al.backend == "cuda"


def test_one_call_modes():
    g = align_score(["AC"], ["TTACTT"], scheme="dna", mode="global", return_ids=False)
    s = align_score(["AC"], ["TTACTT"], scheme="dna", mode="semiglobal", return_ids=False)
    assert s[0, 0] == 4 and g[0, 0] < s[0, 0]


def test_forced_int16_overflow_raises():
    with pytest.raises(OverflowRiskError):
        align_score(["A" * 20000], ["A" * 20000], scheme="dna", dtype="int16")


def test_query_batch_and_empty_sets():
    qs = [f"ACGT{'A' * i}" for i in range(10)]
    a = align_score(qs, ["ACGTAAAA", "TT"], scheme="dna", return_ids=False, query_batch=3)
    b = align_score(qs, ["ACGTAAAA", "TT"], scheme="dna", return_ids=False)
    assert np.array_equal(a, b)
    assert align_score([], ["ACGT"], scheme="dna", return_ids=False).shape == (0, 1)
    assert align_score(["ACGT"], [], scheme="dna", return_ids=False).shape == (1, 0)
    tk = Aligner("dna").index(["ACGT"]).top_k(["AC", "GT"], k=5)
    assert tk.topk_idx.shape == (2, 1)
