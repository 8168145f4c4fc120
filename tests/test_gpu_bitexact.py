"""GPU scores == the reference's oracle, to the integer: golden vectors produced by the
reference itself, the reference's own GPU test cases (tests/test_gpu_bitexact.py), and
seeded random sets against the C oracle -- all through the public API and the C ABI."""
import numpy as np
import pytest

import oracle
from gpusw_b200 import Aligner, Matrix, Scheme, align_pairs, align_score
from gpusw_b200.encode import Encoded, funnel
from tests._util import golden, rand_seqs, scheme_from_spec

pytestmark = pytest.mark.gpu
SCORES = golden("scores.json")


@pytest.mark.parametrize("kind", ["cross", "edges"])
@pytest.mark.parametrize("name", sorted(SCORES["cross"]))
def test_cross_matches_golden(kind, name):
    case = SCORES[kind][name]
    sch = scheme_from_spec(case["scheme"])
    got = align_score(case["queries"], case["refs"], scheme=sch, return_ids=False)
    assert got.dtype == np.int32
    assert got.tolist() == case["scores"]


@pytest.mark.parametrize("kind", ["cross", "edges"])
@pytest.mark.parametrize("name", sorted(SCORES["cross"]))
def test_cross_int32_matches_golden(kind, name):
    case = SCORES[kind][name]
    sch = scheme_from_spec(case["scheme"]).replace(dtype="int32")
    got = align_score(case["queries"], case["refs"], scheme=sch, return_ids=False)
    assert got.tolist() == case["scores"]


@pytest.mark.parametrize("name", sorted(SCORES["pairs"]))
@pytest.mark.parametrize("dtype", ["auto", "int32"])
def test_pairs_match_golden(name, dtype):
    case = SCORES["pairs"][name]
    sch = scheme_from_spec(case["scheme"]).replace(dtype=dtype)
    got = align_pairs(case["queries"], case["refs"], scheme=sch, return_ids=False)
    assert got.tolist() == case["scores"]


@pytest.mark.parametrize("name", sorted(SCORES["edges"]))
def test_pairs_edges_all_combinations(name):
    case = SCORES["edges"][name]
    sch = scheme_from_spec(case["scheme"])
    qs, rs = case["queries"], case["refs"]
    pairs = [(i, j) for i in range(len(qs)) for j in range(len(rs))]
    got = align_pairs(qs, rs, pairs=pairs, scheme=sch, return_ids=False)
    assert got.tolist() == [case["scores"][i][j] for i, j in pairs]


def test_anchors():
    for a in SCORES["anchors"]:
        sch = scheme_from_spec(a["scheme"])
        got = align_score([a["query"]], [a["ref"]], scheme=sch, return_ids=False)
        assert int(got[0, 0]) == a["score"], a


SCHEMES = {
    "dna_local": (Scheme(mode="local"), "ACGTN"),
    "dna_global": (Scheme(mode="global"), "ACGT"),
    "dna_semi_qr": (Scheme(mode="semiglobal"), "ACGT"),
    "dna_semi_q": (Scheme(mode="semiglobal", free_end_gaps_query=True, free_end_gaps_ref=False), "ACGT"),
    "dna_semi_r": (Scheme(mode="semiglobal", free_end_gaps_query=False, free_end_gaps_ref=True), "ACGT"),
    "ednafull_global": (Scheme(mode="global", matrix=Matrix.named("EDNAFULL"), gap_open=-10, gap_extend=-1), "ACGTN"),
    "blosum62_local": (Scheme(mode="local", matrix=Matrix.named("BLOSUM62"), gap_open=-11, gap_extend=-1), "ARNDCQEGHILKMFPSTWYV"),
    "blosum62_global": (Scheme(mode="global", matrix=Matrix.named("BLOSUM62"), gap_open=-11, gap_extend=-1), "ARNDCQEGHILKMFPSTWYVX"),
    "protein_semiglobal": (Scheme(mode="semiglobal", matrix=Matrix.named("BLOSUM62"), gap_open=-11, gap_extend=-1), "ARNDCQEGHILKMFPSTWYV"),
}


@pytest.mark.parametrize("name", list(SCHEMES))
def test_random_cross_vs_c_oracle(name):
    """Lengths spanning every kernel shape (up to 1100 columns) and odd query counts."""
    scheme, alpha = SCHEMES[name]
    rng = np.random.default_rng(sorted(SCHEMES).index(name) + 17)
    queries = rand_seqs(rng, 13, 0, 300, alpha) + rand_seqs(rng, 2, 500, 1100, alpha)
    refs = rand_seqs(rng, 37, 0, 400, alpha)
    got = align_score(queries, refs, scheme=scheme, return_ids=False)
    want = oracle.score_cross(funnel(queries, scheme), funnel(refs, scheme), scheme)
    assert np.array_equal(got.astype(np.int64), want)


@pytest.mark.parametrize("name", list(SCHEMES))
def test_random_pairs_vs_c_oracle(name):
    scheme, alpha = SCHEMES[name]
    rng = np.random.default_rng(sorted(SCHEMES).index(name) + 101)
    qs = rand_seqs(rng, 301, 0, 600, alpha)
    rs = rand_seqs(rng, 301, 0, 600, alpha)
    got = align_pairs(qs, rs, scheme=scheme, return_ids=False)
    want = oracle.score_pairs(funnel(qs, scheme), funnel(rs, scheme), np.arange(301), np.arange(301), scheme)
    assert np.array_equal(got.astype(np.int64), want)


def test_reference_regressions():
    s = Scheme()
    assert int(align_score(["ACGTACGTAC"], ["ACGTACGTAC"], scheme=s, return_ids=False)[0, 0]) == 20
    assert int(align_score(["ACGTACGTAC"], ["TTACGTACGTACTT"], scheme=s, return_ids=False)[0, 0]) == 20


def test_int32_promotion_bitexact():
    scheme = Scheme(mode="local", match=1000, mismatch=-3, gap_open=-5, gap_extend=-2)
    q = r = "ACGT" * 15
    assert scheme.resolve_dtype(len(q), len(r)) == "int32"
    got = align_score([q], [r], scheme=scheme, return_ids=False)
    assert got.dtype == np.int32 and int(got[0, 0]) == 60000


def test_int32_promotion_pairs_bitexact():
    scheme = Scheme(mode="local", match=1000, mismatch=-3, gap_open=-5, gap_extend=-2)
    qs = ["ACGT" * 15, "ACGTAC" * 5, "AAAA"]
    rs = ["ACGT" * 15, "ACGTAC" * 5, "TTTT", "ACGT" * 15]
    pairs = [(0, 0), (1, 1), (2, 2), (0, 3)]
    res = align_pairs(qs, rs, pairs=pairs, scheme=scheme, return_ids=False)
    cpu = oracle.score_cross(funnel(qs, scheme), funnel(rs, scheme), scheme)
    assert res.tolist() == [int(cpu[i, j]) for i, j in pairs]


@pytest.mark.parametrize("mode", ["local", "global", "semiglobal"])
def test_int16_overflow_rescore_mixed(mode):
    """Some pairs overflow int16 and are rescored in int32, the rest stay int16."""
    scheme = Scheme(mode=mode, match=300, mismatch=-7, gap_open=-9, gap_extend=-4)
    rng = np.random.default_rng(5)
    base = rand_seqs(rng, 1, 200, 201, "ACGT")[0]
    qs = [base, base[:40], base[50:170]] + rand_seqs(rng, 9, 1, 200, "ACGT")
    rs = [base, base[10:190]] + rand_seqs(rng, 20, 1, 220, "ACGT")
    al = Aligner(scheme).index(rs).set_queries(qs)
    got = al.score_cross()
    want = oracle.score_cross(funnel(qs, scheme), funnel(rs, scheme), scheme)
    assert np.array_equal(got.astype(np.int64), want)
    assert want.max() > 32767  # the case really exercises the rescoring
    pairs = align_pairs(qs[:3] * 2, rs[:2] * 3, scheme=scheme, return_ids=False)
    qi, rj = np.arange(6) % 3, np.arange(6) % 2
    assert pairs.astype(np.int64).tolist() == [int(want[i, j]) for i, j in zip(qi, rj)]


def test_long_sequences_multipass():
    """Columns beyond the widest single-pass shape go through the multi-pass kernel."""
    rng = np.random.default_rng(9)
    for scheme, alpha in [(Scheme(mode="local"), "ACGT"), (Scheme(mode="global"), "ACGT"),
                          (Scheme(mode="semiglobal", free_end_gaps_ref=False), "ACGT"),
                          (Scheme(mode="local", matrix=Matrix.named("BLOSUM62"), gap_open=-11,
                                  gap_extend=-1), "ARNDCQEGHILKMFPSTWYV")]:
        qs = rand_seqs(rng, 3, 1500, 3000, alpha)
        rs = rand_seqs(rng, 5, 100, 2500, alpha)
        got = align_score(qs, rs, scheme=scheme, return_ids=False)
        want = oracle.score_cross(funnel(qs, scheme), funnel(rs, scheme), scheme)
        assert np.array_equal(got.astype(np.int64), want)
        gp = align_pairs(qs + qs[:2], rs, scheme=scheme, return_ids=False)
        wp = oracle.score_pairs(funnel(qs + qs[:2], scheme), funnel(rs, scheme), np.arange(5), np.arange(5), scheme)
        assert np.array_equal(gp.astype(np.int64), wp)


def test_unequal_row_lengths_in_pairs_semiglobal():
    scheme = Scheme(mode="semiglobal", free_end_gaps_query=True, free_end_gaps_ref=True)
    rng = np.random.default_rng(21)
    qs = rand_seqs(rng, 64, 1, 150, "ACGT")
    rs = rand_seqs(rng, 64, 1, 300, "ACGT")
    got = align_pairs(qs, rs, scheme=scheme, return_ids=False)
    want = oracle.score_pairs(funnel(qs, scheme), funnel(rs, scheme), np.arange(64), np.arange(64), scheme)
    assert np.array_equal(got.astype(np.int64), want)


def test_large_alphabet_eight_bit_codes():
    alpha = "".join(chr(c) for c in range(48, 48 + 40))  # 40 symbols -> 8-bit packing
    arr = (np.arange(40)[:, None] * 7 + np.arange(40)[None, :] * 3) % 11 - 5
    scheme = Scheme(mode="local", matrix=Matrix.from_array(alpha, arr), gap_open=-6, gap_extend=-1,
                    case_insensitive=False)
    rng = np.random.default_rng(3)
    qs = rand_seqs(rng, 5, 1, 90, alpha)
    rs = rand_seqs(rng, 7, 1, 120, alpha)
    got = align_score(qs, rs, scheme=scheme, return_ids=False)
    want = oracle.score_cross(funnel(qs, scheme), funnel(rs, scheme), scheme)
    assert np.array_equal(got.astype(np.int64), want)


@pytest.mark.parametrize("scheme,alpha,hi", [
    (Scheme(mode="local", match=100, mismatch=-60, gap_open=-50, gap_extend=-10), "ACGT", 200),
    (Scheme(mode="semiglobal", free_end_gaps_query=True, free_end_gaps_ref=False), "ACGTN", 400),
    (Scheme(mode="semiglobal", free_end_gaps_query=False, free_end_gaps_ref=True), "ACGTN", 400),
    (Scheme(mode="global"), "ACGT", 400),
    (Scheme(mode="local", matrix=Matrix.named("BLOSUM62"), gap_open=-11, gap_extend=-1),
     "ARNDCQEGHILKMFPSTWYV", 1300),
], ids=["profile_beyond_int8", "semi_free_query_only", "semi_free_ref_only", "global",
        "blosum62_multipass"])
def test_pairs_kernel_paths(scheme, alpha, hi):
    """Every form of the pairs kernel: int8 or s16x2 query tables, the branch-free pass and
    the general one (free query ends without left padding), one or several column passes,
    partners of unequal row lengths."""
    rng = np.random.default_rng(hi + len(alpha))
    qs = rand_seqs(rng, 160, 0, hi, alpha)
    rs = rand_seqs(rng, 160, 0, hi, alpha)
    qi = rng.permutation(160).astype(np.int32)
    rj = rng.integers(0, 160, size=160).astype(np.int32)
    al = Aligner(scheme).index(rs).set_queries(qs)
    got = al.score_pairs(qi, rj)
    want = oracle.score_pairs(funnel(qs, scheme), funnel(rs, scheme), qi, rj, scheme)
    assert np.array_equal(got.astype(np.int64), want)


def _short_set(rng, n, max_len, ncodes, alphabet):
    lengths = rng.integers(0, max_len + 1, size=n).astype(np.int32)
    offsets = np.zeros(n + 1, dtype=np.int32)
    np.cumsum(lengths, out=offsets[1:])
    codes = rng.integers(0, ncodes, size=int(offsets[-1])).astype(np.uint8)
    return Encoded(codes=codes, offsets=offsets, ids=[f"s{i}" for i in range(n)],
                   lengths=lengths, alphabet=alphabet)


@pytest.mark.gpu
@pytest.mark.parametrize("scheme,ncodes", [
    (Scheme(mode="semiglobal", free_end_gaps_query=True, free_end_gaps_ref=True), 4),
    (Scheme(mode="local", matrix=Matrix.named("BLOSUM62"), gap_open=-11, gap_extend=-1), 24),
], ids=["dna_2bit", "protein_5bit"])
def test_many_short_sequences_chunked_upload(scheme, ncodes):
    """Sets of 300,000 sequences (0-32 residues) are packed and copied to the device in
    chunks that overlap; every pair must still score as the oracle says."""
    rng = np.random.default_rng(300_000 + ncodes)
    n = 300_000
    qs = _short_set(rng, n, 32, ncodes, scheme.eff_alphabet)
    rs = _short_set(rng, n, 32, ncodes, scheme.eff_alphabet)
    qi = rng.permutation(n).astype(np.int32)
    rj = rng.integers(0, n, size=n).astype(np.int32)
    al = Aligner(scheme).index(rs).set_queries(qs)
    got = al.score_pairs(qi, rj)
    want = oracle.score_pairs(qs, rs, qi, rj, scheme)
    assert np.array_equal(got.astype(np.int64), want)
