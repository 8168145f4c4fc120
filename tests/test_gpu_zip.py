"""Zipped pairs (``align_pairs`` with ``pairs=None``) through the pipelined engine call
``gpusw_score_pairs_zip``: sets packed and scored chunk by chunk on two streams. Every
score must equal the resident path (upload both sets, then ``gpusw_score_pairs``) and the
C oracle, across chunk boundaries (more than 131,072 pairs), empty and multi-pass sequences,
mixed lengths (several kernel shapes per chunk), int16 overflow rescoring and int32."""
import numpy as np
import pytest

import oracle
from gpusw_b200 import Aligner, Scheme, _native, align_pairs, schemes
from gpusw_b200.encode import funnel
from gpusw_b200.errors import OverflowRiskError
from tests._util import rand_seqs

pytestmark = pytest.mark.gpu


def _zip_vs_resident(qs, rs, sch):
    q, r = funnel(qs, sch), funnel(rs, sch)
    ctx = _native.context(0)
    with ctx.lock:
        ctx.set_scheme(sch)
        got = ctx.score_pairs_zip(q.codes, q.offsets, r.codes, r.offsets, sch.dtype)
    idx = np.arange(len(qs), dtype=np.int32)
    resident = Aligner(sch).index(rs).set_queries(qs).score_pairs(idx, idx)
    want = oracle.score_pairs(q, r, idx, idx, sch)
    assert np.array_equal(got, resident)
    assert np.array_equal(got.astype(np.int64), want)
    return got


def _rand_codes(rng, n, lo, hi, k):
    lens = rng.integers(lo, hi, size=n)
    offs = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(lens, out=offs[1:])
    return rng.integers(0, k, size=int(offs[-1])).astype(np.uint8), offs.astype(np.int32)


@pytest.mark.parametrize("mode", ["local", "global", "semiglobal"])
def test_zip_mixed_lengths_all_modes(mode):
    rng = np.random.default_rng(40 + len(mode))
    sch = schemes.DNA.replace(mode=mode)
    qs = rand_seqs(rng, 700, 0, 700, "ACGT")   # empty .. multi-pass, several shapes
    rs = rand_seqs(rng, 700, 0, 900, "ACGT")
    _zip_vs_resident(qs, rs, sch)


def test_zip_protein_and_int32():
    rng = np.random.default_rng(41)
    qs = rand_seqs(rng, 300, 1, 500, "ARNDCQEGHILKMFPSTWYV")
    rs = rand_seqs(rng, 300, 1, 500, "ARNDCQEGHILKMFPSTWYV")
    _zip_vs_resident(qs, rs, schemes.BLOSUM62)
    _zip_vs_resident(qs, rs, schemes.BLOSUM62.replace(dtype="int32"))


def test_zip_int16_overflow_rescored():
    # match = 1000: identical sequences of 40+ residues pass the int16 guard
    sch = Scheme(mode="local", match=1000, mismatch=-3, gap_open=-5, gap_extend=-2)
    rng = np.random.default_rng(42)
    qs = rand_seqs(rng, 200, 5, 80, "ACGT")
    rs = [q if i % 3 == 0 else s for i, (q, s) in enumerate(zip(qs, rand_seqs(rng, 200, 5, 80, "ACGT")))]
    got = _zip_vs_resident(qs, rs, sch)
    assert got.max() > 32767


def test_zip_many_chunks_equals_oracle():
    """300,000 short pairs: three pipeline chunks over both streams, read/window-like."""
    rng = np.random.default_rng(43)
    sch = schemes.DNA_SEMIGLOBAL
    qc, qo = _rand_codes(rng, 300_000, 0, 48, 4)
    rc, ro = _rand_codes(rng, 300_000, 0, 64, 4)
    ctx = _native.context(0)
    with ctx.lock:
        ctx.set_scheme(sch)
        got = ctx.score_pairs_zip(qc, qo, rc, ro, "auto")
        again = ctx.score_pairs_zip(qc, qo, rc, ro, "auto")
    from gpusw_b200.encode import Encoded

    def enc(c, o):
        return Encoded(c, o, list(range(o.shape[0] - 1)), np.diff(o).astype(np.int32), "ACGT")

    idx = np.arange(300_000, dtype=np.int32)
    want = oracle.score_pairs(enc(qc, qo), enc(rc, ro), idx, idx, sch)
    assert np.array_equal(got.astype(np.int64), want)
    assert np.array_equal(again, got)


def test_align_pairs_zip_api_and_errors():
    # the reference's known answer for zipped pairs (tests/test_api.py of the package)
    assert align_pairs(["ACGT", "TTTT"], ["ACGT", "TTTA"], scheme="dna",
                       return_ids=False).tolist() == [8, 6]
    res = align_pairs(["ACGT", "TTTT"], ["ACGT", "TTTA"], scheme="dna")
    assert res.scores.tolist() == [8, 6] and len(res.query_ids) == 2
    with pytest.raises(ValueError, match="len\\(queries\\)==len\\(refs\\)"):
        align_pairs(["ACGT"], ["ACGT", "AC"], scheme="dna")
    assert align_pairs([], [], scheme="dna", return_ids=False).shape == (0,)
    with pytest.raises(OverflowRiskError):
        align_pairs(["A" * 20000], ["A" * 20000], scheme="dna", mode="global", dtype="int16")
    ctx = _native.context(0)
    with ctx.lock:
        ctx.set_scheme(schemes.DNA)
        codes = np.array([0, 1, 9, 3], dtype=np.uint8)  # 9 >= the DNA table's side
        offs = np.array([0, 4], dtype=np.int32)
        with pytest.raises(ValueError, match="codes exceed"):
            ctx.score_pairs_zip(codes, offs, codes[:2] * 0, np.array([0, 2], dtype=np.int32), "auto")
        with pytest.raises(ValueError, match="non-decreasing"):
            ctx.score_pairs_zip(codes, np.array([3, 1], dtype=np.int32), codes, offs, "auto")
