"""The input funnel and AlignResult, pinned against the reference's outputs
(tests/golden/encode.json, topk.json) and its tests/test_encode.py semantics."""
import gzip

import numpy as np
import pytest

from gpusw_b200 import AlignResult, Scheme
from gpusw_b200.encode import build_lut, funnel, read_fasta
from gpusw_b200.errors import EncodeError
from tests._util import golden

DNA = Scheme(mode="local")
ENC = golden("encode.json")


@pytest.mark.parametrize("case", sorted(ENC))
def test_funnel_matches_reference(case):
    c = ENC[case]
    if case == "bytes":
        e = funnel(c["input_latin1"].encode("latin-1"), DNA)
    elif case == "case_sensitive":
        e = funnel(c["input"], Scheme(mode="local", case_insensitive=False))
    elif case == "pairs":
        e = funnel([tuple(p) for p in c["input"]], DNA)
    else:
        e = funnel(c["input"], DNA)
    assert e.codes.tolist() == c["codes"]
    assert e.offsets.tolist() == c["offsets"]
    assert list(e.ids) == c["ids"]
    assert e.codes.dtype == np.uint8 and e.offsets.dtype == np.int32


def test_lut_and_errors(tmp_path):
    lut, sentinel = build_lut(DNA)
    assert sentinel == 4 and [lut[ord(ch)] for ch in "ACGTacgt"] == [0, 1, 2, 3] * 2
    with pytest.raises(EncodeError):
        funnel(["ACGTN"], Scheme(mode="local", unknown="error"))
    with pytest.raises(EncodeError):
        funnel(b"ACG\xffT", Scheme(mode="local", unknown="error"))
    with pytest.raises(EncodeError):
        funnel("nonexistent_refs.fasta", DNA)
    with pytest.raises(FileNotFoundError):
        read_fasta("/no/such/file.fasta")
    codes = np.array([0, 1, 2, 3], dtype=np.uint8)
    for bad in ([0, 4, 1000], [0, -1, 4], [0, 4, 2]):
        with pytest.raises(EncodeError):
            funnel((codes, np.array(bad, dtype=np.int32)), DNA)
    with pytest.raises(EncodeError):
        funnel(42, DNA)


def test_fasta_paths(tmp_path):
    p = tmp_path / "q.fasta"
    p.write_text(">seqA desc\nACGT\nACGT\n>seqB\nTTTT\n")
    e = funnel(str(p), DNA)
    assert e.ids == ["seqA", "seqB"] and e.lengths.tolist() == [8, 4]
    g = tmp_path / "q.fasta.gz"
    with gzip.open(g, "wt") as fh:
        fh.write(">s1\nACGT\n")
    assert read_fasta(str(g)) == [("s1", "ACGT")]


def test_preencoded_and_records():
    codes = np.array([0, 1, 2, 3, 3, 2], dtype=np.uint8)
    e = funnel((codes, np.array([0, 4, 6], dtype=np.int32)), DNA)
    assert e.n == 2 and e.codes[e.offsets[1]:e.offsets[2]].tolist() == [3, 2]
    assert funnel(e, DNA) is e
    with pytest.raises(EncodeError):
        funnel(e, Scheme(alphabet="ACGU"))

    class Rec:
        def __init__(self, i, s):
            self.id, self.seq = i, s

    e = funnel([Rec("a", "ACGT"), Rec("b", "TT")], DNA)
    assert e.ids == ["a", "b"] and e.lengths.tolist() == [4, 2]


def test_alignresult_topk_matches_reference():
    for case in golden("topk.json"):
        m = np.asarray(case["scores"], dtype=np.int32)
        res = AlignResult(m, [f"q{i}" for i in range(m.shape[0])],
                          [f"r{j}" for j in range(m.shape[1])], None)
        assert [[q, [list(h) for h in hits]] for q, hits in res.top_k(case["k"])] == case["top"]


def test_alignresult_stored_topk_and_dataframe():
    idx = np.array([[2, 0], [1, 2]], dtype=np.int32)
    sc = np.array([[9, 5], [7, 7]], dtype=np.int32)
    res = AlignResult(None, ["a", "b"], ["x", "y", "z"], None, topk_idx=idx, topk_scores=sc)
    assert res.top_k(2) == [("a", [("z", 9), ("x", 5)]), ("b", [("y", 7), ("z", 7)])]
    assert res.best() == [("a", "z", 9), ("b", "y", 7)]
    df = res.to_dataframe()
    assert list(df.columns) == ["query", "reference", "rank", "score"] and len(df) == 4
    with pytest.raises(ValueError):
        AlignResult(np.zeros(3, dtype=np.int32), ["a"], ["x"], None).top_k(1)
