"""The native FASTA reader (gpusw_fasta_parse in the engine library) against the Python
reader and encoder, which restate the reference's read_fasta and encoding loop
(src/gpusw/encode.py:89-120, :196-225). Runs on the CPU: the reader makes no CUDA call.

Every case goes through ``funnel`` (native where it applies) and through
``encode_pairs(read_fasta(...))`` (Python) and must give the same codes, offsets, lengths,
ids and errors."""
import gzip

import numpy as np
import pytest

from gpusw_b200 import Scheme, _native, schemes
from gpusw_b200.encode import build_lut, encode_pairs, funnel, read_fasta
from gpusw_b200.errors import EncodeError

SCHEMES = [schemes.DNA, schemes.BLOSUM62, Scheme(mode="local", unknown="zero"),
           Scheme(mode="global", case_insensitive=False)]


def _same(a, b):
    assert np.array_equal(a.codes, b.codes)
    assert np.array_equal(a.offsets, b.offsets)
    assert np.array_equal(a.lengths, b.lengths)
    assert a.ids == b.ids and a.alphabet == b.alphabet


def _native_used(text: str, sch) -> bool:
    lut, sentinel = build_lut(sch)
    return _native.parse_fasta(text.encode("ascii"), lut, sentinel, False) is not None


def _random_fasta(rng, alpha, n, stray=False):
    eols = ["\n", "\r\n", "\r"]
    # text that does not start with ">" is a raw sequence to funnel, so lines before the
    # first header only occur in files
    out = ["stray line before any header\n", "\n"] if stray else []
    for i in range(n):
        eol = eols[int(rng.integers(0, 3))]
        kind = int(rng.integers(0, 5))
        if kind == 0:
            out.append(">" + eol)                                # bare header -> seq<k>
        elif kind == 1:
            out.append(f">  id{i}\tsome description{eol}")       # blanks before the id
        else:
            out.append(f">id{i} desc {i}{eol}")
        for _ in range(int(rng.integers(0, 4))):
            seq = "".join(rng.choice(list(alpha), int(rng.integers(0, 70))))
            pad_l = " \t"[: int(rng.integers(0, 3))]
            pad_r = "\t "[: int(rng.integers(0, 3))]
            out.append(pad_l + seq + pad_r + eol)
            if rng.random() < 0.2:
                out.append("   " + eol)                          # blank line
    return "".join(out)


@pytest.mark.parametrize("sch", SCHEMES, ids=["dna", "blosum62", "unknown_zero", "case_sensitive"])
def test_random_fasta_text_matches_python_reader(sch):
    rng = np.random.default_rng(5)
    alpha = "ACGTNacgtn" if sch.ns <= 6 else "ARNDCQEGHILKMFPSTWYVXarnd*"
    text = _random_fasta(rng, alpha + " ", 300)             # inner spaces map to the sentinel
    assert _native_used(text, sch)
    if sch.unknown == "error":
        with pytest.raises(EncodeError) as e_py:
            encode_pairs(read_fasta(text), sch)
        with pytest.raises(EncodeError) as e_nat:
            funnel(text, sch)
        assert str(e_nat.value) == str(e_py.value)
    else:
        _same(funnel(text, sch), encode_pairs(read_fasta(text), sch))


def test_files_plain_and_gzip(tmp_path):
    rng = np.random.default_rng(6)
    text = _random_fasta(rng, "ACGT", 200, stray=True)
    plain, gz = tmp_path / "refs.fa", tmp_path / "refs.fa.gz"
    plain.write_bytes(text.encode())
    gz.write_bytes(gzip.compress(text.encode()))
    want = encode_pairs(read_fasta(str(plain)), schemes.DNA)
    _same(funnel(str(plain), schemes.DNA), want)
    _same(funnel(str(gz), schemes.DNA), want)
    empty = tmp_path / "none.fa"
    empty.write_bytes(b"ACGT\nACGT\n")                       # no header: no records
    got = funnel(str(empty), schemes.DNA)
    assert got.n == 0 and got.offsets.tolist() == [0]


def test_unknown_error_message_and_first_bad_symbol():
    sch = Scheme(mode="local", unknown="error")
    text = ">a\nACGT\n>b x\nACZGQ\n>c\nQQ\n"
    with pytest.raises(EncodeError) as e:
        funnel(text, sch)
    assert "'b'" in str(e.value) and "'Z'" in str(e.value)
    lut, sentinel = build_lut(sch)
    with pytest.raises(ValueError) as e2:
        _native.parse_fasta(text.encode(), lut, sentinel, True)
    assert e2.value.bad_record == 1 and e2.value.bad_byte == ord("Z")


@pytest.mark.parametrize("text", [">a\nACéGT\n>b\nAC\n", ">a\nAC\vGT\n", ">a\fb\nACGT\n",
                                  ">a\nAC\x1cGT\n"])
def test_text_the_native_reader_declines_goes_to_python(text):
    sch = Scheme(mode="local", unknown="zero")
    lut, sentinel = build_lut(sch)
    try:
        data = text.encode("ascii")
    except UnicodeEncodeError:
        data = text.encode("utf-8")
    assert _native.parse_fasta(data, lut, sentinel, False) is None
    _same(funnel(text, sch), encode_pairs(read_fasta(text), sch))


def test_large_set_offsets_and_ids():
    rng = np.random.default_rng(7)
    recs = [(f"r{i}", "".join(rng.choice(list("ACGT"), int(rng.integers(1, 300)))))
            for i in range(5000)]
    text = "".join(f">{i} d\n{s[:60]}\n{s[60:]}\n" for i, s in recs)
    got = funnel(text, schemes.DNA)
    assert got.n == 5000 and got.ids[:3] == ["r0", "r1", "r2"]
    _same(got, encode_pairs(recs, schemes.DNA))
