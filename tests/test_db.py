"""Persisted packed sets: the engine's packed image written once and mapped back (format 2),
round trips of codes through the image at every packing width, validation of corrupted
files, reading the first (byte-code) format; on a GPU an Aligner indexes a loaded set
without re-packing it and scores exactly as from the original input."""
import json
import os

import numpy as np
import pytest

import oracle
from gpusw_b200 import Aligner, _native, schemes
from gpusw_b200.db import PackedSet, load_db, save_db, unpack_image
from gpusw_b200.encode import Encoded, funnel
from gpusw_b200.errors import EncodeError


def _native_built():
    return os.path.exists(_native.LIB_PATH)


needs_lib = pytest.mark.skipif(not _native_built(), reason="engine library not built")


@needs_lib
def test_round_trip(tmp_path):
    enc = funnel({"r1": "ACGTN", "r2": "", "r3": "ttgca"}, schemes.DNA)
    save_db(enc, str(tmp_path / "db"), schemes.DNA)
    back = load_db(str(tmp_path / "db"), schemes.DNA)
    assert isinstance(back, PackedSet) and back.bits == 4  # N (code 4) needs 4 bits
    assert back.ids == ["r1", "r2", "r3"]
    assert back.codes.tolist() == enc.codes.tolist()
    assert back.offsets.tolist() == enc.offsets.tolist()
    assert back.lengths.tolist() == [5, 0, 5]
    copy = load_db(str(tmp_path / "db"), mmap=False)
    assert copy.codes.tolist() == enc.codes.tolist()


@needs_lib
@pytest.mark.parametrize("k,bits", [(4, 2), (16, 4), (25, 5), (200, 8)])
def test_pack_image_widths(k, bits):
    rng = np.random.default_rng(k)
    lens = rng.integers(0, 90, size=57)
    offs = np.zeros(58, dtype=np.int32)
    np.cumsum(lens, out=offs[1:])
    codes = rng.integers(0, k, size=int(offs[-1])).astype(np.uint8)
    codes[0] = k - 1
    image, b, nwords = _native.pack_image(codes, offs)
    assert b == bits
    assert np.array_equal(unpack_image(image, b, nwords, np.diff(offs)), codes)
    # DNA: 16 codes per word, every sequence 16-byte aligned
    if bits == 2:
        assert nwords == int(sum(((int(x) + 15) // 16 + 3) // 4 * 4 for x in lens))


@needs_lib
def test_alphabet_mismatch_and_corruption(tmp_path):
    enc = funnel(["ACGT", "GG"], schemes.DNA)
    p = str(tmp_path / "db")
    save_db(enc, p)
    with pytest.raises(EncodeError):
        load_db(p, schemes.BLOSUM62)
    np.array([0, 4, 99], dtype="<i4").tofile(tmp_path / "db" / "offsets.i32")
    with pytest.raises(EncodeError):
        load_db(p)
    save_db(enc, p)
    with open(tmp_path / "db" / "image.bin", "ab") as fh:  # a truncated or padded image
        fh.write(b"\0")
    with pytest.raises(EncodeError):
        load_db(p)


@needs_lib
def test_empty_set(tmp_path):
    enc = funnel([], schemes.DNA)
    save_db(enc, str(tmp_path / "e"))
    back = load_db(str(tmp_path / "e"))
    assert back.n == 0 and back.offsets.tolist() == [0] and back.codes.size == 0


def test_first_format_still_loads(tmp_path):
    enc = funnel({"a": "ACGT", "b": "GGA"}, schemes.DNA)
    p = tmp_path / "old"
    p.mkdir()
    enc.codes.astype(np.uint8).tofile(p / "codes.u8")
    enc.offsets.astype("<i4").tofile(p / "offsets.i32")
    (p / "ids.txt").write_text("a\nb")
    (p / "meta.json").write_text(json.dumps({"format": 1, "n": 2, "residues": 7,
                                             "alphabet": enc.alphabet, "scheme": None}))
    back = load_db(str(p), schemes.DNA)
    assert isinstance(back, Encoded) and back.codes.tolist() == enc.codes.tolist()


@pytest.mark.gpu
@pytest.mark.parametrize("scheme,alpha", [(schemes.DNA, "ACGT"), (schemes.BLOSUM62, "ARNDCQEGHILKMFPSTWYV")])
def test_index_from_loaded_db(tmp_path, scheme, alpha):
    rng = np.random.default_rng(1)
    refs = ["".join(rng.choice(list(alpha), int(rng.integers(50, 300)))) for _ in range(40)]
    qs = ["".join(rng.choice(list(alpha), int(rng.integers(50, 300)))) for _ in range(5)]
    save_db(funnel(refs, scheme, id_prefix="r"), str(tmp_path / "db"), scheme)
    al = Aligner(scheme).index(load_db(str(tmp_path / "db"), scheme))
    got = al.score_cross(qs)
    want = oracle.score_cross(funnel(qs, scheme), funnel(refs, scheme), scheme)
    assert np.array_equal(got.astype(np.int64), want)
    assert al.reference_ids == [f"r{i}" for i in range(40)]
    tk = al.top_k(qs, k=3)
    idx, sc = oracle.topk_stable(want, 3)
    assert np.array_equal(tk.topk_idx, idx) and np.array_equal(tk.topk_scores, sc)
