"""Persisted encoded sets: save/load round trip, memory mapping, validation; on a GPU an
Aligner indexes a loaded set directly and scores exactly as from the original input."""
import numpy as np
import pytest

import oracle
from gpusw_b200 import Aligner, schemes
from gpusw_b200.db import load_db, save_db
from gpusw_b200.encode import funnel
from gpusw_b200.errors import EncodeError


def test_round_trip(tmp_path):
    enc = funnel({"r1": "ACGTN", "r2": "", "r3": "ttgca"}, schemes.DNA)
    save_db(enc, str(tmp_path / "db"), schemes.DNA)
    back = load_db(str(tmp_path / "db"), schemes.DNA)
    assert back.ids == ["r1", "r2", "r3"]
    assert back.codes.tolist() == enc.codes.tolist()
    assert back.offsets.tolist() == enc.offsets.tolist()
    assert back.lengths.tolist() == [5, 0, 5]
    assert funnel(back, schemes.DNA) is back
    copy = load_db(str(tmp_path / "db"), mmap=False)
    assert copy.codes.tolist() == enc.codes.tolist()


def test_alphabet_mismatch_and_corruption(tmp_path):
    enc = funnel(["ACGT", "GG"], schemes.DNA)
    p = str(tmp_path / "db")
    save_db(enc, p)
    with pytest.raises(EncodeError):
        load_db(p, schemes.BLOSUM62)
    np.array([0, 4, 99], dtype="<i4").tofile(tmp_path / "db" / "offsets.i32")
    with pytest.raises(EncodeError):
        load_db(p)


def test_empty_set(tmp_path):
    enc = funnel([], schemes.DNA)
    save_db(enc, str(tmp_path / "e"))
    back = load_db(str(tmp_path / "e"))
    assert back.n == 0 and back.offsets.tolist() == [0]


@pytest.mark.gpu
def test_index_from_loaded_db(tmp_path):
    rng = np.random.default_rng(1)
    refs = ["".join(rng.choice(list("ACGT"), int(rng.integers(50, 300)))) for _ in range(40)]
    qs = ["".join(rng.choice(list("ACGT"), int(rng.integers(50, 300)))) for _ in range(5)]
    save_db(funnel(refs, schemes.DNA, id_prefix="r"), str(tmp_path / "db"), schemes.DNA)
    al = Aligner(schemes.DNA).index(load_db(str(tmp_path / "db"), schemes.DNA))
    got = al.score_cross(qs)
    want = oracle.score_cross(funnel(qs, schemes.DNA), funnel(refs, schemes.DNA), schemes.DNA)
    assert np.array_equal(got.astype(np.int64), want)
    assert al.reference_ids == [f"r{i}" for i in range(40)]
