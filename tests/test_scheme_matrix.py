"""Scheme validation, substitution tables, the int16/int32 envelope and matrices, pinned
against the reference's outputs (tests/golden/tables.json) and its CPU tests
(tests/test_scheme_dtype.py, tests/test_matrix.py of the reference package)."""
import numpy as np
import pytest

from gpusw_b200 import Matrix, Scheme, available_matrices, schemes
from gpusw_b200.errors import OverflowRiskError, SchemeError
from tests._util import golden, scheme_from_spec

TABLES = golden("tables.json")


@pytest.mark.parametrize("name", sorted(TABLES["presets"]))
def test_preset_tables_match_reference(name):
    ref = TABLES["presets"][name]
    s = getattr(schemes, name)
    assert s.ns == ref["ns"] and s.eff_alphabet == ref["alphabet"]
    assert s.substitution_table().tolist() == ref["table"]
    assert scheme_from_spec(ref["scheme"]) == s


def test_resolve_dtype_matches_reference():
    for case in TABLES["dtype"]:
        s = scheme_from_spec(case["scheme"])
        assert s.resolve_dtype(case["maxq"], case["maxr"]) == case["dtype"]


def test_unknown_zero_table():
    assert Scheme(unknown="zero").substitution_table().tolist() == TABLES["unknown_zero"]


def test_defaults_and_validation():
    s = Scheme()
    assert (s.mode, s.match, s.mismatch, s.gap_open, s.gap_extend) == ("local", 2, -3, -5, -2)
    assert s.eff_alphabet == "ACGT" and s.ns == 5
    for bad in (dict(mode="banana"), dict(gap_open=5), dict(unknown="sometimes"),
                dict(dtype="int8"), dict(match=1.5), dict(alphabet="AAC")):
        with pytest.raises(SchemeError):
            Scheme(**bad)


def test_dtype_envelope():
    assert Scheme(match=2, mismatch=-3).resolve_dtype(500, 1500) == "int16"
    assert Scheme(match=2, mismatch=-3).resolve_dtype(20000, 20000) == "int32"
    with pytest.raises(OverflowRiskError):
        Scheme(match=2, mismatch=-3, dtype="int16").resolve_dtype(20000, 20000)
    assert Scheme(dtype="int32").resolve_dtype(10, 10) == "int32"
    assert Scheme(mode="global").resolve_dtype(20000, 20000) == "int32"


def test_table_hash_and_preset_lookup():
    assert Scheme(unknown="mismatch").table_hash() != Scheme(unknown="zero").table_hash()
    assert Scheme.preset("blosum62") is schemes.BLOSUM62
    with pytest.raises(SchemeError):
        Scheme.preset("nope")


def test_matrix_parsing_and_packing():
    m = Matrix.from_match_mismatch(2, -3, "ACGT")
    assert np.array_equal(np.diag(m.array), [2] * 4)
    assert (m.array[~np.eye(4, dtype=bool)] == -3).all()
    b = Matrix.named("BLOSUM62")
    assert np.array_equal(b.array, b.array.T) and b.array[b.alphabet.index("W")] [b.alphabet.index("W")] == 11
    assert Matrix.named("blosum-62").alphabet == b.alphabet
    with pytest.raises(SchemeError):
        Matrix.named("NOPE")
    t = Matrix.from_ncbi("# tiny\n  A  C\nA  1 -1\nC -1  1\n")
    assert t.alphabet == "AC" and t.array.tolist() == [[1, -1], [-1, 1]]
    with pytest.raises(SchemeError):
        Matrix.from_ncbi("  A C\nC 1 2\nA 3 4\n")
    _, pk = m.packed("mismatch")
    assert (pk[4, :] == -3).all() and (pk[:, 4] == -3).all()
    _, pz = m.packed("zero")
    assert (pz[4, :] == 0).all()
    assert m.hash() == Matrix.from_match_mismatch(2, -3, "ACGT").hash() != Matrix.from_match_mismatch(2, -4).hash()
    with pytest.raises(SchemeError):
        Matrix("ACGT", np.zeros((3, 3), dtype=int))
    assert {"BLOSUM62", "BLOSUM80", "PAM250", "EDNAFULL"} <= set(available_matrices())
