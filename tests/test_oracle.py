"""The CPU oracle (tests' checker) pinned against the reference's own outputs.

The golden fixtures were produced by the reference package's ``cpu_reference_score`` /
``cpu_reference_matrix`` (tests/golden/make_golden.py); both oracle forms -- the pure-Python
port and the C restatement -- must reproduce them exactly.
"""
import numpy as np
import pytest

import oracle
from gpusw_b200.encode import funnel
from tests._util import golden, rand_seqs, scheme_from_spec

SCORES = golden("scores.json")


@pytest.mark.parametrize("kind", ["cross", "edges"])
@pytest.mark.parametrize("name", sorted(SCORES["cross"]))
def test_c_oracle_matches_reference_matrix(kind, name):
    case = SCORES[kind][name]
    sch = scheme_from_spec(case["scheme"])
    q = funnel(case["queries"], sch)
    r = funnel(case["refs"], sch)
    got = oracle.score_cross(q, r, sch)
    assert got.tolist() == case["scores"]


@pytest.mark.parametrize("name", sorted(SCORES["pairs"]))
def test_c_oracle_matches_reference_pairs(name):
    case = SCORES["pairs"][name]
    sch = scheme_from_spec(case["scheme"])
    q = funnel(case["queries"], sch)
    r = funnel(case["refs"], sch)
    idx = np.arange(q.n, dtype=np.int32)
    assert oracle.score_pairs(q, r, idx, idx, sch).tolist() == case["scores"]


@pytest.mark.parametrize("name", sorted(SCORES["edges"]))
def test_python_oracle_matches_reference_edges(name):
    case = SCORES["edges"][name]
    sch = scheme_from_spec(case["scheme"])
    for i, qs in enumerate(case["queries"]):
        for j, rs in enumerate(case["refs"]):
            assert oracle.score_py(qs, rs, sch) == case["scores"][i][j]


def test_anchors_both_oracles():
    for a in SCORES["anchors"]:
        sch = scheme_from_spec(a["scheme"])
        assert oracle.score_py(a["query"], a["ref"], sch) == a["score"]
        q, r = funnel([a["query"]], sch), funnel([a["ref"]], sch)
        assert int(oracle.score_cross(q, r, sch)[0, 0]) == a["score"]


def test_known_answers_of_reference_tests():
    # test_reference_oracle.py:89-94, test_gpu_bitexact.py:114-118, test_api.py:40-49,65-68
    vals = {(a["query"], a["ref"], a["scheme"]["mode"], a["scheme"]["match"]): a["score"]
            for a in SCORES["anchors"]}
    assert vals[("ACGT", "ACT", "local", 2)] == 4
    assert vals[("ACGTAC", "ACAC", "global", 2)] == 1
    assert vals[("ACGT", "TTACGTTT", "semiglobal", 2)] == 8
    assert vals[("ACGTACGTAC", "TTACGTACGTACTT", "local", 2)] == 20
    assert vals[("AC", "TTACTT", "semiglobal", 2)] == 4
    assert vals[("ACGT" * 15, "ACGT" * 15, "local", 1000)] == 60000


def test_c_oracle_equals_python_oracle_random():
    from gpusw_b200 import Matrix, Scheme
    rng = np.random.default_rng(11)
    for sch, alpha in [(Scheme(mode="local"), "ACGTN"), (Scheme(mode="global"), "ACGT"),
                       (Scheme(mode="semiglobal", free_end_gaps_query=False), "ACGT"),
                       (Scheme(mode="semiglobal", matrix=Matrix.named("BLOSUM62"), gap_open=-11,
                               gap_extend=-1), "ARNDCQEGHILKMFPSTWYV")]:
        qs = rand_seqs(rng, 5, 0, 30, alpha)
        rs = rand_seqs(rng, 5, 0, 30, alpha)
        c = oracle.score_cross(funnel(qs, sch), funnel(rs, sch), sch)
        py = [[oracle.score_py(q, r, sch) for r in rs] for q in qs]
        assert c.tolist() == py


def test_oracle_topk_matches_reference_order():
    for case in golden("topk.json"):
        m = np.asarray(case["scores"])
        idx, sc = oracle.topk_stable(m, case["k"])
        for qi, (qid, hits) in enumerate(case["top"]):
            assert [f"r{j}" for j in idx[qi]] == [h[0] for h in hits]
            assert sc[qi].tolist() == [h[1] for h in hits]
