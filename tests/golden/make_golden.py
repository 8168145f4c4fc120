"""Generate the golden fixtures of tests/golden/ from the reference package itself.

Runs only where a checkout of the reference package is available: it imports ``gpusw``
(pure NumPy) from the checkout's ``src`` directory, given as the first argument or in the
environment variable ``GPUSW_REFERENCE_SRC``, and only reads it. The outputs are committed so that the tests
-- on machines without the reference -- compare against numbers the reference produced:

* scores.json   : ``cpu_reference_score`` / ``cpu_reference_matrix`` on seeded random sets
                  for the nine schemes of the reference's GPU parity tests, edge-case sets,
                  larger pairs, and the known anchors of its tests;
* tables.json   : ``Scheme.substitution_table()`` and ``resolve_dtype`` of the presets and
                  of the scheme variants used in the tests;
* encode.json   : ``funnel`` codes/offsets/ids for the accepted input forms;
* topk.json     : ``AlignResult.top_k`` on score matrices with ties.

    python tests/golden/make_golden.py <reference checkout>/src
"""
from __future__ import annotations

import json
import os
import pathlib
import sys

import numpy as np



def _ref_src() -> str:
    src = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GPUSW_REFERENCE_SRC")
    if not src:
        raise SystemExit("usage: make_golden.py <reference checkout>/src "
                         "(or set GPUSW_REFERENCE_SRC)")
    return src


OUT = pathlib.Path(__file__).resolve().parent


def rand_seqs(rng, n, lo, hi, alphabet):
    a = np.array(list(alphabet))
    return ["".join(rng.choice(a, int(rng.integers(lo, hi)))) for _ in range(n)]


def scheme_spec(s):
    return {"mode": s.mode, "match": s.match, "mismatch": s.mismatch, "gap_open": s.gap_open,
            "gap_extend": s.gap_extend, "matrix": s.matrix.name if s.matrix is not None else None,
            "alphabet": s.alphabet, "free_end_gaps_query": s.free_end_gaps_query,
            "free_end_gaps_ref": s.free_end_gaps_ref, "unknown": s.unknown,
            "case_insensitive": s.case_insensitive, "dtype": s.dtype}


def main() -> None:
    sys.path.insert(0, _ref_src())
    import gpusw
    from gpusw import Matrix, Scheme, schemes
    from gpusw.encode import funnel
    from gpusw.reference import cpu_reference_matrix, cpu_reference_score

    named = {
        "dna_local": (Scheme(mode="local"), "ACGTN"),
        "dna_global": (Scheme(mode="global"), "ACGT"),
        "dna_semi_qr": (Scheme(mode="semiglobal"), "ACGT"),
        "dna_semi_q": (Scheme(mode="semiglobal", free_end_gaps_query=True, free_end_gaps_ref=False), "ACGT"),
        "dna_semi_r": (Scheme(mode="semiglobal", free_end_gaps_query=False, free_end_gaps_ref=True), "ACGT"),
        "dna_semi_none": (Scheme(mode="semiglobal", free_end_gaps_query=False, free_end_gaps_ref=False), "ACGT"),
        "ednafull_global": (Scheme(mode="global", matrix=Matrix.named("EDNAFULL"), gap_open=-10, gap_extend=-1), "ACGTN"),
        "blosum62_local": (Scheme(mode="local", matrix=Matrix.named("BLOSUM62"), gap_open=-11, gap_extend=-1), "ARNDCQEGHILKMFPSTWYV"),
        "blosum62_global": (Scheme(mode="global", matrix=Matrix.named("BLOSUM62"), gap_open=-11, gap_extend=-1), "ARNDCQEGHILKMFPSTWYVX"),
        "protein_semiglobal": (Scheme(mode="semiglobal", matrix=Matrix.named("BLOSUM62"), gap_open=-11, gap_extend=-1), "ARNDCQEGHILKMFPSTWYV"),
        "dna_open_gt_extend": (Scheme(mode="global", gap_open=-1, gap_extend=-4), "ACGT"),
        "dna_zero_unknown": (Scheme(mode="local", unknown="zero"), "ACGTN"),
        "dna_linear_gap": (Scheme(mode="semiglobal", gap_open=-3, gap_extend=-3), "ACGT"),
    }
    scores = {"cross": {}, "edges": {}, "pairs": {}, "anchors": []}
    for seed, (name, (sch, alpha)) in enumerate(named.items()):
        rng = np.random.default_rng(1000 + seed)
        qs = rand_seqs(rng, 6, 0, 40, alpha)
        rs = rand_seqs(rng, 9, 0, 48, alpha)
        scores["cross"][name] = {"scheme": scheme_spec(sch), "queries": qs, "refs": rs,
                                 "scores": cpu_reference_matrix(qs, rs, sch).tolist()}
        c0 = alpha[0]
        eq = ["", c0, c0 * 30, "".join(alpha[:4]), alpha[:1]]
        er = ["", c0, "".join(reversed(alpha)) * 2, c0 * 25]
        scores["edges"][name] = {"scheme": scheme_spec(sch), "queries": eq, "refs": er,
                                 "scores": cpu_reference_matrix(eq, er, sch).tolist()}
        rng = np.random.default_rng(2000 + seed)
        pq = rand_seqs(rng, 24, 1, 140, alpha)
        pr = rand_seqs(rng, 24, 1, 160, alpha)
        scores["pairs"][name] = {"scheme": scheme_spec(sch), "queries": pq, "refs": pr,
                                 "scores": [int(cpu_reference_score(q, r, sch)) for q, r in zip(pq, pr)]}
    anchors = [
        ("ACGT", "ACT", Scheme(mode="local")),
        ("ACGTAC", "ACAC", Scheme(mode="global")),
        ("ACGT", "TTACGTTT", Scheme(mode="semiglobal", free_end_gaps_query=True, free_end_gaps_ref=False)),
        ("ACGTACGTAC", "ACGTACGTAC", Scheme()),
        ("ACGTACGTAC", "TTACGTACGTACTT", Scheme()),
        ("ACGTACGT", "ACGT", schemes.DNA),
        ("AC", "TTACTT", schemes.DNA.replace(mode="semiglobal")),
        ("AC", "TTACTT", schemes.DNA.replace(mode="global")),
        ("ACGT" * 15, "ACGT" * 15, Scheme(mode="local", match=1000, mismatch=-3, gap_open=-5, gap_extend=-2)),
        ("ACGTAC" * 5, "ACGTAC" * 5, Scheme(mode="local", match=1000, mismatch=-3, gap_open=-5, gap_extend=-2)),
        ("AAAA", "TTTT", Scheme(mode="local", match=1000, mismatch=-3, gap_open=-5, gap_extend=-2)),
        ("ACGT" * 15, "ACGT" * 15, Scheme(mode="global", match=1000, mismatch=-3, gap_open=-5, gap_extend=-2)),
        ("ACGT", "ACGT", schemes.DNA), ("TTTT", "TTTA", schemes.DNA),
        ("ACGTACGTACGT", "ACGTACGTACGT", schemes.DNA), ("ACGTACGTACGT", "TACGGACGTA", schemes.DNA),
        ("ACGGACGT", "TACGGACGTA", schemes.DNA), ("ACGTACGT", "ACGTACGT", schemes.DNA),
    ]
    for q, r, sch in anchors:
        scores["anchors"].append({"query": q, "ref": r, "scheme": scheme_spec(sch),
                                  "score": int(cpu_reference_score(q, r, sch))})
    (OUT / "scores.json").write_text(json.dumps(scores))

    tables = {"presets": {}, "dtype": []}
    for nm in schemes.__all__:
        s = getattr(schemes, nm)
        tables["presets"][nm] = {"scheme": scheme_spec(s), "ns": s.ns, "alphabet": s.eff_alphabet,
                                 "table": s.substitution_table().tolist()}
    for sch, maxq, maxr in [(Scheme(match=2, mismatch=-3), 500, 1500), (Scheme(match=2, mismatch=-3), 20000, 20000),
                            (Scheme(mode="global"), 20000, 20000), (Scheme(dtype="int32"), 10, 10),
                            (schemes.BLOSUM62, 2000, 2000), (schemes.DNA, 253, 1600),
                            (schemes.DNA_SEMIGLOBAL, 150, 200), (schemes.BLOSUM62_GLOBAL, 2000, 2000),
                            (Scheme(mode="local", match=1000), 60, 60)]:
        tables["dtype"].append({"scheme": scheme_spec(sch), "maxq": maxq, "maxr": maxr,
                                "dtype": sch.resolve_dtype(maxq, maxr)})
    tables["unknown_zero"] = Scheme(unknown="zero").substitution_table().tolist()
    (OUT / "tables.json").write_text(json.dumps(tables))

    dna = Scheme(mode="local")
    cases = {
        "list": ["ACGT", "TTGGCC", "A"], "lower": ["acgt", "AcGt"], "empty": ["", "ACGT", ""],
        "dict": {"x": "ACGN", "y": "ttt"}, "pairs": [["a", "ACGT"], ["b", "GG"]],
        "fasta_text": ">s1 desc\nACGT\nAC\n>s2\nTT\n", "raw": "ACGTNX", "unicode": ["ACGµT", "ßAC"],
    }
    enc = {}
    for k, v in cases.items():
        e = funnel(v, dna)
        enc[k] = {"input": v, "codes": e.codes.tolist(), "offsets": e.offsets.tolist(), "ids": list(e.ids)}
    e = funnel(b"ACG\xffT", dna)
    enc["bytes"] = {"input_latin1": "ACGÿT", "codes": e.codes.tolist(), "offsets": e.offsets.tolist(), "ids": list(e.ids)}
    cs = Scheme(mode="local", case_insensitive=False)
    e = funnel(["acgt", "ACgt"], cs)
    enc["case_sensitive"] = {"input": ["acgt", "ACgt"], "codes": e.codes.tolist(), "offsets": e.offsets.tolist(), "ids": list(e.ids)}
    (OUT / "encode.json").write_text(json.dumps(enc))

    from gpusw.result import AlignResult
    rng = np.random.default_rng(7)
    mats = [rng.integers(-3, 4, size=(5, 11)), np.zeros((2, 6), dtype=np.int64), rng.integers(0, 3, size=(4, 40))]
    topk = []
    for m in mats:
        res = AlignResult(m.astype(np.int32), [f"q{i}" for i in range(m.shape[0])],
                          [f"r{j}" for j in range(m.shape[1])], None)
        topk.append({"scores": m.tolist(), "k": 4, "top": res.top_k(4)})
    (OUT / "topk.json").write_text(json.dumps(topk))
    print("golden fixtures written by gpusw", gpusw.__version__)


if __name__ == "__main__":
    main()
