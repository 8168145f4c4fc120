"""CLI over the engine: argument parsing and info need no GPU; the scoring subcommands
produce the reference CLI's CSV layouts (src/gpusw/cli.py of the reference package)."""
import csv

import pytest

from gpusw_b200 import __version__
from gpusw_b200.cli import main


def _fasta(tmp_path, name, recs):
    p = tmp_path / name
    p.write_text("".join(f">{i}\n{s}\n" for i, s in recs))
    return str(p)


def _rows(path):
    with open(path) as fh:
        return list(csv.reader(fh))


def test_info_runs(capsys):
    assert main(["info"]) == 0
    out = capsys.readouterr().out
    assert __version__ in out and "bundled matrices:" in out and "BLOSUM62" in out


def test_missing_required_arg_exits_2():
    with pytest.raises(SystemExit) as e:
        main(["cross", "--refs", "r.fasta"])
    assert e.value.code == 2


def test_no_subcommand_exits():
    with pytest.raises(SystemExit):
        main([])


def test_missing_file_errors(tmp_path):
    r = _fasta(tmp_path, "r.fasta", [("ra", "ACGT")])
    with pytest.raises(FileNotFoundError):
        main(["cross", "--queries", str(tmp_path / "nope.fasta"), "--refs", r, "--scheme", "dna"])


@pytest.mark.gpu
def test_cli_cross_topk_pairs(tmp_path):
    q = _fasta(tmp_path, "q.fasta", [("qa", "ACGTACGT"), ("qb", "TTTT")])
    r = _fasta(tmp_path, "r.fasta", [("ra", "ACGTACGT"), ("rb", "ACGT")])
    out = str(tmp_path / "cross.csv")
    assert main(["cross", "--queries", q, "--refs", r, "--scheme", "dna", "-o", out]) == 0
    rows = _rows(out)
    assert rows[0] == ["query", "reference", "score"] and len(rows) == 5
    assert {(a, b): int(s) for a, b, s in rows[1:]}[("qa", "ra")] == 16
    r3 = _fasta(tmp_path, "r3.fasta", [("ra", "ACGTACGT"), ("rb", "TTTTTTTT"), ("rc", "ACGT")])
    out = str(tmp_path / "topk.csv")
    assert main(["topk", "--queries", q, "--refs", r3, "--scheme", "dna", "-k", "2", "-o", out,
                 "--block", "1"]) == 0
    rows = _rows(out)
    assert rows[0] == ["query", "rank", "reference", "score"] and len(rows) == 1 + 2 * 2
    assert rows[1][0] == "qa" and rows[1][2] == "ra"
    out = str(tmp_path / "topk_coords.csv")
    assert main(["topk", "--queries", q, "--refs", r3, "--scheme", "dna", "-k", "2", "-o", out,
                 "--coords"]) == 0
    rows = _rows(out)
    assert rows[0][4:] == ["query_start", "query_end", "ref_start", "ref_end"]
    assert rows[1][:4] == ["qa", "1", "ra", "16"] and rows[1][4:] == ["0", "8", "0", "8"]
    q2 = _fasta(tmp_path, "q2.fasta", [("qa", "ACGT"), ("qb", "TTTT")])
    r2 = _fasta(tmp_path, "r2.fasta", [("ra", "ACGT"), ("rb", "TTTA")])
    out = str(tmp_path / "pairs.csv")
    assert main(["pairs", "--queries", q2, "--refs", r2, "--scheme", "dna", "-o", out]) == 0
    assert [int(x[2]) for x in _rows(out)[1:]] == [8, 6]
