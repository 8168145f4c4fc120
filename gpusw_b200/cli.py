"""Command-line interface over the B200 engine: score FASTA files.

    python -m gpusw_b200 cross --queries q.fasta --refs r.fasta --scheme dna -o scores.csv
    python -m gpusw_b200 topk  --queries q.fasta --refs r.fasta --scheme blosum62 -k 5 [--coords]
    python -m gpusw_b200 pairs --queries q.fasta --refs r.fasta --scheme dna
    python -m gpusw_b200 info

The subcommand names, option names and CSV layouts are those of the reference package's
CLI (``src/gpusw/cli.py:28-143``), so scripts written for it run unchanged. The top-k
subcommand streams one query block at a time to the CSV and reports GCUPS on stderr; with
``--coords`` it adds the coordinates of each hit's best local alignment (the reference
recovers those by re-aligning on the CPU).
"""
from __future__ import annotations

import argparse
import csv
import os
import sys

from . import (
    __version__,
    _build_scheme,
    align_pairs,
    align_score,
    available_backends,
    available_matrices,
    gpu_available,
)
from .aligner import Aligner
from .encode import read_fasta


# Options shared by the scoring subcommands: (flags, argparse keywords). The option names
# and choices are the reference CLI's interface; everything else here is this package's.
_SCORING_OPTIONS = (
    (("--queries",), dict(required=True, metavar="FASTA", help="query records (FASTA, may be gzipped)")),
    (("--refs",), dict(required=True, metavar="FASTA", help="reference records (FASTA, may be gzipped)")),
    (("--scheme",), dict(default="dna", help="named scoring preset to start from")),
    (("--mode",), dict(choices=("local", "global", "semiglobal"), default=None,
                       help="alignment mode (default: the preset's)")),
    (("--matrix",), dict(default=None, help="bundled substitution matrix replacing the preset's")),
    (("--match",), dict(type=int, default=None, help="score of identical residues")),
    (("--mismatch",), dict(type=int, default=None, help="score of differing residues")),
    (("--gap-open",), dict(type=int, default=None, dest="gap_open",
                           help="cost of a gap's first residue (<= 0)")),
    (("--gap-extend",), dict(type=int, default=None, dest="gap_extend",
                             help="cost of each further gap residue (<= 0)")),
    (("--dtype",), dict(choices=("auto", "int16", "int32"), default=None,
                        help="score width policy (default: the preset's)")),
    (("--threads",), dict(type=int, default=128, help="accepted for compatibility; unused")),
    (("--backend",), dict(choices=("auto", "cuda", "metal"), default="auto",
                          help="accepted for compatibility; only CUDA runs")),
    (("--out", "-o"), dict(default="-", metavar="CSV", help="where to write the CSV (- for stdout)")),
)


def _add_options(p: argparse.ArgumentParser, options) -> None:
    for flags, kw in options:
        p.add_argument(*flags, **kw)


def _scheme_kw(args) -> dict:
    return dict(scheme=args.scheme, mode=args.mode, matrix=args.matrix, match=args.match,
                mismatch=args.mismatch, gap_open=args.gap_open, gap_extend=args.gap_extend,
                dtype=args.dtype)


class _Out:
    def __init__(self, path: str):
        self.fh = sys.stdout if path == "-" else open(path, "w", newline="")
        self.w = csv.writer(self.fh)

    def __enter__(self):
        return self.w

    def __exit__(self, *exc):
        if self.fh is not sys.stdout:
            self.fh.close()


def _cmd_cross(args) -> int:
    res = align_score(read_fasta(args.queries), read_fasta(args.refs), threads=args.threads,
                      backend=args.backend, **_scheme_kw(args))
    with _Out(args.out) as w:
        w.writerow(["query", "reference", "score"])
        for qi, qid in enumerate(res.query_ids):
            for rj, rid in enumerate(res.reference_ids):
                w.writerow([qid, rid, int(res.scores[qi, rj])])
    return 0


def _cmd_topk(args) -> int:
    qs = read_fasta(args.queries)
    if not os.path.exists(args.refs):
        raise FileNotFoundError(f"FASTA file not found: {args.refs}")
    al = Aligner(_build_scheme(**_scheme_kw(args)), threads=args.threads, backend=args.backend)
    al.index(args.refs)  # the path: read and encoded by the engine library's FASTA reader
    block = max(1, args.block)
    head = ["query", "rank", "reference", "score"]
    if args.coords:
        head += ["query_start", "query_end", "ref_start", "ref_end"]
    with _Out(args.out) as w:
        w.writerow(head)
        for b0 in range(0, len(qs), block):
            res = al.top_k(qs[b0:b0 + block], k=args.k)
            loc = al.locate_top(res) if args.coords else None
            for qi, (qid, hits) in enumerate(res.top_k(args.k)):
                for rank, (rid, sc) in enumerate(hits, 1):
                    row = [qid, rank, rid, sc]
                    if loc is not None:
                        row += [int(loc[key][qi, rank - 1])
                                for key in ("query_start", "query_end", "ref_start", "ref_end")]
                    w.writerow(row)
    sys.stderr.write(f"[gpusw_b200] {al.gcups:.1f} GCUPS\n")
    return 0


def _cmd_pairs(args) -> int:
    qs, rs = read_fasta(args.queries), read_fasta(args.refs)
    res = align_pairs(qs, rs, threads=args.threads, backend=args.backend, **_scheme_kw(args))
    with _Out(args.out) as w:
        w.writerow(["query", "reference", "score"])
        for k, sc in enumerate(res.scores):
            w.writerow([qs[k][0], rs[k][0], int(sc)])
    return 0


def _cmd_info(_args) -> int:
    print(f"gpusw_b200 {__version__}")
    backends = available_backends()
    print(f"GPU backends available: {', '.join(backends) if backends else 'none'}")
    if gpu_available():
        from . import _native

        ctx = _native.context(0)
        st = ctx.stats()
        print(f"  cuda device 0: context ready, {st.device_bytes} bytes held")
    print("bundled matrices:", ", ".join(sorted(available_matrices())))
    return 0


# Subcommands: name -> (one-line summary, handler, options of its own).
_COMMANDS = {
    "cross": ("score every query against every reference", _cmd_cross, ()),
    "topk": ("the k best references of each query, streamed in query blocks", _cmd_topk, (
        (("-k",), dict(type=int, default=5, help="hits kept per query")),
        (("--block",), dict(type=int, default=4096, help="queries scored per streamed block")),
        (("--coords",), dict(action="store_true",
                             help="append 0-based, end-exclusive start/end coordinates of each "
                                  "hit's best local alignment (local schemes; -1 for score 0)")),
    )),
    "pairs": ("score the i-th query against the i-th reference", _cmd_pairs, ()),
    "info": ("print the version, the CUDA device status and the bundled matrices", _cmd_info, None),
}


def _parser() -> argparse.ArgumentParser:
    ap = argparse.ArgumentParser(prog="gpusw_b200", description=__doc__,
                                 formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--version", action="version", version=f"gpusw_b200 {__version__}")
    cmds = ap.add_subparsers(dest="cmd", required=True, metavar="COMMAND")
    for name, (summary, handler, extra) in _COMMANDS.items():
        p = cmds.add_parser(name, help=summary, description=summary)
        if extra is not None:  # None: a command that scores nothing takes no scoring options
            _add_options(p, _SCORING_OPTIONS)
            _add_options(p, extra)
        p.set_defaults(func=handler)
    return ap


def main(argv=None) -> int:
    args = _parser().parse_args(argv)
    return args.func(args)


if __name__ == "__main__":  # pragma: no cover
    raise SystemExit(main())
