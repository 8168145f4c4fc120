"""Command-line interface over the B200 engine: score FASTA files.

    python -m gpusw_b200 cross --queries q.fasta --refs r.fasta --scheme dna -o scores.csv
    python -m gpusw_b200 topk  --queries q.fasta --refs r.fasta --scheme blosum62 -k 5 [--coords]
    python -m gpusw_b200 pairs --queries q.fasta --refs r.fasta --scheme dna
    python -m gpusw_b200 info

Same subcommands, options and CSV layouts as the reference package's CLI
(``src/gpusw/cli.py:28-143``); the top-k subcommand streams one query block at a time to
the CSV and reports GCUPS on stderr, and with ``--coords`` adds the coordinates of each
hit's best local alignment (the reference recovers those by re-aligning on the CPU).
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


def _scoring_args(p: argparse.ArgumentParser) -> None:
    p.add_argument("--queries", required=True, help="FASTA file of query sequences")
    p.add_argument("--refs", required=True, help="FASTA file of reference sequences")
    p.add_argument("--scheme", default="dna", help="preset name (dna, blosum62, ...)")
    p.add_argument("--mode", choices=["local", "global", "semiglobal"], default=None)
    p.add_argument("--matrix", default=None, help="named substitution matrix override")
    p.add_argument("--match", type=int, default=None)
    p.add_argument("--mismatch", type=int, default=None)
    p.add_argument("--gap-open", type=int, default=None, dest="gap_open")
    p.add_argument("--gap-extend", type=int, default=None, dest="gap_extend")
    p.add_argument("--dtype", choices=["auto", "int16", "int32"], default=None)
    p.add_argument("--threads", type=int, default=128)
    p.add_argument("--backend", choices=["auto", "cuda", "metal"], default="auto")
    p.add_argument("--out", "-o", default="-", help="output CSV path ('-' = stdout)")


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


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="gpusw_b200", description=__doc__,
                                 formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--version", action="version", version=f"gpusw_b200 {__version__}")
    sub = ap.add_subparsers(dest="cmd", required=True)
    pc = sub.add_parser("cross", help="all-pairs score matrix")
    _scoring_args(pc)
    pc.set_defaults(func=_cmd_cross)
    pt = sub.add_parser("topk", help="per-query top-k references")
    _scoring_args(pt)
    pt.add_argument("-k", type=int, default=5)
    pt.add_argument("--block", type=int, default=4096, help="queries per streamed block")
    pt.add_argument("--coords", action="store_true",
                    help="add 0-based, end-exclusive coordinates of each hit's best local "
                         "alignment (local schemes; -1 where the score is 0)")
    pt.set_defaults(func=_cmd_topk)
    pp = sub.add_parser("pairs", help="score queries vs refs 1:1")
    _scoring_args(pp)
    pp.set_defaults(func=_cmd_pairs)
    pi = sub.add_parser("info", help="environment / GPU info")
    pi.set_defaults(func=_cmd_info)
    args = ap.parse_args(argv)
    return args.func(args)


if __name__ == "__main__":  # pragma: no cover
    raise SystemExit(main())
