"""Regenerate the bundled substitution tables from the reference package's data files.

The scores must be identical to the reference's (``src/gpusw/data/matrices/*.txt``,
public NCBI/Biopython tables), so this script parses each of the reference's files and
writes the same alphabet and integers back out in NCBI text format with a short header of
our own. It needs a checkout of the reference package, whose matrix directory is given as
the argument or in the environment variable ``GPUSW_REFERENCE_MATRICES``:

    python gpusw_b200/data/make_matrices.py <reference checkout>/src/gpusw/data/matrices
"""
from __future__ import annotations

import os
import pathlib
import sys

HERE = pathlib.Path(__file__).resolve().parent / "matrices"


def _read(path: pathlib.Path) -> tuple[list[str], list[list[int]]]:
    header = None
    rows = []
    for line in path.read_text().splitlines():
        s = line.strip()
        if not s or s.startswith("#") or s.startswith("//"):
            continue
        f = s.split()
        if header is None:
            header = f
            continue
        rows.append([int(round(float(v))) for v in f[1:]])
    return header, rows


def main(src_dir: str) -> None:
    src = pathlib.Path(src_dir)
    for path in sorted(src.glob("*.txt")):
        syms, rows = _read(path)
        width = max(len(str(v)) for r in rows for v in r) + 2
        lines = [f"# {path.stem}: integer substitution scores, rows = reference residue,",
                 "# columns = query residue (NCBI text format)"]
        lines.append(" " + "".join(s.rjust(width) for s in syms))
        for sym, row in zip(syms, rows, strict=True):
            lines.append(sym + "".join(str(v).rjust(width) for v in row))
        (HERE / path.name).write_text("\n".join(lines) + "\n")
        print("wrote", HERE / path.name)


if __name__ == "__main__":
    src = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GPUSW_REFERENCE_MATRICES")
    if not src:
        raise SystemExit("usage: make_matrices.py <reference checkout>/src/gpusw/data/matrices")
    main(src)
