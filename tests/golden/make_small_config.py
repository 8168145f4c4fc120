"""Generate tests/golden/small_config.json from the reference package itself.

The small benchmark configuration -- 32 DNA queries x 128 references, lengths U[80, 200],
i.i.d. uniform ACGT (``gpusw_b200.workloads.small``, seed 0), the default 'dna' scheme in
local mode -- is scored in full by the reference's own ``cpu_reference_matrix`` (pure NumPy),
spread over a process pool. The sequences and the (32, 128) score matrix are written out, so
that the GPU test of that exact shape compares against numbers the reference produced.

Needs a checkout of the reference package: its ``src`` directory is the first argument or
the environment variable ``GPUSW_REFERENCE_SRC``; it is only read.

    python tests/golden/make_small_config.py <reference checkout>/src
"""
from __future__ import annotations

import json
import multiprocessing as mp
import os
import pathlib
import sys

import numpy as np

OUT = pathlib.Path(__file__).resolve().parent / "small_config.json"
ROOT = pathlib.Path(__file__).resolve().parents[2]


def _ref_src() -> str:
    src = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GPUSW_REFERENCE_SRC")
    if not src:
        raise SystemExit("usage: make_small_config.py <reference checkout>/src "
                         "(or set GPUSW_REFERENCE_SRC)")
    return src


def _row(args):
    src, q, refs = args
    sys.path.insert(0, src)
    from gpusw import schemes
    from gpusw.reference import cpu_reference_matrix

    return cpu_reference_matrix([q], refs, schemes.DNA)[0].tolist()


def main() -> None:
    src = _ref_src()
    sys.path.insert(0, str(ROOT))
    from gpusw_b200 import workloads

    wl = workloads.small()
    alpha = np.array(list("ACGT"))

    def texts(pair):
        codes, offs = pair
        return ["".join(alpha[codes[offs[i]:offs[i + 1]]]) for i in range(offs.shape[0] - 1)]

    qs, rs = texts(wl.queries), texts(wl.refs)
    with mp.get_context("spawn").Pool(os.cpu_count() or 1) as pool:
        scores = pool.map(_row, [(src, q, rs) for q in qs])
    sys.path.insert(0, src)
    import gpusw

    OUT.write_text(json.dumps({"scheme": "dna (local, 2/-3, gaps -5/-2)", "queries": qs,
                               "refs": rs, "scores": scores,
                               "made_by": f"gpusw {gpusw.__version__} cpu_reference_matrix"}))
    print("wrote", OUT)


if __name__ == "__main__":
    main()
