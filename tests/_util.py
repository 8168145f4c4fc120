"""Helpers shared by the tests: golden fixtures and scheme reconstruction."""
from __future__ import annotations

import json
import os

import numpy as np

from gpusw_b200 import Matrix, Scheme

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden(name: str):
    with open(os.path.join(GOLDEN, name)) as fh:
        return json.load(fh)


def scheme_from_spec(spec: dict) -> Scheme:
    kw = dict(spec)
    m = kw.pop("matrix")
    if m is not None and not m.startswith("match"):
        kw["matrix"] = Matrix.named(m)
    return Scheme(**kw)


def rand_seqs(rng, n, lo, hi, alphabet):
    a = np.array(list(alphabet))
    return ["".join(rng.choice(a, int(rng.integers(lo, hi)))) for _ in range(n)]
