"""Seeded synthetic workloads with the shapes and value distributions of the benchmark
configurations (the reference's own 16S/BV-BRC inputs are not available, so these stand in
for them). Every generator returns encoded sets -- ``(codes uint8, offsets int32)`` in the
scheme's alphabet -- so no string encoding sits between the generator and the engine.

* ``small``    : 32 queries x 128 refs, lengths U[80, 200], i.i.d. uniform ACGT, DNA local.
* ``sixteen_s``: 300 ancestors (GC ~0.53) -> refs mutated 1-15 % substitutions + 0.5 %
                 indels of length 1-3 (20,000 refs of ~1,400-1,600 nt); queries are 250-253
                 nt windows of mutated refs with 1 % more substitutions (2,000); local, k=5.
* ``protein``  : 4,096 x 100,000, lengths log-normal(median 350, sigma 0.7) clipped to
                 [30, 2000], residues i.i.d. from the Robinson & Robinson (1991) amino-acid
                 background frequencies; BLOSUM62 local -11/-1, k=10.
* ``pairs``    : 1,000,000 (read, window) pairs: 200 nt uniform windows, 150 nt reads cut
                 from them with 0.5-2 % substitutions and 0.1 % indels; DNA semiglobal.
* ``requests`` : the serving stream -- 1-512 queries per request (log-uniform count),
                 lengths U[50, 2000], made by the 16S mutation model.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import schemes
from .scheme import Scheme

__all__ = ["Workload", "small", "sixteen_s", "protein", "pairs", "requests", "by_name"]

# Robinson & Robinson (1991) background frequencies, in BLOSUM62's first 20 symbols'
# order ARNDCQEGHILKMFPSTWYV.
AA_BACKGROUND = np.array([0.07805, 0.05129, 0.04487, 0.05364, 0.01925, 0.04264, 0.06295, 0.07377,
                          0.02199, 0.05142, 0.09019, 0.05744, 0.02243, 0.03856, 0.05203, 0.07120,
                          0.05841, 0.01330, 0.03216, 0.06441])
GC_PROBS = np.array([0.235, 0.265, 0.265, 0.235])  # A C G T with GC ~ 0.53


@dataclass
class Workload:
    name: str
    scheme: Scheme
    queries: tuple[np.ndarray, np.ndarray]
    refs: tuple[np.ndarray, np.ndarray]
    k: int = 0
    pairs: tuple[np.ndarray, np.ndarray] | None = None
    seed: int = 0
    note: str = ""

    @property
    def nq(self) -> int:
        return self.queries[1].shape[0] - 1

    @property
    def nr(self) -> int:
        return self.refs[1].shape[0] - 1

    def cells(self) -> float:
        ql = np.diff(self.queries[1]).astype(np.float64)
        rl = np.diff(self.refs[1]).astype(np.float64)
        if self.pairs is not None:
            return float((ql[self.pairs[0]] * rl[self.pairs[1]]).sum())
        return float(ql.sum() * rl.sum())


def _pack(seqs: list[np.ndarray]) -> tuple[np.ndarray, np.ndarray]:
    lens = np.fromiter((len(s) for s in seqs), dtype=np.int64, count=len(seqs))
    offs = np.zeros(len(seqs) + 1, dtype=np.int64)
    np.cumsum(lens, out=offs[1:])
    if offs[-1] >= 2**31:
        raise ValueError("workload exceeds 2**31 residues")
    codes = np.concatenate(seqs).astype(np.uint8) if seqs else np.zeros(0, np.uint8)
    return codes, offs.astype(np.int32)


def _substitute(rng, seq: np.ndarray, rate: float, k: int = 4) -> np.ndarray:
    out = seq.copy()
    hit = rng.random(out.shape[0]) < rate
    # a different symbol: add 1..k-1 modulo k
    out[hit] = (out[hit] + rng.integers(1, k, size=int(hit.sum()))) % k
    return out


def _indels(rng, seq: np.ndarray, rate: float, probs: np.ndarray) -> np.ndarray:
    return _indels_at(rng, seq, np.flatnonzero(rng.random(seq.shape[0]) < rate), probs)


def _indels_at(rng, seq: np.ndarray, sites: np.ndarray, probs: np.ndarray) -> np.ndarray:
    """Insert or delete 1-3 residues (50/50) at each site."""
    n = seq.shape[0]
    if sites.size == 0:
        return seq
    parts = []
    prev = 0
    for s in sites:
        if s < prev:
            continue
        ln = int(rng.integers(1, 4))
        parts.append(seq[prev:s])
        if rng.random() < 0.5:  # insertion before s
            parts.append(rng.choice(len(probs), size=ln, p=probs).astype(np.uint8))
            prev = s
        else:  # deletion of ln residues
            prev = min(n, s + ln)
    parts.append(seq[prev:])
    return np.concatenate(parts)


def small(seed: int = 0) -> Workload:
    rng = np.random.default_rng(seed)
    q = [rng.integers(0, 4, size=int(rng.integers(80, 201))).astype(np.uint8) for _ in range(32)]
    r = [rng.integers(0, 4, size=int(rng.integers(80, 201))).astype(np.uint8) for _ in range(128)]
    return Workload("small", schemes.DNA.replace(dtype="int32"), _pack(q), _pack(r), k=5, seed=seed,
                    note="32 q x 128 r, U[80,200] i.i.d. ACGT, DNA local, int32")


def _mutated_refs(rng, n_refs: int, n_anc: int = 300, lo: int = 1400, hi: int = 1600):
    anc = [rng.choice(4, size=int(rng.integers(lo, hi + 1)), p=GC_PROBS).astype(np.uint8)
           for _ in range(n_anc)]
    refs = []
    for _ in range(n_refs):
        a = anc[int(rng.integers(0, n_anc))]
        s = _substitute(rng, a, float(rng.uniform(0.01, 0.15)))
        refs.append(_indels(rng, s, 0.005, GC_PROBS))
    return refs


def sixteen_s(seed: int = 1, n_queries: int = 2000, n_refs: int = 20000) -> Workload:
    rng = np.random.default_rng(seed)
    refs = _mutated_refs(rng, n_refs)
    qs = []
    for _ in range(n_queries):
        r = refs[int(rng.integers(0, n_refs))]
        ln = int(rng.integers(250, 254))
        st = int(rng.integers(0, max(1, r.shape[0] - ln + 1)))
        qs.append(_substitute(rng, r[st:st + ln], 0.01))
    return Workload("16s", schemes.DNA, _pack(qs), _pack(refs), k=5, seed=seed,
                    note=f"{n_queries} q (250-253 nt) x {n_refs} r (~1400-1600 nt) from 300 "
                         "ancestors; DNA local 2/-3/-5/-2, int16 with int32 rescoring, top-5")


def _lognormal_lengths(rng, n: int) -> np.ndarray:
    return np.clip(np.rint(rng.lognormal(np.log(350.0), 0.7, size=n)), 30, 2000).astype(np.int64)


def _protein_set(rng, n: int) -> tuple[np.ndarray, np.ndarray]:
    lens = _lognormal_lengths(rng, n)
    offs = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(lens, out=offs[1:])
    codes = rng.choice(20, size=int(offs[-1]), p=AA_BACKGROUND / AA_BACKGROUND.sum()).astype(np.uint8)
    return codes, offs.astype(np.int32)


def protein(seed: int = 2, n_queries: int = 4096, n_refs: int = 100000) -> Workload:
    rng = np.random.default_rng(seed)
    return Workload("protein", schemes.BLOSUM62, _protein_set(rng, n_queries),
                    _protein_set(rng, n_refs), k=10, seed=seed,
                    note=f"{n_queries} x {n_refs}, log-normal(350, 0.7) clipped [30,2000], "
                         "background residue frequencies; BLOSUM62 local -11/-1, top-10")


def pairs(seed: int = 3, n: int = 1_000_000) -> Workload:
    rng = np.random.default_rng(seed)
    windows = rng.integers(0, 4, size=(n, 200), dtype=np.uint8)
    starts = rng.integers(0, 51, size=n)
    reads = windows[np.arange(n)[:, None], starts[:, None] + np.arange(150)[None, :]]
    rate = rng.uniform(0.005, 0.02, size=n)[:, None]
    hit = rng.random(reads.shape) < rate
    reads = np.where(hit, (reads + rng.integers(1, 4, size=reads.shape, dtype=np.uint8)) % 4,
                     reads).astype(np.uint8)
    sites = rng.random(reads.shape) < 0.001
    seqs = list(reads)
    uni = np.full(4, 0.25)
    for i in np.flatnonzero(sites.any(axis=1)):
        seqs[i] = _indels_at(rng, reads[i], np.flatnonzero(sites[i]), uni)
    q = _pack(seqs)
    r = (windows.reshape(-1).copy(), (np.arange(n + 1, dtype=np.int64) * 200).astype(np.int32))
    idx = np.arange(n, dtype=np.int32)
    return Workload("pairs", schemes.DNA_SEMIGLOBAL.replace(dtype="int16"), q, r, pairs=(idx, idx),
                    seed=seed, note=f"{n} (150 nt read, 200 nt window) pairs, DNA semiglobal, int16")


def requests(seed: int = 4, n_requests: int = 64, max_queries: int = 512):
    """Serving stream: a list of encoded query sets (one per request)."""
    rng = np.random.default_rng(seed)
    anc = [rng.choice(4, size=2200, p=GC_PROBS).astype(np.uint8) for _ in range(300)]
    out = []
    for _ in range(n_requests):
        nq = int(np.clip(np.rint(np.exp(rng.uniform(0.0, np.log(max_queries)))), 1, max_queries))
        qs = []
        for _ in range(nq):
            a = anc[int(rng.integers(0, 300))]
            ln = int(rng.integers(50, 2001))
            st = int(rng.integers(0, a.shape[0] - ln + 1))
            s = _substitute(rng, a[st:st + ln], float(rng.uniform(0.01, 0.15)))
            qs.append(_indels(rng, s, 0.005, GC_PROBS))
        out.append(_pack(qs))
    return out


def by_name(name: str, **kw) -> Workload:
    return {"small": small, "16s": sixteen_s, "protein": protein, "pairs": pairs}[name](**kw)
