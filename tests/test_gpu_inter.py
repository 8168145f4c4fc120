"""The inter-sequence pairs kernel (pairs_inter_kernel: one thread scores two alignments as the
int16 halves of its registers): explicit int16 pairs of queries up to 160 residues or of 193 to 224 go to it
when the call has enough of them. Every case is checked against the team kernels (the same
call with the kernel switched off) on all pairs and against the C oracle on a sample, across
modes and free-end flags, strip boundaries (1..224 columns), uneven references, empty
sequences, sentinel codes in references, and calls that mix both kernels."""
import numpy as np
import pytest

import oracle
from gpusw_b200 import Scheme, _native, schemes
from gpusw_b200.encode import Encoded

pytestmark = pytest.mark.gpu

# The kernel is used when the items' work is at least twice the largest item's on every
# resident thread (148 SMs x 512 threads here): the sizes below clear that with a margin.


def _set(rng, n, lo, hi, k=4, empty=0.0):
    lens = rng.integers(lo, hi + 1, size=n)
    lens[rng.random(n) < empty] = 0
    offs = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(lens, out=offs[1:])
    return rng.integers(0, k, size=int(offs[-1])).astype(np.uint8), offs.astype(np.int32)


def _enc(codes, offs):
    return Encoded(codes, offs, list(range(offs.shape[0] - 1)), np.diff(offs).astype(np.int32), "ACGT")


def _run(sch, q, r, qi, rj, sample=3000, expect_inter=True):
    ctx = _native.context(0)
    with ctx.lock:
        ctx.set_scheme(sch)
        qd, rd = ctx.upload(*q), ctx.upload(*r)
        try:
            got = [ctx.score_pairs(qd, rd, qi, rj, "auto") for _ in range(3)]  # eager, recorded, replayed
            items = ctx.stats().last_inter_items
            ctx.set_options(inter=False)
            team = ctx.score_pairs(qd, rd, qi, rj, "auto")
            assert ctx.stats().last_inter_items == 0
        finally:
            ctx.set_options()
            ctx.free(qd)
            ctx.free(rd)
    assert (items > 0) == expect_inter
    for g in got:
        assert np.array_equal(g, team)
    idx = np.linspace(0, len(qi) - 1, min(sample, len(qi))).astype(np.int64)
    want = oracle.score_pairs(_enc(*q), _enc(*r), qi[idx], rj[idx], sch)
    assert np.array_equal(got[0][idx].astype(np.int64), want)
    return got[0], items


MODES = [schemes.DNA, schemes.DNA_GLOBAL, schemes.DNA_SEMIGLOBAL,
         schemes.DNA_SEMIGLOBAL.replace(free_end_gaps_ref=False),
         schemes.DNA_SEMIGLOBAL.replace(free_end_gaps_query=False)]


@pytest.mark.parametrize("sch", MODES, ids=["local", "global", "semi", "semi-fq", "semi-fr"])
def test_inter_uniform_short_pairs(sch):
    rng = np.random.default_rng(70)
    n = 400_001
    q, r = _set(rng, n, 60, 64), _set(rng, n, 70, 90)
    idx = np.arange(n, dtype=np.int32)
    _, items = _run(sch, q, r, idx, rng.permutation(n).astype(np.int32))
    assert items >= n // 2


@pytest.mark.parametrize("lo,hi", [(1, 8), (29, 36), (95, 128), (190, 224)],
                         ids=["1-8", "29-36", "95-128", "190-224"])
def test_inter_strip_widths_and_ends(lo, hi):
    """Every last-strip width (1..32 columns, 1..7 strips); references of 100..150 rows and
    0.5 % empty queries and references."""
    rng = np.random.default_rng(71 + lo)
    n = 900_077
    q, r = _set(rng, n, lo, hi, empty=0.005), _set(rng, n, 100, 150, empty=0.005)
    qi = np.arange(n, dtype=np.int32)
    rj = rng.integers(0, n, size=n).astype(np.int32)
    for sch in (schemes.DNA_SEMIGLOBAL, schemes.DNA_GLOBAL, schemes.DNA):
        _run(sch, q, r, qi, rj, sample=1500)


def test_inter_sentinel_rows_and_custom_scores():
    """References with the sentinel code (N), a scheme whose mismatch and gap values differ."""
    rng = np.random.default_rng(72)
    n = 600_005
    q, r = _set(rng, n, 40, 50), _set(rng, n, 40, 60, k=5)
    idx = np.arange(n, dtype=np.int32)
    sch = Scheme(mode="semiglobal", match=5, mismatch=-4, gap_open=-7, gap_extend=-1,
                 free_end_gaps_query=False)
    _run(sch, q, r, idx, idx)
    _run(Scheme(mode="local", match=3, mismatch=-2, gap_open=-4, gap_extend=-3), q, r, idx, idx)


def test_inter_mixed_call_and_routing():
    """Short alignments on the inter kernel, long ones on the team kernels, in one call; a call
    too small to keep every thread busy, and queries with sentinel codes, stay on the teams."""
    rng = np.random.default_rng(73)
    n = 1_000_000
    q, r = _set(rng, n, 20, 120), _set(rng, n, 60, 120)
    ql = np.diff(q[1]).copy()
    long_q = _set(rng, 20_000, 225, 400)
    codes = np.concatenate([q[0], long_q[0]])
    offs = np.concatenate([q[1], long_q[1][1:] + q[1][-1]]).astype(np.int32)
    qi = np.arange(n + 20_000, dtype=np.int32)
    rj = rng.integers(0, n, size=n + 20_000).astype(np.int32)
    got, items = _run(schemes.DNA_SEMIGLOBAL, (codes, offs), r, qi, rj)
    assert 0 < items < (n + 20_000) // 2 + 1 and ql.max() <= 128
    small = np.arange(5000, dtype=np.int32)
    _run(schemes.DNA_SEMIGLOBAL, q, r, small, small, expect_inter=False)
    qn = (q[0].copy(), q[1])
    qn[0][::97] = 4  # sentinel codes in the queries: not a 2-bit set
    idx = np.arange(n, dtype=np.int32)
    _run(schemes.DNA, qn, r, idx, idx, expect_inter=False)
