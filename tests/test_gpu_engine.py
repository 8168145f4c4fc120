"""Engine behaviour on the GPU: plans recorded on a key's second call and replayed as CUDA
graphs afterwards, plan eviction, the plain (one-batch-per-call) form, and stats -- every
result checked against the oracle."""
import numpy as np
import pytest

import oracle
from gpusw_b200 import Aligner, Scheme, _native, schemes
from gpusw_b200.encode import funnel
from tests._util import rand_seqs

pytestmark = pytest.mark.gpu


def _sets(seed, nq=21, nr=300, alpha="ACGT", lo=20, hi=400):
    rng = np.random.default_rng(seed)
    return rand_seqs(rng, nq, lo, hi, alpha), rand_seqs(rng, nr, lo, hi, alpha)


def test_graph_replay_cross_topk_pairs_bitexact():
    qs, rs = _sets(1)
    sch = schemes.DNA
    al = Aligner(sch).index(rs).set_queries(qs)
    want = oracle.score_cross(funnel(qs, sch), funnel(rs, sch), sch)
    # first call runs eagerly, the second records the plan as a graph, the next ones replay it
    for _ in range(4):
        assert np.array_equal(al.score_cross().astype(np.int64), want)
    idx, sc = oracle.topk_stable(want, 7)
    for _ in range(4):
        tk = al.top_k(k=7)
        assert np.array_equal(tk.topk_idx, idx) and np.array_equal(tk.topk_scores, sc)
    qi = np.arange(21) % 21
    rj = (np.arange(21) * 7) % 300
    for _ in range(4):
        got = al.score_pairs(qi, rj)
        assert got.astype(np.int64).tolist() == [int(want[i, j]) for i, j in zip(qi, rj)]
    st = _native.context(0).stats()
    assert st.last_launches > 0 and st.last_kernel_ms > 0


def test_plan_eviction_and_many_keys():
    qs, rs = _sets(2, nq=9, nr=120)
    sch = schemes.DNA
    al = Aligner(sch).index(rs).set_queries(qs)
    want = oracle.score_cross(funnel(qs, sch), funnel(rs, sch), sch)
    for k in (1, 2, 3, 4, 5, 6, 1, 2):  # more keys than cached plans
        tk = al.top_k(k=k)
        idx, sc = oracle.topk_stable(want, k)
        assert np.array_equal(tk.topk_idx, idx) and np.array_equal(tk.topk_scores, sc)


def test_scheme_change_invalidates_plans():
    qs, rs = _sets(3, nq=6, nr=50)
    a = Aligner(schemes.DNA).index(rs).set_queries(qs)
    b = Aligner(schemes.DNA_GLOBAL).index(rs).set_queries(qs)
    for _ in range(2):
        for al, sch in ((a, schemes.DNA), (b, schemes.DNA_GLOBAL)):
            want = oracle.score_cross(funnel(qs, sch), funnel(rs, sch), sch)
            assert np.array_equal(al.score_cross().astype(np.int64), want)


@pytest.mark.parametrize("name,alpha", [("dna", "ACGT"), ("blosum62", "ARNDCQEGHILKMFPSTWYV")])
def test_plain_form_equals_batched(name, alpha):
    sch = schemes.DNA if name == "dna" else schemes.BLOSUM62
    qs, rs = _sets(4, nq=37, nr=211, alpha=alpha, lo=5, hi=1300)
    ctx = _native.context(0)
    al = Aligner(sch).index(rs).set_queries(qs)
    batched = al.top_k(k=10)
    full = al.score_cross()
    try:
        ctx.set_options(plain=True)
        plain = al.top_k(k=10)
        plain_full = al.score_cross()
        plain_pairs = al.score_pairs(np.arange(37), np.arange(37))
    finally:
        ctx.set_options(plain=False)
    want = oracle.score_cross(funnel(qs, sch), funnel(rs, sch), sch)
    assert np.array_equal(full.astype(np.int64), want)
    assert np.array_equal(plain_full.astype(np.int64), want)
    assert np.array_equal(plain.topk_idx, batched.topk_idx)
    assert np.array_equal(plain.topk_scores, batched.topk_scores)
    assert plain_pairs.astype(np.int64).tolist() == [int(want[i, i]) for i in range(37)]


def test_memory_budget_blocks_topk():
    qs, rs = _sets(5, nq=40, nr=500)
    sch = schemes.DNA
    ctx = _native.context(0)
    al = Aligner(sch).index(rs).set_queries(qs)
    try:
        ctx.set_options(plain=False, mem_budget=500 * 4 * 7)  # 7 query rows per block
        tk = al.top_k(k=5)
    finally:
        ctx.set_options(plain=False, mem_budget=0)
    want = oracle.score_cross(funnel(qs, sch), funnel(rs, sch), sch)
    idx, sc = oracle.topk_stable(want, 5)
    assert np.array_equal(tk.topk_idx, idx) and np.array_equal(tk.topk_scores, sc)


def test_overflow_rescore_through_graph_replay():
    sch = Scheme(mode="local", match=300, mismatch=-7, gap_open=-9, gap_extend=-4)
    rng = np.random.default_rng(8)
    base = rand_seqs(rng, 1, 150, 151, "ACGT")[0]
    qs = [base, base[:30]] + rand_seqs(rng, 5, 1, 150, "ACGT")
    rs = [base] + rand_seqs(rng, 30, 1, 200, "ACGT")
    al = Aligner(sch).index(rs).set_queries(qs)
    want = oracle.score_cross(funnel(qs, sch), funnel(rs, sch), sch)
    assert want.max() > 32767
    for _ in range(3):
        assert np.array_equal(al.score_cross().astype(np.int64), want)
        tk = al.top_k(k=3)
        idx, sc = oracle.topk_stable(want, 3)
        assert np.array_equal(tk.topk_idx, idx) and np.array_equal(tk.topk_scores, sc)


def test_autotune_table_and_results_unchanged():
    qs, rs = _sets(6, nq=30, nr=200, alpha="ARNDCQEGHILKMFPSTWYV", lo=10, hi=1500)
    sch = schemes.BLOSUM62
    ctx = _native.context(0)
    al = Aligner(sch).index(rs).set_queries(qs)
    ctx.set_scheme(sch)
    table = ctx.autotune(2)
    assert len(table) >= 10 and all(t > 0 for t in table)
    want = oracle.score_cross(funnel(qs, sch), funnel(rs, sch), sch)
    assert np.array_equal(al.score_cross().astype(np.int64), want)
    try:
        ctx.set_options(autotune=False, graphs=False)
        assert np.array_equal(al.score_cross().astype(np.int64), want)
    finally:
        ctx.set_options()


@pytest.mark.parametrize("name,alpha", [("dna", "ACGT"), ("blosum62", "ARNDCQEGHILKMFPSTWYV")])
def test_overlapping_shape_launches_with_multipass(name, alpha):
    """A call whose query pairs span many streaming-kernel shapes, several of them multi-pass
    (columns beyond 1,024), with enough references to be planned for throughput: its shape
    launches run on several streams at once, each multi-pass launch with its own boundary
    strips. Scores and top-k equal the oracle eagerly, on the recording call and on replay."""
    sch = Scheme.preset(name)
    rng = np.random.default_rng(71)
    qs = rand_seqs(rng, 40, 10, 2600, alpha)
    rs = rand_seqs(rng, 4000, 20, 600, alpha)
    al = Aligner(sch).index(rs).set_queries(qs)
    want = oracle.score_cross(funnel(qs, sch), funnel(rs, sch), sch)
    idx, sc = oracle.topk_stable(want, 7)
    for _ in range(3):  # eager, eager + recorded, graph replay
        assert np.array_equal(al.score_cross().astype(np.int64), want)
        tk = al.top_k(k=7)
        assert np.array_equal(tk.topk_idx, idx) and np.array_equal(tk.topk_scores, sc)
    assert al._ctx().stats().last_launches >= 3


def test_small_calls_latency_shapes():
    """Calls too small to fill the GPU take the latency-planned shapes (few passes of narrow
    register strips): every column length, including multi-pass ones, stays exact."""
    rng = np.random.default_rng(72)
    for lo, hi, nq, nr in [(1, 90, 5, 7), (80, 200, 32, 128), (900, 2300, 3, 9)]:
        qs = rand_seqs(rng, nq, lo, hi, "ACGT")
        rs = rand_seqs(rng, nr, lo, hi, "ACGT")
        for dtype in ("auto", "int32"):
            sch = schemes.DNA.replace(dtype=dtype)
            got = Aligner(sch).index(rs).set_queries(qs).score_cross()
            want = oracle.score_cross(funnel(qs, sch), funnel(rs, sch), sch)
            assert np.array_equal(got.astype(np.int64), want)


def test_global_cross_multi_shape_bins():
    """Global and semiglobal cross products run on the pairs kernel in cross mode: pairs of
    many column lengths land in several bins (one multi-pass) whose launches overlap."""
    rng = np.random.default_rng(73)
    qs = rand_seqs(rng, 24, 5, 1300, "ACGT")
    rs = rand_seqs(rng, 150, 5, 700, "ACGT")
    for sch in (schemes.DNA.replace(mode="global"), schemes.DNA_SEMIGLOBAL):
        al = Aligner(sch).index(rs).set_queries(qs)
        want = oracle.score_cross(funnel(qs, sch), funnel(rs, sch), sch)
        for _ in range(3):
            assert np.array_equal(al.score_cross().astype(np.int64), want)


@pytest.mark.parametrize("sch", [schemes.DNA, schemes.BLOSUM62.replace(dtype="int32"),
                                 Scheme(mode="local", match=900, mismatch=-3, gap_open=-5, gap_extend=-2)],
                         ids=["dna-int16", "blosum62-int32", "int16-overflow"])
def test_one_launch_option_equals_oracle(sch):
    """GPUSW_OPT_ONE_LAUNCH: every streaming shape of a call (single- and multi-pass, query
    lengths 5..2,500) in one persistent launch. Scores and top-k equal the default launches;
    a 3,000-cell sample of the matrix equals the oracle."""
    alpha = "ACGT" if sch.eff_alphabet == "ACGT" else "ARNDCQEGHILKMFPSTWYV"
    rng = np.random.default_rng(61)
    qs = rand_seqs(rng, 200, 5, 2500, alpha)
    rs = rand_seqs(rng, 1000, 5, 400, alpha)
    if sch.match == 900:
        rs[:40] = [q[:300] for q in qs[:40]]  # identical stretches: int16 overflow, rescored
    ctx = _native.context(0)
    al = Aligner(sch).index(rs).set_queries(qs)
    default = al.score_cross()
    dtk = al.top_k(k=9)
    try:
        ctx.set_options(one_launch=True)
        for _ in range(3):  # eager, recorded, replayed
            assert np.array_equal(al.score_cross(), default)
        tk = al.top_k(k=9)
        assert ctx.stats().last_launches >= 1
    finally:
        ctx.set_options()
    assert np.array_equal(tk.topk_idx, dtk.topk_idx) and np.array_equal(tk.topk_scores, dtk.topk_scores)
    qi = rng.integers(0, 200, 3000).astype(np.int32)
    rj = rng.integers(0, 1000, 3000).astype(np.int32)
    qi[:40] = np.arange(40)
    rj[:40] = np.arange(40)
    want = oracle.score_pairs(funnel(qs, sch), funnel(rs, sch), qi, rj, sch)
    assert np.array_equal(default[qi, rj].astype(np.int64), want)
    if sch.match == 900:
        assert default.max() > 32767
