"""Serving: continuous batching over a resident reference set. Each request's top-k must
be the same alone and in the mix (bit-exact, against Aligner.top_k and the oracle);
admission refusals, cancellation and bounded waits behave as documented."""
import numpy as np
import pytest

import oracle
from gpusw_b200 import Aligner, schemes
from gpusw_b200.encode import funnel
from gpusw_b200.errors import GpuSWError
from gpusw_b200.server import CANCELLED, DONE, PENDING, RUNNING, Server
from tests._util import rand_seqs

pytestmark = pytest.mark.gpu


def _db(seed, n=400, lo=50, hi=600):
    rng = np.random.default_rng(seed)
    return rng, rand_seqs(rng, n, lo, hi, "ACGT")


def test_results_same_alone_and_in_the_mix():
    rng, refs = _db(1)
    sch = schemes.DNA
    requests = [rand_seqs(rng, int(rng.integers(1, 30)), 20, 500, "ACGT") for _ in range(24)]
    alone_al = Aligner(sch).index(refs)
    alone = [alone_al.top_k(q, k=7) for q in requests]
    srv_al = Aligner(sch).index(refs)
    with Server(srv_al, k=7, slots=2, max_batch_queries=64) as srv:
        ids = [srv.submit(q) for q in requests]  # all in flight together
        got = [srv.result(i, timeout=120) for i in ids]
        st = srv.stats()
    renc = funnel(refs, sch)
    for q, a, (idx, sc) in zip(requests, alone, got):
        assert np.array_equal(idx, a.topk_idx) and np.array_equal(sc, a.topk_scores)
        want = oracle.score_cross(funnel(q, sch), renc, sch)
        oi, osc = oracle.topk_stable(want, 7)
        assert np.array_equal(idx, oi) and np.array_equal(sc, osc)
    assert st["completed"] == 24 and st["batches"] >= 1
    assert st["p50_ms"] > 0 and st["p99_ms"] >= st["p50_ms"] and st["gcups"] > 0


def test_protein_requests_and_int16_rescore_in_server():
    rng = np.random.default_rng(2)
    alpha = "ARNDCQEGHILKMFPSTWYV"
    refs = rand_seqs(rng, 300, 30, 900, alpha)
    sch = schemes.BLOSUM62
    requests = [rand_seqs(rng, int(rng.integers(1, 12)), 30, 1500, alpha) for _ in range(10)]
    with Server(Aligner(sch).index(refs), k=10, slots=3, max_batch_queries=16) as srv:
        ids = [srv.submit(q) for q in requests]
        got = [srv.result(i, timeout=120) for i in ids]
    renc = funnel(refs, sch)
    for q, (idx, sc) in zip(requests, got):
        oi, osc = oracle.topk_stable(oracle.score_cross(funnel(q, sch), renc, sch), 10)
        assert np.array_equal(idx, oi) and np.array_equal(sc, osc)


def test_cancel_queue_full_budget_and_timeouts():
    rng, refs = _db(3, n=3000, lo=900, hi=1100)
    sch = schemes.DNA
    big = rand_seqs(rng, 512, 900, 1000, "ACGT")
    small = [rand_seqs(rng, 2, 50, 100, "ACGT") for _ in range(4)]
    with Server(Aligner(sch).index(refs), k=3, slots=1, max_batch_queries=512, max_pending=1) as srv:
        a = srv.submit(big)             # occupies the only slot for a while
        import time
        time.sleep(0.05)
        b = srv.submit(small[0])        # waits in the queue
        with pytest.raises(GpuSWError):  # queue (max_pending = 1) is full
            srv.submit(small[1])
        state, _, _ = srv.poll(b, timeout=0.01)
        assert state in (PENDING, RUNNING)
        srv.cancel(b)
        state, _, _ = srv.poll(b)
        assert state in (CANCELLED, RUNNING)
        idx, sc = srv.result(a, timeout=300)
        assert idx.shape == (512, 3)
        with pytest.raises(ValueError):  # released after its result was taken
            srv.poll(a)
        st = srv.stats()
        assert st["rejected"] >= 1
    with Server(Aligner(sch).index(refs), k=3, mem_budget=1 << 20) as tiny:
        with pytest.raises(GpuSWError):  # 512 x 3000 score block exceeds a 1 MiB budget
            tiny.submit(big)
        rid = tiny.submit(small[2])      # a small one still fits
        idx, _ = tiny.result(rid, timeout=60)
        assert idx.shape == (2, 3)


def test_large_request_runs_in_parts_and_small_ones_share_batches():
    """A request above one batch's work is cut into parts (here 1e12 cells per batch, or the
    backlog's share per slot when larger); the parts and the small requests queued behind it
    come back bit-identical to scoring them alone."""
    rng, refs = _db(4, n=3000, lo=950, hi=1050)       # ~3.0e6 reference residues
    sch = schemes.DNA
    big = rand_seqs(rng, 1200, 900, 1000, "ACGT")       # ~3.4e12 cells
    small = [rand_seqs(rng, int(rng.integers(1, 4)), 50, 300, "ACGT") for _ in range(5)]
    al = Aligner(sch).index(refs)
    want_big = al.top_k(big, k=4)
    want_small = [al.top_k(q, k=4) for q in small]
    with Server(Aligner(sch).index(refs), k=4, slots=2, max_batch_queries=2048,
                batch_cells=1e12) as srv:
        ib = srv.submit(big)
        ids = [srv.submit(q) for q in small]
        got_small = [srv.result(i, timeout=300) for i in ids]
        idx, sc = srv.result(ib, timeout=300)
        st = srv.stats()
    assert np.array_equal(idx, want_big.topk_idx) and np.array_equal(sc, want_big.topk_scores)
    for (i2, s2), w in zip(got_small, want_small):
        assert np.array_equal(i2, w.topk_idx) and np.array_equal(s2, w.topk_scores)
    assert st["completed"] == 6 and st["batches"] >= 2
