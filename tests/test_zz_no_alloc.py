"""The no-allocation pairs entry point (gpusw_score_pairs_noalloc).

It serves callers that own all device memory and cannot let a library call cudaMalloc --
a framework's caching allocator, an arena sized at start-up, a plugin host that forbids
allocation in its callbacks. Here the device buffers come from torch, never from the
engine, and two calls in a row (DNA local with multi-pass columns, then protein semiglobal)
must return exactly what the allocating entry point (Aligner.score_pairs, i.e.
gpusw_score_pairs) returns and what the CPU oracle computes: integer scores, so "within
tolerance" means bit-exact. This file is collected last so that a failure here never hides
the other tests.
"""
import ctypes
import dataclasses

import numpy as np
import pytest

import oracle
from gpusw_b200 import Aligner, Scheme, _native, schemes
from gpusw_b200.encode import funnel
from tests._util import rand_seqs

pytestmark = pytest.mark.gpu

MODES = {"local": 0, "global": 1, "semiglobal": 2}


def _dev(a, dtype):
    import torch

    arr = np.ascontiguousarray(a, dtype=dtype)
    if arr.size == 0:
        arr = np.zeros(1, dtype=dtype)
    return torch.from_numpy(arr).to("cuda:0")


def _noalloc(q, r, qi, rj, sch, max_len):
    """Call the entry point on device copies made by torch; returns (rc, scores, msg)."""
    import torch

    torch.cuda.set_device(0)
    tq, tqo = _dev(q.codes, np.uint8), _dev(q.offsets, np.int32)
    tr, tro = _dev(r.codes, np.uint8), _dev(r.offsets, np.int32)
    tqi, trj = _dev(qi, np.int32), _dev(rj, np.int32)
    out = torch.full((len(qi),), -12345, dtype=torch.int32, device="cuda:0")
    sub = np.ascontiguousarray(sch.substitution_table(), dtype=np.int32)
    msg = ctypes.create_string_buffer(256)
    lib = _native.load()
    rc = lib.gpusw_score_pairs_noalloc(
        tq.data_ptr(), tqo.data_ptr(), q.n, tr.data_ptr(), tro.data_ptr(), r.n,
        tqi.data_ptr(), trj.data_ptr(), len(qi), MODES[sch.mode], sch.gap_open, sch.gap_extend,
        int(sch.free_end_gaps_query), int(sch.free_end_gaps_ref), int(sub.shape[0]),
        sub.ctypes.data_as(ctypes.c_void_p), int(max_len), out.data_ptr(),
        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream), msg, 256)
    return rc, out.cpu().numpy(), msg.value.decode()


def _case(seed, sch, alpha, n, lo, hi):
    rng = np.random.default_rng(seed)
    qs = rand_seqs(rng, n, lo, hi, alpha)
    rs = rand_seqs(rng, n, lo, hi, alpha)
    qi = rng.permutation(n).astype(np.int32)
    rj = rng.integers(0, n, size=n).astype(np.int32)
    return qs, rs, qi, rj


def test_noalloc_equals_allocating_entry_two_calls_in_a_row():
    calls = [
        (schemes.DNA, "ACGTN", _case(11, schemes.DNA, "ACGTN", 150, 0, 700)),
        (schemes.PROTEIN_SEMIGLOBAL, "ARNDCQEGHILKMFPSTWYV",
         _case(12, schemes.PROTEIN_SEMIGLOBAL, "ARNDCQEGHILKMFPSTWYV", 90, 1, 400)),
    ]
    for sch, _, (qs, rs, qi, rj) in calls:
        q, r = funnel(qs, sch), funnel(rs, sch)
        rc, got, msg = _noalloc(q, r, qi, rj, sch, max_len=1000)
        assert rc == 0, msg
        want = Aligner(sch).index(rs).set_queries(qs).score_pairs(qi, rj)
        assert np.array_equal(got, want)
        assert np.array_equal(got, oracle.score_pairs(q, r, qi, rj, sch))


def test_noalloc_rejects_bad_inputs_without_touching_outputs():
    sch = Scheme(mode="global")
    qs, rs, qi, rj = _case(13, sch, "ACGT", 20, 5, 60)
    q, r = funnel(qs, sch), funnel(rs, sch)
    bad = rj.copy()
    bad[7] = 20  # one past the last reference: found on the device and skipped
    rc, got, msg = _noalloc(q, r, qi, bad, sch, max_len=100)
    assert rc == _native.E_INVALID and "position 7" in msg
    assert got[7] == -12345
    rc, _, msg = _noalloc(q, r, qi, rj, sch, max_len=400_000)  # strips would not fit
    assert rc == _native.E_MEMORY and "max_len" in msg
    rc, _, msg = _noalloc(q, r, qi, rj, sch, max_len=10**9)  # scores could leave int32
    assert rc == _native.E_OVERFLOW
    rc, got, msg = _noalloc(q, r, qi, rj, sch, max_len=100)  # and the next call is fine
    assert rc == 0, msg
    assert np.array_equal(got, Aligner(sch).index(rs).set_queries(qs).score_pairs(qi, rj))


def _with(enc, **kw):
    return dataclasses.replace(enc, **kw)


def test_noalloc_rejects_bad_codes_and_offsets_before_using_them():
    """A code >= ns would index past the profile and the table; decreasing offsets give a
    negative length. Both are found on the device before use and the pair is skipped."""
    sch = schemes.DNA
    qs, rs, qi, rj = _case(14, sch, "ACGT", 24, 5, 80)
    q, r = funnel(qs, sch), funnel(rs, sch)
    ns = sch.substitution_table().shape[0]
    want = oracle.score_pairs(q, r, qi, rj, sch)
    # a query code past the table (ns + 5) in the query of pair 3
    qc = q.codes.copy()
    qc[q.offsets[qi[3]]] = ns + 5
    rc, got, msg = _noalloc(_with(q, codes=qc), r, qi, rj, sch, max_len=100)
    assert rc == _native.E_INVALID and "code" in msg
    hit = qi == qi[3]
    assert np.all(got[hit] == -12345)
    assert np.array_equal(got[~hit], want[~hit])
    # a reference code of 255 in the reference of pair 5
    rcodes = r.codes.copy()
    rcodes[r.offsets[rj[5]]] = 255
    rc, got, msg = _noalloc(q, _with(r, codes=rcodes), qi, rj, sch, max_len=100)
    assert rc == _native.E_INVALID and "code" in msg
    assert np.all(got[rj == rj[5]] == -12345)
    # decreasing offsets: reference k gets length -1 (k - 1 grows by len(k) + 1 residues,
    # all of them still inside the buffer since k + 1 is not the last reference)
    ro = r.offsets.copy()
    k = next(int(x) for x in rj if 1 <= x < r.n - 1)
    ro[k] = ro[k + 1] + 1
    rc, got, msg = _noalloc(q, _with(r, offsets=ro), qi, rj, sch, max_len=200)
    assert rc == _native.E_INVALID and "offsets" in msg
    assert np.all(got[rj == k] == -12345)
    # the shared scratch holds no trace of the failures
    rc, got, msg = _noalloc(q, r, qi, rj, sch, max_len=100)
    assert rc == 0, msg
    assert np.array_equal(got, want)
