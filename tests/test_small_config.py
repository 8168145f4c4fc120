"""The small benchmark configuration at its exact shape: 32 DNA queries x 128 references,
lengths U[80, 200], the default 'dna' scheme in local mode, scored in full by the reference
package's own cpu_reference_matrix (tests/golden/small_config.json, made by
tests/golden/make_small_config.py). The fixture pins the workload generator and the C oracle
on the CPU; on the GPU every one of the 4,096 scores must match, with dtype "auto" (int16
with int32 rescoring) and with "int32"."""
import numpy as np
import pytest

import oracle
from gpusw_b200 import align_score, schemes, workloads
from gpusw_b200.encode import funnel
from tests._util import golden


def _fixture():
    d = golden("small_config.json")
    return d["queries"], d["refs"], np.array(d["scores"], dtype=np.int64)


def test_fixture_is_the_small_workload():
    qs, rs, want = _fixture()
    wl = workloads.small()
    assert want.shape == (32, 128) == (wl.nq, wl.nr)
    for texts, (codes, offs) in ((qs, wl.queries), (rs, wl.refs)):
        enc = funnel(texts, schemes.DNA)
        assert np.array_equal(enc.codes, codes) and np.array_equal(enc.offsets, offs)
    lens = np.diff(wl.queries[1])
    assert lens.min() >= 80 and lens.max() <= 200


def test_oracle_reproduces_the_reference_on_the_small_config():
    qs, rs, want = _fixture()
    got = oracle.score_cross(funnel(qs, schemes.DNA), funnel(rs, schemes.DNA), schemes.DNA)
    assert np.array_equal(got, want)


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["auto", "int32"])
def test_small_config_on_gpu_equals_reference(dtype):
    qs, rs, want = _fixture()
    res = align_score(qs, rs, scheme="dna", dtype=dtype)
    assert res.scores.dtype == np.int32 and res.scores.shape == (32, 128)
    assert np.array_equal(res.scores.astype(np.int64), want)
