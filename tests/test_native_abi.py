"""The C ABI library: built for sm_100a, loadable, exporting every symbol the header
declares; no GPU is needed (no compute calls are made here)."""
import ctypes
import os
import re

import pytest

from gpusw_b200 import _native
from tests.conftest import HAS_GPU, ROOT

HEADER = os.path.join(ROOT, "include", "gpusw_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(gpusw_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for must in ("gpusw_ctx_create", "gpusw_set_scheme", "gpusw_db_upload", "gpusw_score_cross",
                 "gpusw_topk", "gpusw_score_pairs", "gpusw_last_error", "gpusw_get_stats"):
        assert must in syms


def test_library_exports_every_declared_symbol():
    lib = _native.load()
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    assert lib.gpusw_version() >= 100


def test_python_binding_covers_header():
    bound = set(_native._SIGNATURES)
    assert set(declared_symbols()) <= bound


def test_device_count_without_gpu_is_not_an_error():
    lib = _native.load()
    n = ctypes.c_int(-1)
    assert lib.gpusw_device_count(ctypes.byref(n)) == 0
    assert n.value >= 0


@pytest.mark.skipif(HAS_GPU, reason="checks the no-GPU error path")
def test_no_gpu_paths_raise_nogpuerror():
    import gpusw_b200 as g
    from gpusw_b200.errors import NoGpuError

    assert not g.gpu_available()
    with pytest.raises(NoGpuError):
        _native.Context(0)
    with pytest.raises(NoGpuError):
        g.align_score(["ACGT"], ["ACGT"])
    with pytest.raises(NoGpuError):
        g.Aligner("dna", backend="metal").index(["ACGT"])
    with pytest.raises(ValueError):
        g.Aligner("dna", backend="bogus").index(["ACGT"])
    assert g.metal_available() is False and g.available_backends() == []
