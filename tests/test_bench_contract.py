"""bench.py's reference arm runs on the host cores (the oracle port over the same workload),
so its JSON line can be checked here without a GPU: one line, the contract's keys, and the
reference-arm specifics (impl, cpu_baseline, a zero-copy e2e)."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--workload", "small", "--steps", "1", "--warmup", "1"],
                         capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
                "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == "GCUPS"
    assert d["higher_is_better"] is True and d["n_gpus"] == 1
    assert d["cpu_baseline"]["value"] == d["value"] and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert "workload" in d["config"]


def test_roofline_binds_on_the_alu_pipe():
    """Each int16x2 register of two cells takes 4.5 DPX ops on the ALU pipe and one vadd2
    on the FMA pipe, so the ALU ceiling (rate x 2 / 4.5) is the peak the fraction uses."""
    sys.path.insert(0, ROOT)
    import bench

    rate = 18.48e12
    r = bench.roofline(cells=8.0e12, score_ms=1000.0, dpx=rate)
    assert r["peak_pipe"] == "alu" and r["bound"] == "int"
    assert abs(r["peak"] - rate * 2 / 4.5 / 1e9) < 1e-6
    assert r["ceilings_gcups"]["fma"] > r["peak"]
    assert abs(r["frac"] - 8000.0 / r["peak"]) < 1e-12
    assert r["traffic"] is None  # cross products: L2-resident references, not extrapolated


def test_roofline_of_the_inter_sequence_pairs_kernel():
    """Pairs scored by the inter-sequence kernel are measured against its own ceiling: 4 ALU
    ops per register outside local mode (4.5 with the running maximum), 2 vadd2 on the FMA
    pipe; the pairs workload's traffic is the measured DRAM bytes of that kernel per pair."""
    sys.path.insert(0, ROOT)
    import bench

    rate = 18.48e12
    wl = bench.workload("pairs", nq=1000)
    assert wl.scheme.mode == "semiglobal"
    r = bench.roofline(cells=wl.cells(), score_ms=1.0, dpx=rate, wl=wl, inter=True)
    assert r["kernel"] == "pairs_inter_kernel"
    assert abs(r["peak"] - rate * 2 / 4.0 / 1e9) < 1e-6
    assert abs(r["ceilings_gcups"]["fma"] - rate * 2 / 2.0 / 1e9) < 1e-6
    assert abs(r["traffic"] - 4259.93 * 1000) < 1e-3 and "pairs_inter_kernel" in r["traffic_source"]
    team = bench.roofline(cells=wl.cells(), score_ms=1.0, dpx=rate, wl=wl, inter=False)
    assert team["kernel"] == "team kernels" and abs(team["peak"] - rate * 2 / 4.5 / 1e9) < 1e-6
    assert abs(team["traffic"] - 148.8512 * 1000) < 1e-3
    local = wl.scheme.replace(mode="local")
    wl.scheme = local
    r_local = bench.roofline(cells=1.0, score_ms=1.0, dpx=rate, wl=wl, inter=True)
    assert abs(r_local["peak"] - rate * 2 / 4.5 / 1e9) < 1e-6


def test_reference_code_baseline_matches_the_oracle():
    """The reference package's own cpu_reference_score (installed under baseline/_ref), run
    in a spawn pool, gives the C oracle's scores on a seeded sample of the small workload."""
    import pytest

    sys.path.insert(0, ROOT)
    import numpy as np

    import bench
    import oracle

    if not os.path.isdir(os.path.join(bench.REF_INSTALL, "gpusw")):
        pytest.skip("reference package not installed under baseline/_ref")
    wl = bench.workload("small")
    rec, qi, rj, grid, got = bench.cpu_reference_code(wl, 1.5e6)
    assert rec["kind"] == "reference" and rec["value"] > 0 and rec["cores"] >= 1
    assert grid is not None and got.shape == (len(qi), len(rj))
    q = bench._enc(wl, *wl.queries)
    want = oracle.score_cross(q, bench._enc(wl, *bench.subset(wl.refs, rj)), wl.scheme, qlist=qi)
    assert np.array_equal(got, want)
