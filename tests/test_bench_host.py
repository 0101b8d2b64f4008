"""Host logic of bench.py on CPU: the clock record taken with nvidia-smi
during the timed steps (here a stand-in nvidia-smi on PATH that prints the
queried CSV columns), the peak fallback, the workload description and the
command-line defaults (one GPU, three warm-up steps, the 2N = 61440 workload)."""
import os
import stat
import sys
import time

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def _fake_smi(tmp_path, rows):
    """A stand-in nvidia-smi that prints `rows` (CSV, the bench's query order)
    then idles until it is terminated, as `-lms 200` would."""
    script = tmp_path / "nvidia-smi"
    body = "\n".join(f"echo '{r}'" for r in rows)
    script.write_text(f"#!/bin/bash\n{body}\nexec sleep 30\n")
    script.chmod(script.stat().st_mode | stat.S_IEXEC)
    return str(tmp_path)


@pytest.mark.parametrize("rows,expect", [
    # idle samples before the load are left out of the median
    (["0, 345, 1965, 120.0, 0x0, Not Active, Not Active, Not Active, Not Active",
      "0, 1500, 1965, 990.1, 0x4, Not Active, Not Active, Not Active, Active",
      "0, 1492, 1965, 998.0, 0x4, Not Active, Not Active, Not Active, Active",
      "0, 1485, 1965, 1001.2, 0x4, Not Active, Not Active, Not Active, Active"],
     (1492.0, 1965.0, ["sw_power_cap"], 4)),
    (["0, 1965, 1965, 700.0, 0x0, Not Active, Not Active, Not Active, Not Active",
      "0, 1800, 1965, 900.0, 0x40, Not Active, Active, Not Active, Not Active"],
     (1882.5, 1965.0, ["hw_thermal_slowdown"], 2)),
])
def test_clock_sampler_reads_clocks_and_reasons(tmp_path, monkeypatch, rows, expect):
    import bench
    monkeypatch.setenv("PATH", _fake_smi(tmp_path, rows) + os.pathsep + os.environ["PATH"])
    s = bench.ClockSampler(0)
    time.sleep(0.5)
    c = s.stop()
    assert (c["sm_mhz"], c["sm_max_mhz"], c["reasons"], c["samples"]) == expect


def test_clock_sampler_without_nvidia_smi(tmp_path, monkeypatch):
    import bench
    monkeypatch.setenv("PATH", str(tmp_path))
    c = bench.ClockSampler(0).stop()
    assert c["sm_mhz"] is None and c["reasons"] == ["nvidia-smi unavailable"]


def test_peaks_fall_back_when_the_measured_file_is_absent(tmp_path, monkeypatch):
    import bench
    monkeypatch.setattr(bench, "REPO", str(tmp_path))
    pk, basis = bench.peaks()
    assert basis == "fallback" and pk["hbm_gbs"] == 6650.0 and pk["bf16_tflops"] == 1590.0


def test_defaults_and_workload(monkeypatch):
    import bench
    monkeypatch.setattr(sys, "argv", ["bench.py"])
    a = bench.parse()
    assert (a.gpus, a.warmup, a.impl, a.ref, tuple(a.orient), a.tensor_split) == (1, 3, "bem", 5, (45, 31, 1), 1)
    assert a.warmup >= 3 and a.steps >= 1
    w = bench.workload(a, 61440)
    assert w["unknowns"] == 61440 and w["rhs"] == 2790 and "L2" in w["l2_policy"]
    assert bench._n_rwg_ico(5) == 30720


def test_cpu_dense_path_sample_is_scaled_and_described():
    # the reference's CPU dense path (oracle restatement) on samples of an
    # icosphere of refinement 1: the row sample scales to about the full
    # assembly, the LU sample by n^3, and the description names every sample
    import bench
    from oracle import bem_oracle as bo
    v, t = bo.icosphere(1.0, 1)
    full = bench.cpu_dense_path(v, t, 1.0, 1.3116, 2, 19)
    samp = bench.cpu_dense_path(v, t, 1.0, 1.3116, 2, 19, reps=3, rows=30, n_lu=96, n_ff=1, ff_dirs=7)
    for r in (full, samp):
        assert r["total"] >= r["solve_only"] > 0 and r["cores"] >= 1 and r["n"] == 240
        assert "logical cores" in r["description"] and "OPENBLAS_NUM_THREADS" in r["description"]
    assert "assembly full" in full["description"]
    assert "30 of 120 test rows" in samp["description"] and "median of 3" in samp["description"]
    assert "scaled by (n/96)^3" in samp["description"] and "1 of 2 orientations at 7 of 19" in samp["description"]
    assert 0.2 < samp["assembly"] / full["assembly"] < 5.0


def test_options_and_config_switches(monkeypatch):
    import bench
    monkeypatch.setattr(sys, "argv", ["bench.py", "--option", "residual_pace_epoch=16", "--option",
                                      "residual_pace_lead = 1", "--config", "gemm", "--gemm-shape", "solve"])
    a = bench.parse()
    assert bench.extra_options(a) == {"residual_pace_epoch": 16, "residual_pace_lead": 1}
    assert (a.config, a.gemm_shape, a.gemm_n, a.gemm_ncol, a.gemm_pairs) == ("gemm", "solve", 12288, 2790, 1)


def test_cpu_dense_path_blocked_assembly_covers_every_row():
    # the full-size C2 leg times every assembly row in blocks: the same work
    # as one call, so about the same time, and described as such
    import bench
    from oracle import bem_oracle as bo
    v, t = bo.icosphere(1.0, 1)
    full = bench.cpu_dense_path(v, t, 1.0, 1.3116, 2, 19)
    blk = bench.cpu_dense_path(v, t, 1.0, 1.3116, 2, 19, rows="blocks")
    assert "all 120 test rows in blocks of 256" in blk["description"]
    assert 0.2 < blk["assembly"] / full["assembly"] < 5.0 and blk["total"] > blk["solve_only"] > 0
