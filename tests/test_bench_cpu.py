"""bench.py's host-side pieces on the CPU: the forward step's vector-field
evaluation count behind the FP64 roofline, the reading of the measured-peaks
file, and the reference arm's JSON line (the CPU port of the reference
algorithm on a small grid)."""
import json
import os
import subprocess
import sys

from conftest import ROOT

sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_forward_evaluations_follow_the_shrinking_stage_regions():
    # one 64x32 tile: stages on 70x38, 68x36, 66x34, 64x32
    assert bench.fwd_evaluations(32, 64, 64, 32) == 70 * 38 + 68 * 36 + 66 * 34 + 64 * 32
    # 512x512 in 64x32 tiles: 4.59 evaluations per cell
    n = bench.fwd_evaluations(512, 512, 64, 32)
    assert abs(n / 512 ** 2 - 9400 / 2048) < 1e-12
    # a cut bottom tile (29-row tiles over 512 rows: the last has 19)
    last = sum((64 + 2 * e) * (19 + 2 * e) for e in range(4))
    assert bench.fwd_evaluations(512, 64, 64, 29) == 17 * sum((64 + 2 * e) * (29 + 2 * e) for e in range(4)) + last


def test_measured_peaks_file_is_read_when_present(tmp_path, monkeypatch):
    monkeypatch.setattr(bench, "ROOT", str(tmp_path))
    assert bench.peaks() == (6650.0, "fallback")
    (tmp_path / "MEASURED_PEAKS.json").write_text(json.dumps({"gpu": {"HBM_copy_GBps": 7100.5, "bf16": 1500}}))
    assert bench.peaks() == (7100.5, "measured")
    (tmp_path / "MEASURED_PEAKS.json").write_text(json.dumps({"hbm_gbs": 6900.0}))
    assert bench.peaks() == (6900.0, "measured")
    (tmp_path / "MEASURED_PEAKS.json").write_text("not json")
    assert bench.peaks() == (6650.0, "fallback")


def test_reference_arm_prints_its_line_on_a_small_grid():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--n", "64",
                          "--nt", "40", "--ref-sample-steps", "8", "--steps", "3", "--warmup", "1"],
                         cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["unit"] == "gradients/s" and line["value"] > 0
    # each timed step is one sample of 8 of the 40 steps: steps x ms_per_step is the timed run
    assert line["steps"] == 3 and line["sample_steps"] == 8 and line["extrapolated_to"] == 40
    assert abs(line["steps"] * line["ms_per_step"] / 1000.0 - line["timed_s"]) <= 0.5 * line["timed_s"]
    assert abs(line["value"] - 8 / 40 / (line["ms_per_step"] / 1000.0)) <= 0.5 * line["value"]
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"] == {"value": line["value"], "unit": "gradients/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert line["config"]["grid"] == [64, 64] and line["config"]["nt"] == 40


def test_binding_roof_leads_with_the_larger_fraction():
    roof = {"bound": "hbm", "kernel": "k_fwd_step", "achieved": 850.0, "peak": 6500.0, "unit": "GB/s",
            "frac": 850.0 / 6500.0, "peak_source": "measured", "traffic": 1.0, "bytes_per_launch": 2.0,
            "avg_launch_ms": 0.017, "note": "x",
            "fp64": {"kernel": "k_fwd_step", "achieved": 11.4, "peak": 37.2, "unit": "TFLOP/s", "frac": 11.4 / 37.2,
                     "peak_source": "nominal", "flops_per_launch": 3.0, "avg_launch_ms": 0.017, "flops_source": "y"}}
    out = bench.binding_roof(dict(roof))
    assert out["bound"] == "fp64" and out["unit"] == "TFLOP/s" and out["frac"] == 11.4 / 37.2
    assert out["hbm"]["frac"] == 850.0 / 6500.0 and out["hbm"]["unit"] == "GB/s" and "fp64" not in out
    roof["fp64"]["frac"] = 0.01
    assert bench.binding_roof(dict(roof))["bound"] == "hbm"
