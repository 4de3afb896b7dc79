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
                          "--nt", "40", "--cpu-steps", "4", "--steps", "1", "--warmup", "1"],
                         cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["unit"] == "gradients/s" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"] == {"value": line["value"], "unit": "gradients/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert line["config"]["grid"] == [64, 64] and line["config"]["nt"] == 40
