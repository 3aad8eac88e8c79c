"""bench.py's reference arm (the reference's CPU path on the bench workload)
runs on the host alone: its JSON line keeps the contract of the mixed arm's
line (metric, unit, config) with its own baseline fields."""
import json
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "3"], capture_output=True, text=True, cwd=ROOT, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["higher_is_better"] is True
    assert line["unit"] == "particle-steps/s" and line["metric"].startswith("particle-steps/s")
    cfg = line["config"]
    assert cfg["workload"].startswith("sase: mixed-precision") and cfg["particles"] == 8388608
    assert cfg["slices"] == 1024 and cfg["grid"] == [102, 102] and cfg["iterations"] == [3, 4]
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == line["value"] and cb["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


def test_beam_counts_match_the_loader(fb, tmp_path):
    from felis_b200 import workloads

    cfg = fb.Config(workloads.write_input(str(tmp_path / "c.inp"), kind="sase", slices=24, beamlets=64, nx=21,
                                          sigma_slices=6.0))
    beam = cfg.load_beam(0, seed=2)
    assert np.array_equal(np.diff(beam["offsets"]), cfg.beam_counts(0))
