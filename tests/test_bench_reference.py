"""bench.py's reference arm (the reference's own CPU step loop on the bench
workload) runs on the host alone, without loading the product library: its
JSON line keeps the contract of the GPU arm's line (metric, unit, workload)
with its own baseline fields."""
import json
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


RUN_AND_CHECK_MAPS = """
import runpy, sys
sys.argv = ["bench.py", "--impl", "reference", "--steps", "1", "--warmup", "3"]
runpy.run_path("bench.py", run_name="__main__")
maps = open("/proc/self/maps").read()
print("PRODUCT_LIBRARY_LOADED" if "libfelis_b200" in maps else "PRODUCT_LIBRARY_NOT_LOADED")
"""


def test_reference_arm_line():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import refrun

    r = subprocess.run([sys.executable, "-c", RUN_AND_CHECK_MAPS], capture_output=True, text=True, cwd=ROOT,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    out = r.stdout.strip().splitlines()
    assert out[-1] == "PRODUCT_LIBRARY_NOT_LOADED"
    line = json.loads(out[-2])
    assert line["impl"] == "reference" and line["value"] > 0 and line["higher_is_better"] is True
    assert line["unit"] == "particle-steps/s" and line["metric"].startswith("particle-steps/s")
    cfg = line["config"]
    assert cfg["workload"].startswith("sase: FP64") and cfg["particles"] == 8388608 and line["dtype"] == "f64"
    assert cfg["slices"] == 1024 and cfg["grid"] == [102, 102]
    cb = line["cpu_baseline"]
    assert cb["kind"] == ("reference" if refrun.available("fast") else "port")
    assert cb["cores"] >= 1 and cb["value"] == line["value"] and cb["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


def test_beam_counts_match_the_loader(fb, tmp_path):
    from felis_b200 import workloads

    cfg = fb.Config(workloads.write_input(str(tmp_path / "c.inp"), kind="sase", slices=24, beamlets=64, nx=21,
                                          sigma_slices=6.0))
    beam = cfg.load_beam(0, seed=2)
    assert np.array_equal(np.diff(beam["offsets"]), cfg.beam_counts(0))
