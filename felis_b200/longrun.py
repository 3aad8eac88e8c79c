"""A whole undulator through the FP64 plain path and through the
mixed-precision engine, from the same initial state, with the error of the
mixed run stated per result and both runs timed.

    python -m felis_b200.longrun [--workload gaussian_taper] [--slices S] [--length L] [--out r.json]

The default workload is the mixed-precision long run of felis_b200.workloads
("gaussian_taper": QuadPolar undulator, harmonics 1 and 3, Gaussian current
of 4096 slices, copper wake, 152 x 152 grid, 60 m, linear taper -1 %).
`--slices` scales the bunch (the rms length with it) and `--length` the
undulator for shorter checks.

Results per harmonic (felis_b200.analysis): output power along z (relative
error at the end, and the largest over the iterations after the power passed
1e-3 of its final value), gain length, and the centroid and rms width of the
final spectrum summed over both polarisations.  Timings are CUDA-event device
times of the graph launches (felis_run / felis_batch_run), in chunks of
`--chunk` iterations.
"""
from __future__ import annotations

import argparse
import json
import os
import tempfile
import time

import numpy as np

from . import analysis, workloads


def prepare(workload: str = "gaussian_taper", slices: int | None = None, length: float | None = None, seed: int = 2):
    """Config (with the wake table of this beam when the wake is on), beam and seed field."""
    import felis_b200 as fb

    kw = dict(workloads.WORKLOADS[workload])
    if slices is not None:
        if kw.get("sigma_slices"):
            kw["sigma_slices"] = kw["sigma_slices"] * slices / kw.get("slices", 1024)
        kw["slices"] = slices
    if length is not None:
        kw["total_length"] = length
        kw["units"] = max(1, int(np.ceil(length / kw.get("unit_len", 4.0))))
    d = tempfile.mkdtemp(prefix="felis_longrun_")
    path = workloads.write_input(os.path.join(d, f"{workload}.inp"), **kw)
    cfg = fb.Config(path)
    beam = cfg.load_beam_device(0, seed=seed)  # the per-beamlet work on the GPU
    if cfg.params.wake_on:
        # wakeField.cpp:9-50 from this beam's slice charge (makeDensity)
        cfg.wake(beam["weights"] * np.diff(beam["offsets"]))
    # without a seed laser both engines start from their zeroed fields
    fields = None if kw.get("seed_power", 1.0) == 0.0 else [cfg.load_seed(h) for h in range(cfg.params.num_harmony)]
    return cfg, beam, fields, kw


def _spectra(get_field, H: int) -> list[tuple[np.ndarray, np.ndarray]]:
    out = []
    for h in range(H):
        tot = None
        for pol in (0, 1):
            nu, p = analysis.spectrum(get_field(h, pol)[1:-1])
            tot = p if tot is None else tot + p
        out.append((nu, tot))
    return out


def _moments(nu: np.ndarray, p: np.ndarray) -> tuple[float, float]:
    w = p / p.sum()
    c = float((nu * w).sum())
    return c, float(np.sqrt(((nu - c) ** 2 * w).sum()))


def _chunks(n: int, chunk: int):
    for a in range(0, n, chunk):
        yield a, min(n, a + chunk)


def run_fp64(cfg, beam, fields, steps: int, chunk: int) -> dict:
    import felis_b200 as fb

    p = cfg.params
    h = fb.Handle(p)
    try:
        h.upload_particles(0, beam["x"], beam["y"], beam["px"], beam["py"], beam["theta"], beam["gamma"],
                           beam["offsets"], beam["weights"])
        for k, (ux, uy) in enumerate(fields or []):
            h.upload_field(k, 0, ux)
            h.upload_field(k, 1, uy)
        ms = 0.0
        for a, b in _chunks(steps, chunk):
            h.run(a, b)
            ms += h.last_run_ms()
        e, _, _ = h.diagnostics(0, steps + 1)
        spec = _spectra(h.download_field, p.num_harmony)
    finally:
        h.close()
    return {"energy": e, "spectra": spec, "ms": ms}


def run_mixed(cfg, beam, fields, steps: int, chunk: int, tune_steps: int = 4) -> dict:
    import felis_b200 as fb

    p = cfg.params

    def make():
        b = fb.Batch([p])
        b.upload_particles(0, beam["x"], beam["y"], beam["px"], beam["py"], beam["theta"], beam["gamma"],
                           beam["offsets"], beam["weights"])
        for k, (ux, uy) in enumerate(fields or []):
            b.upload_field(0, k, 0, ux)
            b.upload_field(0, k, 1, uy)
        return b

    # the tuner advances its run, so the measured run starts over with its choice
    b = make()
    b.tune(0, tune_steps)
    launch = b.launch()
    b.close()
    b = make()
    try:
        b.set_launch(*launch)
        ms = 0.0
        for a, c in _chunks(steps, chunk):
            b.run(a, c)
            ms += b.last_run_ms()
        e, _, _ = b.diagnostics(0, 0, steps + 1)
        spec = _spectra(lambda k, pol: b.download_field(0, k, pol), p.num_harmony)
    finally:
        b.close()
    return {"energy": e, "spectra": spec, "ms": ms, "launch": {"push_box_cells": launch[0], "adi_ctas_per_sm": launch[1]}}


def compare(ref: dict, mix: dict, H: int, harmonics: list[int], dz: float) -> dict:
    """Error of the mixed run per harmonic, against the FP64 run."""
    out = {}
    for k in range(H):
        P64 = analysis.output_power(ref["energy"], k)
        P32 = analysis.output_power(mix["energy"], k)
        ok = P64 > 0
        rel = np.zeros_like(P64)
        rel[ok] = np.abs(P32[ok] - P64[ok]) / P64[ok]
        grown = np.flatnonzero(P64 > 1e-3 * P64[-1])
        L64, L32 = analysis.gain_length(P64, dz), analysis.gain_length(P32, dz)
        c64, w64 = _moments(*ref["spectra"][k])
        c32, w32 = _moments(*mix["spectra"][k])
        out[f"H{harmonics[k]}"] = {
            "power_final": float(P64[-1]), "power_final_rel_error": float(rel[-1]),
            "power_max_rel_error_after_1e-3": float(rel[grown[0]:].max()) if grown.size else None,
            "power_max_rel_error_all": float(rel[ok].max()) if ok.any() else None,
            "power_gain": float(P64[-1] / P64[ok][0]) if ok.any() else None,
            "gain_length_m": L64, "gain_length_rel_error": abs(L32 - L64) / L64 if np.isfinite(L64) else None,
            "spectral_centroid": c64, "spectral_width": w64,
            "centroid_error_over_width": abs(c32 - c64) / w64 if w64 > 0 else None,
            "width_rel_error": abs(w32 - w64) / w64 if w64 > 0 else None,
        }
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--workload", default="gaussian_taper")
    ap.add_argument("--slices", type=int, default=None)
    ap.add_argument("--length", type=float, default=None)
    ap.add_argument("--steps", type=int, default=None, help="iterations (default: the whole undulator)")
    ap.add_argument("--chunk", type=int, default=128)
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)

    t0 = time.time()
    cfg, beam, fields, kw = prepare(a.workload, a.slices, a.length)
    p = cfg.params
    steps = a.steps if a.steps is not None else p.max_step
    P = int(beam["offsets"][-1])  # (the beam's device arrays stay referenced until the runs are done)
    cells = p.slice_n * p.nx * p.ny * 2 * p.num_harmony
    harmonics = [p.harmony[i] for i in range(p.num_harmony)]
    dz = p.dz if p.dz > 0 else kw.get("lambda_u_cm", 2.6) * 0.01
    t_setup = time.time() - t0
    ref = run_fp64(cfg, beam, fields, steps, a.chunk)
    mix = run_mixed(cfg, beam, fields, steps, a.chunk)
    res = {
        "workload": a.workload, "slices": p.slice_n, "grid": [p.nx, p.ny], "harmonics": harmonics,
        "particles": P, "steps": steps, "dz_m": dz, "setup_s": t_setup,
        "fp64": {"ms_per_step": ref["ms"] / steps, "particle_steps_per_s": P * steps / (ref["ms"] / 1e3),
                 "adi_cells_per_s": cells * steps / (ref["ms"] / 1e3)},
        "mixed": {"ms_per_step": mix["ms"] / steps, "particle_steps_per_s": P * steps / (mix["ms"] / 1e3),
                  "adi_cells_per_s": cells * steps / (mix["ms"] / 1e3), "launch": mix["launch"]},
        "speedup": ref["ms"] / mix["ms"],
        "errors": compare(ref, mix, p.num_harmony, harmonics, dz),
        "power_curves": {f"H{h}": {"fp64": analysis.output_power(ref["energy"], k)[::16].tolist(),
                                   "mixed": analysis.output_power(mix["energy"], k)[::16].tolist()}
                         for k, h in enumerate(harmonics)},
    }
    txt = json.dumps(res, indent=1)
    if a.out:
        with open(a.out, "w") as f:
            f.write(txt)
    summary = {k: v for k, v in res.items() if k != "power_curves"}
    print(json.dumps(summary, indent=1))
    return res


if __name__ == "__main__":
    main()
