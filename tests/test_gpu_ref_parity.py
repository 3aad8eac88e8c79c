"""The GPU FP64 plain path against the reference itself, at the workload
sizes: config 1 complete (Static, 8192 particles, 102 x 102, 1 MW seed, 1539
steps) and config 2 (Time_Dependent SASE, 1024 slices x 8192 particles,
1539 steps) on its leading slices.

The reference side is oracle/_ref/felis_ref (the reference's unmodified
sources with the MPI/GSL stand-ins of oracle/ref_shim/), run from the input
file with its own loader and tables, when the executable is present; the
golden fixtures of tests/golden/ (made by the same executable,
make_ref_golden.py) otherwise, and always.  The C-library build of the CPU
restatement (liboracle_libm.so) is compared as well.

Tolerance: 1e-10 relative to the largest magnitude of each result (particle
columns, field planes, power per iteration).  The GPU path is bit-identical
to the strict restatement; what remains against the reference is its use of
glibc's sin/cos/atan and two-division complex quotients, measured at
1e-16 .. 5e-13 after the 1539 steps.
"""
import os

import numpy as np
import pytest

import refrun

from conftest import ref_case, rel_err

TOL = 1e-10
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
LIVE_PREFIX_SLICES = 4


def _gpu_run(fb, cfg, beam, fields):
    p = cfg.params
    g = fb.Handle(p)
    g.upload_particles(0, *(beam[k] for k in refrun.KEYS), beam["offsets"], beam["weights"])
    for h, (ux, uy) in enumerate(fields):
        g.upload_field(h, 0, ux)
        g.upload_field(h, 1, uy)
    g.run(0, p.max_step)
    energy = g.diagnostics(0, p.max_step)[0]
    parts = g.download_particles(0)
    ux, uy = g.download_field(0, 0), g.download_field(0, 1)
    g.close()
    return parts, ux, uy, energy


def _report(tag, errs):
    print(f"{tag}: " + ", ".join(f"{k} {v:.2e}" for k, v in errs.items()))
    bad = {k: v for k, v in errs.items() if not v <= TOL}
    assert not bad, f"{tag}: above {TOL}: {bad}"


def _errors(parts, ux, uy, energy, ref_parts, ref_ux, ref_uy, ref_energy, n_particles=None, planes=None):
    n = n_particles if n_particles is not None else ref_parts["x"].size
    errs = {k: rel_err(parts[k][:n], ref_parts[k]) for k in refrun.KEYS}
    sl = slice(1, -1) if planes is None else slice(1, planes + 1)
    errs["Ux"] = rel_err(ux[sl], ref_ux[1:-1])
    errs["Uy"] = rel_err(uy[sl], ref_uy[1:-1]) if np.any(ref_uy) else float(np.max(np.abs(uy[sl])))
    if energy is not None:
        errs["power"] = max(rel_err(energy[i], ref_energy[i]) for i in range(energy.shape[0]))
    return errs


def _golden(name):
    return np.load(os.path.join(GOLDEN, name))


def _golden_errors(gold, parts, ux, uy, energy=None):
    pick = gold["pick"]
    errs = {k: rel_err(parts[k][pick], gold[k]) for k in refrun.KEYS}
    cs = int(gold["cell_stride"])
    S = gold["field_x"].shape[0]
    errs["Ux"] = rel_err(ux[1:S + 1, ::cs, ::cs], gold["field_x"])
    errs["Uy"] = float(np.max(np.abs(uy[1:S + 1, ::cs, ::cs] - gold["field_y"])))
    if energy is not None:
        errs["power"] = max(rel_err(energy[i], gold["energy"][i]) for i in range(energy.shape[0]))
    return errs


def _write_golden_input(tmp_path, gold):
    path = tmp_path / "golden.inp"
    path.write_text(str(gold["input"]))
    return str(path)


@pytest.mark.gpu
def test_config1_complete_against_reference(fb, oracle_mod, tmp_path):
    cfg, beam, fields, path, seed = ref_case(fb, tmp_path, "static")
    p = cfg.params
    assert (p.max_step, int(beam["offsets"][-1]), p.nx, p.ny, p.slice_n) == (1539, 8192, 102, 102, 1)
    parts, ux, uy, energy = _gpu_run(fb, cfg, beam, fields)

    gold = _golden("ref_config1.npz")
    gcfg = fb.Config(_write_golden_input(tmp_path, gold))
    gbeam = gcfg.load_beam(0, seed=int(gold["seed"]))
    for k in refrun.KEYS:  # the fixture's input is this workload's input
        assert np.array_equal(gbeam[k], beam[k]), k
    _report("config 1 vs reference golden", _golden_errors(gold, parts, ux, uy, energy))

    if refrun.available():
        r = refrun.run(path, seed=seed)
        ref_e = np.stack([r["energyX"], r["energyY"]], axis=2).reshape(p.max_step, -1)
        f = r["final"]
        _report("config 1 vs reference", _errors(parts, ux, uy, energy, f["particles"][0], f["Ux"][0], f["Uy"][0],
                                                 ref_e))

    o = oracle_mod.Oracle(p, threads=os.cpu_count() or 4, variant="libm")
    o.set_particles(0, *(beam[k] for k in refrun.KEYS), beam["offsets"], beam["weights"])
    for h, (a, b) in enumerate(fields):
        o.set_field(h, 0, a)
        o.set_field(h, 1, b)
    e, _, _ = o.run(0, p.max_step)
    _report("config 1 vs restatement (glibc libm)",
            _errors(parts, ux, uy, energy, o.get_particles(0), o.get_field(0, 0), o.get_field(0, 1), e))


@pytest.mark.gpu
def test_config2_leading_slices_against_reference(fb, tmp_path):
    """The full 1024-slice SASE run on the GPU; its slices 1..k against the
    reference run on k slices (a closed sub-problem: radiation slips from
    slice s-1 to s only, solveField.cpp:19-47, and there is no wake)."""
    cfg, beam, fields, path, seed = ref_case(fb, tmp_path, "sase")
    p = cfg.params
    assert (p.max_step, p.slice_n, int(beam["offsets"][-1]), p.nx) == (1539, 1024, 8388608, 102)
    assert not p.wake_on
    parts, ux, uy, _ = _gpu_run(fb, cfg, beam, fields)

    gold = _golden("ref_config2_prefix.npz")
    k = gold["field_x"].shape[0]
    gcfg = fb.Config(_write_golden_input(tmp_path, gold))
    gbeam = gcfg.load_beam(0, seed=int(gold["seed"]))
    nk = int(gbeam["offsets"][-1])
    for key in refrun.KEYS:  # the fixture's slices are this run's leading slices
        assert np.array_equal(gbeam[key], beam[key][:nk]), key
    _report(f"config 2 slices 1..{k} vs reference golden", _golden_errors(gold, parts, ux, uy))

    if refrun.available():
        from felis_b200 import workloads

        k = LIVE_PREFIX_SLICES
        kpath = workloads.write_input(str(tmp_path / "prefix.inp"), kind="sase", slices=k)
        r = refrun.run(kpath, seed=seed)
        f = r["final"]
        nk = int(beam["offsets"][k])
        _report(f"config 2 slices 1..{k} vs reference",
                _errors(parts, ux, uy, None, f["particles"][0], f["Ux"][0], f["Uy"][0], None, n_particles=nk,
                        planes=k))
