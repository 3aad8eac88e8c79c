"""[Phase_shifter] (README.md:57-70): parsing and its effect in the CPU
restatement.

The reference documents the block (number, start_position, interval_length,
phase in units of pi; several blocks allowed) but its parser never reads it,
so the loop there has no phase shifter.  This project reads it as a delay of
the electrons against the field: theta -= phase * pi for every particle,
applied after the push or drift of the iteration whose step [it dz,
(it+1) dz) contains the shifter, before the wrap.  A shift of 2 pi is then a
no-op up to the rounding of the wrap; a shift of pi turns the bunching
against the field.
"""
import numpy as np
import pytest

from felis_b200 import workloads

from conftest import rel_err

KEYS = ("x", "y", "px", "py", "theta", "gamma")


def _run(fb, oracle_mod, tmp_path, name, shifters, steps=None):
    path = workloads.write_input(str(tmp_path / f"{name}.inp"), kind="static", beamlets=128, nx=41,
                                 total_length=12.0, phase_shifters=shifters)
    cfg = fb.Config(path)
    p = cfg.params
    beam = cfg.load_beam(0, seed=1)
    ux, uy = cfg.load_seed(0)
    o = oracle_mod.Oracle(p, threads=4)
    o.set_particles(0, *(beam[k] for k in KEYS), beam["offsets"], beam["weights"])
    o.set_field(0, 0, ux)
    o.set_field(0, 1, uy)
    e, _, _ = o.run(0, steps or p.max_step)
    return cfg, e[:, 0] + e[:, 1], o.get_particles(0)


def test_blocks_are_parsed(fb, tmp_path):
    path = workloads.write_input(str(tmp_path / "ps.inp"), kind="static",
                                 phase_shifters=[(3, 3.7, 4.0, 1.0), (1, 21.7, 0.0, 0.5)])
    cfg = fb.Config(path)  # (the params point into the config's arrays)
    p = cfg.params
    assert p.num_phase_shifts == 4
    z = [p.phase_shift_z[k] for k in range(4)]
    ph = [p.phase_shift_phase[k] for k in range(4)]
    assert z == [3.7, 7.7, 11.7, 21.7] and ph == [1.0, 1.0, 1.0, 0.5]
    assert fb.Config(workloads.write_input(str(tmp_path / "none.inp"), kind="static")).params.num_phase_shifts == 0


def test_shift_of_pi_changes_the_power_and_two_pi_does_not(fb, oracle_mod, tmp_path):
    dz = 0.026
    it_ps = int(3.7 / dz)  # the shifter's step (3.7 m, in the first gap)
    _, p0, b0 = _run(fb, oracle_mod, tmp_path, "none", ())
    _, p1, _ = _run(fb, oracle_mod, tmp_path, "pi", [(1, 3.7, 0.0, 1.0)])
    _, p2, b2 = _run(fb, oracle_mod, tmp_path, "two_pi", [(1, 3.7, 0.0, 2.0)])
    # identical up to the shifter; the seeded beam bunches on the field, so a
    # pi shift turns the exchange around and the power after it differs
    assert np.array_equal(p0[: it_ps + 1], p1[: it_ps + 1])
    assert abs(p1[-1] - p0[-1]) > 1e-3 * p0[-1]
    # 2 pi is the same bunch position: only the wrap's rounding differs
    assert rel_err(p2, p0) < 1e-9
    assert rel_err(np.mod(b2["theta"], 2 * np.pi), np.mod(b0["theta"], 2 * np.pi)) < 1e-9


def test_drop_in_sequence_applies_the_shift(fb, oracle_mod, tmp_path):
    """orc_phase_shift between the push and the wrap reproduces orc_run."""
    cfg, _, ref = _run(fb, oracle_mod, tmp_path, "fused", [(1, 0.3, 0.0, 1.0)], steps=20)
    p = cfg.params
    beam = cfg.load_beam(0, seed=1)
    ux, uy = cfg.load_seed(0)
    o = oracle_mod.Oracle(p, threads=4)
    o.set_particles(0, *(beam[k] for k in KEYS), beam["offsets"], beam["weights"])
    o.set_field(0, 0, ux)
    o.set_field(0, 1, uy)
    for it in range(20):
        o.solve_field()
        o.update_lattice(it, 0.0)
        o.transverse_push()
        o.update_lattice(it, 0.5)
        o.transverse_push()
        if o.lattice().drift_flag:
            o.drift_theta_gamma()
        else:
            o.push_theta_gamma()
        o.phase_shift(it)
        o.periodic_particles()
    got = o.get_particles(0)
    for k in KEYS:
        assert np.array_equal(got[k], ref[k]), k
