"""The product's setup and the CPU restatement against the reference itself.

oracle/_ref/felis_ref is the reference's own setup and step loop, compiled
from its unmodified sources (parameterSetting.cpp, boundary.cpp, loadBeam.cpp,
loadSeed.cpp, wakeField.cpp, particlePush.cpp, solveField.cpp,
fieldShareZ.cpp, rearrangeParticles.cpp, updateTotalEnergy.cpp, twiss.cpp,
saveFile.cpp, updateK_quadG.cpp) with project-written stand-ins for MPI (one
rank) and GSL (oracle/ref_shim/).  These tests pin:

* the product's input parser, lattice, tables, seed and beam loader
  (felis_b200 Config) to the reference's parameterSetting / boundary /
  loadSeed / loadBeam / wakeFunction;
* the CPU restatement (oracle/felis_oracle.cpp, both builds) to the
  reference's step loop, from the same initial state.

The GPU path is bit-identical to the restatement (tests/test_gpu_parity.py)
and is compared with felis_ref directly in tests/test_gpu_ref_parity.py.
"""
import os

import numpy as np
import pytest

import refrun

from conftest import ref_case, rel_err

pytestmark = pytest.mark.skipif(not refrun.build(), reason="oracle/_ref is not built and the reference sources are absent")

# (workload kind, options of felis_b200.workloads.input_text)
CASES = {
    "static": ("static", dict(beamlets=256, total_length=12.0)),
    "sase": ("sase", dict(slices=3, beamlets=128, nx=41, total_length=8.0, seed_power=1e6)),
    "quadpolar_h123_wake_quads_taper": ("sase", dict(
        slices=3, beamlets=128, nx=41, total_length=8.0, seed_power=1e6, harmonics=(1, 2, 3),
        undulator="QuadPolar", polarity=0.5, K_und=2.6 / np.sqrt(1.25), wake=True, quads=True,
        linear_taper=-0.005)),
    "gaussian_h13": ("sase", dict(slices=6, beamlets=128, nx=33, total_length=6.0, seed_power=0.0,
                                 harmonics=(1, 3), sigma_slices=2.0, wake=True)),
    "oned_h13_wake": ("sase", dict(slices=6, beamlets=128, total_length=20.0, dimension=1, harmonics=(1, 3),
                                  wake=True, seed_power=1e5)),
}


@pytest.mark.parametrize("name", list(CASES))
def test_setup_matches_reference(fb, tmp_path, name):
    """parameterSetting + boundary + loadSeed + loadBeam + wakeFunction of the
    reference against felis_config_* on the same input file."""
    kind, kw = CASES[name]
    cfg, beam, fields, path, seed = ref_case(fb, tmp_path, kind, **kw)
    p = cfg.params
    r = refrun.run(path, setup=True, initial=True, seed=seed, it1=1, final=False)
    s = r["setup"]
    # Domain scalars: integers exactly, doubles bit for bit
    for ref_key, val in (("nx", p.nx), ("ny", p.ny), ("sliceN", p.slice_n), ("maxStep", p.max_step),
                         ("numHarmony", p.num_harmony), ("nr", p.nr), ("bn", p.bessel_rows),
                         ("BesselMaxOrder", p.bessel_cols), ("abcN", p.abc_n), ("SCLmode", p.scl_mode),
                         ("SCFmode", p.scf_mode), ("numSlice", p.num_slice), ("nSpecies", p.num_species),
                         ("wakeONOFF", p.wake_on), ("dimension", p.dimension)):
        assert int(s[ref_key]) == val, ref_key
    for ref_key, val in (("ks", p.ks), ("lambda0", p.lambda0), ("dz", p.dz), ("dx", p.dx), ("dy", p.dy),
                         ("dr", p.dr), ("minX", p.min_x), ("maxX", p.max_x), ("minZ", p.min_z),
                         ("maxZ", p.max_z), ("gamma0", p.gamma0), ("gamR", p.gam_r), ("dBessel", p.d_bessel),
                         ("abcSig", p.abc_sig), ("K0", p.K0_init), ("ue", p.ue_init), ("lambdaU", p.lambdaU_init),
                         ("spotSigR", p.spot_sig_r)):
        assert s[ref_key] == val, (ref_key, s[ref_key], val)
    # undulator lattice: unit/undulator boundaries and per-unit K
    und = p.undulators[0]
    for n in range(und.numbers):
        assert s[f"und0.{n}"] == [und.unit_start[n], und.unit_end[n], und.und_start[n], und.und_end[n], und.K0[n]]
    # ABC coefficients: the reference divides complex numbers with two real
    # divisions, the product with one reciprocal; they agree to a few ulp
    if p.dimension == 3:
        for mine, theirs in zip(cfg.abc(), r["abc"]):
            assert np.max(np.abs(mine - theirs)) <= 4e-16 * np.max(np.abs(theirs))
    # Bessel J_n: the product's series/Miller recurrence against the stand-in's
    # trapezoidal Bessel integral
    assert np.max(np.abs(cfg.bessel().ravel() - r["bessel"])) < 2e-15
    if p.wake_on:
        assert rel_err(cfg.wake_function(), r["wakeF"]) < 1e-13
        den = beam["weights"] * np.diff(beam["offsets"])
        assert rel_err(cfg.wake(den), r["wakeE"]) < 1e-13
    # initial state: the reference's loader (through the generator stand-ins)
    # and the product's loader give the same bits
    init = r["init"]
    for k in ("x", "y", "px", "py", "theta", "gamma", "offsets", "weights"):
        assert np.array_equal(beam[k], init["particles"][0][k]), k
    for h, (ux, uy) in enumerate(fields):
        assert np.array_equal(ux, init["Ux"][h]) and np.array_equal(uy, init["Uy"][h]), h


@pytest.mark.parametrize("variant", ["strict", "libm"])
@pytest.mark.parametrize("name", list(CASES))
def test_restatement_matches_reference(fb, oracle_mod, tmp_path, name, variant):
    """The CPU restatement's whole run against the reference's step loop from
    the same initial state and tables.  The strict build differs from the
    reference only in its elementary functions (deterministic sin/cos/atan
    instead of glibc's) and complex-division rounding; measured differences
    are 1e-15 .. 3e-13."""
    kind, kw = CASES[name]
    cfg, beam, fields, path, _ = ref_case(fb, tmp_path, kind, **kw)
    p = cfg.params
    r = refrun.run(path, state=([beam], fields), bessel=cfg.bessel())
    o = oracle_mod.Oracle(p, threads=4, variant=variant)
    o.set_particles(0, *(beam[k] for k in ("x", "y", "px", "py", "theta", "gamma")), beam["offsets"],
                    beam["weights"])
    for h, (ux, uy) in enumerate(fields):
        o.set_field(h, 0, ux)
        o.set_field(h, 1, uy)
    e, _, _ = o.run(0, p.max_step)
    mine, theirs = o.get_particles(0), r["final"]["particles"][0]
    for k in ("x", "y", "px", "py", "theta", "gamma"):
        assert rel_err(mine[k], theirs[k]) < 1e-11, k
    for h in range(p.num_harmony):
        assert rel_err(o.get_field(h, 0)[1:-1], r["final"]["Ux"][h][1:-1]) < 1e-11
        assert rel_err(o.get_field(h, 1)[1:-1], r["final"]["Uy"][h][1:-1]) < 1e-11
    ref_e = np.stack([r["energyX"], r["energyY"]], axis=2).reshape(p.max_step, -1)
    assert rel_err(e, ref_e) < 1e-11
