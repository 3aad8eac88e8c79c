"""Host-side setup of the input format (no GPU): parser, Domain scalars,
boundary tables, beam and seed loaders, checked against the reference's
formulas, scipy, and the CPU restatement."""
import math
import os

import numpy as np
import pytest
import scipy.special

from conftest import assert_bits

MC2 = 0.510998918
PLANCK_H = 4.135667696e-15
C_LIGHT = 299792458.0


def _cfg(fb, tmp_path, **kw):
    from felis_b200 import workloads

    path = workloads.write_input(str(tmp_path / "c.inp"), **kw)
    return fb.Config(path)


def test_domain_scalars_sase(fb, tmp_path):
    cfg = _cfg(fb, tmp_path, kind="sase")
    p = cfg.params
    assert (p.nx, p.ny) == (102, 102)  # key nx=101 -> 102 points (parameterSetting.cpp:108-111)
    assert p.dx == pytest.approx(600e-6 / 101, rel=1e-15)
    assert p.global_slice_n == 1024 and p.slice_n == 1024
    assert p.max_step == 1539  # (int)(40 / 0.026 + 1)
    assert p.dz == pytest.approx(0.026, rel=1e-15)
    assert p.gamma0 == pytest.approx(8000 / MC2 + 1, rel=1e-15)
    assert p.gam_r == pytest.approx(p.gamma0, rel=1e-12)  # resonant photon energy
    assert p.nr == int(math.sqrt(2 * 102 * 102)) and p.nr == 144
    assert p.bessel_rows == 2001 and p.bessel_cols == 2
    assert p.mode == fb.TIME_DEPENDENT and p.num_harmony == 1


def test_domain_static_and_harmonics(fb, tmp_path):
    cfg = _cfg(fb, tmp_path, kind="static", harmonics=(1, 3, 5))
    p = cfg.params
    assert p.slice_n == 1 and p.mode == fb.STATIC
    assert p.min_z == 0.0 and p.max_z == pytest.approx(p.lambda0, rel=1e-15)
    assert [p.harmony[i] for i in range(3)] == [1, 3, 5]
    assert p.bessel_cols == (5 + 1) // 2 + 1
    assert p.d_bessel == pytest.approx(5 * 2 * math.pi / 2001, rel=1e-15)


def test_parser_comments_blocks_and_missing(fb, tmp_path):
    from felis_b200 import workloads

    text = workloads.input_text("sase", slices=4)
    # comments, padding and a repeated [Undulator] block (the n-th block is read)
    text = text.replace(" nx=101", " nx  =  101   // grid points").replace("[Domain]", "  [ Domain ]")
    text += "\n[Undulator]\n undulator_type=BiPolar\n polarity=0\n numbers=2\n lambdaU=3.0\n unit_start=40\n" \
            " unit_end=44\n undulator_start=40\n undulator_end=43\n K0=2.0\n"
    path = tmp_path / "x.inp"
    path.write_text(text)
    cfg = fb.Config(str(path))
    assert cfg.params.nx == 102
    assert cfg.params.num_undulators == 2
    u2 = cfg.params.undulators[1]
    assert u2.numbers == 2 and u2.lambdaU == pytest.approx(0.03)
    assert [u2.K0[i] for i in range(2)] == [2.0, 2.0]
    assert [u2.unit_start[i] for i in range(2)] == [40.0, 44.0]
    bad = tmp_path / "bad.inp"
    bad.write_text(text.replace(" photon_energy=", " photon_energyX="))
    with pytest.raises(fb.FelisError) as e:
        fb.Config(str(bad))
    assert e.value.status == fb.NOT_FOUND
    with pytest.raises(fb.FelisError):
        fb.Config(str(tmp_path / "nope.inp"))


def test_taper_and_explicit_k_list(fb, tmp_path):
    cfg = _cfg(fb, tmp_path, kind="sase", linear_taper=-0.01)
    u = cfg.params.undulators[0]
    K = [u.K0[i] for i in range(u.numbers)]
    # K0 + i * linTaper / sqrt(2) (parameterSetting.cpp:383,414)
    assert K == pytest.approx([2.6 + i * (-0.01 / math.sqrt(2.0)) for i in range(10)], rel=1e-15)


def test_bessel_table_vs_scipy(fb, tmp_path):
    cfg = _cfg(fb, tmp_path, kind="static", harmonics=(1, 3, 5, 7))
    B = cfg.bessel()
    p = cfg.params
    x = p.d_bessel * np.arange(p.bessel_rows)
    for order in range(p.bessel_cols):
        ref = scipy.special.jv(order, x)
        np.testing.assert_allclose(B[:, order], ref, rtol=1e-13, atol=1e-15)


def test_abc_tables_match_restatement(fb, oracle_mod, tmp_path):
    cfg = _cfg(fb, tmp_path, kind="sase", slices=2, nx=41)
    o = oracle_mod.Oracle(cfg.params)
    for a, b in zip(cfg.abc(), o.abc()):
        assert_bits(a, b, "ABC table")
    al, alp, be, bep = cfg.abc()
    # interior coefficients are -i dz / (2 ks dx^2 s_i (s_i + s_{i-1})): small, imaginary-dominated
    assert np.all(np.abs(al[1:-1]) < 1e-2) and np.all(np.abs(al[1:-1].imag) > 0)


def test_beam_loader_statistics(fb, tmp_path):
    cfg = _cfg(fb, tmp_path, kind="sase", slices=8, beamlets=1024)
    p = cfg.params
    b = cfg.load_beam(0, seed=2)
    assert b["offsets"][-1] == 8 * 1024 * 4
    g0 = 8000 / MC2 + 1
    sig = math.sqrt(0.4e-6 / g0 * 20.0)  # sqrt(emit / gamma_twiss), alpha = 0
    assert np.std(b["x"]) == pytest.approx(sig, rel=0.03)
    assert np.std(b["y"]) == pytest.approx(sig, rel=0.03)
    assert np.mean(b["gamma"]) == pytest.approx(g0, rel=1e-6)
    assert np.std(b["gamma"]) / g0 == pytest.approx(1e-4, rel=0.05)
    th = b["theta"]
    # Fawley shot-noise kicks: sigma = sqrt(2 / (w * n_beamlet)) ~ 0.4 rad here
    # theta0 in [0, 2pi) plus n * 2pi/4 (loadBeam.cpp:185,240), wrapped only by the loop
    assert th.min() > -2.5 and th.max() < 3.5 * math.pi + 2.5 and abs(np.mean(np.exp(1j * th))) < 0.05
    # weight: peak_current / e / c * lambda0 / particles per slice (loadBeam.cpp:63)
    assert b["weights"][0] == pytest.approx(3000 / 1.60217662e-19 / C_LIGHT * p.lambda0 / 4096, rel=1e-12)


def test_quiet_start_phases(fb, tmp_path):
    cfg = _cfg(fb, tmp_path, kind="static", beamlets=64)
    b = cfg.load_beam(0, seed=1)
    th = b["theta"].reshape(-1, 4)
    np.testing.assert_allclose(np.diff(th, axis=1), 2 * math.pi / 4, rtol=1e-12)
    assert np.all(b["x"].reshape(-1, 4) == b["x"].reshape(-1, 4)[:, :1])
    # quiet start: bunching of the loaded beam vanishes
    assert abs(np.exp(1j * b["theta"]).mean()) < 1e-12


def test_seed_power_normalisation(fb, tmp_path):
    cfg = _cfg(fb, tmp_path, kind="static", seed_power=1e6)
    p = cfg.params
    ux, uy = cfg.load_seed(0)
    assert np.all(uy == 0)  # laser_alpha = 1: x polarisation only
    coef = (9.10938291e-31 * C_LIGHT ** 2 * p.ks / 1.60217662e-19) ** 2 / (2 * 376.730313668) * p.dx * p.dy
    power = np.sum(np.abs(ux[1]) ** 2) * coef  # updateTotalEnergy.cpp:38-45 (static: no dt)
    assert power == pytest.approx(1e6, rel=1e-3)


def test_wake_circular_ac(fb, tmp_path):
    cfg = _cfg(fb, tmp_path, kind="sase", slices=64, wake=True)
    den = np.full(64, 1e6)
    w = cfg.wake(den)
    assert w.shape == (64,) and np.all(np.isfinite(w))
    # causal convolution: the head slice sees its own wake only
    assert abs(w[-1]) <= abs(w).max()


def _sobol_direct(n, dims=3, bits=30):
    """Point n (1-based) of the Gray-code Sobol sequence computed directly:
    XOR of the direction numbers at the set bits of gray(n) = n ^ (n >> 1)
    (Antonov-Saleev), direction numbers of Bratley-Fox for the polynomials
    1, x + 1, x^2 + x + 1 (initial m 1; 1; 1, 3)."""
    m = [[1] * (bits + 1) for _ in range(dims)]
    for k in range(2, bits + 1):
        m[1][k] = (2 * m[1][k - 1]) ^ m[1][k - 1]
    m[2][2] = 3
    for k in range(3, bits + 1):
        m[2][k] = (2 * m[2][k - 1]) ^ (4 * m[2][k - 2]) ^ m[2][k - 2]
    g = n ^ (n >> 1)
    out = []
    for d in range(dims):
        x = 0
        for k in range(1, bits + 1):
            if (g >> (k - 1)) & 1:
                x ^= m[d][k] << (bits - k)
        out.append(x / 2.0 ** bits)
    return out


def test_1d_loader(fb, tmp_path):
    """loadBeam.cpp:271-446: particles without transverse coordinates, the
    phase of each beamlet's first particle and its energy from consecutive
    Sobol points (noise off)."""
    from felis_b200 import workloads

    path = workloads.write_input(str(tmp_path / "d1.inp"), kind="sase", slices=6, beamlets=16, per_beamlet=4,
                                 dimension=1, noise=False, spread_pct=0.01)
    cfg = fb.Config(path)
    p = cfg.params
    b = cfg.load_beam(0, seed=3)
    n = int(b["offsets"][-1])
    assert n == 6 * 16 * 4
    for k in ("x", "y", "px", "py"):
        assert not np.any(b[k])
    dPhi = 2 * math.pi * p.num_slice
    div = 2 * math.pi / 4
    gamma0 = p.gamma0
    dGam = 1e-4 * gamma0  # spread 0.01 % with the flat energy-spread profile
    for beamlet in range(24):
        v = _sobol_direct(beamlet + 1)
        th0 = v[0] * dPhi
        for q in range(4):
            assert b["theta"][beamlet * 4 + q] == th0 + q * div
        expect = gamma0 + dGam * math.sqrt(-2.0 * math.log(v[1])) * math.cos(v[2] * 2.0 * math.pi)
        assert abs(b["gamma"][beamlet * 4] - expect) <= 1e-12 * gamma0
    # 1D seed: one value per slice; the 1D Domain has nx = ny = 1
    ux, uy = cfg.load_seed(0)
    assert ux.shape == (p.slice_n + 2, 1, 1) and np.all(ux[1:-1] != 0) and not np.any(ux[[0, -1]])
