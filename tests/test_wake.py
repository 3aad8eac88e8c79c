"""Wake function and wake field of the host (felis_config_wake,
wakeField.cpp:9-50, 53-159) against the numpy restatement in oracle/wake.py,
and the restatement pinned by the resistive-wall limit W(0+) = Z0 c / (pi a^2)
of the round pipe."""

import numpy as np
import pytest
from scipy import integrate

import wake as wref

RADIUS, COND, CTAU = 5e-3, 5.8e7, 8.1e-6
SHAPES = {"circular_ac": ("Circular", "AC"), "circular_dc": ("Circular", "DC"), "flat_ac": ("Flat", "AC")}


def wake_config(fb, tmp_path, shape, acdc, slices=96):
    from felis_b200 import workloads

    path = workloads.write_input(str(tmp_path / "w.inp"), kind="sase", slices=slices, beamlets=64, nx=21,
                                 wake=True, seed_power=0.0, total_length=4.0)
    text = open(path).read().replace("shape=Circular", f"shape={shape}").replace("ac_dc=AC", f"ac_dc={acdc}")
    open(path, "w").write(text)
    return fb.Config(path)


def density(S, seed=3):
    rng = np.random.default_rng(seed)
    z = np.arange(S)
    return 1e5 * np.exp(-0.5 * ((z - S / 2) / (S / 6)) ** 2) * (1 + 0.1 * rng.random(S))


def test_round_pipe_wake_at_origin():
    """DC round pipe: the integral of the impedance over k, with the analytic
    tail beyond the table's k = 20, is pi, i.e. W(0+) = Z0 c / (pi a^2)."""
    imp, _ = wref.impedance("Circular", "DC", RADIUS, COND, 0.0)
    f = lambda k: 1.0 / np.sqrt(k) / (2.0 / k + 0.25 * k * k - np.sqrt(k))
    tail, _ = integrate.quad(f, wref.MAX_K, np.inf, limit=200)
    # trapezoid end correction of the table's left-point sum
    dK = wref.MAX_K / wref.NUM_K
    total = imp.sum() * dK - 0.5 * imp[-1] * dK + tail
    assert abs(total / np.pi - 1.0) < 2e-3


@pytest.mark.parametrize("name", sorted(SHAPES))
def test_host_wake_matches_restatement(fb, tmp_path, name):
    shape, acdc = SHAPES[name]
    cfg = wake_config(fb, tmp_path, shape, acdc)
    p = cfg.params
    S, dZ = p.global_slice_n, p.num_slice * p.lambda0
    den = density(S)
    we = cfg.wake(den)
    wf = cfg.wake_function()
    ctau = CTAU if acdc == "AC" else 0.0
    wf_ref = wref.wake_function(S, dZ, shape, acdc, RADIUS, COND, ctau)
    np.testing.assert_allclose(wf, wf_ref, rtol=1e-10, atol=1e-10 * np.abs(wf_ref).max())
    np.testing.assert_allclose(we, wref.wake_field(den, wf, dZ), rtol=1e-12, atol=1e-12 * np.abs(we).max())
    assert np.abs(we).max() > 0
