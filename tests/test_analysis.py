"""The figures of merit the mixed-precision error is stated in
(felis_b200/analysis.py, felis_b200/longrun.compare), on inputs whose answers
are known in closed form."""
import numpy as np

from felis_b200 import analysis, longrun


def _energy(power_h1, power_h3=None):
    """energy[it, 2H] with the power split evenly over the polarisations."""
    cols = [power_h1 * 0.5, power_h1 * 0.5]
    if power_h3 is not None:
        cols += [power_h3 * 0.25, power_h3 * 0.75]
    return np.stack(cols, axis=1)


def test_output_power_sums_polarisations():
    e = np.array([[1.0, 2.0, 10.0, 20.0], [3.0, 4.0, 30.0, 40.0]])
    assert np.array_equal(analysis.output_power(e, 0), [3.0, 7.0])
    assert np.array_equal(analysis.output_power(e, 1), [30.0, 70.0])


def test_gain_length_of_an_exponential_with_saturation():
    dz, Lg = 0.026, 1.7
    z = np.arange(2000) * dz
    p = 1e-6 * np.exp(z / Lg)
    p = np.minimum(p, 1e-6 * np.exp(40.0))  # saturated tail is excluded by the window
    assert abs(analysis.gain_length(p, dz) / Lg - 1.0) < 1e-9


def test_gain_length_without_growth_is_infinite():
    assert analysis.gain_length(np.full(100, 2.0), 0.1) == float("inf")


def test_spectrum_of_one_frequency():
    S, k = 64, 5
    s = np.arange(S)
    field = np.exp(2j * np.pi * k * s / S)[:, None, None] * np.ones((1, 3, 4))
    c, w = analysis.spectral_moments(field)
    assert abs(c - k / S) < 1e-12
    assert w < 1e-7
    nu, p = analysis.spectrum(field)
    assert np.all(np.diff(nu) > 0)
    assert abs(p.sum() - (S * 12) * S) < 1e-6 * p.sum()


def test_spectral_moments_of_two_lines():
    S = 128
    s = np.arange(S)
    # equal power at +4/S and -4/S: centroid 0, rms width 4/S
    field = (np.exp(2j * np.pi * 4 * s / S) + np.exp(-2j * np.pi * 4 * s / S))[:, None, None]
    c, w = analysis.spectral_moments(field)
    assert abs(c) < 1e-12
    assert abs(w - 4 / S) < 1e-12


def test_compare_states_the_perturbation():
    """A mixed run whose power is the reference's times (1 + eps) reports eps
    as its power error at every iteration and no gain-length error; identical
    spectra report no centroid or width error."""
    dz, Lg, eps = 0.026, 2.0, 3e-4
    z = np.arange(600) * dz
    p1 = 1e-3 * np.exp(z / Lg)
    p3 = 1e-5 * np.exp(z / (Lg / 2))
    ref_e = _energy(p1, p3)
    mix_e = _energy(p1 * (1 + eps), p3 * (1 - eps))
    S = 32
    s = np.arange(S)
    f = (np.exp(2j * np.pi * 3 * s / S) + 0.5 * np.exp(2j * np.pi * 2 * s / S))[:, None, None] * np.ones((1, 2, 2))
    spec = [analysis.spectrum(f), analysis.spectrum(f)]
    out = longrun.compare({"energy": ref_e, "spectra": spec}, {"energy": mix_e, "spectra": spec}, 2, [1, 3], dz)
    h1, h3 = out["H1"], out["H3"]
    assert abs(h1["power_final_rel_error"] - eps) < 1e-12
    assert abs(h3["power_final_rel_error"] - eps) < 1e-12
    assert abs(h1["power_max_rel_error_all"] - eps) < 1e-12
    assert h1["gain_length_rel_error"] < 1e-9 and h3["gain_length_rel_error"] < 1e-9
    assert abs(h1["gain_length_m"] / Lg - 1) < 1e-9 and abs(h3["gain_length_m"] / (Lg / 2) - 1) < 1e-9
    assert h1["centroid_error_over_width"] == 0.0 and h1["width_rel_error"] == 0.0
