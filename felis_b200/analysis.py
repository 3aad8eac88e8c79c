"""Figures of merit of a FELIS run, used to state the error of the
mixed-precision ensemble against the FP64 plain path.

  output power     sum over polarisations of a harmonic's field energy
                   (the per-iteration sums of updateTotalEnergy.cpp:25-36,
                   unscaled: every comparison here is a ratio)
  gain length      z distance over which the power grows by e, from a
                   least-squares line through ln P(z) over the exponential
                   stretch (between `lo` and `hi` of the final power)
  spectral centroid / bandwidth
                   first and second moments of the transverse-integrated
                   power spectrum over the slices, |FFT_s U(x, y, s)|^2, in
                   units of the slice frequency 1 / (numSlice lambda0)
"""
from __future__ import annotations

import numpy as np


def output_power(energy: np.ndarray, hidx: int = 0) -> np.ndarray:
    """energy[it, 2H] (Ux, Uy interleaved per harmonic) -> P[it] of harmonic hidx."""
    e = np.asarray(energy)
    return e[:, 2 * hidx] + e[:, 2 * hidx + 1]


def gain_length(power: np.ndarray, dz: float, lo: float = 1e-3, hi: float = 0.1) -> float:
    """Gain length [m] of a power curve sampled every dz metres."""
    p = np.asarray(power, dtype=np.float64)
    top = p.max()
    sel = np.flatnonzero((p > lo * top) & (p < hi * top))
    if sel.size < 3:
        sel = np.arange(len(p) // 4, len(p))
    z = sel * dz
    slope = np.polyfit(z, np.log(p[sel]), 1)[0]
    return float(1.0 / slope) if slope > 0 else float("inf")


def spectrum(field: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """field[S, ny, nx] (one harmonic and polarisation, physical slices) ->
    (frequency in units of 1/S per slice, transverse-integrated power)."""
    f = np.asarray(field)
    S = f.shape[0]
    F = np.fft.fft(f, axis=0)
    p = (np.abs(F) ** 2).sum(axis=(1, 2))
    nu = np.fft.fftfreq(S)
    order = np.argsort(nu)
    return nu[order], p[order]


def spectral_moments(field: np.ndarray) -> tuple[float, float]:
    """(centroid, rms bandwidth) of spectrum(field)."""
    nu, p = spectrum(field)
    w = p / p.sum()
    c = float((nu * w).sum())
    return c, float(np.sqrt(((nu - c) ** 2 * w).sum()))


def lag_moments(r) -> tuple[float, float]:
    """(centroid, rms width), in units of the slice frequency, from the
    first-lag moments (R0, Re R1, Im R1) of felis_batch_spectral_moments:
    R1 / R0 = <e^{2 pi i nu}> over the slice spectrum, so the centroid is its
    circular mean arg(R1) / (2 pi) and the width that of the Gaussian line
    with the same |R1| / R0, sqrt(-2 ln(|R1| / R0)) / (2 pi)."""
    r0, re, im = (float(v) for v in r)
    c = np.arctan2(im, re) / (2.0 * np.pi)
    q = min(np.hypot(re, im) / r0, 1.0) if r0 > 0 else 0.0
    w = np.sqrt(-2.0 * np.log(q)) / (2.0 * np.pi) if q > 0 else float("inf")
    return float(c), float(w)
