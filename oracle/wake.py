"""Numpy restatement of the reference's wake function and wake field.

TEST INFRASTRUCTURE ONLY: imported by tests/, never by the felis_b200 package.

    wake_function   wakeField.cpp:53-159 (impedance of the flat or circular
                    resistive pipe, PRAB 18, 034401 (2015), then its cosine
                    transform per slice distance)
    wake_field      wakeField.cpp:9-50 with makeDensity (:161-223)

Vectorised over wavenumbers and slices; the sums use numpy's summation order,
so they agree with the reference's serial sums to rounding (about 1e-14
relative), not bit for bit.  Pinned by the analytic DC limit of the circular
pipe in tests/test_wake.py.
"""
from __future__ import annotations

import numpy as np

Z0 = 376.730313668  # constants.h
NUM_K, MAX_K = 1000, 20.0
NUM_X, MAX_X = 50000, 2000.0


def impedance(shape: str, acdc: str, radius: float, cond: float, ctau: float) -> tuple[np.ndarray, float]:
    """impZ[0..numK] and s0 (wakeField.cpp:63-116)."""
    s0 = (2.0 * radius * radius / Z0 / cond) ** (1.0 / 3.0)
    dK = MAX_K / NUM_K
    k = np.arange(NUM_K + 1) * dK
    imp = np.zeros(NUM_K + 1)
    if shape == "Flat":
        dX = MAX_X / NUM_X
        x = np.arange(NUM_X + 1) * dX
        x = x[x <= 320]  # the terms beyond are zero
        xs = x[1:]
        ch, sh = np.cosh(xs), np.sinh(xs)
        for a in range(1, NUM_K + 1, 100):
            kk = k[a:a + 100][:, None]
            A = 2.0 / (1.0 - 1j) / np.sqrt(kk - 1j * kk * kk * ctau / s0)
            cd = A * ch - 1j * kk * sh / xs
            cal = (1.0 / ch) / cd
            x0 = np.sqrt(kk[:, 0]) / (2.0 + kk[:, 0] ** 3 - 2.0 * np.sqrt(kk[:, 0]) * kk[:, 0])
            imp[a:a + 100] = x0 * dX + (cal.real * dX).sum(axis=1)
    elif shape == "Circular":
        kk = k[1:]
        if acdc == "AC":
            cd = np.sqrt(2.0 * s0 / ctau) / kk * (1j + s0 * 0.5 / kk / ctau) - 1j * 0.5 * kk
            imp[1:] = (1.0 / cd).real
        else:
            dino = 2.0 / kk + 0.25 * kk * kk - np.sqrt(kk)
            imp[1:] = 1.0 / np.sqrt(kk) / dino
    return imp, s0


def wake_function(S: int, dZ: float, shape: str, acdc: str, radius: float, cond: float, ctau: float) -> np.ndarray:
    """wakeF[i] for the slice distance i dZ (wakeField.cpp:128-140)."""
    imp, s0 = impedance(shape, acdc, radius, cond, ctau)
    dK = MAX_K / NUM_K
    k = np.arange(NUM_K + 1) * dK
    coef = Z0 * 3e8 / np.pi / radius / radius / np.pi
    z = (np.arange(S) * dZ) / s0
    return (imp[None, :] * np.cos(k[None, :] * z[:, None]) * dK).sum(axis=1) * coef


def wake_field(den: np.ndarray, wakeF: np.ndarray, dZ: float) -> np.ndarray:
    """wakeE[ii] = sum_{i >= ii} den_n[i] wakeF[i - ii] dZ coef with den_n the
    density normalised to unit integral and coef = total charge count x 1.602e-19."""
    den = np.asarray(den, dtype=np.float64)
    tot = den.sum()
    dn = den / (tot * dZ) if tot > 0 else den
    coef = tot * 1.602e-19
    S = den.size
    out = np.zeros(S)
    for ii in range(S):
        out[ii] = (dn[ii:] * wakeF[:S - ii]).sum() * dZ * coef
    return out
