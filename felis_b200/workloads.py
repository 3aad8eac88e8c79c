"""Input files (FELIS .inp format) for the workloads this library is measured on.

The reference publishes no benchmark inputs; these are the synthetic beams
of the project's workload table, written in the reference's own input format
(README.md:51-187; keys as parsed by parameterSetting.cpp):

  static   Plain FP64 steady-state single slice: 8 GeV, relative energy
           spread 1e-4, normalised emittance 0.4 um, beta 20 m, 3 kA;
           2048 beamlets x 4 quiet-start particles; BiPolar undulator
           lambda_u 2.6 cm, K0 2.6, 10 units of 3.4 m with 0.6 m in-air gaps;
           1 MW Gaussian seed, waist 30 um; 102 x 102 grid over +-300 um,
           ABC_N 10; 40 m (1539 steps of one period).
  sase     Plain FP64 time-dependent SASE: the same beam and undulator,
           flat-top 3 kA over 1024 slices, 8192 particles per slice with
           shot-noise phases, no seed.

The seed is put into the x polarisation (laser_alpha = 1), the one a
K0_alpha = 1 planar undulator couples to; with the reference's default
laser_alpha = -1 it would land in Uy and never interact.
"""
from __future__ import annotations

import math
import os
import tempfile

PLANCK_H = 4.135667696e-15  # [eV s], constants.h
C_LIGHT = 299792458.0
MC2 = 0.510998918


def resonant_photon_energy(energy_mev: float, lambda_u_cm: float, K0: float) -> float:
    gamma = energy_mev / MC2 + 1.0
    lam_u = lambda_u_cm * 0.01
    lam0 = lam_u / (2.0 * gamma * gamma) * (1.0 + 0.5 * K0 * K0)
    return PLANCK_H * C_LIGHT / lam0


def input_text(kind: str = "sase", *, slices: int = 1024, beamlets: int = 2048, per_beamlet: int = 4,
               nx: int = 101, window_um: float = 300.0, total_length: float = 40.0, harmonics=(1,),
               energy_mev: float = 8000.0, spread_pct: float = 0.01, emit_um: float = 0.4, beta: float = 20.0,
               current: float = 3000.0, K0: float = 2.6, lambda_u_cm: float = 2.6, units: int = 10,
               unit_len: float = 4.0, und_len: float = 3.4, seed_power: float = 1e6, seed_sigma_um: float = 30.0,
               noise: bool | None = None, undulator: str = "BiPolar", polarity: float = 0.0,
               linear_taper: float = 0.0, wake: bool = False, quads: bool = False, abc_n: int = 10,
               in_air: bool = True, k_list=None, sigma_slices: float | None = None, profile_nodes: int = 65,
               K_und: float | None = None, dimension: int = 3, phase_shifters=(), bucket: int = 1) -> str:
    """Input text of one workload.  `sigma_slices` switches the flat-top
    current to a Gaussian of that rms length (in slices) centred on the bunch,
    written as a `profile_nodes`-node Polygon so that the energy-spread nodes
    still apply (loadBeam.cpp's Gaussian load type has no spread).  `K0` sets
    the photon energy by the planar resonance; `K_und` (default K0) is the
    undulator's K, e.g. K0 / sqrt(1 + polarity^2) for an elliptical undulator
    on the same resonance (parameterSetting.cpp's default K0).  `dimension` 1
    selects the 1D model (the grid collapses to one cell per slice).
    `phase_shifters` lists [Phase_shifter] blocks as (number, start_position
    [m], interval_length [m], phase [pi]) tuples (README.md:57-70).
    `bucket` sets slices_in_bucket = lambdaUs_in_iteration: each slice spans
    `bucket` wavelengths and one step `bucket` undulator periods, so the field
    still slips one slice per step."""
    static = kind == "static"
    if noise is None:
        noise = not static
    photon = resonant_photon_energy(energy_mev, lambda_u_cm, K0)
    lam0_um = PLANCK_H * C_LIGHT / photon * 1e6
    minZ, maxZ = 0.0, (slices + 0.5) * bucket * lam0_um
    k_line = "" if k_list is None else " K0_list=" + ",".join(repr(float(k)) for k in k_list) + "\n"
    harm = "\n".join(f" harmony{i} = {h}" for i, h in enumerate(harmonics))
    zspan = 1.0e-3
    if sigma_slices is None:
        z_nodes = f" z_nodes=2\n z0={-zspan}\n z1={zspan}\n z_n0=1\n z_n1=1"
    else:
        lam0 = lam0_um * 1e-6 * bucket  # slice length
        centre, sig = 0.5 * slices * lam0, sigma_slices * lam0
        zs = [(-1.0 + (slices + 2.0) * k / (profile_nodes - 1)) * lam0 for k in range(profile_nodes)]
        lines = [f" z_nodes={profile_nodes}"]
        lines += [f" z{k}={z!r}" for k, z in enumerate(zs)]
        lines += [f" z_n{k}={math.exp(-0.5 * ((z - centre) / sig) ** 2)!r}" for k, z in enumerate(zs)]
        z_nodes = "\n".join(lines)
    quad_block = ""
    if quads:
        quad_block = """
[Quad]
 numbers=10
 unit_start = 3.6
 unit_end = 7.6
 quad_start = 3.6
 quad_end = 3.7
 g = 10

[Quad]
 numbers=10
 unit_start = 5.6
 unit_end = 9.6
 quad_start = 5.6
 quad_end = 5.7
 g = -10
"""
    ps_blocks = "".join(f"""
[Phase_shifter]
 number={n}
 start_position={z0!r}
 interval_length={dzs!r}
 phase={ph!r}
""" for n, z0, dzs, ph in phase_shifters)
    return f"""// generated by felis_b200.workloads ({kind})
{ps_blocks}
[Save]
 field_save=OFF
 particle_save=OFF
 total_length={total_length}
 save_step=1000000
 save_start=1000000

[Domain]
 dimension={dimension}
 mode={'Static' if static else 'Time_Dependent'}
 minZ={minZ!r}
 maxZ={maxZ!r}
 minX={-window_um}
 maxX={window_um}
 minY={-window_um}
 maxY={window_um}
 nx={nx}
 ny={nx}
 photon_energy={photon!r}
 num_harmony={len(harmonics)}
{harm}
 slices_in_bucket={bucket}
 lambdaUs_in_iteration={bucket}
 ABC_N={abc_n}
 ABC_coef=1

[Seed]
 power={seed_power}
 rms_duration=1e9
 spot_sigma_R={seed_sigma_um}
 focus=0
 laser_alpha=1

[Undulator]
 undulator_type={undulator}
 polarity={polarity}
 K0_alpha=1
 numbers={units}
 in_air={'ON' if in_air else 'OFF'}
 linear_taper={linear_taper}
 lambdaU={lambda_u_cm}
 unit_start=0.0
 unit_end={unit_len}
 undulator_start=0.0
 undulator_end={und_len}
 K0={K0 if K_und is None else K_und}
{k_line}
[Wake_field]
 activate={'ON' if wake else 'OFF'}
 shape=Circular
 ac_dc=AC
 radius=5e-3
 conductivity=5.8e7
 ctau=8.1e-6
{quad_block}
[EBeam]
 load_type=Polygon
 noise_ONOFF={'ON' if noise else 'OFF'}
 beam_energy={energy_mev}
 energy_spread={spread_pct}
 peak_current={current}
 norm_emittance_x={emit_um}
 norm_emittance_y={emit_um}
 beta_x={beta}
 beta_y={beta}
 alpha_x=0
 alpha_y=0
 beamlets_in_bucket={beamlets}
 number_in_beamlet={per_beamlet}
{z_nodes}
 energy_nodes=2
 energy_z0={-zspan}
 energy_z1={zspan}
 energy_n0=1
 energy_n1=1
 energySpread_nodes=2
 energySpread_z0={-zspan}
 energySpread_z1={zspan}
 energySpread_n0=1
 energySpread_n1=1
 emit_nodes=2
 emit_z0={-zspan}
 emit_z1={zspan}
 emit_n0=1
 emit_n1=1
"""


def write_input(path: str | None = None, kind: str = "sase", **kw) -> str:
    text = input_text(kind, **kw)
    if path is None:
        fd, path = tempfile.mkstemp(prefix=f"felis_{kind}_", suffix=".inp")
        os.close(fd)
    with open(path, "w") as f:
        f.write(text)
    return path


WORKLOADS = {
    "static": dict(kind="static"),
    "sase": dict(kind="sase", seed_power=0.0),
    # mixed-precision long run: QuadPolar (polarity 0.5), harmonics 1 and 3,
    # Gaussian current (rms 600 slices, peak 4 kA, 16384 particles per slice
    # at the peak), copper AC wake in a 5 mm pipe, 151 x 151 grid, 60 m with
    # a linear taper to K = 0.99 K0 in the last of 15 units
    "gaussian_taper": dict(kind="sase", slices=4096, sigma_slices=600.0, current=4000.0, beamlets=4096,
                           per_beamlet=4, nx=151, harmonics=(1, 3), undulator="QuadPolar", polarity=0.5,
                           wake=True, units=15, total_length=60.0, seed_power=0.0,
                           K_und=2.6 / math.sqrt(1.25), linear_taper=-0.01 * 2.6 / math.sqrt(1.25) * math.sqrt(2.0) / 14.0),
}


def ensemble(n: int = 96, seed: int = 20240601) -> list[dict]:
    """The batched SASE ensemble (shot noise, no seed laser): n instances with beam seeds 1..n, slice
    counts uniform in {128, 256, 512, 1024, 2048}, grid keys nx = ny from
    {65, 101, 151}, 1024 beamlets x 4 = 4096 particles per slice, peak current
    uniform in [2, 4] kA and relative energy spread uniform in [0.5, 2]e-4.
    Returns input_text keyword sets with a `beam_seed` entry."""
    import random

    rng = random.Random(seed)
    out = []
    for k in range(n):
        out.append(dict(kind="sase", seed_power=0.0, slices=rng.choice([128, 256, 512, 1024, 2048]), beamlets=1024,
                        per_beamlet=4, nx=rng.choice([65, 101, 151]), current=rng.uniform(2000.0, 4000.0),
                        spread_pct=rng.uniform(0.5e-4, 2e-4) * 100.0, beam_seed=k + 1))
    return out
