"""Mixed-precision ensemble (felis_batch_*) on the GPU.

Two kinds of checks:
  * error against the FP64 plain path (itself bit-identical to the CPU
    restatement, test_gpu_parity.py) on the same initial state, stated per
    figure of merit: output power per iteration, gain length, spectral
    centroid and bandwidth;
  * exact properties of the ensemble: an instance's results do not depend on
    the other instances, on the launch shape or on the run (fixed-point
    deposit, no float atomics).
"""
import numpy as np
import pytest

from conftest import make_case

pytestmark = pytest.mark.gpu

# Tolerances of the mixed path against FP64 (relative unless stated).
POWER_RTOL = 1e-3        # output power at every iteration
GAIN_LENGTH_RTOL = 1e-4  # gain length fitted over the exponential stretch
CENTROID_ATOL = 1e-3     # spectral centroid, in units of the rms bandwidth
BANDWIDTH_RTOL = 1e-3    # rms bandwidth
TWISS_RTOL = 1e-4        # emittance, beta, alpha of the final beam
BUNCHING_RTOL = 1e-3     # |bunching factor| of the final beam

# 1 GeV beam in the 2.6 cm undulator: gain length about 0.8 m, so 10 m show
# four orders of magnitude of seeded gain in 385 iterations.
SEEDED = dict(slices=400, beamlets=64, nx=41, total_length=10.0, seed_power=1e5, units=3, energy_mev=1000.0)


def _upload(fb, b, k, cfg, beam, fields):
    b.upload_particles(k, beam["x"], beam["y"], beam["px"], beam["py"], beam["theta"], beam["gamma"],
                       beam["offsets"], beam["weights"])
    for h, (ux, uy) in enumerate(fields):
        b.upload_field(k, h, 0, ux)
        b.upload_field(k, h, 1, uy)


def _fp64(fb, cfg, beam, fields, steps):
    g = fb.Handle(cfg.params)
    g.upload_particles(0, beam["x"], beam["y"], beam["px"], beam["py"], beam["theta"], beam["gamma"],
                       beam["offsets"], beam["weights"])
    for h, (ux, uy) in enumerate(fields):
        g.upload_field(h, 0, ux)
        g.upload_field(h, 1, uy)
    g.run(0, steps)
    return g


def _state(b, k, H):
    p = b.download_particles(k)
    f = [b.download_field(k, h, pol) for h in range(H) for pol in (0, 1)]
    return p, f


def _same(a, b, what):
    for k in a[0]:
        assert np.array_equal(a[0][k], b[0][k]), f"{what}: particles {k}"
    for i, (x, y) in enumerate(zip(a[1], b[1])):
        assert np.array_equal(x, y), f"{what}: field plane {i}"


@pytest.fixture
def seeded(fb, tmp_path):
    return make_case(fb, tmp_path, kind="sase", **SEEDED)


def test_mixed_vs_fp64_figures_of_merit(fb, seeded):
    from felis_b200 import analysis

    cfg, beam, fields = seeded
    p = cfg.params
    steps = p.max_step
    g = _fp64(fb, cfg, beam, fields, steps)
    b = fb.Batch([p])
    _upload(fb, b, 0, cfg, beam, fields)
    b.run(0, steps)
    e64, t64, bf64 = g.diagnostics(0, steps + 1)
    e32, t32, bf32 = b.diagnostics(0, 0, steps + 1)
    P64, P32 = analysis.output_power(e64), analysis.output_power(e32)
    assert P64[-1] > 1e3 * P64[0], "the seeded case must show gain"
    rel = np.abs(P32 - P64) / P64
    assert rel.max() < POWER_RTOL, f"power: max rel err {rel.max():.3e}"
    lg64, lg32 = analysis.gain_length(P64, p.dz), analysis.gain_length(P32, p.dz)
    assert abs(lg32 / lg64 - 1) < GAIN_LENGTH_RTOL, (lg32, lg64)
    u64 = g.download_field(0, 0)[1:-1]
    u32 = b.download_field(0, 0, 0)[1:-1]
    c64, w64 = analysis.spectral_moments(u64)
    c32, w32 = analysis.spectral_moments(u32)
    assert abs(c32 - c64) < CENTROID_ATOL * w64, (c32, c64, w64)
    assert abs(w32 / w64 - 1) < BANDWIDTH_RTOL, (w32, w64)
    # twiss and bunching of the final state
    np.testing.assert_allclose(t32[-1], t64[-1], rtol=TWISS_RTOL)
    np.testing.assert_allclose(np.hypot(bf32[-1, 0], bf32[-1, 1]), np.hypot(bf64[-1, 0], bf64[-1, 1]),
                               rtol=BUNCHING_RTOL)


def test_mixed_vs_fp64_every_harmonic_and_polarisation(fb, tmp_path):
    """An elliptical undulator (QuadPolar, polarity 0.5) with harmonics 1, 2
    and 3: each harmonic and polarisation has its own source plane (odd
    harmonics one shared plane, even harmonics one per polarisation), and the
    power of every one of the 2 H planes follows FP64."""
    import math

    cfg, beam, fields = make_case(fb, tmp_path, kind="sase", **dict(
        SEEDED, slices=96, harmonics=(1, 2, 3), undulator="QuadPolar", polarity=0.5, K_und=2.6 / math.sqrt(1.25)))
    p = cfg.params
    steps = p.max_step
    g = _fp64(fb, cfg, beam, fields, steps)
    b = fb.Batch([p])
    _upload(fb, b, 0, cfg, beam, fields)
    b.run(0, steps)
    e64, _, _ = g.diagnostics(0, steps + 1)
    e32, _, _ = b.diagnostics(0, 0, steps + 1)
    for col in range(2 * p.num_harmony):
        P64, P32 = e64[:, col], e32[:, col]
        assert P64[-1] > 0 and P32[-1] > 0, f"plane {col}: no field"
        sel = P64 > 1e-6 * P64.max()
        rel = np.abs(P32[sel] - P64[sel]) / P64[sel]
        assert rel.max() < POWER_RTOL, f"plane {col} (harmonic {p.harmony[col // 2]}, pol {col % 2}): {rel.max():.3e}"


def test_initial_diagnostics_match_fp64(fb, seeded):
    cfg, beam, fields = seeded
    g = _fp64(fb, cfg, beam, fields, 1)
    b = fb.Batch([cfg.params])
    _upload(fb, b, 0, cfg, beam, fields)
    b.run(0, 1)
    e64, t64, bf64 = g.diagnostics(0, 2)
    e32, t32, bf32 = b.diagnostics(0, 0, 2)
    # state stored in FP32: energy and twiss agree to FP32 rounding
    np.testing.assert_allclose(e32[0], e64[0], rtol=1e-6)
    np.testing.assert_allclose(t32[0], t64[0], rtol=1e-5)
    np.testing.assert_allclose(bf32[0], bf64[0], rtol=1e-4, atol=1e-6)
    np.testing.assert_allclose(e32[1], e64[1], rtol=1e-4)


def test_instances_independent(fb, tmp_path):
    """An instance gives the same bits whatever the other instances of the
    ensemble are and wherever it sits in it.  (The kernel instance is chosen by
    the ensemble's largest harmonic count; both ensembles here use the one for
    up to 4 harmonics.)"""
    (tmp_path / "a").mkdir()
    (tmp_path / "c").mkdir()
    a = make_case(fb, tmp_path / "a", kind="sase", slices=8, beamlets=128, nx=41, total_length=2.0)
    c = make_case(fb, tmp_path / "c", kind="sase", slices=12, beamlets=64, nx=61, total_length=2.0,
                  harmonics=(1, 2, 3), undulator="QuadPolar", polarity=0.5, seed_power=2e6)
    steps = 30
    pair = fb.Batch([a[0].params, c[0].params])
    for k, case in enumerate((a, c)):
        _upload(fb, pair, k, *case)
    pair.run(0, steps)
    mix = fb.Batch([c[0].params, a[0].params, c[0].params])
    for k, case in enumerate((c, a, c)):
        _upload(fb, mix, k, *case)
    mix.run(0, steps)
    _same(_state(pair, 0, 1), _state(mix, 1, 1), "instance in two different ensembles")
    _same(_state(pair, 1, 3), _state(mix, 0, 3), "instance in two different ensembles")
    _same(_state(mix, 0, 3), _state(mix, 2, 3), "two copies of one instance")


def test_launch_shape_and_rerun_invariant(fb, seeded):
    cfg, beam, fields = seeded
    res = []
    for shape in ((6144, 2), (3072, 1), (1024, 2)):
        b = fb.Batch([cfg.params])
        _upload(fb, b, 0, cfg, beam, fields)
        b.set_launch(*shape)
        b.run(0, 40)
        res.append((_state(b, 0, 1), b.diagnostics(0, 0, 41)))
    for r in res[1:]:
        _same(res[0][0], r[0], "launch shape")
        np.testing.assert_allclose(r[1][0], res[0][1][0], rtol=1e-12)
    # the same shape twice: every bit, diagnostics included
    b = fb.Batch([cfg.params])
    _upload(fb, b, 0, cfg, beam, fields)
    b.set_launch(6144, 2)
    b.run(0, 40)
    _same(res[0][0], _state(b, 0, 1), "rerun")
    for x, y in zip(res[0][1], b.diagnostics(0, 0, 41)):
        assert np.array_equal(x, y)


def test_split_runs_equal_one_run(fb, seeded):
    cfg, beam, fields = seeded
    one = fb.Batch([cfg.params])
    _upload(fb, one, 0, cfg, beam, fields)
    one.run(0, 24)
    two = fb.Batch([cfg.params])
    _upload(fb, two, 0, cfg, beam, fields)
    two.run(0, 10)
    two.run(10, 24)
    _same(_state(one, 0, 1), _state(two, 0, 1), "split run")


def test_static_mode(fb, tmp_path):
    from felis_b200 import analysis

    cfg, beam, fields = make_case(fb, tmp_path, kind="static", beamlets=512, nx=51, total_length=12.0, units=3,
                                  energy_mev=1000.0)
    p = cfg.params
    steps = p.max_step
    g = _fp64(fb, cfg, beam, fields, steps)
    b = fb.Batch([p])
    _upload(fb, b, 0, cfg, beam, fields)
    b.run(0, steps)
    P64 = analysis.output_power(g.diagnostics(0, steps + 1)[0])
    P32 = analysis.output_power(b.diagnostics(0, 0, steps + 1)[0])
    assert P64[-1] > 1e3 * P64[0]
    rel = np.abs(P32 - P64) / P64
    assert rel.max() < POWER_RTOL, rel.max()
    lg64, lg32 = analysis.gain_length(P64, p.dz), analysis.gain_length(P32, p.dz)
    assert abs(lg32 / lg64 - 1) < GAIN_LENGTH_RTOL, (lg32, lg64)


def test_tune_advances_and_caches(fb, seeded):
    cfg, beam, fields = seeded
    b = fb.Batch([cfg.params])
    _upload(fb, b, 0, cfg, beam, fields)
    nxt = b.tune(0, 2)
    # the first deposit, then 2 iterations under each of ADI CTAs/SM 1 and 2 at the
    # one staged source area a 42 x 42 grid needs
    assert nxt == 1 + 2 * 2
    b.run(nxt, nxt + 4)
    ref = fb.Batch([cfg.params])
    _upload(fb, ref, 0, cfg, beam, fields)
    ref.run(0, nxt + 4)
    _same(_state(b, 0, 1), _state(ref, 0, 1), "tuned run")
    again = fb.Batch([cfg.params])
    _upload(fb, again, 0, cfg, beam, fields)
    assert again.tune(0, 2) == 0  # cached: nothing run


def test_download_into_caller_buffers(fb, seeded):
    """download_particles(out=...) fills the given arrays with the same values
    as a download into new arrays; a wrong buffer is refused."""
    cfg, beam, fields = seeded
    b = fb.Batch([cfg.params])
    _upload(fb, b, 0, cfg, beam, fields)
    b.run(0, 6)
    ref = b.download_particles(0)
    n = ref["x"].size
    out = {k: np.full(n, np.nan) for k in ref}
    got = b.download_particles(0, out=out)
    assert got is out
    for k in ref:
        assert np.array_equal(out[k], ref[k]), k
    with pytest.raises(ValueError):
        b.download_particles(0, out=dict(out, x=np.zeros(n, dtype=np.float32)))
    b.close()


@pytest.mark.parametrize("nx", [41, 42])
def test_particles_in_the_edge_cells(fb, tmp_path, nx):
    """Particles in the last grid column and row (cell index nx - 1, outside
    the interior box the deposit accumulates) on odd and even grids: the run
    completes, and its power follows the FP64 path's, which leaves those
    cells' sources out too (the ADI solves interior cells only)."""
    cfg, beam, fields = make_case(fb, tmp_path, kind="sase", slices=6, beamlets=64, nx=nx, total_length=0.5,
                                  seed_power=1e5, energy_mev=1000.0)
    p = cfg.params
    beam = {k: np.array(v) for k, v in beam.items()}
    last_x = p.min_x + (p.nx - 0.5) * p.dx
    last_y = p.min_y + (p.ny - 0.5) * p.dy
    for k in range(0, len(beam["x"]), 7):  # one particle in seven on the edge
        if k % 2:
            beam["x"][k] = last_x
        beam["y"][k] = last_y
    steps = 6
    g = _fp64(fb, cfg, beam, fields, steps)
    b = fb.Batch([p])
    _upload(fb, b, 0, cfg, beam, fields)
    b.run(0, steps)
    P32 = b.diagnostics(0, 0, steps + 1)[0].sum(axis=1)
    P64 = g.diagnostics(0, steps + 1)[0].sum(axis=1)
    assert np.all(np.isfinite(P32))
    assert np.max(np.abs(P32 - P64) / P64) < POWER_RTOL


def test_errors_are_reported(fb, seeded):
    cfg, beam, fields = seeded
    b = fb.Batch([cfg.params])
    with pytest.raises(fb.FelisError):
        b.run(0, 1)  # no particles uploaded
    with pytest.raises(fb.FelisError):
        b.set_launch(100, 1)


def test_grid_classes_and_uneven_instances(fb, tmp_path):
    """Instances of the three ensemble grid sizes (ADI launch per size, the
    largest planes filling one SM's shared memory) with uneven slice counts:
    every instance tracks its own FP64 plain run."""
    from felis_b200 import analysis

    cases = []
    for k, (slices, nx) in enumerate(((24, 65), (8, 151), (16, 101))):
        d = tmp_path / f"g{k}"
        d.mkdir()
        cases.append(make_case(fb, d, kind="sase", slices=slices, beamlets=128, nx=nx, total_length=1.0,
                               seed_power=1e5, energy_mev=1000.0, seed=k + 5))
    steps = 30
    b = fb.Batch([c[0].params for c in cases])
    for k, c in enumerate(cases):
        _upload(fb, b, k, *c)
    b.run(0, steps)
    for k, (cfg, beam, fields) in enumerate(cases):
        g = _fp64(fb, cfg, beam, fields, steps)
        P64 = analysis.output_power(g.diagnostics(0, steps + 1)[0])
        P32 = analysis.output_power(b.diagnostics(k, 0, steps + 1)[0])
        rel = np.abs(P32 - P64) / P64
        assert rel.max() < POWER_RTOL, (k, rel.max())


def test_spectral_moments_match_the_downloaded_field(fb, tmp_path):
    """felis_batch_spectral_moments against the same sums over the downloaded
    fields (slices in bunch order, both polarisations), two instances of
    different length after slippage shifts."""
    from felis_b200 import analysis, workloads

    cfgs, beams = [], []
    for k, S in enumerate((24, 40)):
        path = workloads.write_input(str(tmp_path / f"s{k}.inp"), kind="sase", slices=S, beamlets=64, nx=33,
                                     total_length=1.0, seed_power=1e6)
        cfgs.append(fb.Config(path))
        beams.append(cfgs[-1].load_beam(0, seed=2 + k))
    b = fb.Batch([c.params for c in cfgs])
    for k, (c, beam) in enumerate(zip(cfgs, beams)):
        b.upload_particles(k, *(beam[x] for x in ("x", "y", "px", "py", "theta", "gamma")), beam["offsets"],
                           beam["weights"])
        ux, uy = c.load_seed(0)
        b.upload_field(k, 0, 0, ux)
        b.upload_field(k, 0, 1, uy)
    b.run(0, 17)
    got = b.spectral_moments(0)
    for k in range(2):
        U = [b.download_field(k, 0, pol)[1:-1] for pol in (0, 1)]
        r0 = sum(float(np.sum(np.abs(u) ** 2)) for u in U)
        r1 = sum(complex(np.sum(np.conj(u[:-1]) * u[1:])) for u in U)
        np.testing.assert_allclose(got[k], [r0, r1.real, r1.imag], rtol=1e-9, atol=1e-12 * r0)
        c, w = analysis.lag_moments(got[k])
        assert np.isfinite(c) and w >= 0
    b.close()
