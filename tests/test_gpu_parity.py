"""GPU slice loop vs the CPU restatement, through the C ABI.

The FP64 plain path is designed to be bit-identical to the restatement
(fixed operand order, no FMA contraction, shared deterministic sin/cos/atan,
sources summed in particle order), so particle state, field, source and Ez
are compared with ==.  The diagnostics are tree reductions on the GPU and
sequential sums on the CPU: they are compared at 1e-12 relative.
"""
import numpy as np
import pytest

from conftest import assert_bits, load_both, make_case

pytestmark = pytest.mark.gpu

SMALL = dict(slices=6, beamlets=96, nx=41, total_length=3.0)


def _particles_equal(g, o, what):
    a, b = g.download_particles(0), o.get_particles(0)
    for k in ("x", "y", "px", "py", "theta", "gamma"):
        assert_bits(a[k], b[k], f"{what}: {k}")


def _fields_equal(g, o, H, what):
    for h in range(H):
        for pol in (0, 1):
            assert_bits(g.download_field(h, pol)[1:-1], o.get_field(h, pol)[1:-1], f"{what}: U h{h} pol{pol}")


def _sources_equal(g, o, H, what):
    for h in range(H):
        for pol in (0, 1):
            a = g.download_source(h, pol)[1:-1, 1:-1, 1:-1]
            b = o.get_field(h, 2 + pol)[1:-1, 1:-1, 1:-1]
            assert_bits(a, b, f"{what}: Sc h{h} pol{pol}")


def _set_both(g, o, it, half):
    g.update_lattice(it, half)
    o.update_lattice(it, half)
    lg, lo = g.lattice(), o.lattice()
    for f in ("K0", "ue", "lambdaU", "ku", "g", "K0_alpha", "und_type", "current_flag", "drift_flag"):
        assert getattr(lg, f) == getattr(lo, f), f
    return lg


@pytest.fixture(params=["bipolar_h1", "quadpolar_h123"])
def case(request, fb, tmp_path):
    if request.param == "bipolar_h1":
        kw = dict(SMALL, seed_power=2e6, quads=True)
    else:
        kw = dict(SMALL, harmonics=(1, 2, 3), undulator="QuadPolar", polarity=0.5, seed_power=2e6)
    return make_case(fb, tmp_path, kind="sase", **kw)


def test_lattice_and_transverse_push(fb, oracle_mod, case):
    cfg, beam, fields = case
    g, o = load_both(fb, oracle_mod, cfg, beam, fields)
    # quads overlap z = 3.6..3.7 m in the quad case; walk through them
    for it in (0, 5, 138, 139, 140, 141):
        for half in (0.0, 0.5):
            _set_both(g, o, it, half)
            g.transverse_push(it)
            o.transverse_push()
    _particles_equal(g, o, "transverse push")


def test_solve_field_and_push(fb, oracle_mod, case):
    cfg, beam, fields = case
    H = cfg.params.num_harmony
    g, o = load_both(fb, oracle_mod, cfg, beam, fields)
    lat = _set_both(g, o, 3, 0.5)
    assert lat.current_flag == 1 and lat.drift_flag == 0
    g.solve_field(3)
    o.solve_field()
    _sources_equal(g, o, H, "deposit")
    assert_bits(g.download_ez()[:, 1:-1], o.get_ez()[:, 1:-1], "Ez")
    _fields_equal(g, o, H, "ADI")
    g.push_theta_gamma(3)
    o.push_theta_gamma()
    _particles_equal(g, o, "push_theta_gamma")
    g.periodic_particles(3)
    o.periodic_particles()
    _particles_equal(g, o, "periodicParticles")


def test_drift_and_shift(fb, oracle_mod, case):
    cfg, beam, fields = case
    H = cfg.params.num_harmony
    g, o = load_both(fb, oracle_mod, cfg, beam, fields)
    lat = _set_both(g, o, 140, 0.5)  # z = 3.653 m: in the air gap
    assert lat.drift_flag == 1
    g.drift_theta_gamma(140)
    o.drift_theta_gamma()
    _particles_equal(g, o, "drift")
    g.shift_field(140)
    o.shift_field()
    _fields_equal(g, o, H, "shift")


def test_diagnostics(fb, oracle_mod, case):
    cfg, beam, fields = case
    g, o = load_both(fb, oracle_mod, cfg, beam, fields)
    np.testing.assert_allclose(g.total_energy(), o.total_energy(), rtol=1e-12)
    np.testing.assert_allclose(g.twiss(), o.twiss(), rtol=1e-12)
    np.testing.assert_allclose(g.bfactor(), o.bfactor(), rtol=1e-10, atol=1e-15)


def test_step_loop_bit_exact(fb, oracle_mod, case):
    cfg, beam, fields = case
    H = cfg.params.num_harmony
    n = cfg.params.max_step
    g, o = load_both(fb, oracle_mod, cfg, beam, fields)
    for it in range(n):
        g.step(it)
    e0, t0, b0 = o.run(0, n)
    _particles_equal(g, o, f"{n} steps")
    _fields_equal(g, o, H, f"{n} steps")
    e1, t1, b1 = g.diagnostics(0, n)
    np.testing.assert_allclose(e1, e0, rtol=1e-12, atol=1e-300)
    np.testing.assert_allclose(t1, t0, rtol=1e-11)
    np.testing.assert_allclose(b1, b0, rtol=1e-9, atol=1e-14)


def test_graph_run_equals_steps(fb, oracle_mod, tmp_path):
    cfg, beam, fields = make_case(fb, tmp_path, kind="sase", **dict(SMALL, seed_power=2e6))
    n = cfg.params.max_step
    g1, _ = load_both(fb, oracle_mod, cfg, beam, fields)
    g2, _ = load_both(fb, oracle_mod, cfg, beam, fields)
    for it in range(n):
        g1.step(it)
    g2.run(0, n)
    a, b = g1.download_particles(0), g2.download_particles(0)
    for k in a:
        assert_bits(a[k], b[k], f"graph vs steps: {k}")
    assert_bits(g1.download_field(0, 0), g2.download_field(0, 0), "graph vs steps: Ux")
    d1, d2 = g1.diagnostics(0, n), g2.diagnostics(0, n)
    for x, y in zip(d1, d2):
        assert_bits(x, y, "graph vs steps: diagnostics")
    # the same state downloaded into caller buffers
    out = {k: np.full(a[k].size, np.nan) for k in a}
    assert g2.download_particles(0, out=out) is out
    for k in a:
        assert_bits(out[k], b[k], f"download into caller buffers: {k}")


def test_drop_in_loop_equals_fused(fb, oracle_mod, tmp_path):
    cfg, beam, fields = make_case(fb, tmp_path, kind="sase", **dict(SMALL, seed_power=2e6, total_length=1.0))
    n = cfg.params.max_step
    g1, _ = load_both(fb, oracle_mod, cfg, beam, fields)
    g2, _ = load_both(fb, oracle_mod, cfg, beam, fields)
    g1.run_loop(0, n)
    for it in range(n):
        g2.step(it)
    a, b = g1.download_particles(0), g2.download_particles(0)
    for k in a:
        assert_bits(a[k], b[k], f"per-function vs fused: {k}")
    assert_bits(g1.download_field(0, 0), g2.download_field(0, 0), "per-function vs fused: Ux")


def test_static_seeded_bit_exact(fb, oracle_mod, tmp_path):
    cfg, beam, fields = make_case(fb, tmp_path, kind="static", beamlets=512, nx=61, total_length=6.0)
    n = cfg.params.max_step
    g, o = load_both(fb, oracle_mod, cfg, beam, fields)
    g.run(0, n)
    o.run(0, n)
    _particles_equal(g, o, "static")
    _fields_equal(g, o, 1, "static")


def test_slice_sort_stable(fb):
    rng = np.random.default_rng(7)
    for n, kmax in ((0, 1), (1, 1), (5000, 1), (100000, 1024), (300001, 50000), (70000, 3)):
        keys = rng.integers(0, kmax, size=n).astype(np.int32)
        perm = fb.sort_by_slice(keys)
        assert_bits(perm, np.argsort(keys, kind="stable"), f"sort n={n} kmax={kmax}")
    # already slice-major input (the reference's order) is the identity
    keys = np.repeat(np.arange(300, dtype=np.int32), 97)
    assert_bits(fb.sort_by_slice(keys), np.arange(keys.size), "identity")


@pytest.mark.parametrize("kw", [
    dict(kind="static", beamlets=2048, nx=61, total_length=2.0),
    dict(kind="sase", slices=3, beamlets=1536, nx=51, total_length=1.0, harmonics=(1, 2, 3),
         undulator="QuadPolar", polarity=0.5, seed_power=5e6),
])
def test_multichunk_deposit_bit_exact(fb, oracle_mod, tmp_path, kw):
    """Slices larger than one shared-memory chunk of the ordered deposit."""
    kind = kw.pop("kind")
    cfg, beam, fields = make_case(fb, tmp_path, kind=kind, **kw)
    H = cfg.params.num_harmony
    n = cfg.params.max_step
    g, o = load_both(fb, oracle_mod, cfg, beam, fields)
    g.run(0, n)
    o.run(0, n)
    _particles_equal(g, o, "multichunk")
    _fields_equal(g, o, H, "multichunk")
    assert_bits(g.download_ez()[:, 1:-1], o.get_ez()[:, 1:-1], "multichunk Ez")


@pytest.mark.parametrize("kw", [
    dict(slices=3, beamlets=256, nx=151, total_length=1.0, seed_power=1e6),
    dict(slices=2, beamlets=128, nx=131, total_length=0.6, harmonics=(1, 2), undulator="QuadPolar",
         polarity=0.5, seed_power=1e6),
])
def test_large_grid_adi_bit_exact(fb, oracle_mod, tmp_path, kw):
    """Grids whose FP64 plane exceeds shared memory take the global-memory ADI
    (one scratch plane per CTA); results stay bit-identical."""
    cfg, beam, fields = make_case(fb, tmp_path, kind="sase", **kw)
    H = cfg.params.num_harmony
    n = cfg.params.max_step
    g, o = load_both(fb, oracle_mod, cfg, beam, fields)
    g.run(0, n)
    e0, _, _ = o.run(0, n)
    _particles_equal(g, o, "large grid")
    _fields_equal(g, o, H, "large grid")
    np.testing.assert_allclose(g.diagnostics(0, n)[0], e0, rtol=1e-12, atol=1e-300)
