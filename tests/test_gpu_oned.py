"""The 1D model (dimension = 1) of the FP64 handle against the CPU
restatement (solveField.cpp:409-549, particlePush.cpp:388-524): particle
state and field bit-identical after whole runs, through the fused step (one
CUDA graph per range) and through the per-function drop-in sequence."""
import numpy as np
import pytest

from conftest import assert_bits, load_both, make_case

pytestmark = pytest.mark.gpu

CASES = {
    "sase_h13_wake": dict(kind="sase", slices=48, beamlets=128, nx=21, dimension=1, harmonics=(1, 3), wake=True,
                          sigma_slices=12.0, total_length=6.0, seed_power=0.0),
    "quadpolar_h123": dict(kind="sase", slices=24, beamlets=64, nx=21, dimension=1, harmonics=(1, 2, 3),
                           undulator="QuadPolar", polarity=0.5, seed_power=2e6, total_length=4.5),
    "static_seeded": dict(kind="static", beamlets=1024, nx=21, dimension=1, seed_power=1e4, total_length=12.0,
                          units=3),
}


def _case(fb, tmp_path, kw):
    cfg, beam, fields = make_case(fb, tmp_path, **kw)
    if cfg.params.wake_on:
        cfg.wake(beam["weights"] * np.diff(beam["offsets"]))
    return cfg, beam, fields


def _compare(g, o, H):
    q, r = g.download_particles(0), o.get_particles(0)
    for k in r:
        assert_bits(q[k], r[k], k)
    # the physical slices (the restatement's ghost slot S+1 keeps the slice
    # the last shift moved out, solveField.cpp:19-47; the handle's ring has none)
    for h in range(H):
        for pol in (0, 1):
            assert_bits(g.download_field(h, pol)[1:-1], o.get_field(h, pol)[1:-1], f"field h{h} pol{pol}")


@pytest.mark.parametrize("name", sorted(CASES))
def test_1d_run_bit_exact(fb, oracle_mod, tmp_path, name):
    cfg, beam, fields = _case(fb, tmp_path, CASES[name])
    p = cfg.params
    assert p.dimension == 1 and p.nx == 1 and p.ny == 1
    g, o = load_both(fb, oracle_mod, cfg, beam, fields)
    n = min(p.max_step, 240)
    e0, t0, b0 = o.run(0, n)
    g.run(0, n)
    _compare(g, o, p.num_harmony)
    e1, t1, b1 = g.diagnostics(0, n)
    assert np.abs(e0).max() > 0
    np.testing.assert_allclose(e1, e0, rtol=1e-12, atol=1e-300)
    np.testing.assert_allclose(b1, b0, rtol=1e-9, atol=1e-14)
    np.testing.assert_allclose(t1, t0, rtol=1e-11)  # 0/0 for beams without transverse size, as in the reference
    assert_bits(g.download_ez()[:, 1:-1], o.get_ez()[:, 1:-1], "Ez")


def test_1d_drop_in_sequence_bit_exact(fb, oracle_mod, tmp_path):
    """The per-function calls of main.cpp:117-155 (transverse pushes and the
    drift are no-ops in 1D, as the reference's loop and grid test make them)."""
    cfg, beam, fields = _case(fb, tmp_path, CASES["quadpolar_h123"])
    p = cfg.params
    g, o = load_both(fb, oracle_mod, cfg, beam, fields)
    n = min(p.max_step, 120)
    g.run_loop(0, n)
    o.run(0, n, diagnostics=False)
    _compare(g, o, p.num_harmony)
