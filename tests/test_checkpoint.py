"""Checkpoints (felis_b200.checkpoint) in the layout of the reference's HDF5
dumps (saveFieldHDF.cpp, saveParticleHDF.cpp), and restarts from them.

The CPU restatement is the engine on CPU; the GPU case restores the same
checkpoint into a felis_b200.Handle and into the restatement and runs both on:
a restart must be bit-identical between them, like every other entry point.
"""
import math

import numpy as np
import pytest

from conftest import assert_bits, make_case

RESTART, END = 6, 14


def _oracle(oracle_mod, cfg, beam, fields, threads=1):
    p = cfg.params
    o = oracle_mod.Oracle(p, threads=threads)
    o.set_particles(0, beam["x"], beam["y"], beam["px"], beam["py"], beam["theta"], beam["gamma"], beam["offsets"],
                    beam["weights"])
    for h, (ux, uy) in enumerate(fields):
        o.set_field(h, 0, ux)
        o.set_field(h, 1, uy)
    return o


@pytest.fixture
def case(fb, tmp_path):
    return make_case(fb, tmp_path, kind="sase", slices=9, beamlets=32, per_beamlet=4, nx=21, harmonics=(1, 3),
                     total_length=0.4)


@pytest.fixture(params=[3, 1], ids=["3d", "1d"])
def any_case(request, fb, tmp_path):
    """The same case in the 3D and the 1D model."""
    return make_case(fb, tmp_path, kind="sase", slices=9, beamlets=32, per_beamlet=4, nx=21, harmonics=(1, 3),
                     total_length=0.4, dimension=request.param)


def _state(o, H):
    q = o.get_particles(0)
    return q, [o.get_field(h, pol)[1:-1] for h in range(H) for pol in (0, 1)]


def _same(a, b):
    for k in a[0]:
        assert_bits(a[0][k], b[0][k], k)
    for i, (x, y) in enumerate(zip(a[1], b[1])):
        assert_bits(x, y, f"plane {i}")


def test_layout_matches_the_reference_dump(any_case, oracle_mod, tmp_path):
    from felis_b200 import checkpoint

    cfg, beam, fields = any_case
    p = cfg.params
    o = _oracle(oracle_mod, cfg, beam, fields)
    o.run(0, RESTART)
    checkpoint.save_field(o, p, str(tmp_path), RESTART)
    checkpoint.save_particles(o, p, [(beam["offsets"], beam["weights"])], str(tmp_path), RESTART)
    N = p.nx * p.ny
    with np.load(tmp_path / f"field{RESTART}.npz") as f:
        assert {"Ux1", "Uy1", "Ux3", "Uy3"} <= set(f.files)
        assert f["Ux1"].shape == (p.slice_n, 2 * N)
        u = o.get_field(0, 0)[1:-1].reshape(p.slice_n, N)
        assert_bits(f["Ux1"][:, 0::2], u.real, "re")
        assert_bits(f["Ux1"][:, 1::2], u.imag, "im")
        assert list(f["harmony"]) == [1, 3] and int(f["sliceN"][0]) == p.slice_n
        coef = checkpoint.E_MASS * checkpoint.VELOCITY_C ** 2 * p.ks / checkpoint.E_CHARGE
        # saveFieldHDF.cpp:67-72: the cell area, or in 1D the seed spot area
        area = 2.0 * math.pi * p.spot_sig_r * p.spot_sig_r if p.dimension == 1 else (p.dx * p.dy)
        assert f["powerNorm"][0] == coef * coef / (2.0 * checkpoint.Z0) * area
    with np.load(tmp_path / f"particle{RESTART}.npz") as f:
        rows = f["0"]
        q = o.get_particles(0)
        assert rows.shape == (int(beam["offsets"][-1]), 8) and int(f["numData"][0]) == 8
        for col, k in enumerate(("theta", "x", "y", "gamma", "px", "py")):
            assert_bits(rows[:, col], q[k], k)
        cnt = np.diff(beam["offsets"])
        assert_bits(rows[:, 6], np.repeat(np.arange(p.slice_n), cnt).astype(float), "slice")
        assert_bits(rows[:, 7], np.repeat(beam["weights"], cnt), "weight")
        assert int(f["0/totalCnt"][0]) == rows.shape[0]
        assert f["dPhi"][0] == 2.0 * math.pi * p.num_slice


def test_round_trip_is_exact(any_case, oracle_mod, tmp_path):
    from felis_b200 import checkpoint

    cfg, beam, fields = any_case
    p = cfg.params
    o = _oracle(oracle_mod, cfg, beam, fields)
    o.run(0, RESTART)
    checkpoint.save_field(o, p, str(tmp_path), RESTART)
    checkpoint.save_particles(o, p, [(beam["offsets"], beam["weights"])], str(tmp_path), RESTART)
    r = oracle_mod.Oracle(p, threads=1)
    checkpoint.restore_field(r, p, str(tmp_path), RESTART)
    beams = checkpoint.restore_particles(r, p, str(tmp_path), RESTART)
    _same(_state(o, p.num_harmony), _state(r, p.num_harmony))
    assert_bits(beams[0]["offsets"], beam["offsets"], "offsets")
    assert_bits(beams[0]["weights"], beam["weights"], "weights")


def test_restart_differs_only_by_the_lattice_state(any_case, oracle_mod, tmp_path):
    """A restart resumes from a fresh lattice state, as the reference's does
    (main.cpp:51-58 restores particles and field only); with the lattice state
    of the uninterrupted run put back, the continuation is bit-identical."""
    from felis_b200 import checkpoint

    cfg, beam, fields = any_case
    p = cfg.params
    a = _oracle(oracle_mod, cfg, beam, fields)
    a.run(0, RESTART)
    checkpoint.save_field(a, p, str(tmp_path), RESTART)
    checkpoint.save_particles(a, p, [(beam["offsets"], beam["weights"])], str(tmp_path), RESTART)
    lat = a.lattice()
    a.run(RESTART, END)
    c = oracle_mod.Oracle(p, threads=1)
    checkpoint.restore_field(c, p, str(tmp_path), RESTART)
    checkpoint.restore_particles(c, p, str(tmp_path), RESTART)
    c.set_lattice(lat)
    c.run(RESTART, END)
    _same(_state(a, p.num_harmony), _state(c, p.num_harmony))


def test_wake_recomputed_from_the_restored_beam(fb, oracle_mod, tmp_path):
    from felis_b200 import checkpoint

    cfg, beam, fields = make_case(fb, tmp_path, kind="sase", slices=16, beamlets=32, per_beamlet=4, nx=21,
                                  total_length=0.2, wake=True, sigma_slices=4.0)
    p = cfg.params
    cfg.wake(beam["weights"] * np.diff(beam["offsets"]))
    w0 = np.ctypeslib.as_array(p.wake_e, shape=(p.global_slice_n,)).copy()
    assert np.abs(w0).max() > 0
    o = _oracle(oracle_mod, cfg, beam, fields)
    checkpoint.save_particles(o, p, [(beam["offsets"], beam["weights"])], str(tmp_path), 0)
    cfg2 = fb.Config(str(tmp_path / "sase.inp"))  # the input file make_case wrote
    checkpoint.restore_wake(cfg2, checkpoint.read_particles(cfg2.params, str(tmp_path), 0))
    w1 = np.ctypeslib.as_array(cfg2.params.wake_e, shape=(p.global_slice_n,))
    assert_bits(w1, w0, "wake")


@pytest.mark.gpu
def test_gpu_restart_equals_restatement_restart(fb, case, oracle_mod, tmp_path):
    """Restored from the same checkpoint, the handle and the restatement
    continue bit-identically (both from a fresh lattice state)."""
    from felis_b200 import checkpoint

    cfg, beam, fields = case
    p = cfg.params
    a = _oracle(oracle_mod, cfg, beam, fields)
    a.run(0, RESTART)
    checkpoint.save_field(a, p, str(tmp_path), RESTART)
    checkpoint.save_particles(a, p, [(beam["offsets"], beam["weights"])], str(tmp_path), RESTART)
    o = oracle_mod.Oracle(p, threads=1)
    g = fb.Handle(p)
    for eng in (o, g):
        checkpoint.restore_field(eng, p, str(tmp_path), RESTART)
        checkpoint.restore_particles(eng, p, str(tmp_path), RESTART)
    o.run(RESTART, END)
    g.run(RESTART, END)
    q = g.download_particles(0)
    r = o.get_particles(0)
    for k in r:
        assert_bits(q[k], r[k], k)
    for h in range(p.num_harmony):
        for pol in (0, 1):
            assert_bits(g.download_field(h, pol)[1:-1], o.get_field(h, pol)[1:-1], f"h{h} pol{pol}")
    # and the handle's own checkpoint equals the restatement's
    (tmp_path / "g").mkdir()
    checkpoint.save_field(g, p, str(tmp_path / "g"), END)
    checkpoint.save_field(o, p, str(tmp_path), END)
    with np.load(tmp_path / "g" / f"field{END}.npz") as x, np.load(tmp_path / f"field{END}.npz") as y:
        for k in x.files:
            assert_bits(x[k], y[k], k)
    g.close()
