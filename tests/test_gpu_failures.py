"""Failure detection on the GPU, without a GPU fault.

The reference ends the process where its state goes bad: exit(0) when a
particle's phase step exceeds the bucket (particlePush.cpp:371-374) or its
wrapped phase leaves [0, dTh] (rearrangeParticles.cpp:105-108), MPI_Abort on
an unknown polarisation.  The library raises device error words instead and
returns a status; these tests make each failure on the host (bad values
uploaded through the C ABI), check the status, and check that the handle
keeps working after a clean re-upload: the continued run equals, bit for bit
(FP64) or exactly (the mixed engine is deterministic), that of a handle whose
first iteration succeeded and that was re-uploaded the same way.  Every
kernel involved returns on its own; the library's device waits (the
tensor-core pipeline's mbarrier waits) are bounded, and the self-test makes
one run out on a barrier that nothing completes.
"""
from fractions import Fraction

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KEYS = ("x", "y", "px", "py", "theta", "gamma")


def _case(fb, tmp_path, radial_grids=None):
    from felis_b200 import workloads

    text = workloads.input_text("static", beamlets=64, nx=41, total_length=1.0)
    if radial_grids is not None:
        text = text.replace("[Domain]\n", f"[Domain]\n radial_grids={radial_grids}\n", 1)
    path = tmp_path / "f.inp"
    path.write_text(text)
    cfg = fb.Config(str(path))
    beam = cfg.load_beam(0, seed=1)
    return cfg, beam, cfg.load_seed(0)


def _handle(fb, cfg, beam, field):
    h = fb.Handle(cfg.params)
    _upload(h, beam, field)
    return h


def _upload(h, beam, field, batch=False):
    if batch:
        h.upload_particles(0, *(beam[k] for k in KEYS), beam["offsets"], beam["weights"])
        h.upload_field(0, 0, 0, field[0])
        h.upload_field(0, 0, 1, field[1])
    else:
        h.upload_particles(0, *(beam[k] for k in KEYS), beam["offsets"], beam["weights"])
        h.upload_field(0, 0, field[0])
        h.upload_field(0, 1, field[1])


def _batch(fb, cfg, beam, field):
    b = fb.Batch([cfg.params])
    _upload(b, beam, field, batch=True)
    return b


def _batch_wrap_out_of_range(theta: float, dth: float) -> bool:
    """The mixed engine's wrap of one phase, evaluated both with and without a
    fused multiply-add, exactly: True when both leave [0, dTh]."""
    k = Fraction(np.floor(theta * (1.0 / dth)))
    th = Fraction(theta)
    fused = float(th - Fraction(dth) * k)
    plain = float(th - Fraction(float(Fraction(dth) * k)))
    out = True
    for r in (fused, plain):
        if r >= dth:
            r -= dth
        elif r < 0:
            r += dth
        out = out and (r > dth or r < 0)
    return out


def _bad_state(kind, cfg, beam, field, batch=False):
    beam = {k: np.array(v) for k, v in beam.items()}
    ux, uy = field[0].copy(), field[1].copy()
    dth = 2.0 * np.pi * cfg.params.num_slice
    if kind == "nan":
        beam["theta"][5] = np.nan
    elif kind == "range":
        # a phase so large that the wrap cannot bring it back into [0, dTh],
        # on a particle outside the transverse grid (the push leaves it alone,
        # the wrap does not)
        cands = [1e30 * (1.0 + 1e-3 * j) for j in range(64)]
        beam["theta"][5] = next(t for t in cands if not batch or _batch_wrap_out_of_range(t, dth))
        beam["x"][5] = 500e-6
    elif kind == "overflow":
        # |U|^2 / 2 of 50 makes the phase step dz ks / (2 gamma^2) * 50 ~ 70 > 2 pi
        ux[1:-1] = 10.0
    elif kind == "radial":
        # inside the +-300 um grid, beyond 10 radial cells of 20.2 um
        beam["x"][5], beam["y"][5] = 250e-6, 0.0
    return beam, (ux, uy)


STATUS = {"nan": "NAN", "range": "OUT_OF_RANGE", "overflow": "THETA_OVERFLOW", "radial": "UNSUPPORTED"}


@pytest.mark.parametrize("kind", list(STATUS))
def test_fp64_handle_reports_and_recovers(fb, tmp_path, kind):
    cfg, beam, field = _case(fb, tmp_path, radial_grids=10 if kind == "radial" else None)
    n = 5
    bad_beam, bad_field = _bad_state(kind, cfg, beam, field)
    h = _handle(fb, cfg, bad_beam, bad_field)
    with pytest.raises(fb.FelisError) as e:
        h.run(0, 1)  # every failure shows in the first step
    assert e.value.status == getattr(fb, STATUS[kind]), str(e.value)
    # a clean re-upload continues as a handle whose first iteration succeeded
    # does (the lattice flags of iteration 0 carry into iteration 1 either way)
    _upload(h, beam, field)
    h.run(1, n)
    ref = _handle(fb, cfg, beam, field)
    ref.run(0, 1)
    _upload(ref, beam, field)
    ref.run(1, n)
    a, b = h.download_particles(0), ref.download_particles(0)
    for k in KEYS:
        assert np.array_equal(a[k], b[k]), k
    assert np.array_equal(h.download_field(0, 0), ref.download_field(0, 0))
    h.close()
    ref.close()


@pytest.mark.parametrize("kind", list(STATUS))
def test_mixed_engine_reports_and_recovers(fb, tmp_path, kind):
    cfg, beam, field = _case(fb, tmp_path, radial_grids=10 if kind == "radial" else None)
    n = 5
    bad_beam, bad_field = _bad_state(kind, cfg, beam, field, batch=True)
    b = _batch(fb, cfg, bad_beam, bad_field)
    with pytest.raises(fb.FelisError) as e:
        b.run(0, 1)
    assert e.value.status == getattr(fb, STATUS[kind]), str(e.value)
    _upload(b, beam, field, batch=True)
    b.run(1, n)
    ref = _batch(fb, cfg, beam, field)
    ref.run(0, 1)
    _upload(ref, beam, field, batch=True)
    ref.run(1, n)
    x, y = b.download_particles(0), ref.download_particles(0)
    for k in KEYS:
        assert np.array_equal(x[k], y[k]), k
    b.close()
    ref.close()


def test_bounded_wait_runs_out_and_the_context_stays_usable(fb):
    """The tensor-core pipeline's mbarrier wait, on a phase nothing completes:
    it gives up after its limit and reports FELIS_TIMEOUT; the next
    tensor-core forward on the same context is correct."""
    assert fb.wait_selftest(2000) == fb.TIMEOUT
    m = fb.MLP(38, 256, 33, seed=2)
    x = np.random.default_rng(1).standard_normal((256, 38)).astype(np.float32)
    y1 = m.forward(x)
    assert np.all(np.isfinite(y1))
    assert fb.wait_selftest(2000) == fb.TIMEOUT
    assert np.array_equal(m.forward(x), y1)
    m.close()
