"""The beam loader on the device (felis_config_load_beam_device) against the
host loader (felis_config_load_beam, loadBeam.cpp:28-269).

Counts, offsets and weights are computed by the same host code and must be
equal.  The particles come from the same Halton points and the same noise
stream; the transforms use the device's log / sin / cos, so they agree with
the host's C library to a few ulps (tolerance 1e-13 of each array's scale).
Device arrays then go into a handle or an ensemble without a host copy, and
the uploads must store exactly what the host path stores.
"""
import numpy as np
import pytest

from conftest import assert_bits

pytestmark = pytest.mark.gpu

CASES = [
    ("sase", dict(kind="sase", slices=64, beamlets=256, nx=31), 1),
    ("sase_h13", dict(kind="sase", slices=40, beamlets=128, nx=31, harmonics=(1, 3)), 1),
    ("gaussian", dict(kind="sase", slices=96, beamlets=512, nx=31, sigma_slices=20.0, current=4000.0), 1),
    ("static", dict(kind="static", beamlets=2048, nx=31), 1),
    ("rank1_of_2", dict(kind="sase", slices=50, beamlets=128, nx=31), 2),
]


def _cfg(fb, tmp_path, kw, ranks):
    from felis_b200 import workloads

    path = workloads.write_input(str(tmp_path / "l.inp"), **kw)
    return fb.Config(path, ranks, ranks - 1)


@pytest.mark.parametrize("name,kw,ranks", CASES, ids=[c[0] for c in CASES])
def test_device_loader_matches_host_loader(fb, tmp_path, name, kw, ranks):
    cfg = _cfg(fb, tmp_path, kw, ranks)
    host = cfg.load_beam(0, seed=5)
    dev = cfg.load_beam_device(0, seed=5)
    assert_bits(dev["offsets"], host["offsets"], "offsets")
    assert_bits(dev["weights"], host["weights"], "weights")
    assert host["offsets"][-1] > 0
    for k in ("x", "y", "px", "py", "gamma", "theta"):
        d = dev[k].cpu().numpy()
        h = host[k]
        scale = np.abs(h).max()
        np.testing.assert_allclose(d, h, rtol=1e-13, atol=1e-13 * scale, err_msg=k)


def test_device_arrays_upload_like_host_arrays(fb, tmp_path):
    cfg = _cfg(fb, tmp_path, dict(kind="sase", slices=32, beamlets=128, nx=31, total_length=0.4), 1)
    p = cfg.params
    dev = cfg.load_beam_device(0, seed=5)
    host = {k: (v.cpu().numpy() if hasattr(v, "cpu") else v) for k, v in dev.items()}
    fields = [cfg.load_seed(h) for h in range(p.num_harmony)]
    keys = ("x", "y", "px", "py", "theta", "gamma", "offsets", "weights")
    # FP64 handle
    runs = []
    for beam in (dev, host):
        g = fb.Handle(p)
        g.upload_particles(0, *(beam[k] for k in keys))
        for h, (ux, uy) in enumerate(fields):
            g.upload_field(h, 0, ux)
            g.upload_field(h, 1, uy)
        g.run(0, 8)
        runs.append((g.download_particles(0), g.download_field(0, 0)))
        g.close()
    for k in runs[0][0]:
        assert_bits(runs[0][0][k], runs[1][0][k], k)
    assert_bits(runs[0][1], runs[1][1], "field")
    # mixed ensemble: the FP32 rounding on the device equals the host's
    runs = []
    for beam in (dev, host):
        b = fb.Batch([p])
        b.upload_particles(0, *(beam[k] for k in keys))
        for h, (ux, uy) in enumerate(fields):
            b.upload_field(0, h, 0, ux)
            b.upload_field(0, h, 1, uy)
        runs.append(b.download_particles(0))
        b.run(0, 8)
        runs.append(b.download_particles(0))
        b.close()
    for k in runs[0]:
        assert_bits(runs[0][k], runs[2][k], f"stored {k}")
        assert_bits(runs[1][k], runs[3][k], f"after 8 steps {k}")
