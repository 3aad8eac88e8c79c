"""[Phase_shifter] on the GPU (README.md:57-70; see tests/test_phase_shifter.py
for the reading of the block): the FP64 plain path through shifters is
bit-identical to the CPU restatement, fused (felis_run) and through the
per-function sequence with felis_phase_shift; the mixed engine follows the
FP64 path's power through the shifters within its tolerance, and the power
with a pi shifter differs from the run without."""
import numpy as np
import pytest

from felis_b200 import workloads

from conftest import assert_bits, load_both

pytestmark = pytest.mark.gpu

KEYS = ("x", "y", "px", "py", "theta", "gamma")
SHIFTERS = [(2, 3.7, 4.0, 1.0), (1, 9.75, 0.0, 0.5)]


def _case(fb, tmp_path, shifters, kind="static", **kw):
    opts = dict(beamlets=128, nx=41, total_length=12.0)
    opts.update(kw)
    path = workloads.write_input(str(tmp_path / f"ps{len(shifters)}.inp"), kind=kind, phase_shifters=shifters, **opts)
    cfg = fb.Config(path)
    beam = cfg.load_beam(0, seed=1 if kind == "static" else 2)
    fields = [cfg.load_seed(h) for h in range(cfg.params.num_harmony)]
    return cfg, beam, fields


@pytest.mark.parametrize("kind", ["static", "sase"])
def test_fp64_path_bit_identical_through_shifters(fb, oracle_mod, tmp_path, kind):
    kw = {} if kind == "static" else dict(slices=4, seed_power=1e6)
    cfg, beam, fields = _case(fb, tmp_path, SHIFTERS, kind, **kw)
    assert cfg.params.num_phase_shifts == 3
    n = cfg.params.max_step
    g, o = load_both(fb, oracle_mod, cfg, beam, fields)
    g.run(0, n)
    o.run(0, n)
    a, b = g.download_particles(0), o.get_particles(0)
    for k in KEYS:
        assert_bits(a[k], b[k], k)
    assert_bits(g.download_field(0, 0)[1:-1], o.get_field(0, 0)[1:-1], "Ux")
    # the per-function sequence of the reference's loop with felis_phase_shift
    g2, _ = load_both(fb, oracle_mod, cfg, beam, fields)
    g2.run_loop(0, n)
    c = g2.download_particles(0)
    for k in KEYS:
        assert_bits(c[k], b[k], k)


def test_mixed_engine_follows_fp64_through_shifters(fb, tmp_path):
    cfg, beam, fields = _case(fb, tmp_path, SHIFTERS)
    cfg0, _, _ = _case(fb, tmp_path, ())
    n = cfg.params.max_step - 1  # (diagnostics of iteration n are kept)
    powers = {}
    for name, c in (("shift", cfg), ("none", cfg0)):
        b = fb.Batch([c.params])
        b.upload_particles(0, *(beam[k] for k in KEYS), beam["offsets"], beam["weights"])
        b.upload_field(0, 0, 0, fields[0][0])
        b.upload_field(0, 0, 1, fields[0][1])
        b.run(0, n)
        e = b.diagnostics(0, 0, n + 1)[0]
        powers[name] = e[:, 0] + e[:, 1]
        b.close()
    h = fb.Handle(cfg.params)
    h.upload_particles(0, *(beam[k] for k in KEYS), beam["offsets"], beam["weights"])
    h.upload_field(0, 0, fields[0][0])
    h.upload_field(0, 1, fields[0][1])
    h.run(0, n)
    e64 = h.diagnostics(0, n + 1)[0]
    p64 = e64[:, 0] + e64[:, 1]
    assert np.max(np.abs(powers["shift"] - p64) / p64) < 1e-3
    assert abs(powers["shift"][-1] - powers["none"][-1]) > 1e-2 * powers["none"][-1]
