"""The CPU restatement against the golden fixtures made by the reference's own
step loop (tests/golden/make_ref_golden.py): config 1 complete and config 2's
two leading slices, whole runs of 1539 steps from the input file.  These hold
where oracle/_ref cannot be built (no reference sources); the fixtures store
every 16th particle, every 3rd cell of the field planes and the power of
every iteration."""
import os

import numpy as np
import pytest

from conftest import rel_err

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
KEYS = ("x", "y", "px", "py", "theta", "gamma")


@pytest.mark.parametrize("name", ["ref_config1.npz", "ref_config2_prefix.npz"])
def test_restatement_matches_reference_golden(fb, oracle_mod, tmp_path, name):
    gold = np.load(os.path.join(GOLDEN, name))
    path = tmp_path / "golden.inp"
    path.write_text(str(gold["input"]))
    cfg = fb.Config(str(path))
    p = cfg.params
    beam = cfg.load_beam(0, seed=int(gold["seed"]))
    assert np.array_equal(beam["offsets"], gold["offsets"])
    o = oracle_mod.Oracle(p, threads=os.cpu_count() or 4, variant="strict")
    o.set_particles(0, *(beam[k] for k in KEYS), beam["offsets"], beam["weights"])
    for h in range(p.num_harmony):
        ux, uy = cfg.load_seed(h)
        o.set_field(h, 0, ux)
        o.set_field(h, 1, uy)
    e, _, _ = o.run(0, p.max_step)
    mine = o.get_particles(0)
    pick = gold["pick"]
    for k in KEYS:
        assert rel_err(mine[k][pick], gold[k]) < 1e-11, k
    cs = int(gold["cell_stride"])
    assert rel_err(o.get_field(0, 0)[1:-1, ::cs, ::cs], gold["field_x"]) < 1e-11
    assert np.max(np.abs(o.get_field(0, 1)[1:-1, ::cs, ::cs] - gold["field_y"])) <= 1e-11 * np.max(np.abs(gold["field_x"]))
    assert max(rel_err(e[i], gold["energy"][i]) for i in range(p.max_step)) < 1e-11
