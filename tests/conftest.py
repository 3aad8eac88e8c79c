import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


def _has_gpu() -> bool:
    try:
        import felis_b200 as fb

        fb.device_info()
        return True
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def fb():
    import felis_b200

    return felis_b200


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle

    return oracle


def make_case(fb, tmp_path, kind="sase", seed=None, **kw):
    """Parsed config + initial particles + seed field for a small workload."""
    from felis_b200 import workloads

    path = workloads.write_input(str(tmp_path / f"{kind}.inp"), kind=kind, **kw)
    cfg = fb.Config(path)
    beam = cfg.load_beam(0, seed=(1 if kind == "static" else 2) if seed is None else seed)
    fields = [cfg.load_seed(h) for h in range(cfg.params.num_harmony)]
    return cfg, beam, fields


def ref_case(fb, tmp_path, kind="sase", seed=None, **kw):
    """make_case for a comparison with the reference (oracle/_ref): also the
    input path, the loader seed (GSL_RNG_SEED), and the wake energy loss of
    the loaded beam installed in the parameters (the reference computes it at
    iteration 0 from the same slice charges, wakeField.cpp:9-50)."""
    from felis_b200 import workloads

    path = workloads.write_input(str(tmp_path / f"{kind}.inp"), kind=kind, **kw)
    cfg = fb.Config(path)
    seed = (1 if kind == "static" else 2) if seed is None else seed
    beam = cfg.load_beam(0, seed=seed)
    fields = [cfg.load_seed(h) for h in range(cfg.params.num_harmony)]
    if cfg.params.wake_on:
        cfg.wake(beam["weights"] * np.diff(beam["offsets"]))
    return cfg, beam, fields, path, seed


def rel_err(a, b) -> float:
    """Largest absolute difference relative to the largest magnitude of b."""
    a = np.asarray(a)
    b = np.asarray(b)
    assert a.shape == b.shape
    scale = float(np.max(np.abs(b))) if b.size else 0.0
    d = float(np.max(np.abs(a - b))) if b.size else 0.0
    return d / scale if scale > 0 else d


def load_both(fb, oracle_mod, cfg, beam, fields, threads=4):
    """The same initial state in a GPU handle and in the CPU restatement."""
    p = cfg.params
    g = fb.Handle(p)
    o = oracle_mod.Oracle(p, threads=threads)
    for obj in (g, o):
        up = obj.upload_particles if obj is g else obj.set_particles
        up(0, beam["x"], beam["y"], beam["px"], beam["py"], beam["theta"], beam["gamma"], beam["offsets"], beam["weights"])
    for h, (ux, uy) in enumerate(fields):
        g.upload_field(h, 0, ux)
        g.upload_field(h, 1, uy)
        o.set_field(h, 0, ux)
        o.set_field(h, 1, uy)
    return g, o


def assert_bits(a, b, what=""):
    """Bit-identical comparison (-0.0 == 0.0; no NaN expected)."""
    a = np.asarray(a)
    b = np.asarray(b)
    assert a.shape == b.shape, what
    bad = np.flatnonzero(~(a == b).ravel())
    if bad.size:
        i = bad[0]
        av, bv = a.ravel()[i], b.ravel()[i]
        raise AssertionError(f"{what}: {bad.size} of {a.size} values differ; first at {i}: {av!r} vs {bv!r}")
