"""Slices sharded across processes (felis_b200.shard) against one process.

Two and three gloo processes on CPU run the CPU restatement on their slice
blocks (boundary.cpp:33-46), exchange the slipping slice after every shift
(fieldShareZ.cpp:39-78) and reduce energy and twiss across processes.  The
particles and fields of every block must be bit-identical to the same slices
of a single-process run: each slice's step is local and the exchanged plane is
copied, not computed.  The reduced diagnostics are sums in another order, so
they agree to rounding (rtol 1e-12).
"""
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

from conftest import assert_bits

HERE = os.path.dirname(os.path.abspath(__file__))
IT0, IT1 = 0, 14


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _run_ranks(path, world, tmp_path, engine="oracle", ckpt=None):
    port = _free_port()
    procs, outs = [], []
    for r in range(world):
        out = str(tmp_path / f"rank{r}.npz")
        env = dict(os.environ, RANK=str(r), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                   OMP_NUM_THREADS="1")
        procs.append(subprocess.Popen([sys.executable, os.path.join(HERE, "shard_worker.py"), path, str(IT0), str(IT1),
                                       out, engine] + ([ckpt] if ckpt else []), env=env, stdout=subprocess.PIPE, stderr=subprocess.STDOUT))
        outs.append(out)
    logs = []
    for p in procs:
        try:
            o, _ = p.communicate(timeout=240)
        except subprocess.TimeoutExpired:
            for q in procs:
                q.kill()
            raise
        logs.append(o.decode(errors="replace"))
    for p, log in zip(procs, logs):
        assert p.returncode == 0, log[-3000:]
    return [dict(np.load(o)) for o in outs]


def _single(fb, oracle_mod, tmp, **extra):
    from felis_b200 import workloads

    path = workloads.write_input(str(tmp / "s.inp"), kind="sase", slices=11, beamlets=64, per_beamlet=4, nx=21,
                                 harmonics=(1, 3), total_length=0.2, **extra)
    cfg = fb.Config(path)
    p = cfg.params
    beam = cfg.load_beam(0, seed=2)
    o = oracle_mod.Oracle(p, threads=1)
    o.set_particles(0, beam["x"], beam["y"], beam["px"], beam["py"], beam["theta"], beam["gamma"], beam["offsets"],
                    beam["weights"])
    for h in range(p.num_harmony):
        ux, uy = cfg.load_seed(h)
        o.set_field(h, 0, ux)
        o.set_field(h, 1, uy)
    # bunching sums of the whole bunch before every iteration, as the blocks report them
    E, T, B, sums, shifts = [], [], [], [], 0
    for it in range(IT0, IT1):
        e, t, b = o.run(it, it + 1)
        E.append(e[0]); T.append(t[0]); B.append(b[0])
        shifts += int(not o.lattice().drift_flag)
    res = dict(E=np.array(E), T=np.array(T), B=np.array(B), shifts=shifts, path=path, H=p.num_harmony)
    res.update(o.get_particles(0))
    res["fields"] = {(h, pol): o.get_field(h, pol)[1:-1] for h in range(p.num_harmony) for pol in (0, 1)}
    res["offsets"] = beam["offsets"]
    from felis_b200 import checkpoint

    res["ckpt"] = str(tmp)
    checkpoint.save_field(o, p, str(tmp), IT1)
    checkpoint.save_particles(o, p, [(beam["offsets"], beam["weights"])], str(tmp), IT1)
    return res


@pytest.fixture(scope="module")
def single(fb, oracle_mod, tmp_path_factory):
    return _single(fb, oracle_mod, tmp_path_factory.mktemp("shard"))


@pytest.fixture(scope="module")
def single_1d(fb, oracle_mod, tmp_path_factory):
    return _single(fb, oracle_mod, tmp_path_factory.mktemp("shard1d"), dimension=1)


def test_slice_blocks_match_the_decomposition():
    from felis_b200 import shard

    assert shard.slice_blocks(11, 2) == [(0, 6), (6, 11)]
    assert shard.slice_blocks(11, 3) == [(0, 4), (4, 8), (8, 11)]
    assert shard.slice_blocks(8, 4) == [(0, 2), (2, 4), (4, 6), (6, 8)]


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_loop_equals_single_process(single, world, tmp_path):
    assert single["shifts"] > 4, "the case must slip several slices across the block edges"
    ranks = _run_ranks(single["path"], world, tmp_path)
    off = single["offsets"]
    for r in ranks:
        lo, hi = int(r["lo"]), int(r["hi"])
        a, b = int(off[lo]), int(off[hi])
        for k in ("x", "y", "px", "py", "theta", "gamma"):
            assert_bits(r[k], single[k][a:b], f"{k} slices {lo}:{hi}")
        for (h, pol), U in single["fields"].items():
            assert_bits(r[f"U{h}{pol}"], U[lo:hi], f"field h{h} pol{pol} slices {lo}:{hi}")
        # energy and twiss are whole-bunch values on every process
        np.testing.assert_allclose(r["E"], single["E"], rtol=1e-12, atol=1e-300)
        np.testing.assert_allclose(r["T"], single["T"], rtol=1e-12)
    # the bunching factor is per block; its sums reassemble the whole-bunch value
    tot = sum(r["bsums"] for r in ranks)
    np.testing.assert_allclose(tot[:, :-1] / tot[:, -1:], single["B"], rtol=1e-11, atol=1e-14)


def test_sharded_1d_loop_equals_single_process(single_1d, tmp_path):
    """The 1D model (one field value per slice, harmonic and polarisation)
    sharded over two processes: the hand-over is one value per plane."""
    assert single_1d["shifts"] > 4
    ranks = _run_ranks(single_1d["path"], 2, tmp_path)
    off = single_1d["offsets"]
    for r in ranks:
        lo, hi = int(r["lo"]), int(r["hi"])
        a, b = int(off[lo]), int(off[hi])
        for k in ("x", "y", "px", "py", "theta", "gamma"):
            assert_bits(r[k], single_1d[k][a:b], f"{k} slices {lo}:{hi}")
        for (h, pol), U in single_1d["fields"].items():
            assert_bits(r[f"U{h}{pol}"], U[lo:hi], f"field h{h} pol{pol} slices {lo}:{hi}")
        np.testing.assert_allclose(r["E"], single_1d["E"], rtol=1e-12, atol=1e-300)
    tot = sum(r["bsums"] for r in ranks)
    np.testing.assert_allclose(tot[:, :-1] / tot[:, -1:], single_1d["B"], rtol=1e-11, atol=1e-14)


def test_sharded_checkpoint_equals_single_process(single, tmp_path):
    """Two processes write one checkpoint of their blocks (rank 0 gathers,
    as the reference's collective HDF5 writes assemble one file); it equals
    the single-process checkpoint of the same state entry for entry, except
    the per-process particle counts."""
    d = tmp_path / "ck"
    d.mkdir()
    _run_ranks(single["path"], 2, tmp_path, ckpt=str(d))
    for name in (f"field{IT1}.npz", f"particle{IT1}.npz"):
        with np.load(d / name) as a, np.load(os.path.join(single["ckpt"], name)) as b:
            assert set(a.files) == set(b.files)
            for k in a.files:
                if k.endswith("/cntP"):
                    assert a[k].sum() == b[k].sum() and len(a[k]) == 2
                else:
                    assert_bits(a[k], b[k], f"{name}:{k}")


@pytest.mark.gpu
@pytest.mark.parametrize("exchange", ["host", "device"])
def test_gpu_blocks_equal_single_process(fb, single, exchange):
    """Two felis_b200.Handle blocks in exchange mode on one GPU, the slipping
    slice handed over after every shift -- through host buffers, or in device
    memory on the handles' streams (felis_first_planes_device) -- against the
    single-process CPU run: the FP64 path is bit-exact, so the blocks are too."""
    from felis_b200 import shard

    path, world = single["path"], 2
    glob = fb.Config(path)
    beam = glob.load_beam(0, seed=2)
    fields = [glob.load_seed(h) for h in range(glob.params.num_harmony)]
    blocks = shard.slice_blocks(glob.params.global_slice_n, world)
    cfgs, engines = [], []
    for r, (lo, hi) in enumerate(blocks):
        cfgs.append(fb.Config(path, world, r))
        g = fb.Handle(cfgs[-1].params)
        b = shard.split_beam(beam, lo, hi)
        g.upload_particles(0, b["x"], b["y"], b["px"], b["py"], b["theta"], b["gamma"], b["offsets"], b["weights"])
        for h, (ux, uy) in enumerate(fields):
            g.upload_field(h, 0, shard.split_field(ux, lo, hi))
            g.upload_field(h, 1, shard.split_field(uy, lo, hi))
        engines.append(shard.GpuEngine(g))
    ns = glob.params.num_species
    for k, it in enumerate(range(IT0, IT1)):
        E = sum(e.energy(it) for e in engines)
        S = sum(e.sums(it) for e in engines)
        np.testing.assert_allclose(E, single["E"][k], rtol=1e-12, atol=1e-300)
        np.testing.assert_allclose(shard.twiss_from_sums(S[:7 * ns], ns), single["T"][k], rtol=1e-11)
        np.testing.assert_allclose(S[7 * ns:-1] / S[-1], single["B"][k], rtol=1e-9, atol=1e-14)
        shifted = [e.step(it) for e in engines]
        assert len(set(shifted)) == 1
        if shifted[0] and exchange == "device":
            shard.exchange_in_process(engines)
        elif shifted[0]:
            out = [e.outgoing() for e in engines]
            engines[0].incoming(np.zeros_like(out[0]))
            for r in range(1, world):
                engines[r].incoming(out[r - 1])
    off = single["offsets"]
    for e, (lo, hi) in zip(engines, blocks):
        a, b = int(off[lo]), int(off[hi])
        got = e.h.download_particles(0)
        for k in ("x", "y", "px", "py", "theta", "gamma"):
            assert_bits(got[k], single[k][a:b], f"{k} slices {lo}:{hi}")
        for (h, pol), U in single["fields"].items():
            assert_bits(e.h.download_field(h, pol)[1:-1], U[lo:hi], f"field h{h} pol{pol} slices {lo}:{hi}")
        e.h.close()


@pytest.mark.gpu
def test_gpu_sharded_processes_equal_single_process(single, tmp_path):
    """Two gloo processes, each with its own Handle on cuda:0 (independent
    contexts; no kernel waits on another process)."""
    ranks = _run_ranks(single["path"], 2, tmp_path, engine="gpu")
    off = single["offsets"]
    for r in ranks:
        lo, hi = int(r["lo"]), int(r["hi"])
        a, b = int(off[lo]), int(off[hi])
        for k in ("x", "y", "px", "py", "theta", "gamma"):
            assert_bits(r[k], single[k][a:b], f"{k} slices {lo}:{hi}")
        for (h, pol), U in single["fields"].items():
            assert_bits(r[f"U{h}{pol}"], U[lo:hi], f"field h{h} pol{pol} slices {lo}:{hi}")
        np.testing.assert_allclose(r["E"], single["E"], rtol=1e-12, atol=1e-300)
        np.testing.assert_allclose(r["T"], single["T"], rtol=1e-11)
