"""One process of the sharded slice loop on CPU (gloo), driven by test_shard.py.

argv: input file, iterations it0 it1, output .npz, engine ("oracle": the CPU
restatement; "gpu": a felis_b200.Handle on cuda:0), and optionally a
directory for a checkpoint of the end state written by all processes
together (felis_b200.checkpoint).  RANK, WORLD_SIZE,
MASTER_ADDR and MASTER_PORT come from the environment.  The initial state is
the single-process beam and seed field cut into this process's slice block,
so the blocks together start from exactly the state of the single-process run.
"""
import datetime
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def main():
    path, it0, it1, out = sys.argv[1], int(sys.argv[2]), int(sys.argv[3]), sys.argv[4]
    engine = sys.argv[5] if len(sys.argv) > 5 else "oracle"
    ckpt = sys.argv[6] if len(sys.argv) > 6 else None
    rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])

    import torch.distributed as dist

    import felis_b200 as fb
    import oracle
    from felis_b200 import checkpoint, shard

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        glob = fb.Config(path)
        beam = glob.load_beam(0, seed=2)
        fields = [glob.load_seed(h) for h in range(glob.params.num_harmony)]
        lo, hi = shard.slice_blocks(glob.params.global_slice_n, world)[rank]

        cfg = fb.Config(path, world, rank)
        p = cfg.params
        assert (p.min_i, p.slice_n) == (lo, hi - lo), (p.min_i, p.slice_n, lo, hi)
        b = shard.split_beam(beam, lo, hi)
        if engine == "gpu":
            o = fb.Handle(p)
            put_particles, put_field = o.upload_particles, o.upload_field
            get_particles, get_field = o.download_particles, o.download_field
        else:
            o = oracle.Oracle(p, threads=1)
            put_particles, put_field = o.set_particles, o.set_field
            get_particles, get_field = o.get_particles, o.get_field
        put_particles(0, b["x"], b["y"], b["px"], b["py"], b["theta"], b["gamma"], b["offsets"], b["weights"])
        for h, (ux, uy) in enumerate(fields):
            put_field(h, 0, shard.split_field(ux, lo, hi))
            put_field(h, 1, shard.split_field(uy, lo, hi))

        eng = shard.GpuEngine(o) if engine == "gpu" else shard.OracleEngine(o, p.mode)
        loop = shard.ShardedLoop(eng, dist, rank, world)
        E, T, B = loop.run(it0, it1)
        res = dict(E=E, T=T, B=B, bsums=loop.bunching_sums, lo=lo, hi=hi)
        res.update({k: v for k, v in get_particles(0).items()})
        for h in range(o.H):
            for pol in (0, 1):
                res[f"U{h}{pol}"] = get_field(h, pol)[1:-1]
        np.savez(out, **res)
        if ckpt:
            checkpoint.save_field(o, p, ckpt, it1, dist=dist)
            checkpoint.save_particles(o, p, [(b["offsets"], b["weights"])], ckpt, it1, dist=dist)
        dist.barrier()
    finally:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
