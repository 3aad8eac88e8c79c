"""Checkpoints in the logical layout of the reference's HDF5 dumps.

saveFieldHDF.cpp:34-157 writes `field<it>.h5` with one dataset per harmonic
and polarisation, "Ux<H>" / "Uy<H>", of shape (sliceN, 2 nx ny) (re, im
interleaved, the physical slices without the ghost planes), and the metadata
sliceN, harmony, numHarmony, nx, ny, minZ, dz, bucketZ, powerNorm,
intensityNorm, dx, dy, minX, minY.  saveParticleHDF.cpp:27-170 writes
`particle<it>.h5` with one dataset per species, "<s>", of shape (N, 8) with
the columns theta, x, y, gamma, px, py, global slice index, weight (slice
order), the attributes cntP / totalCnt, and the metadata minZ, dz, bucketZ,
dPhi, lambda0, gamma0, numData, nSpecies, sliceN.

HDF5 is not available to this library, so the same datasets and metadata are
kept in numpy .npz containers (`field<it>.npz`, `particle<it>.npz`; an
attribute A of dataset D is the entry "D/A").  Restoring follows
restoreFieldHDF.cpp / restoreParticleHDF.cpp: the run resumes from a freshly
created handle (so the lattice state machine starts over, as the reference's
restart does: its first solveField after a restart uses the initial current
flag), and the wake is recomputed from the restored beam (main.cpp:51-58).

Engines: a felis_b200.Handle, or anything with the same download/upload
methods (the CPU restatement in the tests).  With a torch.distributed group,
every process passes its slice block and rank 0 writes the whole bunch.
"""
from __future__ import annotations

import math
import os

import numpy as np

# the values of constants.h
E_CHARGE = 1.60217662e-19
E_MASS = 9.10938291e-31
VELOCITY_C = 299792458.0
Z0 = 376.730313668


def _fields(engine, H: int):
    get = getattr(engine, "download_field", None) or engine.get_field
    return [(get(h, 0)[1:-1], get(h, 1)[1:-1]) for h in range(H)]


def _put_field(engine, h: int, pol: int, planes: np.ndarray):
    put = getattr(engine, "upload_field", None) or engine.set_field
    S = planes.shape[0]
    full = np.zeros((S + 2,) + planes.shape[1:], dtype=np.complex128)
    full[1:-1] = planes
    put(h, pol, full)


def _gather(dist, a: np.ndarray) -> np.ndarray:
    """Concatenation of every process's array along axis 0 (rank order)."""
    import torch

    world = dist.get_world_size()
    n = torch.tensor([a.shape[0]], dtype=torch.int64)
    sizes = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
    dist.all_gather(sizes, n)
    sizes = [int(x.item()) for x in sizes]
    tail = a.shape[1:]
    big = max(sizes)
    buf = np.zeros((big,) + tail, dtype=a.dtype)
    buf[:a.shape[0]] = a
    t = torch.from_numpy(buf.view(np.float64) if np.iscomplexobj(buf) else buf)
    parts = [torch.zeros_like(t) for _ in range(world)]
    dist.all_gather(parts, t)
    out = []
    for p, k in zip(parts, sizes):
        v = p.numpy()
        if np.iscomplexobj(a):
            v = v.view(np.complex128)
        out.append(v[:k])
    return np.concatenate(out, axis=0)


def field_meta(p) -> dict:
    """The metadata of saveFieldHDF.cpp:67-88 from a felis_params (the power
    normalisation uses the cell area dx dy, or in 1D the seed spot area
    2 pi spotSigR^2)."""
    area = 2.0 * math.pi * p.spot_sig_r * p.spot_sig_r if p.dimension == 1 else p.dx * p.dy
    coef = E_MASS * VELOCITY_C * VELOCITY_C * p.ks / E_CHARGE
    bucketZ = p.num_slice * p.lambda0
    return {
        "sliceN": np.array([p.global_slice_n], np.int32),
        "harmony": np.array([p.harmony[i] for i in range(p.num_harmony)], np.int32),
        "numHarmony": np.array([p.num_harmony], np.int32),
        "nx": np.array([p.nx], np.int32), "ny": np.array([p.ny], np.int32),
        "minZ": np.array([p.min_z]), "dz": np.array([p.dz]), "bucketZ": np.array([bucketZ]),
        "powerNorm": np.array([coef * coef / (2.0 * Z0) * area]),
        "intensityNorm": np.array([coef * coef / (2.0 * Z0) * bucketZ / VELOCITY_C]),
        "dx": np.array([p.dx]), "dy": np.array([p.dy]), "minX": np.array([p.min_x]), "minY": np.array([p.min_y]),
    }


def save_field(engine, p, directory: str, iteration: int, dist=None) -> str | None:
    """field<iteration>.npz of the engine's field (saveFieldHDF.cpp:34-94)."""
    H, N = p.num_harmony, p.nx * p.ny
    data = {}
    for h, (ux, uy) in enumerate(_fields(engine, H)):
        Hn = p.harmony[h]
        for name, u in ((f"Ux{Hn}", ux), (f"Uy{Hn}", uy)):
            a = np.ascontiguousarray(u.reshape(u.shape[0], N))
            if dist is not None:
                a = _gather(dist, a)
            data[name] = a.view(np.float64).reshape(a.shape[0], 2 * N)
    if dist is not None and dist.get_rank() != 0:
        return None
    data.update(field_meta(p))
    path = os.path.join(directory, f"field{iteration}.npz")
    np.savez(path, **data)
    return path


def save_particles(engine, p, beam_weights, directory: str, iteration: int, dist=None) -> str | None:
    """particle<iteration>.npz (saveParticleHDF.cpp:27-170): per species (N, 8)
    rows theta, x, y, gamma, px, py, global slice, weight.  `beam_weights[s]`
    are the per-slice weights and offsets of species s: (offsets, weights)."""
    get = getattr(engine, "download_particles", None) or engine.get_particles
    data = {}
    for sp in range(p.num_species):
        offsets, weights = beam_weights[sp]
        q = get(sp)
        cnt = np.diff(np.asarray(offsets))
        sl = np.repeat(np.arange(len(cnt)) + p.min_i, cnt).astype(np.float64)
        w = np.repeat(np.asarray(weights, dtype=np.float64), cnt)
        rows = np.stack([q["theta"], q["x"], q["y"], q["gamma"], q["px"], q["py"], sl, w], axis=1)
        local = np.array([rows.shape[0]], np.int64)
        if dist is not None:
            import torch

            t = torch.from_numpy(local.copy())
            parts = [torch.zeros_like(t) for _ in range(dist.get_world_size())]
            dist.all_gather(parts, t)
            cntP = np.array([int(x.item()) for x in parts], np.int64)
            rows = _gather(dist, rows)
        else:
            cntP = local
        data[str(sp)] = rows
        data[f"{sp}/cntP"] = cntP
        data[f"{sp}/totalCnt"] = np.array([rows.shape[0]], np.int64)
    if dist is not None and dist.get_rank() != 0:
        return None
    gamma0 = [p.gamma0] * p.num_species
    data.update({
        "minZ": np.array([p.min_z]), "dz": np.array([p.dz]), "bucketZ": np.array([p.lambda0 * p.num_slice]),
        "dPhi": np.array([2.0 * math.pi * p.num_slice]), "lambda0": np.array([p.lambda0]),
        "gamma0": np.array(gamma0), "numData": np.array([8], np.int32),
        "nSpecies": np.array([p.num_species], np.int32), "sliceN": np.array([p.global_slice_n], np.int32),
    })
    path = os.path.join(directory, f"particle{iteration}.npz")
    np.savez(path, **data)
    return path


def restore_field(engine, p, directory: str, iteration: int):
    """Loads this process's slice block from field<iteration>.npz
    (restoreFieldHDF.cpp): the planes min_i .. min_i + slice_n - 1."""
    with np.load(os.path.join(directory, f"field{iteration}.npz")) as f:
        if int(f["nx"][0]) != p.nx or int(f["ny"][0]) != p.ny or int(f["sliceN"][0]) != p.global_slice_n:
            raise ValueError("checkpoint grid or slice count differs from the parameters")
        for h in range(p.num_harmony):
            Hn = p.harmony[h]
            for pol, name in ((0, f"Ux{Hn}"), (1, f"Uy{Hn}")):
                a = f[name][p.min_i:p.min_i + p.slice_n]
                u = np.ascontiguousarray(a).view(np.complex128).reshape(p.slice_n, p.ny, p.nx)
                _put_field(engine, h, pol, u)


def read_particles(p, directory: str, iteration: int) -> list:
    """This process's particles from particle<iteration>.npz (the rows whose
    slice index lies in the block, restoreParticleHDF.cpp), per species as a
    beam dict (x, y, px, py, theta, gamma, offsets, weights of the block)."""
    out = []
    with np.load(os.path.join(directory, f"particle{iteration}.npz")) as f:
        if int(f["nSpecies"][0]) != p.num_species:
            raise ValueError(f"checkpoint holds {int(f['nSpecies'][0])} species")
        for sp in range(p.num_species):
            rows = f[str(sp)]
            sl = rows[:, 6].astype(np.int64) - p.min_i
            keep = (sl >= 0) & (sl < p.slice_n)
            rows, sl = rows[keep], sl[keep]
            order = np.argsort(sl, kind="stable")
            rows, sl = rows[order], sl[order]
            cnt = np.bincount(sl, minlength=p.slice_n)
            offsets = np.zeros(p.slice_n + 1, np.int64)
            offsets[1:] = np.cumsum(cnt)
            weights = np.zeros(p.slice_n)
            weights[cnt > 0] = rows[offsets[:-1][cnt > 0], 7]
            out.append({"theta": rows[:, 0].copy(), "x": rows[:, 1].copy(), "y": rows[:, 2].copy(),
                        "gamma": rows[:, 3].copy(), "px": rows[:, 4].copy(), "py": rows[:, 5].copy(),
                        "offsets": offsets, "weights": weights})
    return out


def restore_particles(engine, p, directory: str, iteration: int) -> list:
    """Uploads this process's particles from particle<iteration>.npz; returns
    read_particles' beams."""
    put = getattr(engine, "upload_particles", None) or engine.set_particles
    beams = read_particles(p, directory, iteration)
    for sp, b in enumerate(beams):
        put(sp, b["x"], b["y"], b["px"], b["py"], b["theta"], b["gamma"], b["offsets"], b["weights"])
    return beams


def restore_wake(cfg, beams: list):
    """Recomputes the wake table of a Config from restored beams (main.cpp:51-58,
    updateWakeField): the slice charge of every species, then
    felis_config_wake.  Call before creating the handle from cfg.params.
    Only for a single process holding the whole bunch."""
    den = np.zeros(cfg.params.global_slice_n)
    for b in beams:
        den[:len(b["weights"])] += np.asarray(b["weights"]) * np.diff(b["offsets"])
    cfg.wake(den)
