"""Runs the reference's own step loop (oracle/_ref/felis_ref*, compiled from
the reference's unmodified sources with the stand-ins of oracle/ref_shim/).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's reference arm, never by the felis_b200 package.  The executable
is a child process that runs in a scratch directory, because the reference
writes its text outputs (totalEnergy, twissFile, bFactor, ...) into the
current directory and ends the process on its own errors (exit(0) in
particlePush.cpp:373 and rearrangeParticles.cpp:107, MPI_Abort elsewhere).

The executable is built here by `make ref` from the reference's sources; on
a machine without those sources only the prebuilt files in oracle/_ref/ are
used (`available()` tells).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_OUT = os.path.join(HERE, "_ref")
DEFAULT_SOURCES = "/root/reference"
BINARIES = {"strict": "felis_ref", "fast": "felis_ref_fast"}
KEYS = ("x", "y", "px", "py", "theta", "gamma")


def sources() -> str | None:
    src = os.environ.get("FELIS_REFERENCE_SOURCES", DEFAULT_SOURCES)
    return src if os.path.exists(os.path.join(src, "particlePush.cpp")) else None


def binary(variant: str = "strict") -> str:
    return os.path.join(REF_OUT, BINARIES[variant])


def available(variant: str = "strict") -> bool:
    return os.access(binary(variant), os.X_OK)


def build() -> bool:
    """Compiles oracle/_ref when the reference's sources are present; returns
    whether both executables exist afterwards."""
    src = sources()
    if src is not None:
        r = subprocess.run(["make", "-s", "-C", HERE, f"REF={src}", "-j8", "ref"], capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"oracle/_ref build failed:\n{r.stdout}\n{r.stderr}")
    return available("strict") and available("fast")


def write_state(d: str, beams: list[dict], fields: list[tuple[np.ndarray, np.ndarray]]):
    """An initial state in the files felis_ref --state reads: per species the
    six particle columns, slice offsets and weights; per harmonic the (S+2,
    ny, nx) complex fields with ghost planes."""
    os.makedirs(d, exist_ok=True)
    for s, b in enumerate(beams):
        for k in KEYS:
            np.ascontiguousarray(b[k], dtype=np.float64).tofile(os.path.join(d, f"p{s}_{k}.bin"))
        np.ascontiguousarray(b["offsets"], dtype=np.int64).tofile(os.path.join(d, f"p{s}_offsets.bin"))
        np.ascontiguousarray(b["weights"], dtype=np.float64).tofile(os.path.join(d, f"p{s}_weights.bin"))
    for h, (ux, uy) in enumerate(fields):
        np.ascontiguousarray(ux, dtype=np.complex128).tofile(os.path.join(d, f"Ux_{h}.bin"))
        np.ascontiguousarray(uy, dtype=np.complex128).tofile(os.path.join(d, f"Uy_{h}.bin"))


def read_state(d: str, num_harmony: int, num_species: int, shape: tuple[int, int, int]) -> dict:
    out = {"Ux": [], "Uy": [], "particles": []}
    for h in range(num_harmony):
        out["Ux"].append(np.fromfile(os.path.join(d, f"Ux_{h}.bin"), dtype=np.complex128).reshape(shape))
        out["Uy"].append(np.fromfile(os.path.join(d, f"Uy_{h}.bin"), dtype=np.complex128).reshape(shape))
    ez = os.path.join(d, "Ez_0.bin")
    if os.path.exists(ez):
        out["Ez"] = np.fromfile(ez, dtype=np.complex128)
    for s in range(num_species):
        b = {k: np.fromfile(os.path.join(d, f"p{s}_{k}.bin")) for k in KEYS}
        b["offsets"] = np.fromfile(os.path.join(d, f"p{s}_offsets.bin"), dtype=np.int64)
        b["weights"] = np.fromfile(os.path.join(d, f"p{s}_weights.bin"))
        out["particles"].append(b)
    return out


def read_setup(d: str) -> dict:
    vals = {}
    with open(os.path.join(d, "setup.txt")) as f:
        for line in f:
            k, *rest = line.split()
            nums = [float(v) for v in rest]
            vals[k] = nums[0] if len(nums) == 1 else nums
    return vals


def run(input_path: str, *, state: tuple[list[dict], list] | None = None, bessel: np.ndarray | None = None,
        it0: int = 0, it1: int | None = None, setup: bool = False, initial: bool = False, final: bool = True,
        time_warmup: int | None = None, variant: str = "strict", seed: int | None = None,
        ranks: tuple[int, int] | None = None, workdir: str | None = None, keep: bool = False,
        timeout: float | None = None) -> dict:
    """Runs felis_ref on `input_path` and returns its outputs.

    state: (beams per species, fields per harmonic) to start from instead of
    the reference's own loadSeed/loadBeam; bessel: a table to use instead of
    the one boundary() builds; seed: GSL_RNG_SEED for the reference's loader;
    ranks: (n, r) to play rank r of n (timing runs only, no messages cross).
    Returns {'energyX','energyY' (iterations x H), 'final', 'init', 'setup',
    'timing', 'dir', 'stdout'} as requested."""
    exe = binary(variant)
    if not os.access(exe, os.X_OK):
        raise FileNotFoundError(f"{exe} is not built (make -C oracle ref)")
    own = workdir is None
    wd = workdir or tempfile.mkdtemp(prefix="felis_ref_")
    try:
        out_dir = os.path.join(wd, "out")
        args = [exe, os.path.abspath(input_path), out_dir, "--from", str(it0)]
        if it1 is not None:
            args += ["--to", str(it1)]
        if state is not None:
            sd = os.path.join(wd, "state")
            write_state(sd, *state)
            args += ["--state", sd]
        if bessel is not None:
            bf = os.path.join(wd, "bessel.bin")
            np.ascontiguousarray(bessel, dtype=np.float64).tofile(bf)
            args += ["--bessel", bf]
        if setup:
            args.append("--setup")
        if initial:
            args.append("--initial")
        if not final:
            args.append("--no-final")
        if time_warmup is not None:
            args += ["--time", str(time_warmup)]
        env = dict(os.environ)
        env.pop("GSL_RNG_SEED", None)
        if seed is not None:
            env["GSL_RNG_SEED"] = str(seed)
        if ranks is not None:
            env["FELIS_REF_NRANKS"], env["FELIS_REF_RANK"] = str(ranks[0]), str(ranks[1])
        r = subprocess.run(args, cwd=wd, env=env, capture_output=True, text=True, timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError(f"felis_ref failed ({r.returncode}):\n{r.stdout[-2000:]}\n{r.stderr[-2000:]}")
        res = {"dir": wd, "stdout": r.stdout}
        if setup:
            res["setup"] = read_setup(out_dir)
            res["bessel"] = np.fromfile(os.path.join(out_dir, "bessel.bin"))
            res["wakeF"] = np.fromfile(os.path.join(out_dir, "wakeF.bin"))
            if os.path.exists(os.path.join(out_dir, "abc_alpha.bin")):
                res["abc"] = tuple(np.fromfile(os.path.join(out_dir, f"abc_{n}.bin"), dtype=np.complex128)
                                   for n in ("alpha", "alphaP", "beta", "betaP"))
        with open(os.path.join(out_dir, "meta.txt")) as f:
            meta = {k: int(v) for k, v in (ln.split() for ln in f)}
        shape_info = (meta["harmonics"], meta["species"], (meta["slices"] + 2, meta["ny"], meta["nx"]))
        res["meta"] = meta
        if initial:
            res["init"] = read_state(os.path.join(out_dir, "init"), *shape_info)
        if final:
            res["final"] = read_state(out_dir, *shape_info)
        nh = shape_info[0]
        ex = np.fromfile(os.path.join(out_dir, "energyX.bin"))
        ey = np.fromfile(os.path.join(out_dir, "energyY.bin"))
        res["energyX"] = ex.reshape(-1, nh)
        res["energyY"] = ey.reshape(-1, nh)
        res["wakeE"] = np.fromfile(os.path.join(out_dir, "wakeE.bin"))
        tf = os.path.join(out_dir, "timing.txt")
        if os.path.exists(tf):
            with open(tf) as f:
                res["timing"] = {k: float(v) for k, v in (ln.split() for ln in f)}
        return res
    finally:
        if own and not keep:
            shutil.rmtree(wd, ignore_errors=True)

