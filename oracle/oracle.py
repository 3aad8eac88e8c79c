"""ctypes view of the CPU restatement (felis_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, never by the felis_b200 package.
Parity status: pinned to the reference's own step loop (oracle/_ref,
tests/test_ref_pin.py, tests/test_golden_ref.py; see felis_oracle.cpp).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
VARIANTS = {"strict": "liboracle_strict.so", "libm": "liboracle_libm.so", "fast": "liboracle_fast.so"}


def build(variant: str = "strict", out_dir: str | None = None) -> str:
    out_dir = out_dir or BUILD
    target = "fast" if variant == "fast" else "all"
    r = subprocess.run(["make", "-s", "-C", HERE, f"OUT={out_dir}", target], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stdout}\n{r.stderr}")
    return os.path.join(out_dir, VARIANTS[variant])


_dp = C.POINTER(C.c_double)
_i64p = C.POINTER(C.c_int64)
_libs: dict[str, C.CDLL] = {}


def load(variant: str = "strict", out_dir: str | None = None) -> C.CDLL:
    key = f"{variant}:{out_dir}"
    if key in _libs:
        return _libs[key]
    path = os.path.join(out_dir or BUILD, VARIANTS[variant])
    if not os.path.exists(path):
        path = build(variant, out_dir)
    lib = C.CDLL(path)
    vp = C.c_void_p
    sigs = {
        "orc_create": (vp, [vp, C.c_int]),
        "orc_destroy": (None, [vp]),
        "orc_error": (C.c_char_p, [vp]),
        "orc_set_threads": (None, [vp, C.c_int]),
        "orc_set_particles": (C.c_int, [vp, C.c_int, _dp, _dp, _dp, _dp, _dp, _dp, _i64p, _dp]),
        "orc_get_particles": (C.c_int, [vp, C.c_int, _dp, _dp, _dp, _dp, _dp, _dp]),
        "orc_set_field": (C.c_int, [vp, C.c_int, C.c_int, _dp]),
        "orc_get_field": (C.c_int, [vp, C.c_int, C.c_int, _dp]),
        "orc_get_ez": (C.c_int, [vp, _dp]),
        "orc_set_ez": (C.c_int, [vp, _dp]),
        "orc_get_abc": (None, [vp, _dp, _dp, _dp, _dp]),
        "orc_update_lattice": (C.c_int, [vp, C.c_int, C.c_double]),
        "orc_get_lattice": (None, [vp, vp]),
        "orc_set_lattice": (None, [vp, vp]),
        "orc_transverse_push": (C.c_int, [vp]),
        "orc_push_theta_gamma": (C.c_int, [vp]),
        "orc_drift_theta_gamma": (C.c_int, [vp]),
        "orc_solve_field": (C.c_int, [vp]),
        "orc_periodic_particles": (C.c_int, [vp]),
        "orc_phase_shift": (C.c_int, [vp, C.c_int]),
        "orc_shift_field": (C.c_int, [vp]),
        "orc_total_energy": (None, [vp, _dp]),
        "orc_twiss": (None, [vp, _dp]),
        "orc_bfactor": (None, [vp, _dp]),
        "orc_diagnostic_sums": (None, [vp, _dp]),
        "orc_run": (C.c_int, [vp, C.c_int, C.c_int, _dp, _dp, _dp]),
        "orc_build_flags": (C.c_int, []),
    }
    for name, (res, args) in sigs.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _libs[key] = lib
    return lib


def _p(a):
    return a.ctypes.data_as(_dp) if a is not None else None


class Oracle:
    """CPU restatement of the slice loop for one felis_params (a Domain)."""

    def __init__(self, params, threads: int = 1, variant: str = "strict", out_dir: str | None = None):
        self.lib = load(variant, out_dir)
        self.h = self.lib.orc_create(C.byref(params), threads)
        if not self.h:
            raise ValueError("orc_create rejected the parameters")
        self.S = params.slice_n
        self.nx, self.ny = params.nx, params.ny
        self.H = params.num_harmony
        self.species = params.num_species
        self.L, self.F, self.nr = params.scl_mode, params.scf_mode, params.nr
        self.mode = params.mode
        self._counts = [0] * self.species

    def close(self):
        if getattr(self, "h", None):
            self.lib.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def _ck(self, rc):
        if rc != 0:
            raise RuntimeError(f"oracle status {rc}: {self.lib.orc_error(self.h).decode()}")

    def set_threads(self, n: int):
        self.lib.orc_set_threads(self.h, n)

    def set_particles(self, species, x, y, px, py, theta, gamma, offsets, weights):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, px, py, theta, gamma)]
        off = np.ascontiguousarray(offsets, dtype=np.int64)
        w = np.ascontiguousarray(weights, dtype=np.float64)
        self._ck(self.lib.orc_set_particles(self.h, species, *(_p(a) for a in arrs), off.ctypes.data_as(_i64p), _p(w)))
        self._counts[species] = int(off[-1])

    def get_particles(self, species: int = 0) -> dict:
        n = self._counts[species]
        out = {k: np.zeros(n) for k in ("x", "y", "px", "py", "theta", "gamma")}
        self._ck(self.lib.orc_get_particles(self.h, species, *(_p(out[k]) for k in ("x", "y", "px", "py", "theta", "gamma"))))
        return out

    def set_field(self, hidx: int, which: int, data: np.ndarray):
        buf = np.ascontiguousarray(data, dtype=np.complex128).ravel().view(np.float64)
        self._ck(self.lib.orc_set_field(self.h, hidx, which, _p(buf)))

    def get_field(self, hidx: int, which: int) -> np.ndarray:
        n = (self.S + 2) * self.nx * self.ny
        buf = np.zeros(2 * n)
        self._ck(self.lib.orc_get_field(self.h, hidx, which, _p(buf)))
        return (buf[0::2] + 1j * buf[1::2]).reshape(self.S + 2, self.ny, self.nx)

    def get_ez(self) -> np.ndarray:
        n = self.L * (self.S + 2) * self.F * self.nr
        buf = np.zeros(2 * n)
        self._ck(self.lib.orc_get_ez(self.h, _p(buf)))
        return (buf[0::2] + 1j * buf[1::2]).reshape(self.L, self.S + 2, self.F, self.nr)

    def abc(self):
        a = [np.zeros(2 * self.nx), np.zeros(2 * self.nx), np.zeros(2 * self.ny), np.zeros(2 * self.ny)]
        self.lib.orc_get_abc(self.h, *(_p(x) for x in a))
        return tuple(x[0::2] + 1j * x[1::2] for x in a)

    def update_lattice(self, it: int, half: float):
        self.lib.orc_update_lattice(self.h, it, half)

    def lattice(self):
        from felis_b200 import Lattice  # struct layout only

        l = Lattice()
        self.lib.orc_get_lattice(self.h, C.byref(l))
        return l

    def set_lattice(self, l):
        self.lib.orc_set_lattice(self.h, C.byref(l))

    def transverse_push(self):
        self._ck(self.lib.orc_transverse_push(self.h))

    def push_theta_gamma(self):
        self._ck(self.lib.orc_push_theta_gamma(self.h))

    def drift_theta_gamma(self):
        self._ck(self.lib.orc_drift_theta_gamma(self.h))

    def solve_field(self):
        self._ck(self.lib.orc_solve_field(self.h))

    def periodic_particles(self):
        self._ck(self.lib.orc_periodic_particles(self.h))

    def phase_shift(self, it: int):
        self._ck(self.lib.orc_phase_shift(self.h, it))

    def shift_field(self):
        self._ck(self.lib.orc_shift_field(self.h))

    def total_energy(self) -> np.ndarray:
        out = np.zeros(2 * self.H)
        self.lib.orc_total_energy(self.h, _p(out))
        return out

    def twiss(self) -> np.ndarray:
        out = np.zeros(6 * self.species)
        self.lib.orc_twiss(self.h, _p(out))
        return out

    def bfactor(self) -> np.ndarray:
        out = np.zeros(2 * self.H)
        self.lib.orc_bfactor(self.h, _p(out))
        return out

    def diagnostic_sums(self) -> np.ndarray:
        out = np.zeros(7 * self.species + 2 * self.H + 1)
        self.lib.orc_diagnostic_sums(self.h, _p(out))
        return out

    def run(self, it0: int, it1: int, diagnostics: bool = True):
        n = it1 - it0
        e = np.zeros(n * 2 * self.H) if diagnostics else None
        t = np.zeros(n * 6 * self.species) if diagnostics else None
        b = np.zeros(n * 2 * self.H) if diagnostics else None
        self._ck(self.lib.orc_run(self.h, it0, it1, _p(e), _p(t), _p(b)))
        if diagnostics:
            return e.reshape(n, 2 * self.H), t.reshape(n, 6 * self.species), b.reshape(n, 2 * self.H)
        return None
