"""felis_b200 — B200-native FELIS slice loop behind a C ABI.

Python view of include/felis_b200.h (ctypes over the in-tree
libfelis_b200.so).  The library is the product: every compute call here goes
to CUDA kernels; nothing falls back to the CPU.  Importing the package fails
loudly when the shared library has not been built.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libfelis_b200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"felis_b200: {LIB_PATH} is missing; build it with `python felis_b200/_build.py` "
        "(the CUDA extension is required, there is no CPU fallback)")

_lib = C.CDLL(LIB_PATH)

MAX_HARMONY = 8
MAX_SPECIES = 8
ABI_VERSION = 3

OK, BAD_ARG, CUDA_ERROR, THETA_OVERFLOW, OUT_OF_RANGE, NAN, TIMEOUT, UNSUPPORTED, NO_DEVICE, IO, NOT_FOUND = range(11)
STATUS_NAMES = {0: "OK", 1: "BAD_ARG", 2: "CUDA_ERROR", 3: "THETA_OVERFLOW", 4: "OUT_OF_RANGE", 5: "NAN",
                6: "TIMEOUT", 7: "UNSUPPORTED", 8: "NO_DEVICE", 9: "IO", 10: "NOT_FOUND"}
STATIC, TIME_DEPENDENT = 1, 2
KERNEL_KINDS = {"particles": 0, "deposit": 1, "adi": 2, "reduce": 3, "shift": 4}
BATCH_KERNEL_KINDS = {"adi": 0, "push": 1, "reduce": 2}
BIPOLAR, QUADPOLAR = 1, 2
FP64, MIXED = 0, 1

_dp = C.POINTER(C.c_double)
_i64p = C.POINTER(C.c_int64)
_i32p = C.POINTER(C.c_int32)


class Undulator(C.Structure):
    _fields_ = [("type", C.c_int32), ("K0_alpha", C.c_int32), ("numbers", C.c_int32), ("air", C.c_int32),
                ("lambdaU", C.c_double), ("slopeK", C.c_double), ("ue", C.c_double),
                ("unit_start", _dp), ("unit_end", _dp), ("und_start", _dp), ("und_end", _dp), ("K0", _dp)]


class Quad(C.Structure):
    _fields_ = [("numbers", C.c_int32), ("pad_", C.c_int32), ("unit_start", _dp), ("unit_end", _dp),
                ("qd_start", _dp), ("qd_end", _dp), ("g", _dp)]


class Params(C.Structure):
    _fields_ = [
        ("abi_version", C.c_int32), ("precision", C.c_int32), ("dimension", C.c_int32), ("mode", C.c_int32),
        ("num_harmony", C.c_int32), ("harmony", C.c_int32 * MAX_HARMONY),
        ("slice_n", C.c_int32), ("min_i", C.c_int32), ("global_slice_n", C.c_int32),
        ("nx", C.c_int32), ("ny", C.c_int32), ("num_slice", C.c_int32), ("num_lambda_u", C.c_int32),
        ("num_species", C.c_int32), ("scl_mode", C.c_int32), ("scf_mode", C.c_int32), ("nr", C.c_int32),
        ("bessel_rows", C.c_int32), ("bessel_cols", C.c_int32), ("abc_n", C.c_int32), ("wake_on", C.c_int32),
        ("max_step", C.c_int32), ("num_undulators", C.c_int32), ("num_quads", C.c_int32),
        ("ks", C.c_double), ("lambda0", C.c_double), ("dz", C.c_double), ("dx", C.c_double), ("dy", C.c_double),
        ("dr", C.c_double), ("min_x", C.c_double), ("max_x", C.c_double), ("min_y", C.c_double),
        ("max_y", C.c_double), ("min_z", C.c_double), ("max_z", C.c_double),
        ("gamma0", C.c_double), ("gam_r", C.c_double), ("d_bessel", C.c_double), ("abc_sig", C.c_double),
        ("spot_sig_r", C.c_double),
        ("K0_init", C.c_double), ("ue_init", C.c_double), ("lambdaU_init", C.c_double),
        ("K0_alpha_init", C.c_int32), ("und_type_init", C.c_int32),
        ("abc_alpha", _dp), ("abc_alpha_p", _dp), ("abc_beta", _dp), ("abc_beta_p", _dp),
        ("bessel", _dp), ("wake_e", _dp),
        ("undulators", C.POINTER(Undulator)), ("quads", C.POINTER(Quad)),
        ("beam_area", C.c_double * 8),
        ("num_phase_shifts", C.c_int32), ("pad_ps_", C.c_int32),
        ("phase_shift_z", _dp), ("phase_shift_phase", _dp),
    ]


class Lattice(C.Structure):
    _fields_ = [("K0", C.c_double), ("ue", C.c_double), ("lambdaU", C.c_double), ("ku", C.c_double),
                ("g", C.c_double), ("K0_alpha", C.c_int32), ("und_type", C.c_int32),
                ("current_flag", C.c_int32), ("drift_flag", C.c_int32)]


def _sig(name, res, *args):
    f = getattr(_lib, name)
    f.restype = res
    f.argtypes = list(args)
    return f


_vp = C.c_void_p
_sig("felis_create", C.c_int, C.POINTER(Params), C.POINTER(_vp))
_sig("felis_destroy", None, _vp)
_sig("felis_last_error", C.c_char_p, _vp)
_sig("felis_device_info", C.c_int, C.c_char_p, C.c_size_t, _i32p)
_sig("felis_upload_particles", C.c_int, _vp, C.c_int32, _dp, _dp, _dp, _dp, _dp, _dp, _i64p, _dp)
_sig("felis_download_particles", C.c_int, _vp, C.c_int32, _dp, _dp, _dp, _dp, _dp, _dp)
_sig("felis_upload_field", C.c_int, _vp, C.c_int32, C.c_int32, _dp)
_sig("felis_download_field", C.c_int, _vp, C.c_int32, C.c_int32, _dp)
_sig("felis_download_source", C.c_int, _vp, C.c_int32, C.c_int32, _dp)
_sig("felis_download_ez", C.c_int, _vp, _dp)
_sig("felis_update_lattice", C.c_int, _vp, C.c_int32, C.c_double)
_sig("felis_get_lattice", C.c_int, _vp, C.POINTER(Lattice))
_sig("felis_set_lattice", C.c_int, _vp, C.POINTER(Lattice))
for _n in ("felis_update_total_energy", "felis_twiss", "felis_bfactor"):
    _sig(_n, C.c_int, _vp, C.c_int32, _dp)
for _n in ("felis_solve_field", "felis_transverse_push", "felis_push_theta_gamma", "felis_drift_theta_gamma",
           "felis_periodic_particles", "felis_phase_shift", "felis_shift_field", "felis_step"):
    _sig(_n, C.c_int, _vp, C.c_int32)
_sig("felis_run", C.c_int, _vp, C.c_int32, C.c_int32)
_sig("felis_first_planes_device", C.c_int, _vp, C.POINTER(_vp))
_sig("felis_get_stream", C.c_int, _vp, C.POINTER(_vp))
_sig("felis_set_slice_exchange", C.c_int, _vp, C.c_int32)
_sig("felis_get_first_planes", C.c_int, _vp, _dp)
_sig("felis_set_first_planes", C.c_int, _vp, _dp)
_sig("felis_diagnostic_sums", C.c_int, _vp, C.c_int32, _dp)
_sig("felis_get_diagnostics", C.c_int, _vp, C.c_int32, C.c_int32, _dp, _dp, _dp)
_sig("felis_edge_deposit_count", C.c_int, _vp, _i64p)
_sig("felis_sort_by_slice", C.c_int, _i32p, C.c_int64, _i64p)
_sig("felis_sort_by_slice_noalloc", C.c_int, _vp, C.c_int64, _vp, _vp)
_sig("felis_sync", C.c_int, _vp)
_sig("felis_profile", C.c_int, _vp, C.c_int32, C.c_int32)
_sig("felis_kernel_stats", C.c_int, _vp, C.c_int32, _i64p, _dp)
_sig("felis_last_run_ms", C.c_int, _vp, _dp)
_sig("felis_batch_create", C.c_int, C.POINTER(C.POINTER(Params)), C.c_int32, C.POINTER(_vp))
_sig("felis_batch_destroy", None, _vp)
_sig("felis_batch_last_error", C.c_char_p, _vp)
_sig("felis_batch_upload_particles", C.c_int, _vp, C.c_int32, _dp, _dp, _dp, _dp, _dp, _dp, _i64p, _dp)
_sig("felis_batch_download_particles", C.c_int, _vp, C.c_int32, _dp, _dp, _dp, _dp, _dp, _dp)
_sig("felis_batch_upload_field", C.c_int, _vp, C.c_int32, C.c_int32, C.c_int32, _dp)
_sig("felis_batch_download_field", C.c_int, _vp, C.c_int32, C.c_int32, C.c_int32, _dp)
_sig("felis_batch_run", C.c_int, _vp, C.c_int32, C.c_int32)
_sig("felis_batch_get_diagnostics", C.c_int, _vp, C.c_int32, C.c_int32, C.c_int32, _dp, _dp, _dp)
_sig("felis_batch_spectral_moments", C.c_int, _vp, C.c_int32, _dp)
_sig("felis_batch_set_launch", C.c_int, _vp, C.c_int32, C.c_int32)
_sig("felis_batch_get_launch", C.c_int, _vp, _i32p, _i32p)
_sig("felis_batch_tune", C.c_int, _vp, C.c_int32, C.c_int32, _i32p)
_sig("felis_batch_last_run_ms", C.c_int, _vp, _dp)
_sig("felis_batch_profile", C.c_int, _vp, C.c_int32, C.c_int32)
_sig("felis_batch_kernel_stats", C.c_int, _vp, C.c_int32, _i64p, _dp)
_fp = C.POINTER(C.c_float)
_sig("felis_mlp_create", C.c_int, C.c_int32, C.c_int32, C.c_int32, C.c_uint64, C.POINTER(_vp))
_sig("felis_mlp_destroy", None, _vp)
_sig("felis_mlp_last_error", C.c_char_p, _vp)
_sig("felis_mlp_param_count", C.c_int, _vp, _i64p)
_sig("felis_mlp_get_params", C.c_int, _vp, _fp)
_sig("felis_mlp_set_params", C.c_int, _vp, _fp)
_sig("felis_mlp_forward", C.c_int, _vp, _fp, C.c_int64, _fp)
_sig("felis_mlp_last_forward", C.c_int, _vp, _dp, _dp)
_sig("felis_mlp_set_fused", C.c_int, _vp, C.c_int32)
_sig("felis_mlp_gradients", C.c_int, _vp, _fp, _fp, C.c_int64, _fp, _dp)
_sig("felis_mlp_set_data", C.c_int, _vp, _fp, _fp, C.c_int64)
_sig("felis_mlp_train", C.c_int, _vp, C.c_int32, C.c_int32, C.c_float, C.c_float, C.c_uint64, _dp)
_sig("felis_wait_selftest", C.c_int, C.c_int32, _i32p)
_sig("felis_config_load", C.c_int, C.c_char_p, C.c_int32, C.c_int32, C.POINTER(_vp))
_sig("felis_config_free", None, _vp)
_sig("felis_config_params", C.POINTER(Params), _vp)
_sig("felis_config_error", C.c_char_p)
_sig("felis_config_load_beam", C.c_int, _vp, C.c_int32, C.c_uint64, _i64p, _dp, _dp, _dp, _dp, _dp, _dp, _dp)
_sig("felis_config_load_beam_device", C.c_int, _vp, C.c_int32, C.c_uint64, _i64p, _dp, _dp, _dp, _dp, _dp, _dp, _dp)
_sig("felis_config_load_seed", C.c_int, _vp, C.c_int32, _dp, _dp)
_sig("felis_config_wake", C.c_int, _vp, _dp, _dp)
_sig("felis_config_wake_device", C.c_int, _vp, _dp, _dp)
_sig("felis_config_wake_function", C.c_int, _vp, _dp)
_sig("felis_detmath_sincos", None, C.c_double, _dp, _dp)
_sig("felis_detmath_atan", C.c_double, C.c_double)
_sig("felis_detmath_atan2", C.c_double, C.c_double, C.c_double)


class FelisError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def _p(a: np.ndarray):
    return a.ctypes.data_as(_dp) if a is not None else None


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def _arr64(a):
    """(owner, double*) of a host array or of a torch CUDA tensor (whose data
    the uploads copy device to device)."""
    if getattr(a, "is_cuda", False):
        import torch

        t = a.to(torch.float64).contiguous()
        return t, C.cast(C.c_void_p(t.data_ptr()), _dp)
    h = _f64(a)
    return h, _p(h)


class Config:
    """A parsed FELIS input file (felis_config_load) and its setup tables."""

    def __init__(self, path: str, num_ranks: int = 1, rank: int = 0):
        h = _vp()
        st = _lib.felis_config_load(os.fsencode(path), num_ranks, rank, C.byref(h))
        if st != OK:
            raise FelisError(st, _lib.felis_config_error().decode())
        self._h = h
        self.params = _lib.felis_config_params(h).contents

    def close(self):
        if getattr(self, "_h", None) and _lib is not None:  # (interpreter teardown)
            _lib.felis_config_free(self._h)
            self._h = None

    def __del__(self):
        self.close()

    @property
    def N(self) -> int:
        return self.params.nx * self.params.ny

    def harmonics(self) -> list[int]:
        return [self.params.harmony[i] for i in range(self.params.num_harmony)]

    def bessel(self) -> np.ndarray:
        p = self.params
        return np.ctypeslib.as_array(p.bessel, shape=(p.bessel_rows * p.bessel_cols,)).reshape(p.bessel_rows, p.bessel_cols).copy()

    def abc(self) -> tuple[np.ndarray, ...]:
        p = self.params
        out = []
        for name, n in (("abc_alpha", p.nx), ("abc_alpha_p", p.nx), ("abc_beta", p.ny), ("abc_beta_p", p.ny)):
            a = np.ctypeslib.as_array(getattr(p, name), shape=(2 * n,)).copy()
            out.append(a[0::2] + 1j * a[1::2])
        return tuple(out)

    def load_beam(self, species: int = 0, seed: int = 0) -> dict:
        """Initial particles of one species (loadBeam.cpp:28-269)."""
        S = self.params.slice_n
        counts = np.zeros(S, dtype=np.int64)
        st = _lib.felis_config_load_beam(self._h, species, seed, counts.ctypes.data_as(_i64p), *([None] * 7))
        if st != OK:
            raise FelisError(st, _lib.felis_config_error().decode())
        n = int(counts.sum())
        arrs = {k: np.zeros(n) for k in ("x", "y", "px", "py", "theta", "gamma")}
        w = np.zeros(S)
        st = _lib.felis_config_load_beam(self._h, species, seed, counts.ctypes.data_as(_i64p),
                                         *(_p(arrs[k]) for k in ("x", "y", "px", "py", "theta", "gamma")), _p(w))
        if st != OK:
            raise FelisError(st, _lib.felis_config_error().decode())
        off = np.zeros(S + 1, dtype=np.int64)
        off[1:] = np.cumsum(counts)
        arrs["offsets"] = off
        arrs["weights"] = w
        return arrs

    def beam_counts(self, species: int = 0) -> np.ndarray:
        """Particles per slice the loader gives this species (no particle is
        generated, no GPU is needed; 3D beams)."""
        counts = np.zeros(self.params.slice_n, dtype=np.int64)
        st = _lib.felis_config_load_beam_device(self._h, species, 0, counts.ctypes.data_as(_i64p), *([None] * 7))
        if st != OK:
            raise FelisError(st, _lib.felis_config_error().decode())
        return counts

    def load_beam_device(self, species: int = 0, seed: int = 0, device: int = 0) -> dict:
        """load_beam with the per-beamlet work on the GPU: x .. gamma as torch
        CUDA tensors (float64), offsets and weights as host arrays."""
        import torch

        S = self.params.slice_n
        counts = np.zeros(S, dtype=np.int64)
        st = _lib.felis_config_load_beam_device(self._h, species, seed, counts.ctypes.data_as(_i64p), *([None] * 7))
        if st != OK:
            raise FelisError(st, _lib.felis_config_error().decode())
        n = int(counts.sum())
        dev = torch.device("cuda", device)
        arrs = {k: torch.empty(max(n, 1), dtype=torch.float64, device=dev)[:n]
                for k in ("x", "y", "px", "py", "theta", "gamma")}
        w = np.zeros(S)
        with torch.cuda.device(dev):
            st = _lib.felis_config_load_beam_device(
                self._h, species, seed, counts.ctypes.data_as(_i64p),
                *(C.cast(C.c_void_p(arrs[k].data_ptr()), _dp) for k in ("x", "y", "px", "py", "theta", "gamma")),
                _p(w))
        if st != OK:
            raise FelisError(st, _lib.felis_config_error().decode())
        off = np.zeros(S + 1, dtype=np.int64)
        off[1:] = np.cumsum(counts)
        arrs["offsets"] = off
        arrs["weights"] = w
        return arrs

    def load_seed(self, hidx: int) -> tuple[np.ndarray, np.ndarray]:
        """Seed field of harmonic index hidx, reference layout (S+2, ny, nx) complex."""
        p = self.params
        n = (p.slice_n + 2) * p.nx * p.ny
        ux = np.zeros(2 * n)
        uy = np.zeros(2 * n)
        st = _lib.felis_config_load_seed(self._h, hidx, _p(ux), _p(uy))
        if st != OK:
            raise FelisError(st, "load_seed")
        shp = (p.slice_n + 2, p.ny, p.nx)
        return (ux[0::2] + 1j * ux[1::2]).reshape(shp), (uy[0::2] + 1j * uy[1::2]).reshape(shp)

    def wake(self, den: np.ndarray, device: bool = False) -> np.ndarray:
        """Wake energy loss per global slice from the slice charge
        (wakeField.cpp:9-50); `device` computes the wake function (when none
        is cached) and the convolution on the GPU."""
        den = _f64(den)
        out = np.zeros(self.params.global_slice_n)
        fn = _lib.felis_config_wake_device if device else _lib.felis_config_wake
        st = fn(self._h, _p(den), _p(out))
        if st != OK:
            raise FelisError(st, "wake")
        return out

    def wake_function(self) -> np.ndarray:
        """The cached wake function per global slice distance (wakeField.cpp:128-140)."""
        out = np.zeros(self.params.global_slice_n)
        st = _lib.felis_config_wake_function(self._h, _p(out))
        if st != OK:
            raise FelisError(st, "wake_function")
        return out


def _cplx_to_interleaved(a: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.complex128).ravel()
    return a.view(np.float64)


class Handle:
    """One felis_handle: the device-resident slice loop of one GPU."""

    def __init__(self, params: Params):
        h = _vp()
        st = _lib.felis_create(C.byref(params), C.byref(h))
        if st != OK:
            raise FelisError(st, "felis_create failed (see stderr)")
        self._h = h
        self.S = params.slice_n
        self.nx, self.ny = params.nx, params.ny
        self.H = params.num_harmony
        self.species = params.num_species
        self.L, self.F, self.nr = params.scl_mode, params.scf_mode, params.nr
        self.mode = params.mode
        self._counts = [0] * self.species

    def close(self):
        if getattr(self, "_h", None) and _lib is not None:  # (interpreter teardown)
            _lib.felis_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def _ck(self, st: int):
        if st != OK:
            raise FelisError(st, _lib.felis_last_error(self._h).decode())

    # ---- data in / out ----
    def upload_particles(self, species: int, x, y, px, py, theta, gamma, offsets, weights):
        """Host arrays or torch CUDA tensors (Config.load_beam_device)."""
        arrs = [_arr64(a) for a in (x, y, px, py, theta, gamma)]
        off = np.ascontiguousarray(offsets, dtype=np.int64)
        w = _f64(weights)
        self._ck(_lib.felis_upload_particles(self._h, species, *(p for _, p in arrs), off.ctypes.data_as(_i64p), _p(w)))
        self._counts[species] = int(off[-1])

    def download_particles(self, species: int = 0, out: dict | None = None) -> dict:
        """Particle state of one species.  `out` may hold the six arrays to
        fill (contiguous float64 of the particle count, e.g. pinned host
        buffers for full-speed copies); new arrays otherwise."""
        n = self._counts[species]
        keys = ("x", "y", "px", "py", "theta", "gamma")
        if out is None:
            out = {k: np.zeros(n) for k in keys}
        for k in keys:
            a = out[k]
            if a.dtype != np.float64 or a.size != n or not a.flags.c_contiguous:
                raise ValueError(f"out[{k!r}]: contiguous float64 of {n} elements expected")
        self._ck(_lib.felis_download_particles(self._h, species, *(_p(out[k]) for k in keys)))
        return out

    def upload_field(self, hidx: int, pol: int, data: np.ndarray):
        buf = _cplx_to_interleaved(data)
        self._ck(_lib.felis_upload_field(self._h, hidx, pol, _p(buf)))

    def _dl(self, fn, hidx, pol) -> np.ndarray:
        n = (self.S + 2) * self.nx * self.ny
        buf = np.zeros(2 * n)
        self._ck(fn(self._h, hidx, pol, _p(buf)))
        return (buf[0::2] + 1j * buf[1::2]).reshape(self.S + 2, self.ny, self.nx)

    def download_field(self, hidx: int, pol: int) -> np.ndarray:
        return self._dl(_lib.felis_download_field, hidx, pol)

    def download_source(self, hidx: int, pol: int) -> np.ndarray:
        return self._dl(_lib.felis_download_source, hidx, pol)

    def download_ez(self) -> np.ndarray:
        n = self.L * (self.S + 2) * self.F * self.nr
        buf = np.zeros(2 * n)
        self._ck(_lib.felis_download_ez(self._h, _p(buf)))
        return (buf[0::2] + 1j * buf[1::2]).reshape(self.L, self.S + 2, self.F, self.nr)

    # ---- lattice ----
    def update_lattice(self, it: int, half: float):
        self._ck(_lib.felis_update_lattice(self._h, it, half))

    def lattice(self) -> Lattice:
        l = Lattice()
        self._ck(_lib.felis_get_lattice(self._h, C.byref(l)))
        return l

    def set_lattice(self, l: Lattice):
        self._ck(_lib.felis_set_lattice(self._h, C.byref(l)))

    # ---- per-step functions (main.cpp:117-149) ----
    def total_energy(self, it: int = 0) -> np.ndarray:
        out = np.zeros(2 * self.H)
        self._ck(_lib.felis_update_total_energy(self._h, it, _p(out)))
        return out

    def twiss(self, it: int = 0) -> np.ndarray:
        out = np.zeros(6 * self.species)
        self._ck(_lib.felis_twiss(self._h, it, _p(out)))
        return out

    def bfactor(self, it: int = 0) -> np.ndarray:
        out = np.zeros(2 * self.H)
        self._ck(_lib.felis_bfactor(self._h, it, _p(out)))
        return out

    def solve_field(self, it: int = 0):
        self._ck(_lib.felis_solve_field(self._h, it))

    def transverse_push(self, it: int = 0):
        self._ck(_lib.felis_transverse_push(self._h, it))

    def push_theta_gamma(self, it: int = 0):
        self._ck(_lib.felis_push_theta_gamma(self._h, it))

    def drift_theta_gamma(self, it: int = 0):
        self._ck(_lib.felis_drift_theta_gamma(self._h, it))

    def phase_shift(self, it: int = 0):
        self._ck(_lib.felis_phase_shift(self._h, it))

    def periodic_particles(self, it: int = 0):
        self._ck(_lib.felis_periodic_particles(self._h, it))

    def shift_field(self, it: int = 0):
        self._ck(_lib.felis_shift_field(self._h, it))

    def step(self, it: int):
        self._ck(_lib.felis_step(self._h, it))

    def run(self, it0: int, it1: int):
        self._ck(_lib.felis_run(self._h, it0, it1))

    def diagnostics(self, it0: int, it1: int):
        n = it1 - it0
        e = np.zeros(n * 2 * self.H)
        t = np.zeros(n * 6 * self.species)
        b = np.zeros(n * 2 * self.H)
        self._ck(_lib.felis_get_diagnostics(self._h, it0, it1, _p(e), _p(t), _p(b)))
        return e.reshape(n, 2 * self.H), t.reshape(n, 6 * self.species), b.reshape(n, 2 * self.H)

    def set_slice_exchange(self, enable: bool):
        self._ck(_lib.felis_set_slice_exchange(self._h, 1 if enable else 0))

    def first_planes(self) -> np.ndarray:
        """[H][2][ny][nx] complex planes of the block's first slice."""
        buf = np.zeros(2 * self.H * 2 * self.nx * self.ny)
        self._ck(_lib.felis_get_first_planes(self._h, _p(buf)))
        return (buf[0::2] + 1j * buf[1::2]).reshape(self.H, 2, self.ny, self.nx)

    def first_planes_device(self) -> list[int]:
        """Device addresses of the first slice's 2 H planes ([h][pol] order,
        ny*nx complex128 each), valid until the next shift."""
        ptrs = (_vp * (2 * self.H))()
        self._ck(_lib.felis_first_planes_device(self._h, ptrs))
        return [int(p) for p in ptrs]

    def stream(self) -> int:
        """The cudaStream_t the handle queues its work on."""
        s = _vp()
        self._ck(_lib.felis_get_stream(self._h, C.byref(s)))
        return int(s.value or 0)

    def set_first_planes(self, planes: np.ndarray):
        buf = _cplx_to_interleaved(planes)
        self._ck(_lib.felis_set_first_planes(self._h, _p(buf)))

    def diagnostic_sums(self, it: int = 0) -> np.ndarray:
        out = np.zeros(7 * self.species + 2 * self.H + 1)
        self._ck(_lib.felis_diagnostic_sums(self._h, it, _p(out)))
        return out

    def edge_deposit_count(self) -> int:
        c = C.c_int64(0)
        self._ck(_lib.felis_edge_deposit_count(self._h, C.byref(c)))
        return c.value

    def sync(self):
        self._ck(_lib.felis_sync(self._h))

    def profile(self, enable: bool, max_launches: int = 0):
        self._ck(_lib.felis_profile(self._h, 1 if enable else 0, max_launches))

    def kernel_stats(self, kind: int = -1) -> tuple[int, float]:
        n = C.c_int64(0)
        ms = C.c_double(0)
        self._ck(_lib.felis_kernel_stats(self._h, kind, C.byref(n), C.byref(ms)))
        return n.value, ms.value

    def last_run_ms(self) -> float:
        ms = C.c_double(0)
        self._ck(_lib.felis_last_run_ms(self._h, C.byref(ms)))
        return ms.value

    def run_loop(self, it0: int, it1: int):
        """The drop-in sequence of main.cpp:117-155 through the per-function calls."""
        for it in range(it0, it1):
            self.total_energy(it)
            self.twiss(it)
            self.bfactor(it)
            self.solve_field(it)
            self.update_lattice(it, 0.0)
            self.transverse_push(it)
            self.update_lattice(it, 0.5)
            self.transverse_push(it)
            lat = self.lattice()
            if not lat.drift_flag:
                self.push_theta_gamma(it)
            else:
                self.drift_theta_gamma(it)
            self.phase_shift(it)
            self.periodic_particles(it)
            if not lat.drift_flag and self.mode == TIME_DEPENDENT:
                self.shift_field(it)


class Batch:
    """One felis_batch: an ensemble of independent runs in mixed precision
    (FP32 particles, field and ADI; FP64 theta, lattice and sums)."""

    def __init__(self, params: list):
        arr = (C.POINTER(Params) * len(params))(*[C.pointer(p) for p in params])
        b = _vp()
        st = _lib.felis_batch_create(arr, len(params), C.byref(b))
        if st != OK:
            raise FelisError(st, "felis_batch_create failed (see stderr)")
        self._b = b
        self.n = len(params)
        self.S = [p.slice_n for p in params]
        self.nx = [p.nx for p in params]
        self.ny = [p.ny for p in params]
        self.H = [p.num_harmony for p in params]
        self._counts = [0] * self.n

    def close(self):
        if getattr(self, "_b", None) and _lib is not None:  # (interpreter teardown)
            _lib.felis_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        self.close()

    def _ck(self, st: int):
        if st != OK:
            raise FelisError(st, _lib.felis_batch_last_error(self._b).decode())

    def upload_particles(self, inst: int, x, y, px, py, theta, gamma, offsets, weights):
        """Host arrays or torch CUDA tensors (Config.load_beam_device)."""
        arrs = [_arr64(a) for a in (x, y, px, py, theta, gamma)]
        off = np.ascontiguousarray(offsets, dtype=np.int64)
        w = _f64(weights)
        self._ck(_lib.felis_batch_upload_particles(self._b, inst, *(p for _, p in arrs),
                                                   off.ctypes.data_as(_i64p), _p(w)))
        self._counts[inst] = int(off[-1])

    def download_particles(self, inst: int, out: dict | None = None) -> dict:
        """Particle state of one instance (FP64).  `out` may hold the six
        arrays to fill (contiguous float64 of the particle count, e.g. pinned
        host buffers for full-speed copies); new arrays otherwise."""
        n = self._counts[inst]
        keys = ("x", "y", "px", "py", "theta", "gamma")
        if out is None:
            out = {k: np.zeros(n) for k in keys}
        for k in keys:
            a = out[k]
            if a.dtype != np.float64 or a.size != n or not a.flags.c_contiguous:
                raise ValueError(f"out[{k!r}]: contiguous float64 of {n} elements expected")
        self._ck(_lib.felis_batch_download_particles(self._b, inst, *(_p(out[k]) for k in keys)))
        return out

    def upload_field(self, inst: int, hidx: int, pol: int, data: np.ndarray):
        buf = _cplx_to_interleaved(data)
        self._ck(_lib.felis_batch_upload_field(self._b, inst, hidx, pol, _p(buf)))

    def download_field(self, inst: int, hidx: int, pol: int) -> np.ndarray:
        S, nx, ny = self.S[inst], self.nx[inst], self.ny[inst]
        buf = np.zeros(2 * (S + 2) * nx * ny)
        self._ck(_lib.felis_batch_download_field(self._b, inst, hidx, pol, _p(buf)))
        return (buf[0::2] + 1j * buf[1::2]).reshape(S + 2, ny, nx)

    def run(self, it0: int, it1: int):
        self._ck(_lib.felis_batch_run(self._b, it0, it1))

    def diagnostics(self, inst: int, it0: int, it1: int):
        n, H = it1 - it0, self.H[inst]
        e = np.zeros(n * 2 * H)
        t = np.zeros(n * 6)
        b = np.zeros(n * 2 * H)
        self._ck(_lib.felis_batch_get_diagnostics(self._b, inst, it0, it1, _p(e), _p(t), _p(b)))
        return e.reshape(n, 2 * H), t.reshape(n, 6), b.reshape(n, 2 * H)

    def spectral_moments(self, hidx: int = 0) -> np.ndarray:
        """[n, 3]: sum |U|^2, Re and Im of sum conj(U_s) U_{s+1} per instance
        (felis_batch_spectral_moments)."""
        out = np.zeros(3 * self.n)
        self._ck(_lib.felis_batch_spectral_moments(self._b, hidx, _p(out)))
        return out.reshape(self.n, 3)

    def set_launch(self, push_box: int, adi_ctas: int):
        """Launch shape: source cells the push stages in shared memory (512 ..
        6144; 3072 lets seven one-harmonic CTAs share an SM) and ADI CTAs per
        SM (1 or 2).  Results do not depend on it."""
        self._ck(_lib.felis_batch_set_launch(self._b, push_box, adi_ctas))

    def launch(self) -> tuple[int, int]:
        """(push_box cells, adi_ctas)."""
        t, c = C.c_int32(), C.c_int32()
        self._ck(_lib.felis_batch_get_launch(self._b, C.byref(t), C.byref(c)))
        return t.value, c.value

    def tune(self, it0: int, steps: int) -> int:
        nxt = C.c_int32(0)
        self._ck(_lib.felis_batch_tune(self._b, it0, steps, C.byref(nxt)))
        return nxt.value

    def last_run_ms(self) -> float:
        ms = C.c_double(0)
        self._ck(_lib.felis_batch_last_run_ms(self._b, C.byref(ms)))
        return ms.value

    def profile(self, enable: bool, max_launches: int = 0):
        self._ck(_lib.felis_batch_profile(self._b, 1 if enable else 0, max_launches))

    def kernel_stats(self, kind: int = -1) -> tuple[int, float]:
        n = C.c_int64(0)
        ms = C.c_double(0)
        self._ck(_lib.felis_batch_kernel_stats(self._b, kind, C.byref(n), C.byref(ms)))
        return n.value, ms.value


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


def _pf(a: np.ndarray):
    return a.ctypes.data_as(_fp)


class MLP:
    """felis_mlp: the taper-surrogate network (4 linear layers, GELU, BF16
    tensor-core forward and backward, FP32 AdamW)."""

    def __init__(self, n_in: int, width: int, n_out: int, seed: int = 1):
        h = _vp()
        st = _lib.felis_mlp_create(n_in, width, n_out, seed, C.byref(h))
        if st != OK:
            raise FelisError(st, "felis_mlp_create failed (see stderr)")
        self._m = h
        self.n_in, self.width, self.n_out = n_in, width, n_out
        c = C.c_int64(0)
        _lib.felis_mlp_param_count(h, C.byref(c))
        self.n_params = c.value

    def close(self):
        if getattr(self, "_m", None) and _lib is not None:  # (interpreter teardown)
            _lib.felis_mlp_destroy(self._m)
            self._m = None

    def __del__(self):
        self.close()

    def _ck(self, st: int):
        if st != OK:
            raise FelisError(st, _lib.felis_mlp_last_error(self._m).decode())

    def params(self) -> np.ndarray:
        out = np.zeros(self.n_params, dtype=np.float32)
        self._ck(_lib.felis_mlp_get_params(self._m, _pf(out)))
        return out

    def set_params(self, p):
        p = _f32(p)
        assert p.size == self.n_params
        self._ck(_lib.felis_mlp_set_params(self._m, _pf(p)))

    def unflatten(self, p: np.ndarray) -> list:
        """[(W1, b1), ..., (W4, b4)] views of a flat parameter vector."""
        dims = [(self.width, self.n_in), (self.width, self.width), (self.width, self.width), (self.n_out, self.width)]
        out, k = [], 0
        for r, c in dims:
            W = p[k:k + r * c].reshape(r, c)
            k += r * c
            b = p[k:k + r]
            k += r
            out.append((W, b))
        return out

    def last_forward(self) -> tuple[float, float]:
        """(device ms, FLOPs) of the GEMM chain of the last forward chunk."""
        ms, fl = C.c_double(), C.c_double()
        self._ck(_lib.felis_mlp_last_forward(self._m, C.byref(ms), C.byref(fl)))
        return ms.value, fl.value

    def set_fused(self, enable: bool):
        """Inference by the fused four-layer kernel (the default where the
        shape allows it) or by the layer-by-layer GEMM chain."""
        self._ck(_lib.felis_mlp_set_fused(self._m, 1 if enable else 0))

    def forward(self, x) -> np.ndarray:
        x = _f32(x).reshape(-1, self.n_in)
        y = np.zeros((x.shape[0], self.n_out), dtype=np.float32)
        self._ck(_lib.felis_mlp_forward(self._m, _pf(x), x.shape[0], _pf(y)))
        return y

    def gradients(self, x, t) -> tuple[np.ndarray, float]:
        x = _f32(x).reshape(-1, self.n_in)
        t = _f32(t).reshape(-1, self.n_out)
        g = np.zeros(self.n_params, dtype=np.float32)
        loss = C.c_double(0)
        self._ck(_lib.felis_mlp_gradients(self._m, _pf(x), _pf(t), x.shape[0], _pf(g), C.byref(loss)))
        return g, loss.value

    def set_data(self, x, t):
        x = _f32(x).reshape(-1, self.n_in)
        t = _f32(t).reshape(-1, self.n_out)
        self._ck(_lib.felis_mlp_set_data(self._m, _pf(x), _pf(t), x.shape[0]))

    def train(self, epochs: int, batch: int = 512, lr: float = 1e-3, weight_decay: float = 1e-4,
              seed: int = 1) -> np.ndarray:
        hist = np.zeros(epochs)
        self._ck(_lib.felis_mlp_train(self._m, epochs, batch, lr, weight_decay, seed, _p(hist)))
        return hist


def wait_selftest(limit: int = 1000) -> int:
    """The library's bounded device wait on a barrier phase that nothing
    completes (felis_wait_selftest): returns the status (FELIS_TIMEOUT when
    the wait gave up as designed)."""
    out = C.c_int32(0)
    return _lib.felis_wait_selftest(limit, C.byref(out))


def device_info() -> tuple[str, int]:
    name = C.create_string_buffer(256)
    sm = C.c_int32(0)
    st = _lib.felis_device_info(name, 256, C.byref(sm))
    if st != OK:
        raise FelisError(st, "no CUDA device")
    return name.value.decode(), sm.value


def sort_by_slice(keys: np.ndarray) -> np.ndarray:
    """Stable GPU sort of slice keys; returns the permutation (felis_sort_by_slice)."""
    k = np.ascontiguousarray(keys, dtype=np.int32)
    perm = np.zeros(len(k), dtype=np.int64)
    st = _lib.felis_sort_by_slice(k.ctypes.data_as(_i32p), len(k), perm.ctypes.data_as(_i64p))
    if st != OK:
        raise FelisError(st, "felis_sort_by_slice")
    return perm


SORT_NOALLOC_MAX_KEYS = 262144


def sort_by_slice_noalloc(keys_dev_ptr: int, n: int, perm_dev_ptr: int, stream: int = 0) -> int:
    """felis_sort_by_slice_noalloc on caller-owned device buffers (raw
    pointers); queued on `stream`, returns the status without waiting."""
    return _lib.felis_sort_by_slice_noalloc(keys_dev_ptr, n, perm_dev_ptr, stream or None)


def detmath_sincos(x: float) -> tuple[float, float]:
    s, c = C.c_double(), C.c_double()
    _lib.felis_detmath_sincos(x, C.byref(s), C.byref(c))
    return s.value, c.value


def detmath_atan(x: float) -> float:
    return _lib.felis_detmath_atan(x)


def detmath_atan2(y: float, x: float) -> float:
    return _lib.felis_detmath_atan2(y, x)


def library_symbols() -> list[str]:
    """Names of every entry point declared in include/felis_b200.h."""
    import re

    hdr = os.path.join(os.path.dirname(_HERE), "include", "felis_b200.h")
    with open(hdr) as f:
        text = f.read()
    return sorted(set(re.findall(r"\b(felis_[a-z0-9_]+)\s*\(", text)))
