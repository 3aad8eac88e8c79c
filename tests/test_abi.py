"""The C ABI library: loads, exports every declared entry point, and rejects
bad calls with a status (no GPU needed)."""
import ctypes
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_every_declared_symbol_is_exported(fb):
    names = fb.library_symbols()
    assert "felis_create" in names and "felis_step" in names and "felis_sort_by_slice" in names
    lib = ctypes.CDLL(fb.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_library_links_no_torch_and_is_sm100a(fb):
    out = subprocess.run(["ldd", fb.LIB_PATH], capture_output=True, text=True).stdout
    assert "torch" not in out and "libcudart.so" not in out  # static cudart, no torch types
    src = open(os.path.join(ROOT, "felis_b200", "_build.py")).read()
    assert "arch=compute_100a,code=sm_100a" in src and "--fmad=false" in src


def test_header_compiles_as_c(tmp_path):
    c = tmp_path / "t.c"
    c.write_text('#include "felis_b200.h"\nint main(void){felis_params p; (void)p; return FELIS_OK;}\n')
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), "-c", str(c),
                        "-o", str(tmp_path / "t.o")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_bad_arguments_return_status(fb):
    lib = fb._lib
    assert lib.felis_create(None, None) == fb.BAD_ARG
    p = fb.Params()
    p.abi_version = 999
    h = ctypes.c_void_p()
    assert lib.felis_create(ctypes.byref(p), ctypes.byref(h)) == fb.BAD_ARG
    p.abi_version = fb.ABI_VERSION
    p.dimension = 2  # the reference has 1D and 3D models only
    assert lib.felis_create(ctypes.byref(p), ctypes.byref(h)) == fb.UNSUPPORTED
    p.dimension = 1  # 1D with an empty parameter set: rejected, not run
    assert lib.felis_create(ctypes.byref(p), ctypes.byref(h)) == fb.BAD_ARG
    assert lib.felis_sort_by_slice(None, -1, None) == fb.BAD_ARG


def test_no_device_is_reported_not_crashed(fb, tmp_path):
    if fb._lib.felis_device_info(None, 0, None) == fb.OK:
        pytest.skip("a CUDA device is present")
    from felis_b200 import workloads

    cfg = fb.Config(workloads.write_input(str(tmp_path / "a.inp"), kind="sase", slices=2, nx=31))
    with pytest.raises(fb.FelisError) as e:
        fb.Handle(cfg.params)
    assert e.value.status == fb.NO_DEVICE


def test_noalloc_limit_matches_the_header(fb):
    """The Python binding's copy of the allocation-free sort's key limit is the
    header's FELIS_SORT_NOALLOC_MAX_KEYS."""
    import re

    with open(os.path.join(ROOT, "include", "felis_b200.h")) as f:
        m = re.search(r"#define\s+FELIS_SORT_NOALLOC_MAX_KEYS\s+(\d+)", f.read())
    assert m and int(m.group(1)) == fb.SORT_NOALLOC_MAX_KEYS
