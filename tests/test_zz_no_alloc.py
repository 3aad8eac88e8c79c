"""The allocation-free slice sort against the allocating one.

felis_sort_by_slice_noalloc serves callers that must not allocate device
memory (their HBM belongs to another allocator, or cudaMalloc's implicit
synchronisation is not acceptable in their loop): they pass their own device
buffers and the library works in a fixed scratch array of its own.  This file
runs last so that a failure here leaves every other test already run; it
passes alone in a fresh process and after the rest of the suite.
"""
import numpy as np
import pytest

from conftest import assert_bits

pytestmark = pytest.mark.gpu


def _noalloc(fb, keys: np.ndarray) -> np.ndarray:
    import torch

    kd = torch.from_numpy(np.ascontiguousarray(keys, dtype=np.int32)).cuda()
    pd = torch.full((max(len(keys), 1),), -1, dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    st = fb.sort_by_slice_noalloc(kd.data_ptr(), len(keys), pd.data_ptr(), stream)
    assert st == fb.OK, fb.STATUS_NAMES.get(st, st)
    torch.cuda.synchronize()
    return pd[: len(keys)].cpu().numpy()


def test_noalloc_sort_matches_allocating_sort_twice(fb):
    rng = np.random.default_rng(11)
    # two calls in a row: the second reuses the scratch the first left behind
    for n, kmax in ((100_000, 1024), (fb.SORT_NOALLOC_MAX_KEYS, 50_000)):
        keys = rng.integers(0, kmax, size=n).astype(np.int32)
        assert_bits(_noalloc(fb, keys), fb.sort_by_slice(keys), f"n={n}")
    # slice-major input stays in place
    keys = np.repeat(np.arange(64, dtype=np.int32), 1000)
    assert_bits(_noalloc(fb, keys), np.arange(keys.size), "identity")


def test_noalloc_sort_limits(fb):
    import torch

    assert fb.sort_by_slice_noalloc(0, 0, 0, 0) == fb.OK
    kd = torch.zeros(fb.SORT_NOALLOC_MAX_KEYS + 1, dtype=torch.int32, device="cuda")
    pd = torch.zeros(fb.SORT_NOALLOC_MAX_KEYS + 1, dtype=torch.int64, device="cuda")
    assert fb.sort_by_slice_noalloc(kd.data_ptr(), kd.numel(), pd.data_ptr(), 0) == fb.BAD_ARG
    # host buffers are refused before anything is queued
    hk, hp = np.zeros(16, dtype=np.int32), np.zeros(16, dtype=np.int64)
    assert fb.sort_by_slice_noalloc(hk.ctypes.data, 16, hp.ctypes.data, 0) == fb.BAD_ARG
