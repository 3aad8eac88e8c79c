"""Wake function and wake field on the GPU (felis_config_wake_device) against
the numpy restatement and the host entry point (wakeField.cpp:9-50, 53-159)."""
import numpy as np
import pytest

from test_wake import CTAU, COND, RADIUS, SHAPES, density, wake_config
import wake as wref

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", sorted(SHAPES))
def test_device_wake(fb, tmp_path, name):
    shape, acdc = SHAPES[name]
    host = wake_config(fb, tmp_path, shape, acdc)
    dev = wake_config(fb, tmp_path, shape, acdc)
    p = host.params
    S, dZ = p.global_slice_n, p.num_slice * p.lambda0
    den = density(S)
    we_h, we_d = host.wake(den), dev.wake(den, device=True)
    wf_h, wf_d = host.wake_function(), dev.wake_function()
    ctau = CTAU if acdc == "AC" else 0.0
    wf_ref = wref.wake_function(S, dZ, shape, acdc, RADIUS, COND, ctau)
    scale = np.abs(wf_ref).max()
    # the device integral sums in a tree, CUDA's cos/cosh/sinh round differently
    np.testing.assert_allclose(wf_d, wf_ref, rtol=1e-10, atol=1e-10 * scale)
    np.testing.assert_allclose(wf_d, wf_h, rtol=1e-11, atol=1e-11 * scale)
    np.testing.assert_allclose(we_d, we_h, rtol=1e-11, atol=1e-11 * np.abs(we_h).max())
    # the convolution itself, given the host's wake function: bit-identical
    we_hd = host.wake(den, device=True)
    assert np.array_equal(we_hd, we_h)
    # a second call reuses the cached wake function
    assert np.array_equal(dev.wake(den, device=True), we_d)
