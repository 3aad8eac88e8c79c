"""Taper-surrogate network (felis_mlp_*) against a CPU computation of the same
network.

The GPU computes with BF16 weights and activations on the tensor cores and
accumulates in FP32; its GELU (tanh form) uses the hardware tanh.  The CPU
side (numpy, FP64, exact tanh) rounds to BF16 at the same places -- inputs,
weights, hidden activations, and the backward operands dz -- so the forward
outputs agree up to the BF16 roundings that accumulation order and the
hardware tanh flip, and the gradients to a few BF16 ulps in norm.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N_IN, WIDTH, N_OUT = 38, 256, 33
FWD_ATOL = 3e-3      # forward, relative to the largest |output| (BF16 roundings flipped by
                     # accumulation order and by the hardware tanh's ~2^-11 error)
GRAD_RTOL = 1e-2     # gradient blocks, relative in norm


def bf16(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


GELU_C, GELU_A = np.sqrt(2.0 / np.pi), 0.044715


def gelu(z):
    """The network's GELU, tanh form."""
    return 0.5 * z * (1.0 + np.tanh(GELU_C * (z + GELU_A * z ** 3)))


def gelu_grad(z):
    t = np.tanh(GELU_C * (z + GELU_A * z ** 3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * GELU_C * (1.0 + 3.0 * GELU_A * z * z)


def cpu_forward(layers, x):
    a = bf16(x)
    zs, acts = [], [a]
    for k, (W, b) in enumerate(layers):
        z = a @ bf16(W).T + b.astype(np.float64)
        zs.append(z)
        if k < len(layers) - 1:
            a = bf16(gelu(z))
            acts.append(a)
    return zs, acts


def cpu_gradients(layers, x, t):
    zs, acts = cpu_forward(layers, x)
    n, n_out = t.shape
    y = zs[-1]
    loss = np.mean((y - t) ** 2)
    dz = bf16(2.0 / (n * n_out) * (y - t))
    grads = [None] * len(layers)
    for k in range(len(layers) - 1, -1, -1):
        W, _ = layers[k]
        gW = dz.T @ acts[k]
        gb = dz.sum(axis=0)
        grads[k] = (gW, gb)
        if k == 0:
            break
        da = dz @ bf16(W)
        dz = bf16(da * gelu_grad(zs[k - 1]))
    return grads, loss, y


def random_params(m, rng, scale=1.0):
    p = []
    for (W, b) in m.unflatten(np.zeros(m.n_params, dtype=np.float32)):
        fan_in = W.shape[1]
        p.append(rng.normal(0, scale * np.sqrt(2.0 / fan_in), W.shape).ravel())
        p.append(rng.normal(0, 0.1, b.shape))
    return np.concatenate(p).astype(np.float32)


@pytest.fixture
def net(fb):
    m = fb.MLP(N_IN, WIDTH, N_OUT, seed=3)
    yield m
    m.close()


def test_forward_matches_cpu(net):
    rng = np.random.default_rng(11)
    p = random_params(net, rng)
    net.set_params(p)
    for n in (1, 300, 1024):
        x = rng.normal(0, 1, (n, N_IN)).astype(np.float32)
        y = net.forward(x)
        zs, _ = cpu_forward(net.unflatten(p), x)
        ref = zs[-1]
        np.testing.assert_allclose(y, ref, rtol=0, atol=FWD_ATOL * np.abs(ref).max())


def test_gradients_match_cpu(net):
    rng = np.random.default_rng(12)
    p = random_params(net, rng)
    net.set_params(p)
    x = rng.normal(0, 1, (384, N_IN)).astype(np.float32)
    t = rng.normal(0, 1, (384, N_OUT)).astype(np.float32)
    g, loss = net.gradients(x, t)
    ref, ref_loss, _ = cpu_gradients(net.unflatten(p), x, t)
    np.testing.assert_allclose(loss, ref_loss, rtol=1e-3)
    for k, ((gW, gb), (rW, rb)) in enumerate(zip(net.unflatten(g), ref)):
        ew = np.linalg.norm(gW - rW) / np.linalg.norm(rW)
        eb = np.linalg.norm(gb - rb) / np.linalg.norm(rb)
        assert ew < GRAD_RTOL, (k, "W", ew)
        assert eb < GRAD_RTOL, (k, "b", eb)


def test_gradients_ragged_batch(net):
    """A batch that is not a multiple of 128: the padding rows carry no loss."""
    rng = np.random.default_rng(13)
    p = random_params(net, rng)
    net.set_params(p)
    x = rng.normal(0, 1, (200, N_IN)).astype(np.float32)
    t = rng.normal(0, 1, (200, N_OUT)).astype(np.float32)
    g, loss = net.gradients(x, t)
    ref, ref_loss, _ = cpu_gradients(net.unflatten(p), x, t)
    np.testing.assert_allclose(loss, ref_loss, rtol=1e-3)
    gW, _ = net.unflatten(g)[0]
    assert np.linalg.norm(gW - ref[0][0]) / np.linalg.norm(ref[0][0]) < GRAD_RTOL


def test_training_fits_a_smooth_map(fb):
    """AdamW on the device fits a smooth 38 -> 33 map: the loss falls by an
    order of magnitude and held-out samples follow."""
    rng = np.random.default_rng(14)
    A = rng.normal(0, 1, (N_IN, 8)) / np.sqrt(N_IN)
    B = rng.normal(0, 1, (8, N_OUT))

    def f(x):
        return np.tanh(x @ A) @ B / 2.0

    x = rng.normal(0, 1, (8192, N_IN)).astype(np.float32)
    y = f(x).astype(np.float32)
    m = fb.MLP(N_IN, WIDTH, N_OUT, seed=5)
    m.set_data(x, y)
    hist = m.train(epochs=40, batch=512, lr=1e-3, weight_decay=1e-4)
    assert hist[-1] < 0.1 * hist[0], hist
    xt = rng.normal(0, 1, (1000, N_IN)).astype(np.float32)
    err = np.mean((m.forward(xt) - f(xt)) ** 2) / np.mean(f(xt) ** 2)
    assert err < 0.1, err
    m.close()


@pytest.mark.parametrize("fused", [True, False])
def test_large_batch_forward_and_timing(net, fused):
    """200,000 rows: 1,563 tiles of 128 rows over the persistent kernels'
    CTAs, so every CTA alternates its two tensor-memory accumulators (tile
    slots) and wraps its shared-memory stage ring many times.  Rows spread
    over the batch match the CPU product; the device time of the fused kernel
    and of the layer-by-layer GEMM chain is reported."""
    rng = np.random.default_rng(15)
    p = random_params(net, rng)
    net.set_params(p)
    net.set_fused(fused)
    x = rng.normal(0, 1, (200_000, N_IN)).astype(np.float32)
    y = net.forward(x)
    ms, flops = net.last_forward()
    assert ms > 0 and flops == 2.0 * 200_064 * (WIDTH * 48 + 2 * WIDTH * WIDTH + 48 * WIDTH)
    pick = np.concatenate([np.arange(0, 200_000, 997), np.arange(199_872, 200_000)])
    zs, _ = cpu_forward(net.unflatten(p), x[pick])
    ref = zs[-1]
    np.testing.assert_allclose(y[pick], ref, rtol=0, atol=FWD_ATOL * np.abs(ref).max())
    what = "fused kernel" if fused else "GEMM chain"
    print(f"forward {what}, 200,000 rows: {ms:.3f} ms, {flops / ms / 1e9:.1f} TFLOP/s")


@pytest.mark.parametrize("rows", [1, 127, 129, 5000, 37_003])
def test_fused_inference_equals_the_layer_chain(net, rows):
    """The fused kernel rounds where the chain rounds (BF16 hidden
    activations, FP32 accumulation over the same K order, the same GELU), so
    both give the same bits, for ragged batches (the last tile padded) and
    for batches where CTAs hold an odd number of tiles."""
    rng = np.random.default_rng(rows)
    net.set_params(random_params(net, rng))
    x = rng.normal(0, 1, (rows, N_IN)).astype(np.float32)
    net.set_fused(True)
    a = net.forward(x)
    net.set_fused(False)
    b = net.forward(x)
    net.set_fused(True)
    assert np.array_equal(a, b)


def test_fused_rejects_shapes_it_does_not_cover(fb):
    m = fb.MLP(38, 128, 33, seed=1)
    with pytest.raises(fb.FelisError):
        m.set_fused(True)
    m.set_fused(False)
    m.close()
