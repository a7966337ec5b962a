"""The warm-start U-Net on the GPU (BF16 tensor-core convolutions, FP32
accumulation) against the FP64 numpy reference ``unet_ref.py``: the
prediction, the loss and the gradient of every layer, at the tolerances the
first test states.  Then training reduces the loss, and the warm-start entry
point of the solver equals the manual path (back-propagate, predict, set the
initial volume)."""
import numpy as np
import pytest

import unet_ref as U

pytestmark = pytest.mark.gpu


def sample(seed, shape):
    rng = np.random.default_rng(seed)
    xbp = (rng.normal(size=shape) + 1j * rng.normal(size=shape)).astype(np.complex64)
    mask = rng.random(shape) < 0.1
    xstar = (0.5 * xbp * mask + 0.01 * (rng.normal(size=shape) + 1j * rng.normal(size=shape))).astype(np.complex64)
    return xbp, xstar


def rel(a, b):
    return float(np.linalg.norm(np.ravel(a - b)) / max(np.linalg.norm(np.ravel(b)), 1e-300))


@pytest.mark.parametrize("shape", [(8, 16, 16), (4, 12, 20)])
def test_prediction_and_gradients_match_reference(rihvr, shape):
    """Against the reference with BF16-rounded convolution operands (what the
    kernels compute): 2e-3 on the prediction and loss, 1e-2 on every layer's
    gradient.  Against the exact FP64 reference: 2e-2 on the prediction and
    loss, 1e-1 on the gradients (BF16 rounding of activations and gradients
    accumulates along the backward chain; the deepest layer sits near 6e-2 on
    this small volume)."""
    params = U.init_params(7).astype(np.float32)
    xbp, xstar = sample(8, shape)
    with rihvr.UNet(*shape) as net:
        assert net.param_count() == params.size
        net.set_params(params)
        assert np.array_equal(net.params(), params)
        x0 = net.predict(xbp).cpu().numpy()
        loss, grad = net.gradients(xbp, xstar)
    p64, a64, s64 = params.astype(np.float64), xbp.astype(np.complex128), xstar.astype(np.complex128)
    for emulate, tol_x, tol_g in ((True, 2e-3, 1e-2), (False, 2e-2, 1e-1)):
        U.emulate_bf16(emulate)
        try:
            rx0, _ = U.forward(p64, a64)
            rloss, rgrad = U.loss_and_grad(p64, a64, s64)
        finally:
            U.emulate_bf16(False)
        assert rel(x0, rx0) < tol_x, (emulate, rel(x0, rx0))
        assert abs(loss - rloss) / rloss < tol_x, (emulate, loss, rloss)
        off = 0
        for i, (cin, cout, _) in enumerate(U.LAYERS):
            m = cout * 27 * cin + cout
            e = rel(grad[off:off + m], rgrad[off:off + m])
            assert e < tol_g, (emulate, i, e)
            off += m
        assert rel(grad[off:], rgrad[off:]) < tol_g, (emulate, "head")


def test_training_reduces_the_loss(rihvr):
    shape = (8, 32, 32)
    xbp, xstar = sample(9, shape)
    with rihvr.UNet(*shape, seed=1) as net:
        first = net.train_step(xbp, xstar, lr=3e-3)
        for _ in range(60):
            last = net.train_step(xbp, xstar, lr=3e-3)
    assert np.isfinite(last) and last < 0.7 * first


def test_warm_start_equals_manual_path(rihvr, synthmod, cache_dir):
    cfg = synthmod.small_config(W=64, H=64, Nz=8, seed=12)
    _, b = synthmod.make_hologram(cfg, cache_dir=cache_dir)
    p = rihvr.params_from_config(cfg)
    with rihvr.UNet(8, 64, 64, seed=2) as net, rihvr.SparseCompressiveHolo(p, 64, 64) as s:
        s.setHologram(b)
        xbp = s.backpropagate()
        x0 = net.predict(xbp).cpu().numpy()
        s.setInitialVolume(x0)
        s.iterate(5)
        manual = s.getVolume()
        s.setHologram(b)
        s.warmStart(net)
        s.iterate(5)
        direct = s.getVolume()
    assert rel(direct, manual) < 1e-4
