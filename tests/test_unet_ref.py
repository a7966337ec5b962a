"""CPU checks of the FP64 U-Net reference (``unet_ref.py``): its analytic
gradient against central finite differences, and the parameter count against
the library's."""
import numpy as np

import unet_ref as U


def sample(seed, shape=(4, 8, 8)):
    rng = np.random.default_rng(seed)
    xbp = rng.normal(size=shape) + 1j * rng.normal(size=shape)
    xstar = 0.3 * xbp * (rng.random(shape) < 0.2) + 0.01 * (rng.normal(size=shape) + 1j * rng.normal(size=shape))
    return xbp, xstar


def test_reference_gradient_matches_finite_differences():
    params = U.init_params(3)
    xbp, xstar = sample(4)
    loss, grad = U.loss_and_grad(params, xbp, xstar)
    assert np.isfinite(loss) and loss > 0
    rng = np.random.default_rng(5)
    _, _, _, n = U.unpack(params)
    # parameters of every layer (first layer: input channel 0 only), the head and alpha
    idx = []
    off = 0
    for i, (cin, cout, _) in enumerate(U.LAYERS):
        m = cout * 27 * cin
        w = rng.integers(0, m, 3)
        if i == 0:
            w = w - (w % cin)  # channel 0
        idx += list(off + w) + [off + m + int(rng.integers(0, cout))]
        off += m + cout
    idx += [n - 18, n - 3, n - 2, n - 1]
    h = 1e-6
    for i in idx:
        p1, p2 = params.copy(), params.copy()
        p1[i] += h
        p2[i] -= h
        fd = (U.loss_and_grad(p1, xbp, xstar)[0] - U.loss_and_grad(p2, xbp, xstar)[0]) / (2 * h)
        assert abs(fd - grad[i]) <= 1e-5 * max(1e-3, abs(fd)), (i, fd, grad[i])


def test_parameter_count_matches_library(rihvr):
    """The reference's layout has 359 762 parameters; the library's count for
    a live network is checked against it on the GPU (test_gpu_unet.py).  On
    the CPU, a NULL network has none."""
    _, _, _, n = U.unpack(np.zeros(10 ** 6))
    assert n == 359762
    L = rihvr.load_library()
    assert L.rihvr_unet_param_count(None) == 0
