"""The U-Net's 5th-generation tensor-core convolutions (tcgen05.mma with
accumulators in tensor memory, layers whose width is a multiple of 128)
against the FP64 numpy reference and against the warp-level mma.sync kernels
(RIHVR_UNET_MMA=sync, in a separate process: the choice is read once per
process); and the inference path with BF16 activations (widths that are
multiples of 512: TMA-fed tcgen05 convolutions at every level, the head fused
into the last)."""
import os
import subprocess
import sys

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


def test_tcgen05_layers_match_reference(rihvr):
    """Width 128: the full-resolution layers take the tcgen05 path.  Same
    tolerances as the mma.sync kernels against the reference with BF16-rounded
    operands: 2e-3 on the prediction and loss, 1e-2 on every layer's gradient."""
    shape = (4, 8, 128)
    params = U.init_params(11).astype(np.float32)
    xbp, xstar = sample(12, shape)
    with rihvr.UNet(*shape) as net:
        net.set_params(params)
        x0 = net.predict(xbp).cpu().numpy()
        loss, grad = net.gradients(xbp, xstar)
    p64, a64, s64 = params.astype(np.float64), xbp.astype(np.complex128), xstar.astype(np.complex128)
    U.emulate_bf16(True)
    try:
        rx0, _ = U.forward(p64, a64)
        rloss, rgrad = U.loss_and_grad(p64, a64, s64)
    finally:
        U.emulate_bf16(False)
    assert rel(x0, rx0) < 2e-3
    assert abs(loss - rloss) / rloss < 2e-3
    off = 0
    for i, (cin, cout, _) in enumerate(U.LAYERS):
        m = cout * 27 * cin + cout
        assert rel(grad[off:off + m], rgrad[off:off + m]) < 1e-2, i
        off += m


_SCRIPT = """
import sys, importlib, numpy as np
sys.path.insert(0, sys.argv[1])
R = importlib.import_module(sys.argv[2])
shape = tuple(int(v) for v in sys.argv[3:6])
rng = np.random.default_rng(5)
xbp = (rng.normal(size=shape) + 1j * rng.normal(size=shape)).astype(np.complex64)
xs = (0.3 * xbp * (rng.random(shape) < 0.1)).astype(np.complex64)
with R.UNet(*shape, seed=3) as net:
    x0 = net.predict(xbp).cpu().numpy()
    loss, grad = net.gradients(xbp, xs)
np.savez(sys.argv[6], x0=x0, loss=loss, grad=grad)
"""


def test_tcgen05_matches_mma_sync(tmp_path):
    """Width 256: levels 0 and 1 on tcgen05, level 2 on mma.sync; against the
    all-mma.sync network on the same weights and input.  The BF16 operands are
    the same; only the FP32 accumulation order differs."""
    from conftest import PKG_NAME, ROOT

    script = tmp_path / "unet.py"
    script.write_text(_SCRIPT)
    out = {}
    for mode in ("tc", "sync"):
        env = dict(os.environ)
        env.pop("RIHVR_UNET_MMA", None)
        if mode == "sync":
            env["RIHVR_UNET_MMA"] = "sync"
        f = tmp_path / f"{mode}.npz"
        r = subprocess.run([sys.executable, str(script), ROOT, PKG_NAME, "8", "16", "256", str(f)], env=env,
                           capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        out[mode] = np.load(f)
    a, b = out["tc"], out["sync"]
    assert rel(a["x0"], b["x0"]) < 1e-4
    assert abs(float(a["loss"]) - float(b["loss"])) < 1e-4 * abs(float(b["loss"]))
    assert rel(a["grad"], b["grad"]) < 1e-3


def test_bf16_inference_path_matches_reference(rihvr):
    """Width 512: predict runs with BF16 activations.  Against the reference
    that rounds the stored activations as that path does (BF16 operands and
    FP32 accumulation are the only other difference: 2e-3), and against the
    FP32-activation reference (the pools then average unrounded values:
    1e-2)."""
    shape = (16, 32, 512)
    params = U.init_params(21).astype(np.float32)
    xbp, _ = sample(22, shape)
    with rihvr.UNet(*shape) as net:
        net.set_params(params)
        assert net.activation_bits() == 16
        x0 = net.predict(xbp).cpu().numpy()
        x0b = net.predict(xbp).cpu().numpy()
    assert np.array_equal(x0, x0b)  # deterministic
    p64, a64 = params.astype(np.float64), xbp.astype(np.complex128)
    U.emulate_bf16(True)
    try:
        rs, _ = U.forward(p64, a64, store_bf16=True)
        rf, _ = U.forward(p64, a64)
    finally:
        U.emulate_bf16(False)
    assert rel(x0, rs) < 2e-3
    assert rel(x0, rf) < 1e-2


def test_small_widths_keep_fp32_activations(rihvr):
    with rihvr.UNet(8, 16, 128) as net:
        assert net.activation_bits() == 32
    with rihvr.UNet(8, 16, 256) as net:
        assert net.activation_bits() == 32


_PREDICT = """
import sys, importlib, numpy as np
sys.path.insert(0, sys.argv[1])
R = importlib.import_module(sys.argv[2])
shape = tuple(int(v) for v in sys.argv[3:6])
rng = np.random.default_rng(9)
xbp = (rng.normal(size=shape) + 1j * rng.normal(size=shape)).astype(np.complex64)
with R.UNet(*shape, seed=4) as net:
    assert net.activation_bits() == 16
    x0 = net.predict(xbp).cpu().numpy()
np.save(sys.argv[6], x0)
"""


def test_z_walking_convolutions_equal_per_tile_ones(tmp_path):
    """The z-walking BF16 convolutions (a block walks z over one tile with a
    ring of three input planes; the layers with 16 input channels) issue the same MMAs
    in the same order as the per-tile kernel, so the prediction is bit-equal
    with RIHVR_UNET_ZWALK=0 (separate processes: the choice is read once).
    Depth 36 splits into ragged z-ranges, and the second level's 22 rows are
    not a multiple of its 4-row tiles."""
    from conftest import PKG_NAME, ROOT

    script = tmp_path / "predict.py"
    script.write_text(_PREDICT)
    out = {}
    for mode in ("zwalk", "tile"):
        env = dict(os.environ)
        env.pop("RIHVR_UNET_ZWALK", None)
        if mode == "tile":
            env["RIHVR_UNET_ZWALK"] = "0"
        f = tmp_path / f"{mode}.npy"
        r = subprocess.run([sys.executable, str(script), ROOT, PKG_NAME, "36", "44", "512", str(f)], env=env,
                           capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        out[mode] = np.load(f)
    assert np.all(np.isfinite(out["zwalk"]))
    assert np.array_equal(out["zwalk"].view(np.uint32), out["tile"].view(np.uint32))
