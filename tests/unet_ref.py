"""FP64 numpy restatement of the warm-start 3-D U-Net (forward and backward),
the CPU reference for the GPU kernels' outputs and gradients.

Same architecture and parameter layout as the library's network
(``rihvr_unet_get_params``): for each of the ten 3x3x3 convolutions the
weights [cout][27][cin] (tap k = (dz+1)*9 + (dy+1)*3 + (dx+1)) then the bias
[cout]; then the head's 16 weights, its bias and alpha.  Activations are
channels-last [z][y][x][c]; the input has 16 channels, channel 0 = |xbp| /
rms(|xbp|).
"""
import numpy as np

LAYERS = [(16, 16, 0), (16, 16, 0), (16, 32, 1), (32, 32, 1), (32, 64, 2), (64, 64, 2),
          (96, 32, 1), (32, 32, 1), (48, 16, 0), (16, 16, 0)]  # (cin, cout, level)


def unpack(params):
    p = np.asarray(params, np.float64)
    off = 0
    Ws, bs = [], []
    for cin, cout, _ in LAYERS:
        n = cout * 27 * cin
        Ws.append(p[off:off + n].reshape(cout, 27, cin))
        off += n
        bs.append(p[off:off + cout])
        off += cout
    head = p[off:off + 18]
    return Ws, bs, head, off + 18


def bf16(a):
    """Round to the nearest BF16 value (ties to even), returned as float64: the
    rounding the tensor-core convolutions apply to their operands."""
    f = np.asarray(a, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


ROUND = {"on": False}  # round convolution operands to BF16 (set by emulate_bf16)


def emulate_bf16(on: bool):
    ROUND["on"] = bool(on)


def _r(a):
    return bf16(a) if ROUND["on"] else a


def offsets():
    return [(k // 9 - 1, (k // 3) % 3 - 1, k % 3 - 1) for k in range(27)]


def _shift(Xp, dz, dy, dx, D, H, W):
    return Xp[1 + dz:1 + dz + D, 1 + dy:1 + dy + H, 1 + dx:1 + dx + W]


def conv_fwd(X, Wt, b):
    D, H, W, _ = X.shape
    X, Wt = _r(X), _r(Wt)
    Xp = np.pad(X, ((1, 1), (1, 1), (1, 1), (0, 0)))
    Y = np.zeros((D, H, W, Wt.shape[0]))
    for k, (dz, dy, dx) in enumerate(offsets()):
        Y += _shift(Xp, dz, dy, dx, D, H, W) @ Wt[:, k, :].T
    return Y + b


def conv_back(X, Wt, dY):
    """Gradients of Y = conv(X) + b: (dX, dW, db)."""
    D, H, W, cin = X.shape
    db = dY.reshape(-1, Wt.shape[0]).sum(0)
    X, Wt, dY = _r(X), _r(Wt), _r(dY)
    Xp = np.pad(X, ((1, 1), (1, 1), (1, 1), (0, 0)))
    dYp = np.pad(dY, ((1, 1), (1, 1), (1, 1), (0, 0)))
    dW = np.zeros_like(Wt)
    dX = np.zeros_like(X)
    for k, (dz, dy, dx) in enumerate(offsets()):
        dW[:, k, :] = dY.reshape(-1, Wt.shape[0]).T @ _shift(Xp, dz, dy, dx, D, H, W).reshape(-1, cin)
        dX += _shift(dYp, -dz, -dy, -dx, D, H, W) @ Wt[:, k, :]
    return dX, dW, db


def pool(X):
    D, H, W, C = X.shape
    return X.reshape(D // 2, 2, H // 2, 2, W // 2, 2, C).mean(axis=(1, 3, 5))


def pool_back(dY):
    return np.repeat(np.repeat(np.repeat(dY, 2, 0), 2, 1), 2, 2) / 8.0


def up(X):
    return np.repeat(np.repeat(np.repeat(X, 2, 0), 2, 1), 2, 2)


def up_back(dY):
    D, H, W, C = dY.shape
    return dY.reshape(D // 2, 2, H // 2, 2, W // 2, 2, C).sum(axis=(1, 3, 5))


def net_input(xbp):
    a = np.abs(xbp)
    rms = np.sqrt(np.mean(a * a))
    X = np.zeros(xbp.shape + (16,))
    X[..., 0] = a / rms
    return X


def forward(params, xbp, store_bf16=False):
    """x0 and the intermediate tensors.  `store_bf16` models the inference
    path with BF16 activations: every stored activation (input, layer
    outputs but the last, pooled tensors) is rounded to BF16; the pools
    average the rounded values."""
    Ws, bs, head, _ = unpack(params)
    c = {}
    relu = lambda z: np.maximum(z, 0.0)
    st = bf16 if store_bf16 else (lambda v: v)
    c["in"] = st(net_input(xbp))
    a = [None] * 10
    a[0] = st(relu(conv_fwd(c["in"], Ws[0], bs[0])))
    a[1] = st(relu(conv_fwd(a[0], Ws[1], bs[1])))
    c["p1"] = st(pool(a[1]))
    a[2] = st(relu(conv_fwd(c["p1"], Ws[2], bs[2])))
    a[3] = st(relu(conv_fwd(a[2], Ws[3], bs[3])))
    c["p2"] = st(pool(a[3]))
    a[4] = st(relu(conv_fwd(c["p2"], Ws[4], bs[4])))
    a[5] = st(relu(conv_fwd(a[4], Ws[5], bs[5])))
    c["c2"] = np.concatenate([up(a[5]), a[3]], axis=-1)
    a[6] = st(relu(conv_fwd(c["c2"], Ws[6], bs[6])))
    a[7] = st(relu(conv_fwd(a[6], Ws[7], bs[7])))
    c["c1"] = np.concatenate([up(a[7]), a[1]], axis=-1)
    a[8] = st(relu(conv_fwd(c["c1"], Ws[8], bs[8])))
    a[9] = relu(conv_fwd(a[8], Ws[9], bs[9]))
    z = a[9] @ head[:16] + head[16]
    g = 1.0 / (1.0 + np.exp(-z))
    x0 = g * head[17] * xbp
    c["a"], c["g"] = a, g
    return x0, c


def loss_and_grad(params, xbp, xstar):
    Ws, bs, head, n = unpack(params)
    x0, c = forward(params, xbp)
    a, g = c["a"], c["g"]
    S = np.sum(np.abs(xstar) ** 2)
    e = x0 - xstar
    loss = np.sum(np.abs(e) ** 2) / S
    grad = np.zeros(n)
    gW = [None] * 10
    gb = [None] * 10
    proj = (e.real * xbp.real + e.imag * xbp.imag)
    dg = 2.0 / S * head[17] * proj
    dz = dg * g * (1 - g)
    ghead = np.zeros(18)
    ghead[:16] = (dz[..., None] * a[9]).reshape(-1, 16).sum(0)
    ghead[16] = dz.sum()
    ghead[17] = np.sum(2.0 / S * g * proj)
    d = dz[..., None] * head[:16]

    def back(i, X, dY):
        dY = dY * (a[i] > 0)
        dX, gW[i], gb[i] = conv_back(X, Ws[i], dY)
        return dX

    d = back(9, a[8], d)
    dc1 = back(8, c["c1"], d)
    d7 = up_back(dc1[..., :32])
    ds1 = dc1[..., 32:]
    d = back(7, a[6], d7)
    dc2 = back(6, c["c2"], d)
    d5 = up_back(dc2[..., :64])
    ds2 = dc2[..., 64:]
    d = back(5, a[4], d5)
    dp2 = back(4, c["p2"], d)
    d3 = pool_back(dp2) + ds2
    d = back(3, a[2], d3)
    dp1 = back(2, c["p1"], d)
    d1 = pool_back(dp1) + ds1
    d = back(1, a[0], d1)
    back(0, c["in"], d)
    off = 0
    for i, (cin, cout, _) in enumerate(LAYERS):
        m = cout * 27 * cin
        grad[off:off + m] = gW[i].ravel()
        off += m
        grad[off:off + cout] = gb[i]
        off += cout
    grad[off:off + 18] = ghead
    return loss, grad


def init_params(seed):
    """A parameter vector with the library's initialisation scheme (He normal,
    only channel 0 of the first layer's input used, small head, alpha 1)."""
    rng = np.random.default_rng(seed)
    parts = []
    for i, (cin, cout, _) in enumerate(LAYERS):
        cin_real = 1 if i == 0 else cin
        W = np.zeros((cout, 27, cin))
        W[:, :, :cin_real] = rng.normal(0, np.sqrt(2.0 / (27 * cin_real)), (cout, 27, cin_real))
        parts += [W.ravel(), rng.normal(0, 0.05, cout)]
    head = np.concatenate([rng.normal(0, 0.1, 16), [0.1, 1.0]])
    return np.concatenate(parts + [head])
