"""Independent numpy restatement of the reconstruction iteration.

Test infrastructure: a second, vectorised implementation of the same algorithm
as ``oracle/rihvr_oracle.c`` (written against numpy.fft instead of the
oracle's own FFT) so that the C oracle's loop logic is cross-checked by code
that shares nothing with it.  Small sizes only.

References (RIHVR source tree): forward ``sparse_compressive_holo.cu:1935-2077``,
adjoint ``sparse_gradient.cu:47-165``, 2-D TV prox ``:3652-3732``, 3-D prox
``:3422-3475, 3832-4018``, objective ``:2838-2899``, line search ``:4307-4390``,
restart ``:4393-4482``, momentum ``:4484-4642``, outer loop ``:173-633``.
"""
import numpy as np


def freqs(n):
    i = np.arange(n)
    return (((i + n // 2) % n) - n // 2) / n


def phase_coeff(H, W, dx, lam):
    fy = freqs(H)[:, None]
    fx = freqs(W)[None, :]
    a = (lam / dx) ** 2 * (fx ** 2 + fy ** 2)
    s = np.sqrt(np.maximum(0.0, 1.0 - a))
    return 2 * np.pi / lam * (s - 1.0)


def forward(vol, z, c):
    S = np.zeros(vol.shape[1:], np.complex128)
    for k in range(vol.shape[0]):
        S += np.exp(1j * z[k] * c) * np.fft.fft2(vol[k])
    return np.fft.ifft2(S).real


def adjoint(r, z, c):
    R = np.fft.fft2(r)
    return np.stack([np.fft.ifft2(np.exp(-1j * zz * c) * R) for zz in z])


def shrink(v, T, faithful):
    if T <= 0:
        return v
    if faithful:
        re = np.sign(v.real) * np.maximum(np.abs(v.real) - T, 0)
        im = np.sign(v.imag) * np.maximum(np.abs(v.imag) - T, 0)
        return re + 1j * im
    a = np.abs(v)
    return np.where(a > T, v * (np.maximum(a - T, 0) / np.where(a > 0, a, 1)), 0)


def tv2d_prox(xh, mu, s, n_tv):
    """axes: (..., H, W); forward-periodic div, backward-periodic grad."""
    gx = np.zeros_like(xh)
    gy = np.zeros_like(xh)
    for it in range(n_tv + 1):
        div = np.roll(gx, -1, -1) - gx + np.roll(gy, -1, -2) - gy
        y = xh - mu * div
        if it == n_tv:
            return y
        px = gx + s * (np.roll(y, 1, -1) - y)
        py = gy + s * (np.roll(y, 1, -2) - y)
        n = np.sqrt(px.real ** 2 + px.imag ** 2 + py.real ** 2 + py.imag ** 2)
        n = np.maximum(n, 1.0)
        gx, gy = px / n, py / n


def prox(X, G, t, l1, tv, n_tv, mode, faithful):
    if tv == 0:
        mode = 5
    if mode == 5:
        return shrink(X - t * G, t * l1, faithful)
    mu = t * tv
    s = 1.0 / (12.0 * t * tv)
    if mode == 7:
        y = tv2d_prox(X - t * G, mu, s, n_tv)
        return shrink(y, t * l1, faithful) if l1 > 0 else y
    # mode 6
    x1 = shrink(X - t * G, t * l1 / 2, faithful)
    gx = np.zeros_like(x1); gy = np.zeros_like(x1); gz = np.zeros_like(x1)
    for it in range(n_tv + 1):
        div = (np.roll(gx, -1, 2) - gx + np.roll(gy, -1, 1) - gy + np.roll(gz, -1, 0) - gz)
        y = x1 - mu * div
        if it == n_tv:
            break
        gx = gx + s * (np.roll(y, 1, 2) - y)
        gy = gy + s * (np.roll(y, 1, 1) - y)
        gz = gz + s * (np.roll(y, 1, 0) - y)
    return shrink(y, t * l1 / 2, faithful)


def norms(X, mode, tv):
    if tv == 0:
        mode = 5
    l1 = np.abs(X).sum()
    if mode == 7:
        a = np.roll(X, 1, 2) - X
        b = np.roll(X, 1, 1) - X
        tvn = np.sqrt(np.abs(a) ** 2 + np.abs(b) ** 2).sum()
    elif mode == 6:
        a = np.roll(X, 1, 2) - X
        b = np.roll(X, 1, 1) - X
        c = np.roll(X, 1, 0) - X
        tvn = np.sqrt(np.abs(a) ** 2 + np.abs(b) ** 2 + np.abs(c) ** 2).sum()
    else:
        tvn = 0.0
    return l1, tvn


def restart_weights(H, W, faithful):
    i = np.arange(H * W).reshape(H, W)
    if not faithful:
        return np.ones((H, W)), np.ones((H, W))
    first = (i & 1023) < 512
    return np.where(first, 1.0, 0.0), np.where(first, 2.0, 1.0)


def solve(b, z, dx, lam, l1, tv, n_tv, mode, faithful, n_iter, max_bt=2, t0=0.0):
    Nz = len(z)
    H, W = b.shape
    c = phase_coeff(H, W, dx, lam)
    X = np.zeros((Nz, H, W), np.complex128)
    Y0 = np.zeros_like(X)
    dX = np.zeros((H, W)); dY0 = np.zeros((H, W))
    t = t0 if t0 > 0 else 1.0 / Nz
    alpha1 = 1.0
    r = dX - b
    prev = 0.5 * (r ** 2).sum()
    G = adjoint(r, z, c)
    wr, wi = restart_weights(H, W, faithful)
    log = []
    for it in range(n_iter):
        alpha0 = alpha1
        bt = 0
        while True:
            P = prox(X, G, t, l1, tv, n_tv, mode, faithful)
            dP = forward(P, z, c)
            fr = 0.5 * ((dP - b) ** 2).sum()
            D = P - X
            lim = (D.real * G.real + D.imag * G.imag).sum() + (np.abs(D) ** 2).sum() / (2 * t)
            ratio = fr / (prev + lim)
            if ((ratio > 1) or (ratio < 0)) and bt < max_bt:
                t *= 0.5
                bt += 1
                continue
            break
        a = X - P
        bb = P - Y0
        rs = (wr * a.real * bb.real + wi * a.imag * bb.imag).sum()
        restarted = rs > 0
        if restarted:
            alpha0 = 1.0
        alpha1 = (1 + np.sqrt(1 + 4 * alpha0 ** 2)) / 2
        beta = (alpha0 - 1) / alpha1
        X = P + beta * (P - Y0)
        Y0 = P
        dX = dP + beta * (dP - dY0)
        dY0 = dP
        r = dX - b
        prev = 0.5 * (r ** 2).sum()
        G = adjoint(r, z, c)
        l1x, tvx = norms(X, mode, tv)
        log.append(dict(f_resid_prox=fr, lim=lim, ratio=ratio, t=t, beta=beta,
                        f_x=prev + l1 * l1x + tv * tvx, backtracks=bt, restarted=int(restarted),
                        restart_sum=rs))
    return log, X, Y0, dX
