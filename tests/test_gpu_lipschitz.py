"""FP64 Lipschitz power iteration on the device (rihvr_lipschitz) against the
same power iteration run with the FP64 oracle's operators from the same start
vector, and against the known answer L = num_planes."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def splitmix64(z):
    with np.errstate(over="ignore"):
        z = z + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def start_vector(shape, seed):
    """The device's x_0: uniform [-1, 1) from the top 24 bits of splitmix64."""
    n = int(np.prod(shape))
    i = np.arange(n, dtype=np.uint64)
    with np.errstate(over="ignore"):
        k = np.uint64(seed) * np.uint64(0x100000001B3) + np.uint64(2) * i
    def unit(r):
        return ((r >> np.uint64(40)).astype(np.float64) / 16777216.0 * 2.0 - 1.0).astype(np.float32)
    return (unit(splitmix64(k)) + 1j * unit(splitmix64(k + np.uint64(1)))).astype(np.complex64).reshape(shape)


def test_power_iteration_matches_oracle_and_known_answer(rihvr, synthmod):
    side, nz, iters, seed = 64, 6, 12, 12345
    cfg = synthmod.small_config(W=side, H=side, Nz=nz, seed=1)
    _, b = synthmod.make_hologram(cfg)
    p = rihvr.params_from_config(cfg)
    with rihvr.SparseCompressiveHolo(p, side, side) as s:
        s.setHologram(b)
        L, hist = s.estimateLipschitz(iters, seed)
        # the solve restarts from x = 0 afterwards
        s.iterate(4)
        after = s.getVolume()
    with rihvr.SparseCompressiveHolo(p, side, side) as t:
        t.setHologram(b)
        t.iterate(4)
        assert np.array_equal(t.getVolume(), after)

    op = O.OracleParams(W=side, H=side, z=rihvr.plane_list(p), dx=cfg.dx(), lam=cfg.lam(), l1=cfg.l1(),
                        tv=cfg.tv(), n_tv=cfg.num_tv_iterations, mode=7, faithful=1)
    x = start_vector((nz, side, side), seed).astype(np.complex128)
    ref = []
    for _ in range(iters):
        ax = O.forward(op, x)
        ref.append(float(np.sum(ax * ax) / np.sum(np.abs(x) ** 2)))
        y = O.adjoint(op, ax)
        x = y / np.linalg.norm(y)
    ref = np.asarray(ref)
    assert np.max(np.abs(hist - ref) / ref) < 1e-4, (hist, ref)
    assert L == hist[-1]
    # Rayleigh quotients rise towards L = num_planes and never pass it
    assert np.all(np.diff(hist) > -1e-6 * nz)
    assert hist[-1] <= nz * (1 + 1e-5)
    assert hist[-1] > hist[0]


def test_power_iteration_converges_to_num_planes(rihvr):
    """A start vector close to the top eigenvector (a volume constant in x, y
    and z is one) is not needed: from a random start the quotients approach
    num_planes within a few per cent in a few dozen steps at a small size."""
    side, nz = 32, 4
    p = rihvr.default_params()
    p.start_plane, p.plane_stepsize, p.num_planes = 100.0, 40.0, nz
    p.wavelength, p.resolution, p.zero_padding = 0.632, 2.0, 0
    with rihvr.SparseCompressiveHolo(p, side, side) as s:
        s.setHologram(np.zeros((side, side), np.float32))
        L, hist = s.estimateLipschitz(60, 7)
    assert 0.9 * nz < L <= nz * (1 + 1e-5), hist
