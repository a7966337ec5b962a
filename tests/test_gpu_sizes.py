"""Plane sizes outside the register-resident FFT set: any even width and height
from 16 to 4096 with prime factors 2, 3, 5 and 7 (generic Stockham passes),
rectangular planes included, against the FP64 oracle through the C ABI."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

TOL_F32 = 1e-4


def rel(a, b):
    a = np.asarray(a, np.complex128)
    b = np.asarray(b, np.complex128)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def make(rihvr, nz, **kw):
    p = rihvr.default_params()
    p.start_plane, p.plane_stepsize, p.num_planes = 100.0, 40.0, nz
    p.wavelength, p.resolution = 0.632, 2.0
    p.regularization_param, p.regularization_TV_param, p.num_tv_iterations = 0.01, 0.02, 5
    p.zero_padding = 0
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def oparams(rihvr, p, W, H):
    return O.OracleParams(W=W, H=H, z=rihvr.plane_list(p), dx=float(np.float32(p.resolution)),
                          lam=float(np.float32(p.wavelength)), l1=float(np.float32(p.regularization_param)),
                          tv=float(np.float32(p.regularization_TV_param)), n_tv=p.num_tv_iterations, mode=p.mode,
                          faithful=p.faithful, t0=p.initial_step)


SIZES = [(1280, 1280, 1), (96, 64, 3), (64, 96, 3), (48, 80, 2), (210, 100, 2), (1536, 16, 2), (2560, 2560, 1),
         (640, 512, 2)]


@pytest.mark.parametrize("W,H,nz", SIZES)
def test_forward_and_adjoint(rihvr, W, H, nz):
    p = make(rihvr, nz)
    rng = np.random.default_rng(W * 7 + H)
    vol = (0.05 * (rng.standard_normal((nz, H, W)) + 1j * rng.standard_normal((nz, H, W)))).astype(np.complex64)
    r = rng.standard_normal((H, W)).astype(np.float32)
    with rihvr.SparseCompressiveHolo(p, W, H) as s:
        d = s.forward(vol)
        g = s.adjoint(r)
    op = oparams(rihvr, p, W, H)
    assert rel(d, O.forward(op, vol.astype(np.complex128))) < TOL_F32
    assert rel(g, O.adjoint(op, r.astype(np.float64))) < TOL_F32


@pytest.mark.parametrize("W,H,nz,ntv", [(96, 64, 3, 5), (640, 128, 2, 3), (100, 210, 2, 8), (16, 16, 2, 10),
                                        (32, 16, 2, 7), (16, 48, 2, 3)])
def test_tv_prox_rectangular(rihvr, W, H, nz, ntv):
    p = make(rihvr, nz, num_tv_iterations=ntv)
    rng = np.random.default_rng(W + 3 * H)
    x = (0.05 * (rng.standard_normal((nz, H, W)) + 1j * rng.standard_normal((nz, H, W)))).astype(np.complex64)
    r = rng.standard_normal((H, W)).astype(np.float32)
    with rihvr.SparseCompressiveHolo(p, W, H) as s:
        out, sums = s.prox_step(x, r, 0.3)
    ref, rsums = O.prox_from(oparams(rihvr, p, W, H), x.astype(np.complex128), x.astype(np.complex128),
                             r.astype(np.float64), 0.3)
    assert rel(out, ref) < TOL_F32
    assert abs(sums[1] - rsums[1]) < 1e-4 * abs(rsums[1])


def test_solve_rectangular(rihvr, synthmod, cache_dir):
    cfg = synthmod.small_config(W=96, H=64, Nz=4, seed=21)
    _, b = synthmod.make_hologram(cfg, cache_dir=cache_dir)
    assert b.shape == (64, 96)
    p = rihvr.params_from_config(cfg)
    with rihvr.SparseCompressiveHolo(p, 96, 64) as s:
        s.setHologram(b)
        s.iterate(12)
        log = s.iterations()
        X = s.getVolume()
    olog, OX, _, _, _ = O.solve(oparams(rihvr, p, 96, 64), b.astype(np.float64), 12,
                                forced_bt=log["backtracks"], forced_rs=log["restarted"])
    gap = np.abs(log["f_x"] - olog["f_x"]) / np.abs(olog["f_x"])
    assert gap.max() < TOL_F32, gap
    assert rel(X, OX) < 10 * TOL_F32
