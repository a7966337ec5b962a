"""cuFFT as the comparator of the hand-written FFT passes.

The forward and adjoint operators are formed a second time with cuFFT
(torch.fft, FP32 complex) and the same FP64 transfer function, and both FP32
results are measured against the FP64 oracle: the hand-written passes must be
as accurate as cuFFT on the same planes (within a small factor) and within the
FP32 tolerance."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

TOL_F32 = 1e-4


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def setup(rihvr, side, nz):
    p = rihvr.default_params()
    p.start_plane, p.plane_stepsize, p.num_planes = 100.0, 40.0, nz
    p.wavelength, p.resolution, p.zero_padding = 0.632, 2.0, 0
    op = O.OracleParams(W=side, H=side, z=rihvr.plane_list(p), dx=float(np.float32(p.resolution)),
                        lam=float(np.float32(p.wavelength)))
    c = O.phase_table(side, side, op.dx, op.lam)  # rad per unit length, FP64
    H = np.stack([np.exp(1j * np.remainder(z * c, 2 * np.pi)) for z in op.z]).astype(np.complex64)
    return p, op, H


@pytest.mark.parametrize("side,nz", [(256, 4), (384, 3), (1024, 2), (640, 2), (2304, 2)])
def test_operators_as_accurate_as_cufft(rihvr, side, nz):
    import torch

    p, op, H = setup(rihvr, side, nz)
    rng = np.random.default_rng(side + nz)
    vol = (0.05 * (rng.standard_normal((nz, side, side)) + 1j * rng.standard_normal((nz, side, side)))).astype(
        np.complex64)
    r = rng.standard_normal((side, side)).astype(np.float32)
    with rihvr.SparseCompressiveHolo(p, side, side) as s:
        d_ours = s.forward(vol)
        g_ours = s.adjoint(r)
    dev = torch.device("cuda", 0)
    Ht = torch.from_numpy(H).to(dev)
    X = torch.fft.fft2(torch.from_numpy(vol).to(dev))
    d_cufft = torch.fft.ifft2((Ht * X).sum(dim=0)).real.cpu().numpy()
    R = torch.fft.fft2(torch.from_numpy(r).to(dev).to(torch.complex64))
    g_cufft = torch.fft.ifft2(torch.conj(Ht) * R.unsqueeze(0)).cpu().numpy()
    d_orc = O.forward(op, vol.astype(np.complex128))
    g_orc = O.adjoint(op, r.astype(np.float64))
    e_fwd, e_fwd_cufft = rel(d_ours, d_orc), rel(d_cufft, d_orc)
    e_adj, e_adj_cufft = rel(g_ours, g_orc), rel(g_cufft, g_orc)
    assert e_fwd < TOL_F32 and e_adj < TOL_F32
    assert e_fwd < 4 * e_fwd_cufft + 1e-7, (e_fwd, e_fwd_cufft)
    assert e_adj < 4 * e_adj_cufft + 1e-7, (e_adj, e_adj_cufft)
