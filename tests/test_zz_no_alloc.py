"""The allocation-free adjoint (rihvr_adjoint_noalloc) against the context
adjoint (rihvr_adjoint), through the C ABI.

rihvr_adjoint_noalloc is for callers that cannot allocate device memory
(plugin hosts that own all device memory through their own pool, real-time
loops that cannot take an allocation's latency): it takes caller-owned device
buffers and keeps its scratch in a fixed device array that all calls share.
Two calls in a row with different residuals check that the shared scratch
carries nothing over from one call to the next.  This file is
collected last so that a run stopping at the first failure has run everything
else already; it also passes when run alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_F32 = 1e-4


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def params(rihvr, nz):
    p = rihvr.default_params()
    p.start_plane, p.plane_stepsize, p.num_planes = 150.0, 25.0, nz
    p.wavelength, p.resolution = 0.632, 1.5
    p.zero_padding = 0
    return p


def free_device_bytes():
    """cudaMemGetInfo's free bytes on the current device (the driver's view,
    which includes allocations made outside torch's caching allocator)."""
    import torch

    torch.cuda.synchronize()
    return torch.cuda.mem_get_info()[0]


# side 512 holds 4 planes a chunk of the fixed intermediate region, so 5 planes
# exercise a full chunk followed by a partial one (plane offsets of the output)
@pytest.mark.parametrize("side,nz", [(64, 5), (512, 5), (1024, 3)])
def test_adjoint_noalloc_matches_context_adjoint(rihvr, side, nz):
    import torch

    p = params(rihvr, nz)
    rng = np.random.default_rng(side * 7 + nz)
    r1 = rng.standard_normal((side, side)).astype(np.float32)
    r2 = rng.standard_normal((side, side)).astype(np.float32)
    with rihvr.SparseCompressiveHolo(p, side, side) as s:
        ref1 = s.adjoint(r1)
        ref2 = s.adjoint(r2)
    dev = torch.device("cuda", 0)
    d_r = torch.empty((side, side), dtype=torch.float32, device=dev)
    d_out = torch.empty((nz, side, side, 2), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def call(r):
        d_r.copy_(torch.from_numpy(r))
        d_out.fill_(float("nan"))  # stale output must not survive
        rihvr.adjoint_noalloc(p, side, side, d_r.data_ptr(), d_out.data_ptr(), stream.cuda_stream)
        torch.cuda.synchronize(dev)
        return d_out.cpu().numpy().view(np.complex64)[..., 0]

    # one untimed pass first, so that loading modules (ours and torch's fill
    # kernel) is not mistaken for an allocation by the calls under test
    call(r2)
    free_before = free_device_bytes()
    for r, ref in ((r1, ref1), (r2, ref2)):
        got = call(r)
        assert got.shape == ref.shape
        assert np.all(np.isfinite(got))
        assert rel(got, ref) < TOL_F32
    assert free_device_bytes() == free_before  # the calls allocated nothing


def test_adjoint_noalloc_rejects_sizes_beyond_its_limits(rihvr):
    L = rihvr.load_library()
    p = params(rihvr, 4)
    dummy = ctypes.c_void_p(16)  # never dereferenced: sizes are checked first
    assert L.rihvr_adjoint_noalloc(ctypes.byref(p), 2048, 2048, dummy, dummy, None) == rihvr.ERR_UNSUPPORTED_SIZE
    assert b"1024" in L.rihvr_last_error()
    p.num_planes = 5000
    assert L.rihvr_adjoint_noalloc(ctypes.byref(p), 64, 64, dummy, dummy, None) == rihvr.ERR_UNSUPPORTED_SIZE
    assert b"num_planes" in L.rihvr_last_error()
    p.num_planes = 4
    assert L.rihvr_adjoint_noalloc(ctypes.byref(p), 64, 48, dummy, dummy, None) == rihvr.ERR_UNSUPPORTED_SIZE
    assert b"square" in L.rihvr_last_error()
