"""Failure handling through the C ABI, with the failures made on the host: no
GPU fault, trap or hang is provoked.

* Non-finite holograms (host or device memory) are refused with
  RIHVR_ERR_INVALID_DATA, and the context keeps working afterwards.
* An injected allocation failure at every allocation of rihvr_create returns
  RIHVR_ERR_OUT_OF_MEMORY and frees everything allocated before it.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def small(rihvr, side=64, nz=4):
    p = rihvr.default_params()
    p.start_plane, p.plane_stepsize, p.num_planes = 100.0, 40.0, nz
    p.wavelength, p.resolution, p.zero_padding = 0.632, 2.0, 0
    p.regularization_param, p.regularization_TV_param, p.num_tv_iterations = 0.01, 0.02, 5
    return p


def free_bytes():
    import torch

    torch.cuda.synchronize()
    return torch.cuda.mem_get_info()[0]


@pytest.mark.parametrize("bad", [np.nan, np.inf, -np.inf])
@pytest.mark.parametrize("on_device", [False, True])
def test_non_finite_hologram_is_refused(rihvr, bad, on_device):
    import torch

    side = 64
    p = small(rihvr, side)
    rng = np.random.default_rng(0)
    good = (0.1 * rng.standard_normal((side, side))).astype(np.float32)
    poisoned = good.copy()
    poisoned[17, 33] = bad
    L = rihvr.load_library()
    with rihvr.SparseCompressiveHolo(p, side, side) as s:
        s.setHologram(good)
        s.iterate(3)
        before = s.getVolume()
        if on_device:
            d = torch.from_numpy(poisoned).cuda()
            rc = L.rihvr_set_hologram(s._h, ctypes.c_void_p(d.data_ptr()), 1)
        else:
            rc = L.rihvr_set_hologram(s._h, poisoned.ctypes.data_as(ctypes.c_void_p), 0)
        assert rc == rihvr.ERR_INVALID_DATA
        assert b"non-finite" in L.rihvr_last_error()
        # the refused call left the solve as it was
        assert np.array_equal(s.getVolume(), before)
        s.iterate(2)
        cont = s.getVolume()
    # ... and it continues exactly as an undisturbed solve of the good hologram
    with rihvr.SparseCompressiveHolo(p, side, side) as t:
        t.setHologram(good)
        t.iterate(5)
        assert np.array_equal(t.getVolume(), cont)


def test_allocation_failure_at_every_step_frees_everything(rihvr):
    L = rihvr.load_library()
    side = 128
    p = small(rihvr, side, nz=6)
    # warm the context and the module once, so that lazily created driver
    # resources do not count as leaks
    with rihvr.SparseCompressiveHolo(p, side, side):
        pass
    base = free_bytes()
    out = ctypes.c_void_p()
    failures = 0
    try:
        for n in range(200):
            L.rihvr_debug_fail_allocations_after(n)
            rc = L.rihvr_create(ctypes.byref(p), side, side, ctypes.byref(out))
            if rc == rihvr.OK:
                L.rihvr_debug_fail_allocations_after(-1)
                L.rihvr_destroy(out)
                break
            assert rc == rihvr.ERR_OUT_OF_MEMORY, (n, rc)
            assert not out.value
            failures += 1
            assert free_bytes() == base, f"allocation {n} failed and leaked device memory"
        else:
            pytest.fail("rihvr_create never succeeded")
    finally:
        L.rihvr_debug_fail_allocations_after(-1)
    assert failures >= 20  # every device and pinned allocation of the context was tried
    assert free_bytes() == base
