"""Host side of z-slab sharding on CPU: the slab partition, and the reducer
that sums a slab's exchange buffers over processes, run as two gloo ranks
(host-staged, as rihvr_slab_iterate calls it between the GPU passes)."""
import ctypes
import datetime
import importlib
import os

import numpy as np
import pytest

from conftest import PKG_NAME
from test_multiframe import free_port


def _slabs():
    return importlib.import_module(PKG_NAME + ".slabs")


def test_slab_bounds_tile_the_planes():
    slabs = _slabs()
    for nz in range(1, 40):
        for n in range(1, min(nz, 9) + 1):
            b = [slabs.slab_bounds(nz, n, i) for i in range(n)]
            assert b[0][0] == 0 and all(b[i][0] + b[i][1] == b[i + 1][0] for i in range(n - 1))
            assert b[-1][0] + b[-1][1] == nz
            assert max(c for _, c in b) - min(c for _, c in b) <= 1
    for bad in ((3, 4, 0), (5, 2, 2), (5, 0, 0)):
        with pytest.raises(ValueError):
            slabs.slab_bounds(*bad)


def test_reducer_reports_failures_as_status():
    slabs = _slabs()

    def boom(a):
        raise RuntimeError("no peer")

    r = slabs.SlabReducer(boom)
    a = np.ones(4, np.float64)
    assert r.struct.sum(None, a.ctypes.data, 4, slabs.DTYPE_F64, 0) == 1
    assert r.struct.host_staged == 1 and "no peer" in r.errors[-1]
    # device data to a host-only reducer is an error, not a crash
    assert r.struct.sum(None, 0, 4, slabs.DTYPE_F32, 1) == 1


def _worker(rank, world, port, out):
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import torch.distributed as dist

    slabs = importlib.import_module(PKG_NAME + ".slabs")
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        red = slabs.torch_reducer()
        # a partial spectrum (interleaved complex FP32) and the eight FP64 sums
        spec = (np.arange(16, dtype=np.float32) + 100 * rank).copy()
        sums = np.array([0.5, -1.0, 2.0, 3.0, 4.0, 5.0, 6.0, 7.0]) * (rank + 1)
        fn = red.struct.sum
        rc1 = fn(None, spec.ctypes.data, spec.size, slabs.DTYPE_F32, 0)
        rc2 = fn(None, sums.ctypes.data, sums.size, slabs.DTYPE_F64, 0)
        out.put((rank, rc1, rc2, red.struct.host_staged, spec.copy(), sums.copy()))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_gloo_ranks_sum_slab_buffers():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=120) for _ in procs), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want_spec = 2 * np.arange(16, dtype=np.float32) + 100
    want_sums = np.array([0.5, -1.0, 2.0, 3.0, 4.0, 5.0, 6.0, 7.0]) * 3
    for rank, rc1, rc2, staged, spec, sums in res:
        assert (rc1, rc2, staged) == (0, 0, 1)
        assert np.array_equal(spec, want_spec) and np.array_equal(sums, want_sums)
