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


def _oracle_slab_solve(rank, world, cfg, b, n_iter, sum_fn):
    """FISTA of one z-slab with the FP64 oracle as the compute: the exchange
    rihvr_slab_iterate makes (the slab's share of the forward operator and
    the line-search and restart sums, summed over the slabs), the decisions of
    inverseReconstruct (sparse_compressive_holo.cu:299-611) on the sums."""
    import oracle as O

    slabs = _slabs()
    z0, nz = slabs.slab_bounds(cfg.num_planes, world, rank)
    z = cfg.plane_list()
    p = O.OracleParams(W=cfg.W, H=cfg.H, z=z[z0:z0 + nz], dx=cfg.dx(), lam=cfg.lam(), l1=cfg.l1(), tv=cfg.tv(),
                       n_tv=cfg.num_tv_iterations, mode=7, faithful=1, n_threads=1)
    b = b.astype(np.float64)
    X = np.zeros((nz, cfg.H, cfg.W), np.complex128)
    Y0 = np.zeros_like(X)
    dX = np.zeros_like(b)
    dY0 = np.zeros_like(b)
    r = dX - b
    prev_f = 0.5 * float(np.sum(r * r))
    t = 1.0 / cfg.num_planes  # the whole volume's first step
    alpha1 = 1.0
    log = []
    for _ in range(n_iter):
        alpha0, bt = alpha1, 0
        while True:
            P, s3 = O.prox_from(p, X, Y0, r, t)
            d = sum_fn(O.forward(p, P))  # the slab's share of A P, summed over the slabs
            s3 = sum_fn(s3)
            f_resid = 0.5 * float(np.sum((d - b) ** 2))
            lim = s3[0] + s3[1] / (2.0 * t)
            ratio = f_resid / (prev_f + lim)
            if (ratio > 1.0 or ratio < 0.0) and bt < p.max_backtracks:
                t *= 0.5
                bt += 1
                continue
            break
        restarted = s3[2] > 0.0
        if restarted:
            alpha0 = 1.0
        alpha1 = (1.0 + np.sqrt(1.0 + 4.0 * alpha0 * alpha0)) / 2.0
        beta = (alpha0 - 1.0) / alpha1
        X = P + beta * (P - Y0)
        Y0 = P
        dX = d + beta * (d - dY0)
        dY0 = d
        r = dX - b
        prev_f = 0.5 * float(np.sum(r * r))
        log.append((bt, int(restarted), f_resid, prev_f))
    return log, Y0


def _oracle_slab_worker(rank, world, port, out):
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for p in (root, os.path.join(root, "oracle"), os.path.join(root, "tests")):
        sys.path.insert(0, p)
    import torch
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        cfg, b = _tiny_case()

        def sum_fn(a):
            t = torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64).copy())
            dist.all_reduce(t)
            return t.numpy()

        out.put((rank,) + _oracle_slab_solve(rank, world, cfg, b, 8, sum_fn))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def _tiny_case():
    synth = importlib.import_module(PKG_NAME + ".synth")
    cfg = synth.small_config(W=32, H=32, Nz=7, seed=41, num_inverse_iterations=8)
    _, b = synth.make_hologram(cfg)
    return cfg, b


def test_two_gloo_ranks_solve_one_hologram_by_slabs():
    """Two ranks hold 4 and 3 of the 7 planes and exchange per attempt only
    the forward share and three sums (FP64 oracle compute, gloo sums); their
    solve is the single-process oracle solve of all planes: the same
    backtracking and restart decisions, objective terms within 1e-9 and the
    volume within 1e-9 (only the order of FP64 sums differs)."""
    import oracle as O
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_oracle_slab_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=300) for _ in procs), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, log0, P0), (_, log1, P1) = res
    assert log0 == log1  # every rank takes the same decisions on the same sums
    cfg, b = _tiny_case()
    op = O.OracleParams(W=cfg.W, H=cfg.H, z=cfg.plane_list(), dx=cfg.dx(), lam=cfg.lam(), l1=cfg.l1(), tv=cfg.tv(),
                        n_tv=cfg.num_tv_iterations, mode=7, faithful=1, n_threads=1)
    ref, _, P, _, _ = O.solve(op, b.astype(np.float64), 8)
    assert [x[0] for x in log0] == list(ref["backtracks"])
    assert [x[1] for x in log0] == list(ref["restarted"])
    assert np.allclose([x[2] for x in log0], ref["f_resid_prox"], rtol=1e-9, atol=0)
    assert np.allclose([x[3] for x in log0], ref["f_resid_x"], rtol=1e-9, atol=0)
    Ps = np.concatenate([P0, P1])
    assert Ps.shape == P.shape
    assert np.linalg.norm(Ps - P) <= 1e-9 * np.linalg.norm(P)
