"""Z-slab sharding of one hologram (rihvr_create_slab, rihvr_slab_iterate):
slabs that split the planes reproduce one context over all of them, within
the FP32 order of the spectrum sum, with the same decisions; one slab of every
plane reproduces rihvr_iterate bit for bit; slabs in two processes, summed
over a process group, equal the same slabs in one process bit for bit."""
import ctypes
import importlib
import os

import numpy as np
import pytest

from conftest import PKG_NAME

pytestmark = pytest.mark.gpu


def _slabs():
    return importlib.import_module(PKG_NAME + ".slabs")


def _records_bits(rec):
    return np.ascontiguousarray(rec).tobytes()


def _solve_one(rihvr, p, W, H, b, *calls):
    with rihvr.SparseCompressiveHolo(p, W, H) as s:
        s.setHologram(b)
        for n in calls:
            s.iterate(n)
        return s.iterations(), s.getVolume()


def test_one_slab_of_every_plane_equals_iterate(rihvr, synthmod, cache_dir):
    c = synthmod.small_config(W=128, H=128, Nz=12, seed=31, num_inverse_iterations=15)
    b = synthmod.make_hologram(c, cache_dir=cache_dir)[1]
    p = rihvr.params_from_config(c)
    # each call settles its last record's x-terms with the norm kernel, so the
    # reference run makes the same two calls
    rec, X = _solve_one(rihvr, p, c.W, c.H, b, 7, 8)
    with rihvr.SparseCompressiveHolo(p, c.W, c.H, z_first=0, z_count=c.num_planes) as s:
        s.setHologram(b)
        _slabs().slab_iterate([s], 7)
        _slabs().slab_iterate([s], 8)  # two calls continue the same solve
        assert _records_bits(s.iterations()) == _records_bits(rec)
        assert np.array_equal(s.getVolume(), X)


@pytest.mark.parametrize("storage,tv,n_slabs,n_tv", [(0, None, 3, 5), (2, None, 2, 5), (0, 0.0, 4, 5),
                                                     (0, None, 2, 7)])
def test_slabs_match_one_context(rihvr, synthmod, cache_dir, storage, tv, n_slabs, n_tv):
    """Mode 7 in FP32 and FP16 storage, mode 5 (no TV), and 7 TV iterations
    (the prox in two launches with its dual stored in each slab's buffers)."""
    kw = dict(W=128, H=128, Nz=25, seed=32, num_inverse_iterations=20, num_tv_iterations=n_tv)
    if tv is not None:
        kw["regularization_TV_param"] = tv
    c = synthmod.small_config(**kw)
    b = synthmod.make_hologram(c, cache_dir=cache_dir)[1]
    p = rihvr.params_from_config(c)
    p.storage = storage
    rec, X = _solve_one(rihvr, p, c.W, c.H, b, 20)
    g = _slabs().SlabSolve(p, c.W, c.H, n_slabs)
    try:
        assert [s.depth for s in g.solvers] == [
            _slabs().slab_bounds(c.num_planes, n_slabs, i)[1] for i in range(n_slabs)]
        g.setHologram(b)
        g.iterate(20)
        rs = g.iterations()
        for s in g.solvers[1:]:  # every slab keeps the whole solve's log
            assert _records_bits(s.iterations()) == _records_bits(rs)
        assert np.array_equal(rs["backtracks"], rec["backtracks"])
        assert np.array_equal(rs["restarted"], rec["restarted"])
        # The spectrum's FP32 sum runs in another order, so the iterates differ
        # in their last bits (FP32 storage) or in roundings to 11 bits (FP16).
        tol = 1e-5 if storage == 0 else 1e-3
        for k in ("f_x", "f_prox", "f_resid_prox", "t", "beta"):
            assert np.allclose(rs[k], rec[k], rtol=tol, atol=0), k
        # lim = lim1 + lim2 / 2t is a difference of larger terms; it enters the
        # test ratio = f_resid / (f_resid(x) + lim), held to its own scale
        den = np.concatenate([[np.inf], rec["f_resid_x"][:-1]]) + rec["lim"]
        den[0] = abs(rec["lim"][0]) + rec["f_resid_prox"][0]
        dl = np.abs(rs["lim"] - rec["lim"]) / np.abs(den)
        assert dl.max() <= tol, dl.max()
        assert np.allclose(rs["ratio"], rec["ratio"], rtol=tol, atol=0)
        Xs = g.getVolume()
        assert Xs.shape == X.shape
        assert np.linalg.norm(Xs - X) <= tol * np.linalg.norm(X)
    finally:
        g.destroy()


def test_slab_contexts_refuse_whole_volume_calls(rihvr, synthmod, cache_dir):
    c = synthmod.small_config(W=64, H=64, Nz=6, seed=33, num_inverse_iterations=3)
    b = synthmod.make_hologram(c, cache_dir=cache_dir)[1]
    p = rihvr.params_from_config(c)
    with pytest.raises(rihvr.RihvrError) as e:
        rihvr.SparseCompressiveHolo(p, 64, 64, z_first=4, z_count=3)
    assert e.value.code == rihvr.ERR_INVALID_ARGUMENT
    with pytest.raises(rihvr.RihvrError):
        rihvr.SparseCompressiveHolo(p, 64, 64, z_first=-1, z_count=2)
    p6 = rihvr.params_from_config(c)
    p6.mode, p6.regularization_TV_param = 6, 0.01
    with pytest.raises(rihvr.RihvrError) as e:
        rihvr.SparseCompressiveHolo(p6, 64, 64, z_first=0, z_count=3)
    assert e.value.code == rihvr.ERR_UNKNOWN_MODE
    a = rihvr.SparseCompressiveHolo(p, 64, 64, z_first=0, z_count=3)
    z = rihvr.SparseCompressiveHolo(p, 64, 64, z_first=3, z_count=3)
    other = rihvr.SparseCompressiveHolo(p, 64, 64, z_first=2, z_count=4)
    try:
        L = rihvr.load_library()
        f0, nz = ctypes.c_int(), ctypes.c_int()
        assert L.rihvr_slab_range(z._h, ctypes.byref(f0), ctypes.byref(nz)) == 0 and (f0.value, nz.value) == (3, 3)
        for s in (a, z):
            s.setHologram(b)
        for call in (lambda: a.iterate(1), lambda: a.inverseReconstruct(), lambda: a.calcObjectiveFunction(),
                     lambda: a.estimateLipschitz(2), lambda: a.initialEstimate(),
                     lambda: a.setInitialVolume(np.zeros((3, 64, 64), np.complex64))):
            with pytest.raises(rihvr.RihvrError) as e:
                call()
            assert e.value.code == rihvr.ERR_INVALID_STATE
        # the slabs must tile the planes in order
        with pytest.raises(rihvr.RihvrError):
            _slabs().slab_iterate([z, a], 1)
        with pytest.raises(rihvr.RihvrError):
            _slabs().slab_iterate([a], 1)
        other.setHologram(b)
        with pytest.raises(rihvr.RihvrError):
            _slabs().slab_iterate([a, other], 1)
        # a slab whose hologram differs is refused before any work
        z.setHologram(b * 0.5)
        with pytest.raises(rihvr.RihvrError) as e:
            _slabs().slab_iterate([a, z], 1)
        assert e.value.code == rihvr.ERR_INVALID_STATE
        z.setHologram(b)
        _slabs().slab_iterate([a, z], 2)
        assert len(a.iterations()) == 2 and a.getVolume().shape == (3, 64, 64)
        # the forward operator of a slab gives its planes' share of the hologram
        X = np.concatenate([a.getVolume(), z.getVolume()])
        with rihvr.SparseCompressiveHolo(p, 64, 64) as w:
            full = w.forward(X)
        part = a.forward(X[:3]) + z.forward(X[3:])
        assert np.allclose(part, full, rtol=0, atol=1e-5 * np.abs(full).max())
    finally:
        for s in (a, z, other):
            s.destroy()


def _rank_worker(rank, world, port, p_bytes, W, H, b, n, out):
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import datetime

    import torch.distributed as dist

    rihvr = importlib.import_module(PKG_NAME)
    slabs = importlib.import_module(PKG_NAME + ".slabs")
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        p = rihvr.RihvrParams.from_buffer_copy(p_bytes)
        z0, nz = slabs.slab_bounds(p.num_planes, world, rank)
        red = slabs.torch_reducer()
        with rihvr.SparseCompressiveHolo(p, W, H, z_first=z0, z_count=nz) as s:
            s.setHologram(b)
            slabs.slab_iterate([s], n, red)
            out.put((rank, _records_bits(s.iterations()), s.getVolume()))
    except Exception as e:
        out.put((rank, repr(e), None))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_processes_one_slab_each_equal_one_process(rihvr, synthmod, cache_dir):
    """Two processes (gloo, host-staged sums), one slab each, on one GPU;
    no kernel waits on the other process.  For two slabs every sum is one
    addition of the same two values, so the result is bit-identical to the
    in-process group."""
    import torch.multiprocessing as mp

    from test_multiframe import free_port

    c = synthmod.small_config(W=64, H=64, Nz=9, seed=34, num_inverse_iterations=12)
    b = synthmod.make_hologram(c, cache_dir=cache_dir)[1]
    p = rihvr.params_from_config(c)
    g = _slabs().SlabSolve(p, c.W, c.H, 2)
    try:
        g.setHologram(b)
        g.iterate(12)
        rec, X = _records_bits(g.iterations()), g.getVolume()
    finally:
        g.destroy()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank_worker, args=(r, 2, port, bytes(p), c.W, c.H, b, 12, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    res = sorted((q.get(timeout=300) for _ in procs), key=lambda t: t[0])
    for pr in procs:
        pr.join(timeout=120)
        assert pr.exitcode == 0
    for r, recs, vol in res:
        assert vol is not None, recs
        assert recs == rec
    assert np.array_equal(np.concatenate([res[0][2], res[1][2]]), X)


def _nccl_worker(port, p_bytes, W, H, b, n, out):
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import datetime

    import torch
    import torch.distributed as dist

    rihvr = importlib.import_module(PKG_NAME)
    slabs = importlib.import_module(PKG_NAME + ".slabs")
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60),
                            device_id=torch.device("cuda", 0))
    try:
        p = rihvr.RihvrParams.from_buffer_copy(p_bytes)
        red = slabs.torch_reducer()
        with rihvr.SparseCompressiveHolo(p, W, H, z_first=0, z_count=p.num_planes) as s:
            s.setHologram(b)
            slabs.slab_iterate([s], n, red)
            out.put((red.struct.host_staged, _records_bits(s.iterations()), s.getVolume()))
    except Exception as e:
        out.put((None, repr(e), None))
    finally:
        dist.destroy_process_group()


def test_nccl_reducer_sums_the_spectrum_in_device_memory(rihvr, synthmod, cache_dir):
    """The NCCL reducer takes the device path (the spectrum all-reduced in
    place on the slab's device); over one rank it is the identity, so one slab
    of every plane equals rihvr_iterate bit for bit."""
    import torch.multiprocessing as mp

    from test_multiframe import free_port

    c = synthmod.small_config(W=64, H=64, Nz=6, seed=35, num_inverse_iterations=9)
    b = synthmod.make_hologram(c, cache_dir=cache_dir)[1]
    p = rihvr.params_from_config(c)
    rec, X = _solve_one(rihvr, p, c.W, c.H, b, 9)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    pr = ctx.Process(target=_nccl_worker, args=(free_port(), bytes(p), c.W, c.H, b, 9, q))
    pr.start()
    staged, recs, vol = q.get(timeout=300)
    pr.join(timeout=120)
    assert pr.exitcode == 0
    assert vol is not None, recs
    assert staged == 0
    assert recs == _records_bits(rec)
    assert np.array_equal(vol, X)


def test_slab_checkpoints_resume_the_group(rihvr, synthmod, cache_dir, tmp_path):
    """Each slab saves its own state (rihvr_save_state); new slab contexts
    loading them continue the group's solve bit for bit.  A state file names
    its plane range, so slab 1's file does not load into slab 0 although their
    sizes agree."""
    c = synthmod.small_config(W=64, H=64, Nz=8, seed=36, num_inverse_iterations=9)
    b = synthmod.make_hologram(c, cache_dir=cache_dir)[1]
    p = rihvr.params_from_config(c)
    ref = _slabs().SlabSolve(p, c.W, c.H, 2)
    g = _slabs().SlabSolve(p, c.W, c.H, 2)
    h = _slabs().SlabSolve(p, c.W, c.H, 2)
    try:
        ref.setHologram(b)
        ref.iterate(4)
        ref.iterate(5)
        g.setHologram(b)
        g.iterate(4)
        files = [str(tmp_path / f"slab{i}.state") for i in range(2)]
        for s, f in zip(g.solvers, files):
            s.saveState(f)
        with pytest.raises(rihvr.RihvrError) as e:
            h.solvers[0].loadState(files[1])
        assert e.value.code == rihvr.ERR_INVALID_FILE
        for s, f in zip(h.solvers, files):
            s.loadState(f)
        h.iterate(5)
        assert _records_bits(h.iterations()) == _records_bits(ref.iterations())
        assert np.array_equal(h.getVolume(), ref.getVolume())
    finally:
        for x in (ref, g, h):
            x.destroy()
