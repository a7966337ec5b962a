"""Multi-rank frame sharding on CPU: two gloo ranks, as bench.py --gpus 2 runs
them on GPUs (one process per GPU, independent frames, max-over-ranks timing)."""
import importlib
import os
import socket

import pytest

from conftest import PKG_NAME


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import torch.distributed as dist

    frames = importlib.import_module(PKG_NAME + ".frames")
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        mine = frames.rank_frames(7, world, rank)
        seeds = [frames.frame_seed(100, f) for f in mine]
        elapsed = 10.0 + 5.0 * rank  # ms: rank 1 is the slowest
        mx = frames.reduce_max(elapsed)
        total = frames.reduce_sum(len(mine) * 1000)
        out.put((rank, mine, seeds, mx, total, frames.weak_throughput(total * 3, mx)))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_frames_and_agree_on_timing():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, f0, s0, m0, t0, v0), (r1, f1, s1, m1, t1, v1) = res
    assert f0 == [0, 1, 2, 3] and f1 == [4, 5, 6]  # disjoint and complete
    assert set(s0).isdisjoint(s1)
    assert m0 == m1 == 15.0  # the slowest rank's time
    assert t0 == t1 == 7000
    assert v0 == v1 == pytest.approx(7000 * 3 / 0.015)


def test_rank_frames_partition(rihvr):
    frames = importlib.import_module(PKG_NAME + ".frames")
    for n in range(0, 20):
        for w in range(1, 6):
            parts = [frames.rank_frames(n, w, r) for r in range(w)]
            flat = [i for p in parts for i in p]
            assert flat == list(range(n))
            assert max(map(len, parts)) - min(map(len, parts)) <= 1
    with pytest.raises(ValueError):
        frames.rank_frames(3, 2, 2)


def _tiny_series(n):
    """Small frames of the advected tracer series (32 x 32, 4 planes), for CPU runs."""
    synth = importlib.import_module(PKG_NAME + ".synth")
    cfgs = synth.series_frames(n, iterations=4)
    for c in cfgs:
        c.width = c.height = 32
        c.num_planes = 4
        c.n_disks = 6
        c.name = c.name + "_tiny"
    return cfgs


def _solve_frame(cfg):
    import numpy as np

    import oracle as O

    synth = importlib.import_module(PKG_NAME + ".synth")
    _, b = synth.make_hologram(cfg, cache_dir=os.environ.get("RIHVR_TEST_CACHE"))
    op = O.OracleParams(W=cfg.W, H=cfg.H, z=cfg.plane_list(), dx=cfg.dx(), lam=cfg.lam(), l1=cfg.l1(), tv=cfg.tv(),
                        n_tv=cfg.num_tv_iterations, mode=7, faithful=1, n_threads=1)
    log, _, _, _, _ = O.solve(op, b.astype(np.float64), cfg.num_inverse_iterations, want_volumes=False)
    return float(log["f_x"][-1])


def _reconstruct_worker(rank, world, port, n, out):
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for p in (root, os.path.join(root, "oracle")):
        sys.path.insert(0, p)
    import datetime

    import torch.distributed as dist

    frames = importlib.import_module(PKG_NAME + ".frames")
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        cfgs = _tiny_series(n)
        mine = frames.rank_frames(n, world, rank)
        objs = {i: _solve_frame(cfgs[i]) for i in mine}
        gathered = [None] * world
        dist.all_gather_object(gathered, objs)  # each rank learns every frame's objective
        total = frames.reduce_sum(sum(objs.values()))
        out.put((rank, mine, gathered, total))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_gloo_ranks_reconstruct_their_frames(tmp_path, monkeypatch):
    """Each rank reconstructs its own frames of the advected series (the FP64
    oracle stands in for the GPU solve on CPU); the frames' objectives, gathered
    over the ranks, equal a single-process run over all frames bit for bit."""
    import torch.multiprocessing as mp

    monkeypatch.setenv("RIHVR_TEST_CACHE", str(tmp_path))  # inherited by the spawned ranks
    n = 5
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_reconstruct_worker, args=(r, 2, port, n, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, f0, g0, t0), (_, f1, g1, t1) = res
    assert f0 == [0, 1, 2] and f1 == [3, 4]
    merged = {**g0[0], **g0[1]}
    assert g0 == g1 and sorted(merged) == list(range(n))
    single = {i: _solve_frame(c) for i, c in enumerate(_tiny_series(n))}
    assert merged == single
    assert t0 == t1 == sum(single[i] for i in f0) + sum(single[i] for i in f1)
