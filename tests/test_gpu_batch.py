"""Several frames reconstructed at once (rihvr_reconstruct_batch) give the
results of the sequential calls bit for bit, for frames of different sizes and
parameters."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_batch_equals_sequential(rihvr, synthmod, cache_dir):
    cfgs = [synthmod.small_config(W=64, H=64, Nz=5, seed=11, num_inverse_iterations=8),
            synthmod.small_config(W=128, H=128, Nz=4, seed=12, num_inverse_iterations=6, num_tv_iterations=3),
            synthmod.small_config(W=32, H=32, Nz=7, seed=13, num_inverse_iterations=10),
            synthmod.small_config(W=64, H=64, Nz=3, seed=14, num_inverse_iterations=5,
                                  regularization_TV_param=0.0)]
    holos = [synthmod.make_hologram(c, cache_dir=cache_dir)[1] for c in cfgs]
    seq = []
    for c, b in zip(cfgs, holos):
        with rihvr.SparseCompressiveHolo(rihvr.params_from_config(c), c.W, c.H) as s:
            f = s.inverseReconstruct(b)
            seq.append((f, s.getVolume(), s.iterations()))
    solvers = [rihvr.SparseCompressiveHolo(rihvr.params_from_config(c), c.W, c.H) for c in cfgs]
    try:
        fs = rihvr.reconstruct_batch(solvers, holos)
        for (f, X, log), fb, s in zip(seq, fs, solvers):
            assert fb == f
            assert np.array_equal(s.getVolume(), X)
            assert np.array_equal(s.iterations()["f_x"], log["f_x"])
        # a second batch on the same contexts starts again from x = 0
        fs2 = rihvr.reconstruct_batch(solvers, holos)
        assert fs2 == fs
    finally:
        for s in solvers:
            s.destroy()


def test_batch_reports_the_failing_frame(rihvr, synthmod, cache_dir):
    c = synthmod.small_config(W=64, H=64, Nz=3, seed=15, num_inverse_iterations=2)
    b = synthmod.make_hologram(c, cache_dir=cache_dir)[1]
    s1 = rihvr.SparseCompressiveHolo(rihvr.params_from_config(c), 64, 64)
    s2 = rihvr.SparseCompressiveHolo(rihvr.params_from_config(c), 64, 64)
    try:
        with pytest.raises(ValueError):
            rihvr.reconstruct_batch([s1, s2], [b, b[:32]])
        with pytest.raises(ValueError):
            rihvr.reconstruct_batch([s1], [b, b])
        fs = rihvr.reconstruct_batch([s1, s2], [b, b])
        assert fs[0] == fs[1]
    finally:
        s1.destroy()
        s2.destroy()


def test_batch_as_one_graph_per_iteration(rihvr, synthmod, cache_dir):
    """Batch mode 1: frames of different sizes, TV settings and storage but the
    same iteration count run as one graph launch per iteration (each frame a
    branch with its own device-side backtracking loop); every frame's volume,
    objective and iteration log equal its sequential run bit for bit, on cold
    contexts (eager first iteration) and again on warm ones."""
    cfgs = [synthmod.small_config(W=64, H=64, Nz=5, seed=21, num_inverse_iterations=9),
            synthmod.small_config(W=128, H=128, Nz=4, seed=22, num_inverse_iterations=9, num_tv_iterations=3),
            synthmod.small_config(W=32, H=32, Nz=7, seed=23, num_inverse_iterations=9),
            synthmod.small_config(W=64, H=64, Nz=3, seed=24, num_inverse_iterations=9, regularization_TV_param=0.0)]
    storage = [0, 0, 2, 1]  # BF16 only with faithful = 0
    holos = [synthmod.make_hologram(c, cache_dir=cache_dir)[1] for c in cfgs]
    seq = []
    for c, b, sto in zip(cfgs, holos, storage):
        with rihvr.SparseCompressiveHolo(rihvr.params_from_config(c, storage=sto, faithful=int(sto != 1)), c.W,
                                         c.H) as s:
            f = s.inverseReconstruct(b)
            seq.append((f, s.getVolume(), s.iterations()))
    solvers = [rihvr.SparseCompressiveHolo(rihvr.params_from_config(c, storage=sto, faithful=int(sto != 1)), c.W,
                                           c.H) for c, sto in zip(cfgs, storage)]
    rihvr.set_batch_mode(1)
    try:
        for _ in range(2):
            fs = rihvr.reconstruct_batch(solvers, holos)
            assert rihvr.batch_last_combined() == 1
            for (f, X, log), fb, s in zip(seq, fs, solvers):
                assert fb == f
                assert np.array_equal(s.getVolume(), X)
                got = s.iterations()
                for name in ("f_x", "f_prox", "t", "beta", "backtracks", "restarted"):
                    assert np.array_equal(got[name], log[name]), name
    finally:
        rihvr.set_batch_mode(0)
        for s in solvers:
            s.destroy()
    with pytest.raises(rihvr.RihvrError):
        rihvr.set_batch_mode(3)


def test_batch_whole_solves_as_one_graph(rihvr, synthmod, cache_dir):
    """Batch mode 2: frames of different sizes, TV settings, storage and
    iteration counts run their whole solves as one graph launch (each frame a
    branch looping on the device, its rotation picked by a switch node); every
    frame's volume, objective and iteration log equal its sequential run bit
    for bit, on cold contexts and again on warm ones.  One frame runs more
    than 256 iterations, so its solve takes two launches."""
    cfgs = [synthmod.small_config(W=64, H=64, Nz=5, seed=31, num_inverse_iterations=9),
            synthmod.small_config(W=128, H=128, Nz=4, seed=32, num_inverse_iterations=14, num_tv_iterations=3),
            synthmod.small_config(W=32, H=32, Nz=7, seed=33, num_inverse_iterations=300),
            synthmod.small_config(W=64, H=64, Nz=3, seed=34, num_inverse_iterations=2, regularization_TV_param=0.0)]
    storage = [0, 0, 2, 1]  # BF16 only with faithful = 0
    holos = [synthmod.make_hologram(c, cache_dir=cache_dir)[1] for c in cfgs]
    seq = []
    for c, b, sto in zip(cfgs, holos, storage):
        with rihvr.SparseCompressiveHolo(rihvr.params_from_config(c, storage=sto, faithful=int(sto != 1)), c.W,
                                         c.H) as s:
            f = s.inverseReconstruct(b)
            seq.append((f, s.getVolume(), s.iterations()))
    solvers = [rihvr.SparseCompressiveHolo(rihvr.params_from_config(c, storage=sto, faithful=int(sto != 1)), c.W,
                                           c.H) for c, sto in zip(cfgs, storage)]
    rihvr.set_batch_mode(2)
    try:
        # cold contexts, warm ones (the kept graph is launched again), and after
        # one context was replaced by a new one (the kept graph is not reused)
        for rnd in range(3):
            if rnd == 2:
                solvers[1].destroy()
                c, sto = cfgs[1], storage[1]
                solvers[1] = rihvr.SparseCompressiveHolo(rihvr.params_from_config(c, storage=sto,
                                                                                   faithful=int(sto != 1)), c.W, c.H)
            fs = rihvr.reconstruct_batch(solvers, holos)
            assert rihvr.batch_last_combined() == 2
            for (f, X, log), fb, s in zip(seq, fs, solvers):
                assert fb == f
                assert np.array_equal(s.getVolume(), X)
                got = s.iterations()
                assert got.shape == log.shape
                for name in ("f_x", "f_prox", "t", "beta", "backtracks", "restarted"):
                    assert np.array_equal(got[name], log[name]), name
    finally:
        rihvr.set_batch_mode(0)
        for s in solvers:
            s.destroy()


def test_uneven_iteration_counts_run_frame_by_frame(rihvr, synthmod, cache_dir):
    """Batch mode 1 with frames at different iteration counts falls back to one
    loop per frame."""
    cfgs = [synthmod.small_config(W=64, H=64, Nz=3, seed=25, num_inverse_iterations=4),
            synthmod.small_config(W=64, H=64, Nz=3, seed=26, num_inverse_iterations=6)]
    holos = [synthmod.make_hologram(c, cache_dir=cache_dir)[1] for c in cfgs]
    solvers = [rihvr.SparseCompressiveHolo(rihvr.params_from_config(c), c.W, c.H) for c in cfgs]
    rihvr.set_batch_mode(1)
    try:
        rihvr.reconstruct_batch(solvers, holos)
        assert not rihvr.batch_last_combined()
        assert [s.iterations().shape[0] for s in solvers] == [4, 6]
    finally:
        rihvr.set_batch_mode(0)
        for s in solvers:
            s.destroy()
