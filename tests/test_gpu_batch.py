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
