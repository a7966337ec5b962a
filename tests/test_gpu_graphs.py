"""Captured iterations: after the first iteration the attempts and the momentum
step run as CUDA graphs (one per rotation of the three volumes); the eager
path (profiling mode) must give the same bits."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode,side", [(7, 128), (5, 64), (7, 96)])
def test_graph_replay_equals_eager(rihvr, synthmod, cache_dir, mode, side):
    cfg = synthmod.small_config(W=side, H=side, Nz=5, seed=41 + side)
    _, b = synthmod.make_hologram(cfg, cache_dir=cache_dir)
    out = {}
    for eager in (True, False):
        p = rihvr.params_from_config(cfg, mode=mode)
        with rihvr.SparseCompressiveHolo(p, side, side) as s:
            s.set_profiling(eager)
            s.setHologram(b)
            s.iterate(9)
            n0 = s.launch_count()
            s.iterate(3)
            out[eager] = (s.iterations(), s.getVolume(), s.launch_count() - n0)
    (le, xe, ne), (lg, xg, ng) = out[True], out[False]
    assert np.array_equal(xe, xg)
    for k in ("f_x", "backtracks", "restarted", "t"):
        assert np.array_equal(le[k], lg[k]), k
    assert ne == ng  # the graphs hold the same kernels
