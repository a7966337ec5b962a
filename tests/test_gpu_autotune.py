"""Launch-shape autotuner (rihvr_autotune): tuned shapes keep the solve within
FP32 rounding of the untuned one, and a second context of the same shape
reuses the cached choice."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_autotune_keeps_the_solution(rihvr, synthmod, cache_dir):
    cfg = synthmod.small_config(W=256, H=256, Nz=12, seed=31)
    _, b = synthmod.make_hologram(cfg, cache_dir=cache_dir)
    runs = {}
    for tune in (0, 1):
        p = rihvr.params_from_config(cfg, autotune=tune)
        with rihvr.SparseCompressiveHolo(p, cfg.W, cfg.H) as s:
            s.setHologram(b)  # tunes when autotune = 1
            tun = s.tuning()
            s.iterate(10)
            runs[tune] = (s.iterations(), s.getVolume(), tun)
    (l0, x0, t0), (l1, x1, t1) = runs[0], runs[1]
    assert t0 == {"adj_chunks": 0, "fwd_chunks": t0["fwd_chunks"], "tv_runs": 0, "tv_kernel": 0}
    assert t1["tv_kernel"] in (0, 1, 2) and 1 <= t1["fwd_chunks"] <= 16
    assert np.array_equal(l0["backtracks"], l1["backtracks"])
    assert np.array_equal(l0["restarted"], l1["restarted"])
    assert np.max(np.abs(l0["f_x"] - l1["f_x"]) / np.abs(l0["f_x"])) < 1e-5
    assert np.linalg.norm(x1 - x0) <= 1e-4 * np.linalg.norm(x0)


def test_autotune_cache(rihvr, synthmod, cache_dir):
    cfg = synthmod.small_config(W=128, H=128, Nz=9, seed=32)
    _, b = synthmod.make_hologram(cfg, cache_dir=cache_dir)
    p = rihvr.params_from_config(cfg)
    with rihvr.SparseCompressiveHolo(p, cfg.W, cfg.H) as s:
        s.setHologram(b)
        t = time.perf_counter()
        ms = s.autotune()
        first = time.perf_counter() - t
        choice = s.tuning()
    assert ms > 0
    with rihvr.SparseCompressiveHolo(p, cfg.W, cfg.H) as s2:
        s2.setHologram(b)
        t = time.perf_counter()
        assert s2.autotune() == ms
        second = time.perf_counter() - t
        assert s2.tuning() == choice
    assert second < first
