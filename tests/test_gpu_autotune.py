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
    # evenly spaced planes: the untuned adjoint evaluates directly, the forward uses Horner's scheme
    assert t0 == {"adj_chunks": 0, "fwd_chunks": t0["fwd_chunks"], "tv_runs": 0, "tv_kernel": 0,
                  "adj_recurrence": 0, "fwd_horner": 3}
    assert t1["tv_kernel"] in (0, 1, 2, 3) and 1 <= t1["fwd_chunks"] <= 16 and t1["adj_recurrence"] in (0, 1, 2, 3)
    assert t1["fwd_horner"] in (0, 1, 2, 3)
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


def test_column_variants_only_for_evenly_spaced_planes(rihvr):
    """The recurrence and Horner variants need z_{k+1} - z_k equal for every k
    (in FP64, from the float plane list): dz = 0.1 gives uneven float
    positions, dz = 2 even ones."""
    def tuned(z0, dz, side=128, nz=6):
        p = rihvr.default_params()
        p.start_plane, p.plane_stepsize, p.num_planes = z0, dz, nz
        p.wavelength, p.resolution, p.zero_padding = 0.632, 2.0, 0
        with rihvr.SparseCompressiveHolo(p, side, side) as s:
            t = s.tuning()
            return t["adj_recurrence"], t["fwd_horner"]

    assert tuned(2500.0, 2.0) == (0, 3)  # untuned: direct adjoint, TMA-fed Horner forward
    z = np.float32(100.0) + np.arange(6, dtype=np.float32) * np.float32(0.1)
    assert len(set(np.diff(z.astype(np.float64)))) > 1  # uneven in FP64
    assert tuned(100.0, 0.1) == (0, 0)
    assert tuned(2500.0, 2.0, side=384) == (0, 3)  # 48 elements a thread: the table-twiddle forms only
