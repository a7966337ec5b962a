"""Warm start (rihvr_set_initial_volume): FISTA continues from a given volume.
From its own solution the objective keeps decreasing; from the solution of a
neighbouring frame (same particles, a different noise realisation) it reaches
the plain solve's objective in far fewer iterations than from zero."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _solve(rihvr, cfg, b, n, x0=None):
    p = rihvr.params_from_config(cfg)
    with rihvr.SparseCompressiveHolo(p, cfg.W, cfg.H) as s:
        s.setHologram(b)
        if x0 is not None:
            s.setInitialVolume(x0)
        s.iterate(n)
        return s.iterations()["f_x"], s.getVolume()


def test_warm_start_from_own_solution(rihvr, synthmod, cache_dir):
    cfg = synthmod.small_config(W=128, H=128, Nz=6, seed=51)
    _, b = synthmod.make_hologram(cfg, cache_dir=cache_dir)
    f, X = _solve(rihvr, cfg, b, 40)
    fw, _ = _solve(rihvr, cfg, b, 10, x0=X)
    assert fw[-1] <= f[-1] * (1 + 1e-6)


def test_warm_start_from_neighbouring_frame(rihvr, synthmod, cache_dir):
    a = synthmod.small_config(W=128, H=128, Nz=6, seed=52, noise_sigma=0.010)
    c = synthmod.small_config(W=128, H=128, Nz=6, seed=52, noise_sigma=0.013)
    _, ba = synthmod.make_hologram(a, cache_dir=cache_dir)
    _, bc = synthmod.make_hologram(c, cache_dir=cache_dir)
    assert not np.array_equal(ba, bc)
    n = 60
    _, Xa = _solve(rihvr, a, ba, n)
    fc, _ = _solve(rihvr, c, bc, n)
    target = fc[-1]
    band = 1e-3 * abs(target)
    k_cold = int(np.nonzero(np.abs(fc - target) <= band)[0][0]) + 1
    fw, _ = _solve(rihvr, c, bc, n, x0=Xa)
    hits = np.nonzero(fw - target <= band)[0]
    assert len(hits), (fw[-5:], target)
    k_warm = int(hits[0]) + 1
    print(f"iterations to within 1e-3 of the {n}-iteration objective: cold {k_cold}, warm {k_warm}")
    assert k_warm * 2 <= k_cold
