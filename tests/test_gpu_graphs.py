"""Captured iterations.  After the first iteration of a context, whole
iterations run as CUDA graphs with the backtracking decided on the device (a
conditional WHILE node around the backtracking attempt); RIHVR_ITER_LOOP=host
selects the host-synchronised loop of captured attempts instead.  The eager
path (profiling mode), the host loop and the device loop must give the same
bits, with and without backtracks."""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# the device loop adds four one-thread control kernels an iteration: the
# attempt's scalars, the backtracking test, the momentum factor, the record
CONTROL_KERNELS = 4


@pytest.mark.parametrize("mode,side,t0", [(7, 128, 0.0), (5, 64, 0.0), (7, 96, 0.0), (7, 64, 6.0), (5, 64, 6.0)])
def test_graph_replay_equals_eager(rihvr, synthmod, cache_dir, mode, side, t0):
    cfg = synthmod.small_config(W=side, H=side, Nz=5, seed=41 + side)
    _, b = synthmod.make_hologram(cfg, cache_dir=cache_dir)
    out = {}
    for eager in (True, False):
        p = rihvr.params_from_config(cfg, mode=mode, initial_step=t0 / cfg.num_planes if t0 else 0.0)
        with rihvr.SparseCompressiveHolo(p, side, side) as s:
            s.set_profiling(eager)
            s.setHologram(b)
            s.iterate(9)
            n0 = s.launch_count()
            s.iterate(3)
            out[eager] = (s.iterations(), s.getVolume(), s.launch_count() - n0)
    (le, xe, ne), (lg, xg, ng) = out[True], out[False]
    assert np.array_equal(xe, xg)
    for k in ("f_x", "f_prox", "lim", "ratio", "beta", "backtracks", "restarted", "t"):
        assert np.array_equal(le[k], lg[k]), k
    if t0:
        assert le["backtracks"].sum() > 0  # the backtracking attempt ran
    assert ng == ne + CONTROL_KERNELS * 3  # the same operator kernels, plus the control kernels


_LOOP_SCRIPT = r"""
import importlib, sys
import numpy as np
root, pkg, out, t0, rec = sys.argv[1], sys.argv[2], sys.argv[3], float(sys.argv[4]), int(sys.argv[5])
sys.path.insert(0, root)
rihvr = importlib.import_module(pkg)
synth = importlib.import_module(pkg + ".synth")
cfg = synth.small_config(W=96, H=96, Nz=6, seed=77)
_, b = synth.make_hologram(cfg)
p = rihvr.params_from_config(cfg, initial_step=t0 / cfg.num_planes if t0 else 0.0, record_objective=rec)
with rihvr.SparseCompressiveHolo(p, 96, 96) as s:
    s.setHologram(b)
    s.iterate(14)
    log = s.iterations()
    X = s.getVolume()
np.savez(out, X=X, **{k: log[k] for k in log.dtype.names})
"""


@pytest.mark.parametrize("t0,rec", [(0.0, 0), (6.0, 0), (6.0, 1)])
def test_host_loop_equals_device_loop(rihvr, tmp_path, t0, rec):
    from conftest import PKG_NAME, ROOT

    script = tmp_path / "loop.py"
    script.write_text(_LOOP_SCRIPT)
    res = {}
    for loop in ("host", "device"):
        env = dict(os.environ)
        env.pop("RIHVR_ITER_LOOP", None)
        if loop == "host":
            env["RIHVR_ITER_LOOP"] = "host"
        f = tmp_path / f"{loop}.npz"
        r = subprocess.run([sys.executable, str(script), ROOT, PKG_NAME, str(f), str(t0), str(rec)], env=env,
                           capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        res[loop] = dict(np.load(f))
    h, d = res["host"], res["device"]
    assert np.array_equal(h["X"].view(np.uint32), d["X"].view(np.uint32))
    for k in h:
        if k != "X":
            assert np.array_equal(h[k], d[k]), k
    if t0:
        assert h["backtracks"].sum() > 0
