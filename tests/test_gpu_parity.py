"""GPU parity of the sm_100a path against the FP64 oracle, through the C ABI.

Tolerances (relative L2 error / relative objective gap): 1e-4 for FP32 volume
storage and 1e-2 for BF16/FP16 storage.  Operators are compared elementwise on
random inputs; solves are compared iteration by iteration (same backtracking
and restart decisions, objective within tolerance) and on the final volume.
"""
import hashlib
import os

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

TOL_F32 = 1e-4
TOL_LOW = 1e-2
GOLD_C1 = os.path.join(os.path.dirname(__file__), "golden", "oracle_c1_384x384x40.npz")


def rel(a, b):
    a = np.asarray(a, np.complex128)
    b = np.asarray(b, np.complex128)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def make(rihvr, side, nz, **kw):
    p = rihvr.default_params()
    p.start_plane, p.plane_stepsize, p.num_planes = 100.0, 40.0, nz
    p.wavelength, p.resolution = 0.632, 2.0
    p.regularization_param, p.regularization_TV_param, p.num_tv_iterations = 0.01, 0.02, 5
    p.zero_padding = 0
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def oparams(rihvr, p, side, **kw):
    d = dict(W=side, H=side, z=rihvr.plane_list(p), dx=float(np.float32(p.resolution)),
             lam=float(np.float32(p.wavelength)), l1=float(np.float32(p.regularization_param)),
             tv=float(np.float32(p.regularization_TV_param)), n_tv=p.num_tv_iterations, mode=p.mode,
             faithful=p.faithful, t0=p.initial_step)
    d.update(kw)
    return O.OracleParams(**d)


def rand_volume(rng, nz, side, scale=0.05):
    return (scale * (rng.standard_normal((nz, side, side)) + 1j * rng.standard_normal((nz, side, side)))).astype(
        np.complex64)


@pytest.mark.parametrize("side,nz", [(32, 3), (48, 4), (64, 5), (128, 4), (256, 2), (384, 3), (512, 2), (768, 2),
                                     (1024, 2), (2304, 2), (640, 3)])
def test_forward_matches_oracle(rihvr, side, nz):
    p = make(rihvr, side, nz)
    rng = np.random.default_rng(side + nz)
    vol = rand_volume(rng, nz, side)
    with rihvr.SparseCompressiveHolo(p, side, side) as s:
        d = s.forward(vol)
    ref = O.forward(oparams(rihvr, p, side), vol.astype(np.complex128))
    assert rel(d, ref) < TOL_F32


@pytest.mark.parametrize("side,nz", [(32, 3), (48, 4), (64, 5), (128, 2), (256, 2), (384, 3), (512, 2), (768, 2),
                                     (1024, 2), (2304, 3), (640, 5)])
def test_adjoint_matches_oracle(rihvr, side, nz):
    p = make(rihvr, side, nz)
    rng = np.random.default_rng(7 * side + nz)
    r = rng.standard_normal((side, side)).astype(np.float32)
    with rihvr.SparseCompressiveHolo(p, side, side) as s:
        g = s.adjoint(r)
    ref = O.adjoint(oparams(rihvr, p, side), r.astype(np.float64))
    assert rel(g, ref) < TOL_F32


def test_adjoint_identity_on_gpu(rihvr):
    """<A x, r> = <x, A^H r> in FP32 (testAdjoint, sparse_compressive_holo.cu:2533-2652)."""
    side, nz = 128, 6
    p = make(rihvr, side, nz)
    rng = np.random.default_rng(5)
    x = rand_volume(rng, nz, side, 1.0)
    r = rng.standard_normal((side, side)).astype(np.float32)
    with rihvr.SparseCompressiveHolo(p, side, side) as s:
        lhs = float(np.sum(s.forward(x).astype(np.float64) * r))
        g = s.adjoint(r).astype(np.complex128)
    rhs = float(np.sum(x.real * g.real + x.imag * g.imag))
    assert abs(lhs - rhs) < 1e-5 * max(abs(lhs), abs(rhs))


@pytest.mark.parametrize("mode", [5, 6, 7])
@pytest.mark.parametrize("faithful", [1, 0])
def test_prox_step_matches_oracle(rihvr, mode, faithful):
    side, nz = 64, 4
    p = make(rihvr, side, nz, mode=mode, faithful=faithful)
    rng = np.random.default_rng(mode * 10 + faithful)
    x = rand_volume(rng, nz, side, 0.05)
    r = rng.standard_normal((side, side)).astype(np.float32)
    t = 0.2
    with rihvr.SparseCompressiveHolo(p, side, side) as s:
        out, sums = s.prox_step(x, r, t)
    op = oparams(rihvr, p, side)
    ref, rsums = O.prox_from(op, x.astype(np.complex128), x.astype(np.complex128), r.astype(np.float64), t)
    assert rel(out, ref) < TOL_F32
    assert abs(sums[0] - rsums[0]) < 1e-4 * max(abs(rsums[0]), 1e-6 * abs(rsums[1]) + 1e-12)
    assert abs(sums[1] - rsums[1]) < 1e-4 * abs(rsums[1])
    # the restart statistic against y0 = x: with the reference's weights (faithful) it is
    # a weighted -|p - x|^2, bounded by twice the plain one
    assert abs(sums[2] - rsums[2]) < 2e-4 * abs(rsums[1])
    assert rsums[2] < 0


@pytest.mark.parametrize("side,nz,n_tv", [(32, 3, 5), (128, 3, 1), (128, 2, 2), (384, 2, 3), (256, 2, 6),
                                         (128, 2, 7), (256, 2, 10), (64, 3, 0), (128, 2, 12)])
def test_tv_prox_iteration_counts(rihvr, side, nz, n_tv):
    """Streaming TV prox (1..10 Chambolle iterations) and the tiled one (other
    counts) against the oracle, on planes with several strips and runs."""
    p = make(rihvr, side, nz, mode=7, faithful=1, num_tv_iterations=n_tv)
    rng = np.random.default_rng(side * 10 + n_tv)
    x = rand_volume(rng, nz, side, 0.05)
    r = rng.standard_normal((side, side)).astype(np.float32)
    t = 0.3
    with rihvr.SparseCompressiveHolo(p, side, side) as s:
        out, sums = s.prox_step(x, r, t)
    ref, rsums = O.prox_from(oparams(rihvr, p, side), x.astype(np.complex128), x.astype(np.complex128),
                             r.astype(np.float64), t)
    assert rel(out, ref) < TOL_F32
    assert abs(sums[1] - rsums[1]) < 1e-4 * abs(rsums[1])


_TILES_SCRIPT = """
import sys, numpy as np
sys.path.insert(0, sys.argv[1])
import importlib
R = importlib.import_module(sys.argv[2])
side, nz, ntv, st = (int(v) for v in sys.argv[3:7])
p = R.default_params()
p.start_plane, p.plane_stepsize, p.num_planes = 100.0, 40.0, nz
p.wavelength, p.resolution, p.zero_padding = 0.632, 2.0, 0
p.regularization_param, p.regularization_TV_param, p.num_tv_iterations = 0.01, 0.02, ntv
p.storage = st
p.faithful = int(st != 1)  # BF16 storage only with faithful = 0
rng = np.random.default_rng(11)
x = (0.05 * (rng.standard_normal((nz, side, side)) + 1j * rng.standard_normal((nz, side, side)))).astype(np.complex64)
r = rng.standard_normal((side, side)).astype(np.float32)
with R.SparseCompressiveHolo(p, side, side) as s:
    out, sums = s.prox_step(x, r, 0.3)
np.save(sys.argv[7], out)
"""


@pytest.mark.parametrize("side,nz,ntv,storage", [(1024, 3, 5, 0), (384, 4, 3, 0), (768, 2, 6, 1), (256, 3, 4, 2),
                                                 (512, 2, 10, 2), (640, 2, 8, 0), (1024, 2, 7, 0), (2304, 1, 9, 2)])
def test_streaming_prox_bits_equal_tiled(rihvr, tmp_path, side, nz, ntv, storage):
    """The streaming TV prox, in 2- and 4-warp blocks, and for 6-10 TV
    iterations in two launches (the default, its dual stored between them)
    or one, reproduces the tiled kernel's P_new bit for bit (run lengths odd
    and even, every storage type)."""
    import subprocess
    import sys

    from conftest import PKG_NAME, ROOT

    script = tmp_path / "prox.py"
    script.write_text(_TILES_SCRIPT)
    outs = {}
    for kern in ("tiles", "strip", "strip4", "strip1"):
        env = dict(os.environ)
        env.pop("RIHVR_TV_KERNEL", None)
        if kern != "strip":
            env["RIHVR_TV_KERNEL"] = kern
        f = tmp_path / f"{kern}.npy"
        r = subprocess.run([sys.executable, str(script), ROOT, PKG_NAME, str(side), str(nz), str(ntv), str(storage),
                            str(f)], env=env, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        outs[kern] = np.load(f)
    assert np.array_equal(outs["tiles"].view(np.uint32), outs["strip"].view(np.uint32))
    assert np.array_equal(outs["tiles"].view(np.uint32), outs["strip4"].view(np.uint32))
    assert np.array_equal(outs["tiles"].view(np.uint32), outs["strip1"].view(np.uint32))


def run_gpu(rihvr, p, side, b, n):
    with rihvr.SparseCompressiveHolo(p, side, side) as s:
        s.setHologram(b)
        s.iterate(n)
        log = s.iterations()
        X = s.getVolume()
        f, terms = s.calcObjectiveFunction()
        est = s.getEstimate()
    return log, X, f, terms, est


@pytest.mark.parametrize("mode,faithful,t0", [(7, 1, 0.0), (7, 0, 0.0), (7, 1, 3.0), (5, 1, 3.0), (6, 1, 2.0)])
def test_solve_matches_oracle(rihvr, synthmod, cache_dir, mode, faithful, t0):
    side, nz, n = 64, 6, 20
    cfg = synthmod.small_config(W=side, H=side, Nz=nz, seed=2)
    _, b = synthmod.make_hologram(cfg, cache_dir=cache_dir)
    p = rihvr.params_from_config(cfg, mode=mode, faithful=faithful, initial_step=t0 / nz if t0 else 0.0)
    log, X, f, terms, est = run_gpu(rihvr, p, side, b, n)
    op = oparams(rihvr, p, side)
    # replay the GPU's decisions so that the trajectories are comparable even
    # if a ratio lands within rounding of a threshold
    olog, OX, OP, oest, f0 = O.solve(op, b.astype(np.float64), n, forced_bt=log["backtracks"],
                                     forced_rs=log["restarted"])
    free, _, _, _, _ = O.solve(op, b.astype(np.float64), n, want_volumes=False)
    # every decision of the oracle's own run equals the GPU's (measured: all
    # five cases, objective gap <= 7.5e-7, volume <= 8.4e-7)
    assert np.array_equal(free["backtracks"], log["backtracks"]), (free["backtracks"], log["backtracks"])
    assert np.array_equal(free["restarted"], log["restarted"]), (free["restarted"], log["restarted"])
    gap = np.abs(log["f_x"] - olog["f_x"]) / np.abs(olog["f_x"])
    assert gap.max() < TOL_F32, gap
    assert rel(X, OX) < TOL_F32
    assert abs(f - olog["f_x"][-1]) / abs(olog["f_x"][-1]) < TOL_F32
    assert rel(est, oest) < TOL_F32


def test_objective_recording_does_not_change_the_solve(rihvr, synthmod, cache_dir):
    """record_objective = 0 runs the prox without the norm terms (another
    kernel instantiation); the iterates must not change."""
    side, nz, n = 128, 5, 12
    cfg = synthmod.small_config(W=side, H=side, Nz=nz, seed=6)
    _, b = synthmod.make_hologram(cfg, cache_dir=cache_dir)
    out = {}
    for rec in (1, 0):
        p = rihvr.params_from_config(cfg, record_objective=rec)
        with rihvr.SparseCompressiveHolo(p, side, side) as s:
            s.setHologram(b)
            s.iterate(n)
            out[rec] = (s.getVolume(), s.iterations(), s.calcObjectiveFunction()[0])
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1]["backtracks"], out[1][1]["backtracks"])
    assert np.array_equal(out[0][1]["restarted"], out[1][1]["restarted"])
    assert out[0][2] == out[1][2]


@pytest.mark.parametrize("storage", [1, 2])
def test_reduced_precision_storage(rihvr, synthmod, cache_dir, storage):
    """FP16 in faithful mode; BF16 only with faithful = 0 (refused otherwise)."""
    side, nz, n = 64, 6, 20
    cfg = synthmod.small_config(W=side, H=side, Nz=nz, seed=4)
    _, b = synthmod.make_hologram(cfg, cache_dir=cache_dir)
    p = rihvr.params_from_config(cfg, storage=storage, faithful=0 if storage == 1 else 1)
    log, X, f, terms, est = run_gpu(rihvr, p, side, b, n)
    olog, OX, _, _, _ = O.solve(oparams(rihvr, p, side), b.astype(np.float64), n)
    assert abs(f - olog["f_x"][-1]) / abs(olog["f_x"][-1]) < TOL_LOW
    assert rel(X, OX) < 10 * TOL_LOW


def test_c1_workload_matches_oracle_fixture(rihvr, synthmod):
    """384x384x40, 100 FISTA / 5 TV iterations against the committed oracle
    run: the same backtracking and restart decisions at every iteration, the
    objective within 1e-4 at every iteration, the per-plane L1 norms and
    cropped volume values within 1e-4 (measured: 3.7e-7, 1.8e-6, 5.2e-6)."""
    g = np.load(GOLD_C1)
    cfg = synthmod.config1()
    _, b = synthmod.make_hologram(cfg)
    assert hashlib.sha1(b.tobytes()).digest() == bytes(g["b_sha1"]), "synthetic hologram differs from the fixture's"
    p = rihvr.params_from_config(cfg)
    log, X, f, terms, est = run_gpu(rihvr, p, cfg.W, b, cfg.num_inverse_iterations)
    assert np.array_equal(log["backtracks"], g["backtracks"])
    assert np.array_equal(log["restarted"], g["restarted"])
    gap = np.abs(log["f_x"] - g["f_x"]) / np.abs(g["f_x"])
    assert gap.max() < TOL_F32, gap.max()
    l1 = np.abs(X).sum(axis=(1, 2))
    assert np.abs(l1 - g["plane_l1"]).sum() / g["plane_l1"].sum() < TOL_F32
    crops = X[list(g["crop_planes"])][..., 160:224, 160:224]
    assert rel(crops, g["crops"]) < TOL_F32


def test_errors_are_status_codes(rihvr):
    p = make(rihvr, 64, 2)
    with rihvr.SparseCompressiveHolo(p, 64, 64) as s:
        with pytest.raises(rihvr.RihvrError) as e:
            s.iterate(1)  # no hologram yet
        assert e.value.code == rihvr.ERR_MISSING_DATA
        with pytest.raises(rihvr.RihvrError) as e:
            s.getPlane(5)
        assert e.value.code == rihvr.ERR_INVALID_ARGUMENT
        s.setHologram(np.zeros((64, 64), np.float32))
        s.iterate(2)  # a zero hologram is a valid (trivial) problem
        assert np.all(s.getVolume() == 0)


@pytest.mark.parametrize("side,nz", [(1024, 20), (512, 37), (256, 50), (64, 19), (768, 20), (384, 18), (2304, 3)])
@pytest.mark.parametrize("adj,fwd", [("direct", "direct"), ("recurrence", "horner"),
                                     ("recurrence_hoisted", "horner"), ("recurrence_table", "horner_onebuf"),
                                     ("recurrence_hoisted", "horner_tma")])
def test_column_pass_variants_match_oracle(rihvr, monkeypatch, side, nz, adj, fwd):
    """Every column-pass variant for evenly spaced planes (selected by name,
    as the autotuner would pick them) against the FP64 oracle: the adjoint's
    recurrence (re-anchored every 16 planes) and the forward's Horner sum, on
    enough planes to cross several anchors and z-chunks.  Sides 384, 768 and
    2304 (48 elements a thread) have only the table-twiddle forms; a variant a
    size does not have runs the direct pass."""
    monkeypatch.setenv("RIHVR_ADJ_COL", adj)
    monkeypatch.setenv("RIHVR_FWD_COL", fwd)
    p = make(rihvr, side, nz)
    p.start_plane, p.plane_stepsize = 2500.0, 2.0  # evenly spaced in float
    rng = np.random.default_rng(side * 3 + nz)
    vol = rand_volume(rng, nz, side)
    r = rng.standard_normal((side, side)).astype(np.float32)
    with rihvr.SparseCompressiveHolo(p, side, side) as s:
        d = s.forward(vol)
        g = s.adjoint(r)
    op = oparams(rihvr, p, side)
    assert rel(d, O.forward(op, vol.astype(np.complex128))) < TOL_F32
    assert rel(g, O.adjoint(op, r.astype(np.float64))) < TOL_F32


@pytest.mark.parametrize("side,nz", [(1024, 20), (512, 37), (256, 50), (64, 19)])
def test_table_twiddle_variants_bits_equal_register_forms(rihvr, monkeypatch, side, nz):
    """The three-blocks-an-SM column passes (twiddles from a shared table; the
    forward pass's strip staged in the exchange buffer, by cp.async or by TMA)
    compute the same FP32
    operations as the register-resident forms.  The forward sums are
    bit-equal.  The adjoint's default z-chunks differ between the two (more
    blocks resident, more chunks), and the recurrence re-anchors every 16
    planes from each chunk's first plane, so its last bits may differ."""
    p = make(rihvr, side, nz)
    p.start_plane, p.plane_stepsize = 2500.0, 2.0
    rng = np.random.default_rng(side * 5 + nz)
    vol = rand_volume(rng, nz, side)
    r = rng.standard_normal((side, side)).astype(np.float32)
    out = []
    for adj, fwd in (("recurrence_hoisted", "horner"), ("recurrence_table", "horner_onebuf"),
                     ("recurrence_table", "horner_tma")):
        monkeypatch.setenv("RIHVR_ADJ_COL", adj)
        monkeypatch.setenv("RIHVR_FWD_COL", fwd)
        with rihvr.SparseCompressiveHolo(p, side, side) as s:
            out.append((s.forward(vol), s.adjoint(r)))
    (d0, g0), (d1, g1), (d2, _) = out
    assert np.array_equal(d0, d1)
    assert np.array_equal(d0, d2)
    assert rel(g1, g0) < 2e-6


def test_volume_device_pointer_is_the_volume(rihvr, synthmod, cache_dir):
    """rihvr_get_volume_ptr hands out the momentum-point volume in device
    memory: the same values rihvr_get_volume copies out, for FP32 and FP16
    storage."""
    cfg = synthmod.small_config(W=64, H=64, Nz=5, seed=7)
    _, b = synthmod.make_hologram(cfg, cache_dir=cache_dir)
    for storage in (0, 2):
        p = rihvr.params_from_config(cfg, storage=storage)
        with rihvr.SparseCompressiveHolo(p, cfg.W, cfg.H) as s:
            s.setHologram(b)
            s.iterate(6)
            X = s.getVolume()
            V = s.volume_device().cpu().numpy()
        assert V.shape == X.shape
        assert np.array_equal(V, X)
        assert np.abs(X).max() > 0


@pytest.mark.parametrize("storage,record", [(0, 1), (2, 0)])
def test_checkpoint_resumes_bit_for_bit(rihvr, synthmod, cache_dir, tmp_path, storage, record):
    """rihvr_save_state after 5 iterations and rihvr_load_state into a new
    context, then 7 more iterations: the same iteration log and volume as 5
    and then 7 iterations in one context, bit for bit (with and without
    objective recording, FP32 and FP16 storage).  (Each rihvr_iterate call
    settles its last record's objective terms with a pass of its own, so the
    reference is two calls, not one of 12.)  A state file is refused by a
    context of another size or with other parameters."""
    cfg = synthmod.small_config(W=64, H=64, Nz=6, seed=17, num_inverse_iterations=12)
    _, b = synthmod.make_hologram(cfg, cache_dir=cache_dir)
    p = rihvr.params_from_config(cfg, storage=storage, record_objective=record)
    with rihvr.SparseCompressiveHolo(p, cfg.W, cfg.H) as s:
        s.setHologram(b)
        s.iterate(5)
        s.iterate(7)
        log12, X12 = s.iterations(), s.getVolume()
    path = str(tmp_path / "state.bin")
    with rihvr.SparseCompressiveHolo(p, cfg.W, cfg.H) as s:
        s.setHologram(b)
        s.iterate(5)
        s.saveState(path)
    with rihvr.SparseCompressiveHolo(p, cfg.W, cfg.H) as s:
        s.loadState(path)
        s.iterate(7)
        log, X = s.iterations(), s.getVolume()
    assert log.shape == log12.shape
    for name in log12.dtype.names:
        assert np.array_equal(log[name], log12[name]), name
    assert np.array_equal(X, X12)
    q = rihvr.params_from_config(cfg, storage=storage, record_objective=record)
    q.regularization_param = q.regularization_param * 2
    with rihvr.SparseCompressiveHolo(q, cfg.W, cfg.H) as s:
        with pytest.raises(rihvr.RihvrError) as e:
            s.loadState(path)
        assert e.value.code == rihvr.ERR_INVALID_FILE
    with rihvr.SparseCompressiveHolo(p, 32, 32) as s:
        with pytest.raises(rihvr.RihvrError) as e:
            s.loadState(path)
        assert e.value.code == rihvr.ERR_INVALID_FILE
