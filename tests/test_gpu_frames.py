"""Camera frames on the GPU: rihvr_set_hologram_frame (the driver's
preprocessing, main_sparse_inverse.cu:106-124, from raw 8/16-bit samples),
rihvr_background_mean and rihvr_background_median5 (main_create_background.cu)
and the create-background program, against the restatement in
oracle/frames.py.  Integer and FP32 elementwise work is compared bit for bit;
the background statistics (FP64 sums in another order) to 1e-12."""
import math
import os
import subprocess

import numpy as np
import pytest

import frames as FR

pytestmark = pytest.mark.gpu


def seq(seed, n, shape, dtype=np.uint8, hi=256):
    rng = np.random.default_rng(seed)
    return rng.integers(0, hi, (n,) + tuple(shape)).astype(dtype)


def ctx_params(rihvr, pad=0, nz=3):
    p = rihvr.default_params()
    p.start_plane, p.plane_stepsize, p.num_planes = 100.0, 40.0, nz
    p.wavelength, p.resolution, p.zero_padding = 0.632, 2.0, pad
    p.num_inverse_iterations = 3
    return p


def files_for(rihvr, roi=None, rect=None, background=False):
    fp = rihvr.FileParams()
    fp.roi_x = fp.roi_y = fp.roi_size = -1
    if roi:
        fp.roi_x, fp.roi_y, fp.roi_size = roi
    if rect:
        fp.roi_rect_x, fp.roi_rect_y, fp.roi_rect_w, fp.roi_rect_h = rect
    fp.remove_background = int(background)
    return fp


@pytest.mark.parametrize("dt,hi", [(np.uint8, 256), (np.uint16, 65536), (np.float32, 256)])
@pytest.mark.parametrize("case", ["whole", "rect", "centre_edge", "background"])
def test_frame_preprocessing_bit_exact(rihvr, dt, hi, case):
    """Against the restatement and the host path (rihvr_preprocess), for
    frames in host memory and as CUDA tensors; 64 x 64 holograms cut from
    larger or equal frames, padded by 8 where the crop is 48 wide."""
    import torch

    roi = rect = None
    kw = {}
    pad = 0
    shape = (64, 64)
    if case == "rect":
        shape, rect, pad = (70, 90), (30, 11, 48, 48), 8
        kw["rect"] = rect
    elif case == "centre_edge":
        shape, roi, pad = (60, 77), (70, 5, 48), 8
        kw.update(roi_x=70, roi_y=5, roi_size=48)
    f = seq(1, 1, shape, dt, hi)[0]
    bg = seq(2, 1, shape, dt, hi)[0] if case == "background" else None
    fp = files_for(rihvr, roi, rect, bg is not None)
    want = FR.preprocess(f, background=bg, pad=pad, **kw)
    host = rihvr.preprocess(f.astype(np.float32), pad, background=None if bg is None else bg.astype(np.float32),
                            files=fp)
    assert np.array_equal(host, want)
    with rihvr.SparseCompressiveHolo(ctx_params(rihvr, pad), 64, 64) as s:
        s.setHologramFrame(f, background=bg, files=fp)
        assert np.array_equal(s.getHologram(), want)
        ft = torch.from_numpy(f).cuda()
        bt = None if bg is None else torch.from_numpy(bg).cuda()
        s.setHologramFrame(ft, background=bt, files=fp)
        assert np.array_equal(s.getHologram(), want)


def test_frame_then_solve_equals_float_hologram(rihvr, synthmod, tmp_path):
    """A solve from the raw frame equals the solve from the host-preprocessed
    hologram bit for bit."""
    cfg = synthmod.small_config(W=64, H=64, Nz=5, seed=3, zero_padding=4)
    img, _ = synthmod.make_hologram(cfg, cache_dir=str(tmp_path))
    p = rihvr.params_from_config(cfg)
    b = rihvr.preprocess(img.astype(np.float32), cfg.zero_padding)
    W = img.shape[1] + 2 * cfg.zero_padding
    H = img.shape[0] + 2 * cfg.zero_padding
    with rihvr.SparseCompressiveHolo(p, W, H) as a, rihvr.SparseCompressiveHolo(p, W, H) as c:
        a.setHologram(b)
        c.setHologramFrame(img)
        a.iterate(4)
        c.iterate(4)
        assert np.array_equal(a.getVolume(), c.getVolume())
        assert np.array_equal(a.iterations()["f_x"], c.iterations()["f_x"])


def test_frame_refusals_keep_the_context(rihvr):
    f = seq(5, 1, (64, 64))[0]
    with rihvr.SparseCompressiveHolo(ctx_params(rihvr), 64, 64) as s:
        s.setHologramFrame(f)
        before = s.getHologram()
        bad = f.astype(np.float32)
        bad[3, 4] = 1.5  # not an 8/16-bit sample
        with pytest.raises(rihvr.RihvrError) as e:
            s.setHologramFrame(bad)
        assert e.value.code == rihvr.ERR_INVALID_DATA
        nan = f.astype(np.float32)
        nan[0, 0] = np.nan
        with pytest.raises(rihvr.RihvrError) as e:
            s.setHologramFrame(nan)
        assert e.value.code == rihvr.ERR_INVALID_DATA
        with pytest.raises(rihvr.RihvrError) as e:
            s.setHologramFrame(np.zeros((64, 64), np.uint8))  # mean zero
        assert e.value.code == rihvr.ERR_INVALID_DATA
        with pytest.raises(rihvr.RihvrError) as e:
            s.setHologramFrame(seq(6, 1, (64, 66))[0])  # does not fit the context
        assert e.value.code == rihvr.ERR_INVALID_ARGUMENT
        with pytest.raises(rihvr.RihvrError) as e:
            s.setHologramFrame(f, files=files_for(rihvr, background=True))  # no background given
        assert e.value.code == rihvr.ERR_MISSING_DATA
        assert np.array_equal(s.getHologram(), before)


@pytest.mark.parametrize("dt,hi", [(np.uint8, 256), (np.uint16, 65536), (np.float32, 256)])
def test_background_mean(rihvr, dt, hi):
    import torch

    fr = seq(7, 13, (37, 53), dt, hi)
    bg, st = rihvr.background_mean(fr)
    wbg, (alpha, beta, minimum, average) = FR.background_mean(fr)
    assert np.array_equal(bg, wbg)
    assert math.isclose(st["alpha"], alpha, rel_tol=1e-12, abs_tol=1e-9)
    assert math.isclose(st["beta"], beta, rel_tol=1e-12)
    assert st["minimum"] == minimum == 0.0
    assert math.isclose(st["average"], average, rel_tol=1e-12)
    dbg, dst = rihvr.background_mean(torch.from_numpy(fr).cuda())
    assert np.array_equal(dbg.cpu().numpy(), wbg) and dst == st


@pytest.mark.parametrize("n", [5, 6, 7, 16])
def test_background_median5(rihvr, n):
    import torch

    fr = seq(8 + n, n, (29, 41))
    fr[:, 0, :3] = 17  # ties
    want = FR.background_median5(fr)
    got = rihvr.background_median5(fr)
    assert got.shape == (n - 2, 29, 41) and np.array_equal(got, want)
    dev = rihvr.background_median5(torch.from_numpy(fr.astype(np.uint16)).cuda())
    assert np.array_equal(dev.cpu().numpy(), want)
    with pytest.raises(rihvr.RihvrError):
        rihvr.background_median5(fr[:4])


def test_create_background_program(rihvr, tmp_path):
    """create-background -F: background.png and background_stats.txt in mean
    mode, background_XXXX.png in median mode, from PNG frames on disk."""
    cv2 = pytest.importorskip("cv2")
    fr = seq(21, 12, (33, 47))
    d = tmp_path / "frames"
    d.mkdir()
    for k in range(len(fr)):
        assert cv2.imwrite(str(d / f"f_{100 + k:04d}.png"), fr[k])
    out = tmp_path / "out"
    out.mkdir()
    exe = os.path.join(os.path.dirname(rihvr.CLI_PATH), "create-background")
    base = f"image_file 2001 {d}/f_%04d.png\noutput_path 2004 {out}\n"
    (tmp_path / "mean.param").write_text(base + "start_image 1002 100\nimage_count 1001 9\n")
    r = subprocess.run([exe, "-F", str(tmp_path / "mean.param")], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    ids = FR.mean_frame_ids(100, 9)
    wbg, stats = FR.background_mean(fr[[i - 100 for i in ids]])
    got = cv2.imread(str(out / "background.png"), cv2.IMREAD_UNCHANGED)
    assert np.array_equal(got, FR.to_u8(wbg))
    lines = (out / "background_stats.txt").read_text().split()
    assert [float(v) for v in lines] == pytest.approx([float(f"{v:f}") for v in stats], abs=1.5e-6)

    (tmp_path / "med.param").write_text(base + "background_start 1003 101\nbackground_end 1004 111\n"
                                               "median 7006 true\n")
    r = subprocess.run([exe, "-F", str(tmp_path / "med.param")], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    want = FR.background_median5(fr[1:11])
    for j in range(8):
        got = cv2.imread(str(out / f"background_{101 + j:04d}.png"), cv2.IMREAD_UNCHANGED)
        assert np.array_equal(got, FR.to_u8(want[j])), j
    assert not (out / "background_0109.png").exists()
