"""CPU tests of the frame preprocessing and background generation: the
restatement (oracle/frames.py) pinned against OpenCV's Python bindings (the
library the reference calls), the host preprocessing against it bit for bit,
PNG reading and writing against OpenCV, and the background parameter codes."""
import math

import numpy as np
import pytest

import frames as FR

cv2 = pytest.importorskip("cv2")


def seq(seed, n, shape=(23, 31), dtype=np.uint8, hi=256):
    rng = np.random.default_rng(seed)
    return rng.integers(0, hi, (n,) + shape).astype(dtype)


def test_mat_divide_is_fp32_multiply_by_fp32_reciprocal():
    """``Mat /= n`` is ``convertTo`` with alpha 1/n.  cv2.normalize with
    NORM_INF runs the same convertTo with alpha = a / max|x|; with max|x| =
    1024 and a = 1024 / n that alpha is exactly fl64(1/n)."""
    rng = np.random.default_rng(1)
    for n in (3, 7, 13, 199, 200, 333, 499):
        acc = (rng.random((41, 37)) * 1000).astype(np.float32)
        acc[0, 0] = 1024.0
        via_cv = cv2.normalize(acc, None, alpha=1024.0 / n, norm_type=cv2.NORM_INF)
        assert np.array_equal(via_cv, (acc * np.float32(1.0 / n)).astype(np.float32)), n


def test_background_mean_restatement_matches_opencv():
    fr = seq(2, 9)
    bg, (alpha, beta, minimum, average) = FR.background_mean(fr)
    acc = np.zeros(fr.shape[1:], np.float32)
    for k in range(len(fr)):
        acc = cv2.add(acc, fr[k].astype(np.float32))
    assert np.array_equal(acc * np.float32(1.0 / len(fr)), bg)
    # cv::mean of an FP32 image keeps FP32 partial sums within its SIMD
    # blocks, so it sits about 1e-10 (relative) off the exact mean; the
    # stats file prints 6 decimals
    assert math.isclose(cv2.mean(bg)[0], average, rel_tol=1e-8)
    ms = [cv2.meanStdDev((f.astype(np.float32) - bg).astype(np.float32)) for f in fr]
    mean_mean = np.mean([m[0][0, 0] for m in ms])
    mean_std = np.mean([m[1][0, 0] for m in ms])
    assert math.isclose(alpha, mean_mean - 5 * mean_std, rel_tol=1e-12, abs_tol=1e-12)
    assert math.isclose(beta, 255 / (2 * mean_std * 5), rel_tol=1e-12)
    assert minimum == 0.0


def test_median_stack_follows_the_reference_loop(rihvr):
    """The five-frame stack of median_background_calc, simulated literally:
    frames 0-4 loaded, three backgrounds written, then frame i overwrites
    plane (i - 3) % 5 for 3 <= i < n - 2; against the library's table."""
    for n in (5, 6, 7, 8, 12, 40):
        planes = [0, 1, 2, 3, 4]
        expect = [list(planes)] * 3
        for i in range(3, n - 2):
            planes[(i - 3) % 5] = i
            expect.append(list(planes))
        assert np.array_equal(FR.median5_frames(n), np.array(expect))
        assert np.array_equal(rihvr.median5_frames(n), np.array(expect))
    fr = seq(3, 10).astype(np.float32)
    med = FR.background_median5(fr)
    assert med.shape == (8,) + fr.shape[1:]
    for j, s in enumerate(FR.median5_frames(10)):
        assert np.array_equal(med[j], np.sort(fr[s], axis=0)[2])


def test_mean_frame_choice():
    assert FR.mean_frame_ids(4, 10) == list(range(4, 14))
    assert FR.mean_frame_ids(0, 0, 10, 20) == list(range(10, 19))  # background_end - start - 1 frames
    ids = FR.mean_frame_ids(0, 1000)
    assert ids[:3] == [0, 5, 10] and len(ids) == 200


def test_unit_mean_is_the_correctly_rounded_mean():
    """The exact mean agrees with cv::mean, whose FP32 partial sums put it
    about 1e-11 (relative) off, and the FP32 mean the preprocessing divides
    by is the same (a 1-ulp difference needs the exact mean within 1e-11 of
    an FP32 rounding boundary)."""
    for seed, dt, hi in ((4, np.uint8, 256), (5, np.uint16, 65536)):
        f = seq(seed, 1, (61, 67), dt, hi)[0]
        m = FR.unit_mean(f)
        cvm = cv2.mean(FR.unit(f))[0]
        assert math.isclose(m, cvm, rel_tol=1e-9)
        assert np.float32(m) == np.float32(cvm)


@pytest.mark.parametrize("case", ["whole", "pad", "rect", "centre", "centre_edge", "centre_big", "rect_out"])
@pytest.mark.parametrize("dt", [np.uint8, np.uint16])
def test_host_preprocess_matches_restatement(rihvr, case, dt):
    hi = 256 if dt == np.uint8 else 65536
    f = seq(6, 1, (40, 52), dt, hi)[0]
    fp = rihvr.FileParams()
    fp.roi_x = fp.roi_y = fp.roi_size = -1
    kw = {}
    pad = 0
    if case == "pad":
        pad = 3
    elif case == "rect":
        fp.roi_rect_x, fp.roi_rect_y, fp.roi_rect_w, fp.roi_rect_h = 5, 7, 20, 16
        kw["rect"] = (5, 7, 20, 16)
    elif case == "rect_out":  # partly outside the frame: zeros there
        fp.roi_rect_x, fp.roi_rect_y, fp.roi_rect_w, fp.roi_rect_h = 40, -3, 20, 16
        kw["rect"] = (40, -3, 20, 16)
    elif case.startswith("centre"):
        x, y, s = {"centre": (20, 18, 16), "centre_edge": (50, 2, 16), "centre_big": (10, 10, 48)}[case]
        fp.roi_x, fp.roi_y, fp.roi_size = x, y, s
        kw.update(roi_x=x, roi_y=y, roi_size=s)
        pad = 2
    got = rihvr.preprocess(f.astype(np.float32), pad, files=fp)
    want = FR.preprocess(f, pad=pad, **kw)
    assert got.shape == want.shape and np.array_equal(got, want)


def test_host_background_division_matches_restatement(rihvr):
    f = seq(7, 1)[0]
    b = seq(8, 1)[0]
    b[0, :5] = [0, 1, 2, 3, 255]  # sqrt(B/255) below 0.1 takes 0.1
    got = rihvr.preprocess(f.astype(np.float32), 4, background=b.astype(np.float32))
    assert np.array_equal(got, FR.preprocess(f, background=b, pad=4))


def test_png_written_reads_in_opencv(rihvr, tmp_path):
    img = seq(9, 1, (37, 53))[0]
    p = str(tmp_path / "a.png")
    rihvr.write_png8(p, img)
    assert np.array_equal(cv2.imread(p, cv2.IMREAD_UNCHANGED), img)
    back, bits = rihvr.read_image(p)
    assert bits == 8 and np.array_equal(back, img.astype(np.float32))


@pytest.mark.parametrize("level", [0, 1, 9])
def test_reads_opencv_pngs(rihvr, tmp_path, level):
    """Gray 8 and 16 bit and RGB, as cv2.imwrite writes them (its row filters
    vary with the content and the level)."""
    rng = np.random.default_rng(level)
    smooth = (np.add.outer(np.arange(45), np.arange(61)) * 2 % 256).astype(np.uint8)
    cases = {
        "g8": rng.integers(0, 256, (45, 61), dtype=np.uint8),
        "g8s": smooth,
        "g16": rng.integers(0, 65536, (33, 47), dtype=np.uint16),
        "g16s": (smooth.astype(np.uint16) * 257),
    }
    for name, img in cases.items():
        p = str(tmp_path / f"{name}_{level}.png")
        assert cv2.imwrite(p, img, [cv2.IMWRITE_PNG_COMPRESSION, level])
        back, bits = rihvr.read_image(p)
        assert bits == img.dtype.itemsize * 8
        assert np.array_equal(back, img.astype(np.float32)), name
    bgr = rng.integers(0, 256, (19, 27, 3), dtype=np.uint8)
    p = str(tmp_path / f"rgb_{level}.png")
    assert cv2.imwrite(p, bgr, [cv2.IMWRITE_PNG_COMPRESSION, level])
    back, _ = rihvr.read_image(p)
    expect = cv2.cvtColor(cv2.imread(p, cv2.IMREAD_UNCHANGED), cv2.COLOR_BGR2GRAY)
    assert np.array_equal(back, expect.astype(np.float32))


def test_png_errors(rihvr, tmp_path):
    rgba = np.zeros((8, 8, 4), np.uint8)
    p = str(tmp_path / "rgba.png")
    assert cv2.imwrite(p, rgba)
    with pytest.raises(rihvr.RihvrError):
        rihvr.read_image(p)
    good = str(tmp_path / "g.png")
    rihvr.write_png8(good, np.arange(64, dtype=np.uint8).reshape(8, 8))
    raw = bytearray(open(good, "rb").read())
    raw[40] ^= 0xFF  # inside IDAT: the chunk CRC no longer matches
    bad = tmp_path / "bad.png"
    bad.write_bytes(bytes(raw))
    with pytest.raises(rihvr.RihvrError):
        rihvr.read_image(str(bad))


def test_background_param_codes(rihvr, tmp_path):
    f = tmp_path / "bg.param"
    f.write_text("image_filename 2001 frames/f_%04d.png\noutput_path 2004 out\n"
                 "background_start 1003 12\nbackground_end 1004 40\nmedian 7006 true\n")
    p, files = rihvr.read_param_file(str(f))
    assert (files.background_start, files.background_end, files.use_median_background) == (12, 40, 1)
    f.write_text("image_filename 2001 x\n")
    p, files = rihvr.read_param_file(str(f))
    assert (files.background_start, files.background_end, files.use_median_background) == (-1, -1, 0)
