"""CPU tests of the image I/O and hologram preprocessing in the native library
(the OpenCV parts of the reference's Hologram class on the reconstruction
path), checked against OpenCV's Python bindings and numpy restatements."""
import numpy as np
import pytest

cv2 = pytest.importorskip("cv2")


@pytest.fixture(scope="module")
def frames():
    rng = np.random.default_rng(9)
    img8 = rng.integers(0, 256, (37, 53), dtype=np.uint8)
    img16 = rng.integers(0, 65536, (29, 41), dtype=np.uint16)
    return img8, img16


def test_tiff8_round_trip(rihvr, tmp_path, frames):
    img8, _ = frames
    p = str(tmp_path / "a.tif")
    rihvr.write_tiff8(p, img8)
    back, bits = rihvr.read_image(p)
    assert bits == 8 and np.array_equal(back, img8.astype(np.float32))
    # OpenCV reads what we write
    assert np.array_equal(cv2.imread(p, cv2.IMREAD_UNCHANGED), img8)


@pytest.mark.parametrize("compression", [1, 5, 32773])  # none, LZW, PackBits
def test_reads_opencv_tiffs(rihvr, tmp_path, frames, compression):
    img8, img16 = frames
    for img in (img8, img16):
        p = str(tmp_path / f"c{compression}_{img.dtype}.tif")
        assert cv2.imwrite(p, img, [cv2.IMWRITE_TIFF_COMPRESSION, compression])
        back, bits = rihvr.read_image(p)
        assert bits == img.dtype.itemsize * 8
        assert np.array_equal(back, img.astype(np.float32))


def test_reads_rgb_as_gray(rihvr, tmp_path):
    rng = np.random.default_rng(3)
    bgr = rng.integers(0, 256, (16, 24, 3), dtype=np.uint8)
    p = str(tmp_path / "rgb.tif")
    assert cv2.imwrite(p, bgr, [cv2.IMWRITE_TIFF_COMPRESSION, 1])
    back, _ = rihvr.read_image(p)
    expect = cv2.cvtColor(cv2.imread(p, cv2.IMREAD_UNCHANGED), cv2.COLOR_BGR2GRAY)
    assert np.array_equal(back, expect.astype(np.float32))


def test_reads_pgm(rihvr, tmp_path, frames):
    img8, _ = frames
    p = tmp_path / "a.pgm"
    p.write_bytes(b"P5\n# c\n%d %d\n255\n" % (img8.shape[1], img8.shape[0]) + img8.tobytes())
    back, bits = rihvr.read_image(str(p))
    assert np.array_equal(back, img8.astype(np.float32))


def test_preprocess_matches_synthetic_pipeline(rihvr, synthmod, frames):
    img8, _ = frames
    for pad in (0, 5):
        b = rihvr.preprocess(img8, pad)
        ref = synthmod.preprocess(img8, pad)
        assert b.shape == ref.shape == (37 + 2 * pad, 53 + 2 * pad)
        assert np.abs(b - ref).max() <= 2 * np.finfo(np.float32).eps


def test_preprocess_background_division(rihvr, frames):
    img8, _ = frames
    rng = np.random.default_rng(5)
    bg = rng.integers(0, 256, img8.shape, dtype=np.uint8)
    b = rihvr.preprocess(img8, 2, background=bg)
    I = img8.astype(np.float32) / np.float32(255)
    B = bg.astype(np.float32) / np.float32(255)
    ref = (I - B) / np.maximum(np.sqrt(B), np.float32(0.1))
    assert np.abs(b[2:-2, 2:-2] - ref).max() < 1e-6
    assert np.all(b[:2] == 0) and np.all(b[:, :2] == 0)


def test_preprocess_crop(rihvr, frames):
    img8, _ = frames
    fp = rihvr.FileParams()
    fp.roi_x, fp.roi_y, fp.roi_size = 10, 10, 16  # centre crop, clamped into the frame
    b = rihvr.preprocess(img8, 0, files=fp)
    full = rihvr.preprocess(img8, 0)
    assert b.shape == (16, 16)
    assert np.array_equal(b, full[2:18, 2:18])
    fp = rihvr.FileParams()
    fp.roi_size = -1
    fp.roi_rect_x, fp.roi_rect_y, fp.roi_rect_w, fp.roi_rect_h = 50, 30, 8, 10  # runs past the edge: zeros
    b = rihvr.preprocess(img8, 0, files=fp)
    assert b.shape == (10, 8)
    assert np.array_equal(b[:7, :3], full[30:37, 50:53]) and np.all(b[7:] == 0) and np.all(b[:, 3:] == 0)


def test_bad_image_is_an_error(rihvr, tmp_path):
    p = tmp_path / "junk.tif"
    p.write_bytes(b"not an image at all")
    with pytest.raises(rihvr.RihvrError):
        rihvr.read_image(str(p))
