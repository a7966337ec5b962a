"""CPU checks of the segmentation oracle (``orc_segment``) and of the centroid
file writer.

The oracle is pinned against ``seg_ref.py``, a literal restatement of the
reference's segmentation program (COO planes, counting morphology, sorted
index search, minimum sweeps, first-appearance objects, swap filter), field
for field and bit for bit, and independently against scipy.ndimage's
binary morphology and 26-connected labelling.
"""
import os

import numpy as np
import pytest

import oracle as O
import seg_ref


def random_stack(seed, nz, h, w, density=0.06, scale=100.0):
    rng = np.random.default_rng(seed)
    I = np.zeros((nz, h, w), np.float32)
    m = rng.random(I.shape) < density
    I[m] = (rng.random(int(m.sum())) * scale).astype(np.float32)
    return I


def blob_stack(seed, nz, h, w, nblobs):
    """Intensity blobs (Gaussian bumps) plus sparse noise."""
    rng = np.random.default_rng(seed)
    z, y, x = np.meshgrid(np.arange(nz), np.arange(h), np.arange(w), indexing="ij")
    I = np.zeros((nz, h, w), np.float64)
    for _ in range(nblobs):
        c = rng.uniform([0, 0, 0], [nz, h, w])
        r = rng.uniform(0.8, 2.5)
        I += rng.uniform(10, 100) * np.exp(-((z - c[0]) ** 2 + (y - c[1]) ** 2 + (x - c[2]) ** 2) / (2 * r * r))
    I[I < 0.5] = 0
    I = I.astype(np.float32)
    m = rng.random(I.shape) < 0.01
    I[m] += (rng.random(int(m.sum())) * 20).astype(np.float32)
    return I


def as_rows(objs):
    return [tuple(np.asarray(list(o)).tolist()) for o in objs]


def same_bits(a, b):
    """Field-by-field equality, floats compared by bit pattern (NaN == NaN)."""
    assert len(a) == len(b)
    for ra, rb in zip(a, b):
        for fa, fb in zip(ra, rb):
            if isinstance(fb, (float, np.floating)):
                assert np.float32(fa).tobytes() == np.float32(fb).tobytes(), (ra, rb)
            else:
                assert int(fa) == int(fb), (ra, rb)


CASES = [
    # seed, (nz, h, w), min_intensity, close_size, min_area, faithful, kind
    (0, (5, 12, 14), 1.0, 0, 1, 1, "random"),
    (1, (5, 12, 14), 1.0, 1, 1, 1, "random"),
    (2, (6, 10, 13), 30.0, 0, 2, 1, "random"),
    (3, (6, 10, 13), 30.0, 0, 2, 0, "random"),
    (4, (7, 14, 16), 20.0, 1, 2, 1, "blobs"),
    (5, (7, 14, 16), 20.0, 2, 1, 0, "blobs"),
    (6, (9, 16, 15), 10.0, 1, 3, 1, "blobs"),
]


@pytest.mark.parametrize("seed,shape,mi,cs,ma,faithful,kind", CASES)
def test_oracle_matches_literal_restatement(seed, shape, mi, cs, ma, faithful, kind):
    I = random_stack(seed, *shape, density=0.25) if kind == "random" else blob_stack(seed, *shape, nblobs=6)
    ref, (rmax, rthr) = seg_ref.segment(I, mi, cs, ma, faithful)
    got, (gmax, gthr) = O.segment(I, mi, cs, ma, faithful)
    assert gmax == rmax and gthr == rthr
    assert len(ref) > 0
    same_bits(as_rows(got), ref)


def test_faithful_neighbourhood_continues_on_the_next_row():
    """The reference's in-plane offsets are linear: a voxel at the end of a row
    touches the start of the next row (sparse_segmentation.cu:493-511)."""
    I = np.zeros((3, 6, 8), np.float32)
    I[1, 2, 7] = 50.0  # row end
    I[1, 3, 0] = 60.0  # next row's start
    got_f, _ = O.segment(I, 1.0, 0, 1, 1)
    got_g, _ = O.segment(I, 1.0, 0, 1, 0)
    ref_f, _ = seg_ref.segment(I, 1.0, 0, 1, 1)
    assert len(got_f) == 1 and got_f[0]["num_voxels"] == 2
    assert len(got_g) == 2
    same_bits(as_rows(got_f), ref_f)


def test_closing_and_labels_match_scipy():
    """Independent pin: the closing equals scipy's binary dilation then
    erosion with the same ball (outside the volume is off), and the
    geometric labelling equals scipy's 26-connected components."""
    ndi = pytest.importorskip("scipy.ndimage")
    I = blob_stack(11, 10, 20, 22, nblobs=10)
    cs, mi = 2, 15.0
    got, (mx, thr) = O.segment(I, mi, cs, 1, 0)
    s = np.sqrt(I)
    q = (s * s).astype(np.float32)
    on = q.astype(np.float64) > thr
    zz, yy, xx = np.mgrid[-cs:cs + 1, -cs:cs + 1, -cs:cs + 1]
    ballm = zz * zz + yy * yy + xx * xx <= cs * cs
    closed = ndi.binary_erosion(ndi.binary_dilation(on, structure=ballm, border_value=0), structure=ballm,
                                border_value=0)
    lab, n = ndi.label(closed, structure=np.ones((3, 3, 3), bool))
    assert len(got) == n
    # objects come in order of their smallest linear index
    flat = lab.ravel()
    first = [int(np.flatnonzero(flat == k)[0]) for k in range(1, n + 1)]
    order = np.argsort(first)
    for o, k in zip(got, order + 1):
        zi, yi, xi = np.nonzero(lab == k)
        assert o["num_voxels"] == len(zi)
        assert (o["xmin"], o["xmax"], o["ymin"], o["ymax"], o["zmin"], o["zmax"]) == (
            xi.min(), xi.max(), yi.min(), yi.max(), zi.min(), zi.max())
        assert o["x"] == np.float32(np.float32(xi.sum()) / np.float32(len(xi)))


def test_size_filter_swaps_in_the_last_object():
    """ObjectCloud::blobSizeFilter (object_cloud.cu:313-328) replaces a small
    object with the current last one and re-tests that slot."""
    I = np.zeros((1, 4, 40), np.float32)
    sizes = [1, 3, 1, 2, 4, 1]
    x = 0
    for k, n in enumerate(sizes):
        I[0, 1, x:x + n] = 10.0 + k
        x += n + 2
    got, _ = O.segment(I, 1.0, 0, 2, 0)
    ref, _ = seg_ref.segment(I, 1.0, 0, 2, 0)
    # order before the filter: sizes 1,3,1,2,4,1 -> slot 0 takes the last (1),
    # fails again and takes the 4; slot 2 takes the 2
    assert [o["num_voxels"] for o in got] == [4, 3, 2]
    same_bits(as_rows(got), ref)


def test_write_centroids_formats(rihvr, tmp_path):
    objs = np.zeros(2, rihvr.OBJECT_DTYPE)
    objs[0] = (1.5, 2.25, 3.0, 1.4, 2.2, 3.1, 7, 12.5, 3.25, 0, 3, 1, 4, 2, 4)
    objs[1] = (10.0, 0.125, 5.5, 10.5, 0.25, 5.0, 2, 0.001, 0.0005, 9, 11, 0, 1, 5, 6)
    for weighted, verbose, name in ((0, 0, "c.csv"), (1, 0, "cw.csv"), (0, 1, "cv.csv")):
        path = str(tmp_path / name)
        rihvr.write_centroids(path, objs, weighted=weighted, verbose=verbose)
        lines = open(path).read().splitlines()
        if not verbose:
            assert lines[0] == "x (pixels), y (pixels), z (planes), # of voxels"
            for o, ln in zip(objs, lines[1:]):
                c = (o["wx"], o["wy"], o["wz"]) if weighted else (o["x"], o["y"], o["z"])
                assert ln == "%f, %f, %f, %d" % (float(c[0]), float(c[1]), float(c[2]), o["num_voxels"])
        else:
            assert lines[0].startswith("x (pixels), y (pixels), z (planes), weighted x")
            o = objs[1]
            assert lines[2] == ("%f, %f, %f, %f, %f, %f, %d, %e, %e, %d, %d, %d, %d, %d, %d" % (
                float(o["x"]), float(o["y"]), float(o["z"]), float(o["wx"]), float(o["wy"]), float(o["wz"]),
                o["num_voxels"], float(o["max_value"]), float(o["mean_value"]), o["xmin"], o["xmax"], o["ymin"],
                o["ymax"], o["zmin"], o["zmax"]))


def test_segment_arguments_are_checked_before_the_gpu(rihvr):
    import ctypes

    L = rihvr.load_library()
    sp = rihvr.segment_params()
    assert (sp.min_intensity, sp.close_size, sp.min_area, sp.faithful) == (1.0, 3, 2, 1)
    n = ctypes.c_int()
    assert L.rihvr_segment_intensity(None, 4, 4, 4, 0, ctypes.byref(sp), None, 0, ctypes.byref(n), None) == \
        rihvr.ERR_INVALID_ARGUMENT
    dummy = ctypes.c_void_p(4096)
    assert L.rihvr_segment_intensity(dummy, 0, 4, 4, 1, ctypes.byref(sp), None, 0, ctypes.byref(n), None) == \
        rihvr.ERR_INVALID_ARGUMENT


def test_param_file_reads_segmentation_settings(rihvr, tmp_path):
    f = tmp_path / "seg.param"
    f.write_text("segment_min_area 5009 4\nsegment_min_intensity 5010 12.5\nsegment_close_size 5011 2\n")
    _, fp = rihvr.read_param_file(str(f))
    assert (fp.segment_min_area, fp.segment_min_intensity, fp.segment_close_size) == (4, 12.5, 2)
    g = tmp_path / "plain.param"
    g.write_text("num_planes 3003 10\n")
    _, fp = rihvr.read_param_file(str(g))
    assert (fp.segment_min_area, fp.segment_min_intensity, fp.segment_close_size) == (2, 1.0, 3)
