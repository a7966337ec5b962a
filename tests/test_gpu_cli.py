"""End-to-end test of the sparse-inverse-recon driver (the reference's CLI,
main_sparse_inverse.cu:43-198): .param file in, the reference's output files
out, the volume identical to the one the library computes from the same frame."""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

cv2 = pytest.importorskip("cv2")


def test_cli_end_to_end(rihvr, synthmod, tmp_path):
    cfg = synthmod.small_config(W=64, H=64, Nz=5, seed=7, zero_padding=0)
    img, b = synthmod.make_hologram(cfg, cache_dir=str(tmp_path / "cache"))
    frame = tmp_path / "holo_0007.tif"
    assert cv2.imwrite(str(frame), img)  # LZW-compressed, as OpenCV writes by default
    out = tmp_path / "out"
    out.mkdir()
    n_iter = 6
    param = tmp_path / "run.param"
    param.write_text(
        f"image_file 2001 {tmp_path}/holo_%04d.tif\n"
        f"output_path 2004 {out}/\n"
        "start_image 1002 7\n"
        f"start_plane 3001 {cfg.start_plane}\n"
        f"plane_stepsize 3002 {cfg.plane_stepsize}\n"
        f"num_planes 3003 {cfg.num_planes}\n"
        f"wavelength 3004 {cfg.wavelength}\n"
        f"resolution 3005 {cfg.resolution}\n"
        "zero_padding 3010 0\n"
        f"num_inverse_iterations 6001 {n_iter}\n"
        f"sparsity 6002 {cfg.regularization_param}\n"
        f"tv 6004 {cfg.regularization_TV_param}\n"
        f"tv_iterations 6005 {cfg.num_tv_iterations}\n"
        "output_planes 7001 true\n"
        "output_steps 7005 true\n")
    r = subprocess.run([rihvr.CLI_PATH, "-F", str(param), "-S", "0"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    for name in ("enh.tif", "initial_measured.tif", "estimate_initial.tif", "initial_residual.tif",
                 "estimate_final.tif", "residual_final.tif", "inverse_0000.tif", "inverse_phase_0004.tif",
                 "inverse_real_0002.tif", "inverse_imag_0003.tif", "cmb_xy.tif", "cmb_xz.tif", "cmb_yz.tif",
                 "inverse_voxels.csv", "all_metrics.csv"):
        assert (out / name).exists(), name
    assert cv2.imread(str(out / "cmb_xz.tif"), cv2.IMREAD_UNCHANGED).shape == (cfg.num_planes, 64)
    metrics = (out / "all_metrics.csv").read_text().strip().splitlines()
    assert metrics[0] == "it, f, sparsity, stepsize, total_backtracks" and len(metrics) == 1 + n_iter

    # the same reconstruction through the library
    p, _ = rihvr.read_param_file(str(param))
    raw, _ = rihvr.read_image(str(frame))
    bb = rihvr.preprocess(raw, p.zero_padding)
    assert np.abs(bb - b).max() <= 2 * np.finfo(np.float32).eps
    with rihvr.SparseCompressiveHolo(p, 64, 64) as s:
        s.setHologram(bb)
        s.iterate(n_iter)
        X = s.getVolume()
        log = s.iterations()
    rows = np.loadtxt(out / "inverse_voxels.csv", delimiter=",", skiprows=1, ndmin=2)
    I = np.abs(X) ** 2
    nz = np.argwhere(X != 0)
    assert rows.shape[0] == nz.shape[0]
    xi, yi, zi = rows[:, 0].astype(int), rows[:, 1].astype(int), rows[:, 2].astype(int)
    assert np.allclose(rows[:, 3], I[zi, yi, xi], rtol=1e-5)
    f_cli = float(metrics[-1].split(",")[1])
    assert abs(f_cli - log["f_x"][-1]) <= 1e-5 * abs(log["f_x"][-1]) + 1e-6


def test_cli_errors(rihvr, tmp_path):
    r = subprocess.run([rihvr.CLI_PATH], capture_output=True, text=True, timeout=60)
    assert r.returncode != 0 and "-F" in r.stdout
    bad = tmp_path / "bad.param"
    bad.write_text("image_file 2001 /nonexistent_%04d.tif\n")
    r = subprocess.run([rihvr.CLI_PATH, "-F", str(bad)], capture_output=True, text=True, timeout=60)
    assert r.returncode != 0


def _write_param(path, frame_pattern, out, cfg, n_iter, extra=""):
    path.write_text(
        f"image_file 2001 {frame_pattern}\n"
        f"output_path 2004 {out}/\n"
        "start_image 1002 7\n"
        f"start_plane 3001 {cfg.start_plane}\n"
        f"plane_stepsize 3002 {cfg.plane_stepsize}\n"
        f"num_planes 3003 {cfg.num_planes}\n"
        f"wavelength 3004 {cfg.wavelength}\n"
        f"resolution 3005 {cfg.resolution}\n"
        "zero_padding 3010 0\n"
        f"num_inverse_iterations 6001 {n_iter}\n"
        f"sparsity 6002 {cfg.regularization_param}\n"
        f"tv 6004 {cfg.regularization_TV_param}\n"
        f"tv_iterations 6005 {cfg.num_tv_iterations}\n"
        "output_planes 7001 false\n" + extra)


def test_cli_segmentation(rihvr, synthmod, tmp_path):
    """sparse-inverse-recon -G 1 segments the final volume in device memory;
    sparse-segmentation reads the voxel file as the reference's segmentation
    program does.  The first matches the library's segmentation of the same
    volume, the second the oracle's segmentation of the file's values, both
    to the byte in the three centroid files."""
    import oracle as O

    cfg = synthmod.small_config(W=64, H=64, Nz=8, seed=3, zero_padding=0)
    img, _ = synthmod.make_hologram(cfg, cache_dir=str(tmp_path / "cache"))
    frame = tmp_path / "holo_0007.tif"
    assert cv2.imwrite(str(frame), img)
    seg = "segment_min_area 5009 2\nsegment_min_intensity 5010 4\nsegment_close_size 5011 1\n"
    out = tmp_path / "out"
    out.mkdir()
    param = tmp_path / "run.param"
    _write_param(param, f"{tmp_path}/holo_%04d.tif", out, cfg, 10, seg)
    r = subprocess.run([rihvr.CLI_PATH, "-F", str(param), "-G", "1"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    names = ("centroids_0007.csv", "centroids_weighted_0007.csv", "centroids_verbose_0007.csv")
    for n in names:
        assert (out / n).exists(), n

    # the library on the same frame
    p, fp = rihvr.read_param_file(str(param))
    raw, _ = rihvr.read_image(str(frame))
    bb = rihvr.preprocess(raw, p.zero_padding)
    sp = rihvr.segment_params(min_intensity=fp.segment_min_intensity, close_size=fp.segment_close_size,
                              min_area=fp.segment_min_area)
    with rihvr.SparseCompressiveHolo(p, 64, 64) as s:
        s.setHologram(bb)
        s.iterate(10)
        objs, _ = s.segment(sp)
    assert len(objs) > 0
    lib_dir = tmp_path / "lib"
    lib_dir.mkdir()
    for n, (wt, vb) in zip(names, ((0, 0), (1, 0), (0, 1))):
        rihvr.write_centroids(str(lib_dir / n), objs, weighted=wt, verbose=vb)
        assert (lib_dir / n).read_text() == (out / n).read_text(), n

    # the reference's file round trip: voxel file -> segmentation program
    seg_out = tmp_path / "seg"
    seg_out.mkdir()
    (seg_out / "inverse_voxels_0007.csv").write_text((out / "inverse_voxels.csv").read_text())
    param2 = tmp_path / "seg.param"
    _write_param(param2, f"{tmp_path}/holo_%04d.tif", seg_out, cfg, 10, seg)
    r = subprocess.run([rihvr.SEGMENT_CLI_PATH, "-F", str(param2)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    import ctypes

    libc = ctypes.CDLL(None)
    libc.strtof.restype = ctypes.c_float
    libc.strtof.argtypes = [ctypes.c_char_p, ctypes.c_void_p]
    rows = np.loadtxt(seg_out / "inverse_voxels_0007.csv", delimiter=",", skiprows=1, ndmin=2, dtype=str)
    I = np.zeros((cfg.num_planes, 64, 64), np.float32)
    for x, y, z, v in rows:
        I[int(z), int(y), int(x)] = libc.strtof(v.strip().encode(), None)  # fscanf's direct decimal to float
    ref, _ = O.segment(I, fp.segment_min_intensity, fp.segment_close_size, fp.segment_min_area, 1)
    orc_dir = tmp_path / "orc"
    orc_dir.mkdir()
    for n, (wt, vb) in zip(names, ((0, 0), (1, 0), (0, 1))):
        rihvr.write_centroids(str(orc_dir / n), ref.astype(rihvr.OBJECT_DTYPE), weighted=wt, verbose=vb)
        assert (orc_dir / n).read_text() == (seg_out / n).read_text(), n


def _circular_u8_diff(a, b):
    d = np.abs(a.astype(np.int16) - b.astype(np.int16))
    return np.minimum(d, 256 - d)


def test_cli_images_match_the_reference_scaling(rihvr, synthmod, tmp_path):
    """The 8-bit plane images (inverse_XXXX, _phase_, _real_, _imag_) and the
    max projections (cmb_xy/xz/yz) the driver writes, against the restatement
    of savePlanes and saveProjections (oracle/outputs.py) on the same volume.
    OpenCV's own magnitude and phase (a fast arctangent) feed the restatement;
    the driver uses sqrt and atan2 in float, so a pixel may sit one level away
    where a value falls within rounding of a level boundary."""
    import outputs as OUT

    cfg = synthmod.small_config(W=64, H=64, Nz=6, seed=11, zero_padding=0)
    img, _ = synthmod.make_hologram(cfg, cache_dir=str(tmp_path / "cache"))
    frame = tmp_path / "holo_0007.tif"
    assert cv2.imwrite(str(frame), img)
    out = tmp_path / "out"
    out.mkdir()
    param = tmp_path / "run.param"
    _write_param(param, f"{tmp_path}/holo_%04d.tif", out, cfg, 12)
    param.write_text(param.read_text().replace("output_planes 7001 false", "output_planes 7001 true"))
    r = subprocess.run([rihvr.CLI_PATH, "-F", str(param)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    p, _ = rihvr.read_param_file(str(param))
    raw, _ = rihvr.read_image(str(frame))
    with rihvr.SparseCompressiveHolo(p, 64, 64) as s:
        s.setHologram(rihvr.preprocess(raw, p.zero_padding))
        s.iterate(12)
        X = s.getVolume()
    assert np.count_nonzero(X) > 0
    planes = OUT.save_planes(X)
    for kind, tag in (("mag", ""), ("phase", "_phase"), ("real", "_real"), ("imag", "_imag")):
        got = np.stack([cv2.imread(str(out / f"inverse{tag}_{z:04d}.tif"), cv2.IMREAD_UNCHANGED)
                        for z in range(cfg.num_planes)])
        d = _circular_u8_diff(got, planes[kind]) if kind == "phase" else np.abs(
            got.astype(np.int16) - planes[kind].astype(np.int16))
        assert d.max() <= 1, (kind, int(d.max()))
        assert np.mean(d != 0) < 2e-3, (kind, float(np.mean(d != 0)))
    proj = OUT.save_projections(X)
    for tag in ("xy", "xz", "yz"):
        got = cv2.imread(str(out / f"cmb_{tag}.tif"), cv2.IMREAD_UNCHANGED)
        assert got.shape == proj[tag].shape
        d = np.abs(got.astype(np.int16) - proj[tag].astype(np.int16))
        assert d.max() <= 1 and np.mean(d != 0) < 2e-3, (tag, int(d.max()))
