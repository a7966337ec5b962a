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
