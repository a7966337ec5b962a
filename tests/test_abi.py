"""CPU checks of the C ABI library: it loads, exports every entry point the
header declares, and the host-only logic (defaults, the .param reader, the
float plane list, argument validation) behaves like the reference's."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "rihvr.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(rihvr_[a-z_0-9]+)\s*\(", text)))


def test_header_declares_expected_symbols(rihvr):
    assert set(declared_functions()) == set(rihvr.EXPORTED)


def test_library_exports_every_declared_symbol(rihvr):
    L = rihvr.load_library()
    for name in declared_functions():
        assert hasattr(L, name), name


def test_defaults_match_reference(rihvr):
    p = rihvr.default_params()
    # HoloUi::HoloUi (holo_ui.cpp:10-62)
    assert p.num_inverse_iterations == 500 and p.num_tv_iterations == 5
    assert np.isclose(p.regularization_param, 0.01) and p.regularization_TV_param == 0.0
    assert p.num_planes == 256 and p.zero_padding == 256
    assert p.mode == 7 and p.faithful == 1 and p.max_backtracks == 2


def test_param_file_parsing(rihvr, tmp_path):
    f = tmp_path / "run.param"
    f.write_text(
        "% comment line\n"
        "# another\n"
        "image_file 2001 /data/holo_%04d.tif\n"
        "output_path 2004 /tmp/out\n"
        "start_image 1002 7\n"
        "start_plane 3001 2500\n"
        "plane_stepsize 3002 2\n"
        "num_planes 3003 1000\n"
        "wavelength 3004 0.632\n"
        "resolution 3005 1.1\n"
        "zero_padding 3010 0\n"
        "\n"
        "num_inverse_iterations 6001 100\n"
        "sparsity 6002 0.15\n"
        "tv 6004 0.1\n"
        "tv_iterations 6005 5\n"
        "output_planes 7001 true\n"
        "output_steps 7005 0\n")
    p, fp = rihvr.read_param_file(str(f))
    assert p.start_plane == 2500 and p.plane_stepsize == 2 and p.num_planes == 1000
    assert np.float32(p.wavelength) == np.float32(0.632) and np.float32(p.resolution) == np.float32(1.1)
    assert p.zero_padding == 0 and p.num_inverse_iterations == 100 and p.num_tv_iterations == 5
    assert np.float32(p.regularization_param) == np.float32(0.15)
    assert fp.image_filename.decode() == "/data/holo_%04d.tif"
    assert fp.output_path.decode() == "/tmp/out" and fp.start_image == 7
    assert fp.output_planes == 1 and fp.output_steps == 0


def test_param_file_errors(rihvr, tmp_path):
    with pytest.raises(rihvr.RihvrError) as e:
        rihvr.read_param_file(str(tmp_path / "missing.param"))
    assert e.value.code == rihvr.ERR_BAD_FILENAME
    f = tmp_path / "bad.param"
    f.write_text("bogus 9999 1\n")
    with pytest.raises(rihvr.RihvrError) as e:
        rihvr.read_param_file(str(f))
    assert e.value.code == rihvr.ERR_INVALID_FILE


def test_plane_list_is_float(rihvr):
    p = rihvr.default_params()
    p.start_plane, p.plane_stepsize, p.num_planes = 0.1, 0.3, 50
    z = rihvr.plane_list(p)
    expect = np.array([np.float32(np.float32(0.1) + np.float32(np.float32(i) * np.float32(0.3)))
                       for i in range(50)], np.float32).astype(np.float64)
    assert np.array_equal(z, expect)


def test_create_validates_arguments_before_touching_the_gpu(rihvr):
    L = rihvr.load_library()
    h = ctypes.c_void_p()
    p = rihvr.default_params()
    p.num_planes = 4
    # sides must be even, 16..4096, with prime factors 2, 3, 5 and 7 only
    for w, hh in ((88, 88), (64, 22), (15, 16), (8, 8), (5000, 64), (64, 4802)):
        assert L.rihvr_create(ctypes.byref(p), w, hh, ctypes.byref(h)) == rihvr.ERR_UNSUPPORTED_SIZE, (w, hh)
    p.mode = 4
    assert L.rihvr_create(ctypes.byref(p), 64, 64, ctypes.byref(h)) == rihvr.ERR_UNKNOWN_MODE
    p.mode = 7
    p.num_tv_iterations = 50
    assert L.rihvr_create(ctypes.byref(p), 64, 64, ctypes.byref(h)) == rihvr.ERR_INVALID_ARGUMENT
    assert h.value is None


def test_status_strings(rihvr):
    L = rihvr.load_library()
    assert L.rihvr_status_string(0) == b"ok"
    assert L.rihvr_status_string(7) == b"invalid argument"
    assert L.rihvr_status_string(22) == b"unsupported size"


def test_batch_validates_before_touching_contexts(rihvr):
    """rihvr_reconstruct_batch rejects empty batches and repeated contexts
    without dereferencing them (the pointers below are never valid)."""
    import ctypes

    L = rihvr.load_library()
    fake = (ctypes.c_void_p * 2)(ctypes.c_void_p(4096), ctypes.c_void_p(4096))
    holo = (ctypes.c_void_p * 2)(ctypes.c_void_p(8192), ctypes.c_void_p(8192))
    assert L.rihvr_reconstruct_batch(fake, 0, holo, 0, None, None) == rihvr.ERR_INVALID_ARGUMENT
    assert L.rihvr_reconstruct_batch(None, 1, holo, 0, None, None) == rihvr.ERR_INVALID_ARGUMENT
    assert L.rihvr_reconstruct_batch(fake, 2, holo, 0, None, None) == rihvr.ERR_INVALID_ARGUMENT
    assert b"twice" in L.rihvr_last_error()
    nul = (ctypes.c_void_p * 1)(None)
    assert L.rihvr_reconstruct_batch(nul, 1, holo, 0, None, None) == rihvr.ERR_INVALID_ARGUMENT


def test_batch_mode_setting(rihvr):
    """rihvr_set_batch_mode takes 0, 1 or 2 only; a rejected batch ran no
    frame as a combined graph."""
    L = rihvr.load_library()
    assert L.rihvr_set_batch_mode(3) == rihvr.ERR_INVALID_ARGUMENT
    assert L.rihvr_set_batch_mode(-1) == rihvr.ERR_INVALID_ARGUMENT
    assert L.rihvr_set_batch_mode(1) == rihvr.OK
    assert L.rihvr_reconstruct_batch(None, 1, None, 0, None, None) == rihvr.ERR_INVALID_ARGUMENT
    assert L.rihvr_batch_last_combined() == 0
    assert L.rihvr_set_batch_mode(2) == rihvr.OK
    assert L.rihvr_set_batch_mode(0) == rihvr.OK


def test_header_compiles_as_plain_c(tmp_path):
    """include/rihvr.h is a C header: a C99 translation unit that includes it
    and names its types builds with -pedantic -Werror."""
    import shutil
    import subprocess

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    src = tmp_path / "use.c"
    src.write_text('#include "rihvr.h"\n'
                   "static int sum(void* u, void* d, long long n, int t, int dev) {\n"
                   "  (void)u; (void)d; (void)n; (void)t; (void)dev; return 0;\n}\n"
                   "int use(void) {\n"
                   "  rihvr_params p; rihvr_iter_record r; rihvr_slab_reducer red = {sum, 0, 1};\n"
                   "  (void)p; (void)r; (void)red; return RIHVR_OK + RIHVR_DTYPE_F64;\n}\n")
    res = subprocess.run([cc, "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", f"-I{os.path.dirname(HEADER)}",
                          "-c", str(src), "-o", str(tmp_path / "use.o")], capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
