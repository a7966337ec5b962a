"""B200-native reconstruction core for digital inline holography.

Python mirror of RIHVR's reconstruction entry points (``umnholo::
SparseCompressiveHolo``, src/core/sparse_compressive_holo.h:30-96, and the
``Parameters``/``HoloUi`` pair, src/core/holo_ui.h:83-214) over the C ABI in
``include/rihvr.h``.  The compute runs in ``librihvr_b200.so`` (hand-written
sm_100a CUDA); there is no fallback: loading fails loudly if the library is
missing or no GPU is visible.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "librihvr_b200.so")
CLI_PATH = os.path.join(_HERE, "sparse-inverse-recon")
SEGMENT_CLI_PATH = os.path.join(_HERE, "sparse-segmentation")

# status codes (include/rihvr.h)
OK = 0
ERR_INVALID_ARGUMENT = 7
ERR_UNKNOWN_MODE = 6
ERR_MISSING_DATA = 3
ERR_INVALID_STATE = 4
ERR_INVALID_FILE = 9
ERR_INVALID_DATA = 10
ERR_BAD_FILENAME = 2
ERR_OUT_OF_MEMORY = 5
ERR_CUDA = 20
ERR_NO_DEVICE = 21
ERR_UNSUPPORTED_SIZE = 22

MODE_FASTA_L1 = 5
MODE_FASTA_FUSED_LASSO = 6
MODE_FASTA_FUSED_LASSO_2D = 7
STORE_F32, STORE_BF16, STORE_F16 = 0, 1, 2

SUPPORTED_SIDES = (32, 48, 64, 128, 256, 384, 512, 640, 768, 1024, 2304)


class RihvrParams(ctypes.Structure):
    """``rihvr_params`` (include/rihvr.h); first block = umnholo::Parameters."""
    _fields_ = [
        ("start_plane", ctypes.c_float),
        ("plane_stepsize", ctypes.c_float),
        ("num_planes", ctypes.c_int),
        ("wavelength", ctypes.c_float),
        ("resolution", ctypes.c_float),
        ("zero_padding", ctypes.c_int),
        ("num_inverse_iterations", ctypes.c_int),
        ("regularization_param", ctypes.c_float),
        ("regularization_TV_param", ctypes.c_float),
        ("num_tv_iterations", ctypes.c_int),
        ("mode", ctypes.c_int),
        ("storage", ctypes.c_int),
        ("faithful", ctypes.c_int),
        ("max_backtracks", ctypes.c_int),
        ("initial_step", ctypes.c_double),
        ("record_objective", ctypes.c_int), ("autotune", ctypes.c_int),
    ]


class IterRecord(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in
                ("f_prox", "f_resid_prox", "lim", "ratio", "t", "beta", "f_x", "f_resid_x", "l1_x", "tv_x",
                 "restart_sum")] + [("backtracks", ctypes.c_int), ("restarted", ctypes.c_int)]


ITER_DTYPE = np.dtype([(n, "f8") for n in ("f_prox", "f_resid_prox", "lim", "ratio", "t", "beta", "f_x",
                                             "f_resid_x", "l1_x", "tv_x", "restart_sum")]
                      + [("backtracks", "i4"), ("restarted", "i4")])


class FileParams(ctypes.Structure):
    _fields_ = [
        ("image_filename", ctypes.c_char * 4096),
        ("image_path", ctypes.c_char * 4096),
        ("image_formatted_name", ctypes.c_char * 4096),
        ("output_path", ctypes.c_char * 4096),
        ("background_filename", ctypes.c_char * 4096),
        ("remove_background", ctypes.c_int),
        ("image_count", ctypes.c_int),
        ("start_image", ctypes.c_int),
        ("roi_x", ctypes.c_int), ("roi_y", ctypes.c_int), ("roi_size", ctypes.c_int),
        ("roi_rect_x", ctypes.c_int), ("roi_rect_y", ctypes.c_int), ("roi_rect_w", ctypes.c_int),
        ("roi_rect_h", ctypes.c_int),
        ("output_planes", ctypes.c_int),
        ("output_steps", ctypes.c_int),
        ("segment_min_area", ctypes.c_int),
        ("segment_min_intensity", ctypes.c_double),
        ("segment_close_size", ctypes.c_int),
        ("background_start", ctypes.c_int),
        ("background_end", ctypes.c_int),
        ("use_median_background", ctypes.c_int),
    ]


class SegmentParams(ctypes.Structure):
    """rihvr_segment_params: segment_min_intensity (5010), segment_close_size
    (5011), segment_min_area (5009) and the neighbourhood switch."""
    _fields_ = [
        ("min_intensity", ctypes.c_double),
        ("close_size", ctypes.c_int),
        ("min_area", ctypes.c_int),
        ("faithful", ctypes.c_int),
    ]


class SegmentInfo(ctypes.Structure):
    _fields_ = [
        ("max_intensity", ctypes.c_double),
        ("threshold", ctypes.c_double),
        ("closed_voxels", ctypes.c_longlong),
        ("labelled_objects", ctypes.c_longlong),
        ("strel_size", ctypes.c_int),
        ("kernel_launches", ctypes.c_longlong),
    ]


# rihvr_object, one row per segmented object (ObjectCloud::writeCentroids fields)
OBJECT_DTYPE = np.dtype([
    ("x", "f4"), ("y", "f4"), ("z", "f4"), ("wx", "f4"), ("wy", "f4"), ("wz", "f4"),
    ("num_voxels", "i4"), ("max_value", "f4"), ("mean_value", "f4"),
    ("xmin", "i4"), ("xmax", "i4"), ("ymin", "i4"), ("ymax", "i4"), ("zmin", "i4"), ("zmax", "i4"),
])


# every symbol include/rihvr.h declares
EXPORTED = (
    "rihvr_params_default", "rihvr_read_param_file", "rihvr_plane_list", "rihvr_create", "rihvr_destroy",
    "rihvr_debug_fail_allocations_after", "rihvr_set_hologram", "rihvr_reconstruct", "rihvr_reconstruct_batch", "rihvr_set_batch_mode",
    "rihvr_batch_last_combined", "rihvr_autotune", "rihvr_tuning", "rihvr_reset",
    "rihvr_set_initial_volume",
    "rihvr_iterate",
    "rihvr_iterate_timed",
    "rihvr_iteration_count", "rihvr_objective", "rihvr_get_iterations", "rihvr_get_plane", "rihvr_get_volume",
    "rihvr_get_volume_ptr", "rihvr_save_state", "rihvr_load_state",
    "rihvr_create_slab", "rihvr_slab_range", "rihvr_slab_iterate",
    "rihvr_get_estimate", "rihvr_get_residual", "rihvr_forward", "rihvr_adjoint", "rihvr_prox_step",
    "rihvr_adjoint_noalloc", "rihvr_sparsity", "rihvr_initial_estimate", "rihvr_lipschitz",
    "rihvr_set_hologram_frame", "rihvr_get_hologram", "rihvr_background_mean", "rihvr_background_median5",
    "rihvr_background_median5_frames",
    "rihvr_read_image", "rihvr_write_tiff8", "rihvr_write_png8", "rihvr_preprocess", "rihvr_io_error",
    "rihvr_segment_params_default", "rihvr_segment", "rihvr_segment_intensity", "rihvr_write_centroids",
    "rihvr_unet_create", "rihvr_unet_destroy", "rihvr_unet_param_count", "rihvr_unet_get_params",
    "rihvr_unet_set_params", "rihvr_unet_predict", "rihvr_unet_gradients", "rihvr_unet_train_step",
    "rihvr_unet_launch_count", "rihvr_unet_activation_bits", "rihvr_backpropagate", "rihvr_warm_start",
    "rihvr_set_profiling", "rihvr_kernel_times", "rihvr_get_stream", "rihvr_launch_count", "rihvr_device_bytes",
    "rihvr_status_string", "rihvr_last_error",
)

_lib = None


class RihvrError(RuntimeError):
    def __init__(self, code: int, where: str):
        L = _lib
        msg = ""
        if L is not None:
            msg = (L.rihvr_last_error() or b"").decode(errors="replace")
            name = (L.rihvr_status_string(code) or b"").decode()
        else:
            name = str(code)
        super().__init__(f"{where}: status {code} ({name}) {msg}".strip())
        self.code = code


def load_library(path: str = LIB_PATH):
    """Load the native library (built in-tree by build.py); raises if missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"native library missing: {path} (run build.py); there is no fallback path")
    L = ctypes.CDLL(path)
    vp, ip, dp, fp = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.POINTER(ctypes.c_float)
    P = ctypes.POINTER
    L.rihvr_params_default.argtypes = [P(RihvrParams)]
    L.rihvr_read_param_file.argtypes = [ctypes.c_char_p, P(RihvrParams), P(FileParams)]
    L.rihvr_plane_list.argtypes = [P(RihvrParams), P(ctypes.c_double)]
    L.rihvr_create.argtypes = [P(RihvrParams), ip, ip, P(vp)]
    L.rihvr_create_slab.argtypes = [P(RihvrParams), ip, ip, ip, ip, P(vp)]
    L.rihvr_slab_range.argtypes = [vp, P(ctypes.c_int), P(ctypes.c_int)]
    L.rihvr_slab_iterate.argtypes = [P(vp), ip, ip, vp]
    L.rihvr_destroy.argtypes = [vp]
    L.rihvr_debug_fail_allocations_after.argtypes = [ip]
    L.rihvr_destroy.restype = None
    L.rihvr_set_hologram.argtypes = [vp, vp, ip]
    L.rihvr_set_hologram_frame.argtypes = [vp, vp, ip, ip, ip, vp, P(FileParams), ip]
    L.rihvr_get_hologram.argtypes = [vp, vp, ip]
    L.rihvr_background_mean.argtypes = [vp, ip, ip, ip, ip, ip, vp, P(ctypes.c_double)]
    L.rihvr_background_median5.argtypes = [vp, ip, ip, ip, ip, ip, vp]
    L.rihvr_background_median5_frames.argtypes = [ip, P(ctypes.c_int)]
    L.rihvr_reconstruct.argtypes = [vp, P(ctypes.c_double)]
    L.rihvr_reconstruct_batch.argtypes = [P(vp), ip, P(vp), ip, P(ctypes.c_double), P(ctypes.c_int)]
    L.rihvr_set_batch_mode.argtypes = [ip]
    L.rihvr_batch_last_combined.argtypes = []
    L.rihvr_autotune.argtypes = [vp, P(ctypes.c_double)]
    L.rihvr_tuning.argtypes = [vp, P(ctypes.c_int), P(ctypes.c_int), P(ctypes.c_int), P(ctypes.c_int),
                               P(ctypes.c_int), P(ctypes.c_int)]
    L.rihvr_reset.argtypes = [vp]
    L.rihvr_set_initial_volume.argtypes = [vp, vp, ip]
    L.rihvr_iterate.argtypes = [vp, ip]
    L.rihvr_iterate_timed.argtypes = [vp, ip, fp]
    L.rihvr_iteration_count.argtypes = [vp]
    L.rihvr_objective.argtypes = [vp, P(ctypes.c_double), P(ctypes.c_double)]
    L.rihvr_get_iterations.argtypes = [vp, vp, ip, P(ctypes.c_int)]
    for n in ("rihvr_get_plane",):
        getattr(L, n).argtypes = [vp, ip, vp, ip]
    for n in ("rihvr_get_volume", "rihvr_get_estimate", "rihvr_get_residual"):
        getattr(L, n).argtypes = [vp, vp, ip]
    L.rihvr_get_volume_ptr.argtypes = [vp, P(vp), P(ctypes.c_int)]
    L.rihvr_save_state.argtypes = [vp, ctypes.c_char_p]
    L.rihvr_load_state.argtypes = [vp, ctypes.c_char_p]
    L.rihvr_forward.argtypes = [vp, vp, vp, ip]
    L.rihvr_adjoint.argtypes = [vp, vp, vp, ip]
    L.rihvr_prox_step.argtypes = [vp, vp, vp, dp, vp, P(ctypes.c_double), ip]
    L.rihvr_adjoint_noalloc.argtypes = [P(RihvrParams), ip, ip, vp, vp, vp]
    L.rihvr_sparsity.argtypes = [vp, P(ctypes.c_double)]
    L.rihvr_lipschitz.argtypes = [vp, ip, ctypes.c_ulonglong, P(ctypes.c_double), vp]
    L.rihvr_read_image.argtypes = [ctypes.c_char_p, vp, P(ctypes.c_int), P(ctypes.c_int), P(ctypes.c_int)]
    L.rihvr_write_tiff8.argtypes = [ctypes.c_char_p, vp, ip, ip]
    L.rihvr_write_png8.argtypes = [ctypes.c_char_p, vp, ip, ip]
    L.rihvr_preprocess.argtypes = [vp, ip, ip, vp, P(FileParams), ip, vp, P(ctypes.c_int), P(ctypes.c_int)]
    L.rihvr_io_error.restype = ctypes.c_char_p
    L.rihvr_segment_params_default.argtypes = [P(SegmentParams)]
    L.rihvr_segment.argtypes = [vp, P(SegmentParams), vp, ip, P(ctypes.c_int), P(SegmentInfo)]
    L.rihvr_segment_intensity.argtypes = [vp, ip, ip, ip, ip, P(SegmentParams), vp, ip, P(ctypes.c_int),
                                          P(SegmentInfo)]
    L.rihvr_write_centroids.argtypes = [ctypes.c_char_p, vp, ip, ip, ip]
    L.rihvr_unet_create.argtypes = [ip, ip, ip, ctypes.c_ulonglong, P(vp)]
    L.rihvr_unet_destroy.argtypes = [vp]
    L.rihvr_unet_destroy.restype = None
    L.rihvr_unet_param_count.argtypes = [vp]
    L.rihvr_unet_param_count.restype = ctypes.c_longlong
    L.rihvr_unet_get_params.argtypes = [vp, vp]
    L.rihvr_unet_set_params.argtypes = [vp, vp]
    L.rihvr_unet_predict.argtypes = [vp, vp, vp]
    L.rihvr_unet_gradients.argtypes = [vp, vp, vp, vp, P(ctypes.c_double)]
    L.rihvr_unet_train_step.argtypes = [vp, vp, vp, ctypes.c_float, P(ctypes.c_double)]
    L.rihvr_unet_launch_count.argtypes = [vp]
    L.rihvr_unet_launch_count.restype = ctypes.c_longlong
    L.rihvr_unet_activation_bits.argtypes = [vp]
    L.rihvr_backpropagate.argtypes = [vp, vp, ip]
    L.rihvr_warm_start.argtypes = [vp, vp]
    L.rihvr_initial_estimate.argtypes = [vp, vp, ip]
    L.rihvr_set_profiling.argtypes = [vp, ip]
    L.rihvr_kernel_times.argtypes = [vp, P(ctypes.c_char_p), P(ctypes.c_double), P(ctypes.c_int), ip,
                                     P(ctypes.c_int)]
    L.rihvr_get_stream.argtypes = [vp]
    L.rihvr_get_stream.restype = vp
    L.rihvr_launch_count.argtypes = [vp]
    L.rihvr_launch_count.restype = ctypes.c_longlong
    L.rihvr_device_bytes.argtypes = [vp]
    L.rihvr_device_bytes.restype = ctypes.c_size_t
    L.rihvr_status_string.argtypes = [ip]
    L.rihvr_status_string.restype = ctypes.c_char_p
    L.rihvr_last_error.restype = ctypes.c_char_p
    _lib = L
    return L


def _check(rc: int, where: str):
    if rc != OK:
        raise RihvrError(rc, where)


def default_params() -> RihvrParams:
    """HoloUi defaults (holo_ui.cpp:10-62) plus mode 7 / FP32 / faithful."""
    p = RihvrParams()
    _check(load_library().rihvr_params_default(ctypes.byref(p)), "rihvr_params_default")
    return p


def read_param_file(path: str):
    """HoloUi::readFile (holo_ui.cpp:171-486) -> (RihvrParams, FileParams)."""
    p = default_params()
    f = FileParams()
    _check(load_library().rihvr_read_param_file(path.encode(), ctypes.byref(p), ctypes.byref(f)),
           "rihvr_read_param_file")
    return p, f


def plane_list(p: RihvrParams) -> np.ndarray:
    z = np.empty(p.num_planes, np.float64)
    _check(load_library().rihvr_plane_list(ctypes.byref(p), z.ctypes.data_as(ctypes.POINTER(ctypes.c_double))),
           "rihvr_plane_list")
    return z


def adjoint_noalloc(params: RihvrParams, width: int, height: int, residual_dev: int, volume_dev: int,
                    stream: int = 0):
    """Allocation-free adjoint over caller-owned device buffers (raw pointers):
    for callers that cannot allocate device memory.  Asynchronous on `stream`."""
    _check(load_library().rihvr_adjoint_noalloc(ctypes.byref(params), int(width), int(height),
                                                 ctypes.c_void_p(residual_dev), ctypes.c_void_p(volume_dev),
                                                 ctypes.c_void_p(stream)), "rihvr_adjoint_noalloc")


def segment_params(**kw) -> SegmentParams:
    """Segmentation settings: the HoloUi defaults (holo_ui.cpp:44-46) with
    any field overridden by keyword."""
    sp = SegmentParams()
    _check(load_library().rihvr_segment_params_default(ctypes.byref(sp)), "rihvr_segment_params_default")
    for k, v in kw.items():
        setattr(sp, k, v)
    return sp


def _segment_call(call, where: str, max_objects: int):
    """Run a segmentation entry point, growing the object buffer once if needed."""
    for _ in range(2):
        out = np.zeros(max(1, max_objects), OBJECT_DTYPE)
        n = ctypes.c_int()
        info = SegmentInfo()
        rc = call(out.ctypes.data, len(out), ctypes.byref(n), ctypes.byref(info))
        if rc == ERR_INVALID_ARGUMENT and n.value > len(out):
            max_objects = n.value
            continue
        _check(rc, where)
        info_d = {k: getattr(info, k) for k, _ in SegmentInfo._fields_}
        return out[:n.value].copy(), info_d
    raise RihvrError(ERR_INVALID_ARGUMENT, where)


def segment_intensity(intensity, sp: SegmentParams | None = None, max_objects: int = 1 << 16):
    """Segment a stack of voxel intensities (num_planes x height x width: a
    numpy array, or a CUDA torch tensor used in place).  Returns (objects as
    an OBJECT_DTYPE array in the reference's order, info dict)."""
    sp = sp or segment_params()
    if hasattr(intensity, "is_cuda") and intensity.is_cuda:
        t = intensity.contiguous()
        if t.dtype.itemsize != 4 or t.dim() != 3:
            raise ValueError("expected a float32 tensor of shape (planes, height, width)")
        nz, h, w = t.shape
        ptr, dev = t.data_ptr(), 1
        keep = t
    else:
        keep = np.ascontiguousarray(intensity, dtype=np.float32)
        if keep.ndim != 3:
            raise ValueError("expected shape (planes, height, width)")
        nz, h, w = keep.shape
        ptr, dev = keep.ctypes.data, 0
    L = load_library()
    res = _segment_call(lambda o, m, n, i: L.rihvr_segment_intensity(ctypes.c_void_p(ptr), w, h, nz, dev,
                                                                     ctypes.byref(sp), o, m, n, i),
                        "rihvr_segment_intensity", max_objects)
    del keep
    return res


def write_centroids(path: str, objects: np.ndarray, weighted: bool = False, verbose: bool = False):
    """ObjectCloud::writeCentroids (object_cloud.cu:408-470)."""
    objs = np.ascontiguousarray(objects, dtype=OBJECT_DTYPE)
    _check(load_library().rihvr_write_centroids(path.encode(), objs.ctypes.data if len(objs) else None, len(objs),
                                                int(bool(weighted)), int(bool(verbose))), "rihvr_write_centroids")


def _dev_complex(a):
    """A CUDA complex64 tensor holding `a` (numpy array or tensor), contiguous."""
    import torch

    if isinstance(a, torch.Tensor):
        t = a.to(device="cuda", dtype=torch.complex64)
    else:
        t = torch.from_numpy(np.ascontiguousarray(a, dtype=np.complex64)).cuda()
    return t.contiguous()


class UNet:
    """The learned warm start (rihvr_unet_*): a 3-D U-Net mapping the
    back-propagated volume xbp = t A^H b (depth x height x width complex) to an
    initial iterate x0 = g * alpha * xbp.  Volumes may be numpy arrays or CUDA
    tensors; results are CUDA complex64 tensors."""

    def __init__(self, depth: int, height: int, width: int, seed: int = 0):
        self._L = load_library()
        self._h = ctypes.c_void_p()
        _check(self._L.rihvr_unet_create(int(depth), int(height), int(width), int(seed), ctypes.byref(self._h)),
               "rihvr_unet_create")
        self.shape = (depth, height, width)

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.destroy()

    def destroy(self):
        if self._h:
            self._L.rihvr_unet_destroy(self._h)
            self._h = ctypes.c_void_p()

    def param_count(self) -> int:
        return int(self._L.rihvr_unet_param_count(self._h))

    def params(self) -> np.ndarray:
        out = np.empty(self.param_count(), np.float32)
        _check(self._L.rihvr_unet_get_params(self._h, _ptr(out)), "rihvr_unet_get_params")
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.size != self.param_count():
            raise ValueError(f"{p.size} parameters, the network has {self.param_count()}")
        _check(self._L.rihvr_unet_set_params(self._h, _ptr(p)), "rihvr_unet_set_params")

    def activation_bits(self) -> int:
        """16 when predict runs with BF16 activations (tcgen05 at every
        level), 32 on the FP32 path."""
        return int(self._L.rihvr_unet_activation_bits(self._h))

    def predict(self, xbp):
        import torch

        a = _dev_complex(xbp)
        out = torch.empty_like(a)
        _check(self._L.rihvr_unet_predict(self._h, ctypes.c_void_p(a.data_ptr()), ctypes.c_void_p(out.data_ptr())),
               "rihvr_unet_predict")
        return out

    def gradients(self, xbp, xstar):
        a, b = _dev_complex(xbp), _dev_complex(xstar)
        g = np.empty(self.param_count(), np.float32)
        loss = ctypes.c_double()
        _check(self._L.rihvr_unet_gradients(self._h, ctypes.c_void_p(a.data_ptr()), ctypes.c_void_p(b.data_ptr()),
                                            _ptr(g), ctypes.byref(loss)), "rihvr_unet_gradients")
        return loss.value, g

    def train_step(self, xbp, xstar, lr: float = 1e-3) -> float:
        a, b = _dev_complex(xbp), _dev_complex(xstar)
        loss = ctypes.c_double()
        _check(self._L.rihvr_unet_train_step(self._h, ctypes.c_void_p(a.data_ptr()), ctypes.c_void_p(b.data_ptr()),
                                             float(lr), ctypes.byref(loss)), "rihvr_unet_train_step")
        return loss.value

    def save(self, path: str):
        np.save(path, self.params())

    def load(self, path: str):
        self.set_params(np.load(path))


def reconstruct_batch(solvers, holograms):
    """Run several frames at once (rihvr_reconstruct_batch): frame i sets
    solvers[i]'s hologram to holograms[i] and reconstructs from x = 0.  Returns
    the final objectives; raises RihvrError with the first failing frame."""
    n = len(solvers)
    if n != len(holograms):
        raise ValueError("one hologram per solver")
    bufs = []
    for s, b in zip(solvers, holograms):
        b = np.ascontiguousarray(b, dtype=np.float32)
        if b.shape != (s.height, s.width):
            raise ValueError(f"hologram shape {b.shape} != {(s.height, s.width)}")
        bufs.append(b)
    ctxs = (ctypes.c_void_p * n)(*[s._h for s in solvers])
    ptrs = (ctypes.c_void_p * n)(*[b.ctypes.data for b in bufs])
    f = (ctypes.c_double * n)()
    st = (ctypes.c_int * n)()
    _check(load_library().rihvr_reconstruct_batch(ctxs, n, ptrs, 0, f, st), "rihvr_reconstruct_batch")
    return [f[i] for i in range(n)]


def set_batch_mode(mode: int):
    """rihvr_set_batch_mode: 0 = one host thread and stream per frame
    (default), 1 = one graph launch per iteration for all frames, 2 = one graph
    launch for the whole solves of all frames."""
    _check(load_library().rihvr_set_batch_mode(int(mode)), "rihvr_set_batch_mode")


def batch_last_combined() -> int:
    """How the last reconstruct_batch on this thread ran its frames
    (rihvr_batch_last_combined): 1 one graph launch per iteration, 2 one graph
    launch for the whole solves, 0 one loop per frame."""
    return int(load_library().rihvr_batch_last_combined())


def _io_check(rc: int, where: str):
    if rc != OK:
        msg = (load_library().rihvr_io_error() or b"").decode(errors="replace")
        raise RihvrError(rc, f"{where}: {msg}")


def read_image(path: str):
    """Hologram::read: (pixels float32 [H, W] as stored, bits per sample)."""
    L = load_library()
    w, h, bits = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    _io_check(L.rihvr_read_image(path.encode(), None, ctypes.byref(w), ctypes.byref(h), ctypes.byref(bits)),
              "rihvr_read_image")
    out = np.empty((h.value, w.value), np.float32)
    _io_check(L.rihvr_read_image(path.encode(), _ptr(out), ctypes.byref(w), ctypes.byref(h), None),
              "rihvr_read_image")
    return out, bits.value


def write_tiff8(path: str, img: np.ndarray):
    img = np.ascontiguousarray(img, dtype=np.uint8)
    _io_check(load_library().rihvr_write_tiff8(path.encode(), _ptr(img), img.shape[1], img.shape[0]),
              "rihvr_write_tiff8")


def write_png8(path: str, img: np.ndarray):
    img = np.ascontiguousarray(img, dtype=np.uint8)
    _io_check(load_library().rihvr_write_png8(path.encode(), _ptr(img), img.shape[1], img.shape[0]),
              "rihvr_write_png8")


_SAMPLE_BITS = {np.dtype(np.uint8): 8, np.dtype(np.uint16): 16, np.dtype(np.float32): 32}


def _frames_arg(frames):
    """(pointer, bits, is_device, keep-alive) for camera frames: a numpy array
    of uint8, uint16 or float32 samples, or a CUDA tensor of those types."""
    try:
        import torch
    except ImportError:  # pragma: no cover - torch is part of the image
        torch = None
    if torch is not None and isinstance(frames, torch.Tensor):
        t = frames.contiguous()
        bits = {torch.uint8: 8, torch.uint16: 16, torch.float32: 32}.get(t.dtype)
        if bits is None or not t.is_cuda:
            raise ValueError("frames must be a CUDA tensor of uint8, uint16 or float32")
        return ctypes.c_void_p(t.data_ptr()), bits, 1, t
    a = np.asarray(frames)
    if a.dtype not in _SAMPLE_BITS:
        a = a.astype(np.float32)
    a = np.ascontiguousarray(a)
    return _ptr(a), _SAMPLE_BITS[a.dtype], 0, a


def median5_frames(count: int) -> np.ndarray:
    """The five frames behind each median background (count - 2 rows)."""
    out = np.empty((count - 2, 5), np.int32)
    _check(load_library().rihvr_background_median5_frames(int(count), out.ctypes.data_as(
        ctypes.POINTER(ctypes.c_int))), "rihvr_background_median5_frames")
    return out


def background_mean(frames):
    """Mean background of frames [count, H, W] (HoloSequence::
    useBackgroundSubtraction) on the GPU: (background float32 [H, W],
    stats dict alpha, beta, minimum, average)."""
    ptr, bits, dev, keep = _frames_arg(frames)
    k, h, w = keep.shape
    stats = (ctypes.c_double * 4)()
    if dev:
        import torch

        out = torch.empty((h, w), dtype=torch.float32, device=keep.device)
        optr = ctypes.c_void_p(out.data_ptr())
    else:
        out = np.empty((h, w), np.float32)
        optr = _ptr(out)
    _check(load_library().rihvr_background_mean(ptr, bits, w, h, k, dev, optr, stats), "rihvr_background_mean")
    return out, dict(zip(("alpha", "beta", "minimum", "average"), stats[:]))


def background_median5(frames):
    """Running median-of-five backgrounds (median_background_calc) of frames
    [count, H, W] on the GPU: float32 [count - 2, H, W]."""
    ptr, bits, dev, keep = _frames_arg(frames)
    k, h, w = keep.shape
    if dev:
        import torch

        out = torch.empty((max(k - 2, 0), h, w), dtype=torch.float32, device=keep.device)
        optr = ctypes.c_void_p(out.data_ptr())
    else:
        out = np.empty((max(k - 2, 0), h, w), np.float32)
        optr = _ptr(out)
    _check(load_library().rihvr_background_median5(ptr, bits, w, h, k, dev, optr), "rihvr_background_median5")
    return out


def preprocess(holo: np.ndarray, zero_padding: int, background: np.ndarray | None = None,
               files: FileParams | None = None) -> np.ndarray:
    """The reference preprocessing (rescale, normalise or background divide,
    crop, zero pad) of a raw frame; returns the measured hologram b."""
    L = load_library()
    holo = np.ascontiguousarray(holo, dtype=np.float32)
    bg = None if background is None else np.ascontiguousarray(background, dtype=np.float32)
    if bg is not None and files is None:
        files = FileParams()
        files.remove_background = 1
        files.roi_size = -1
    fp = ctypes.byref(files) if files is not None else None
    w, h = ctypes.c_int(), ctypes.c_int()
    args = (_ptr(holo), holo.shape[1], holo.shape[0], _ptr(bg) if bg is not None else None, fp, int(zero_padding))
    _io_check(L.rihvr_preprocess(*args, None, ctypes.byref(w), ctypes.byref(h)), "rihvr_preprocess")
    out = np.empty((h.value, w.value), np.float32)
    _io_check(L.rihvr_preprocess(*args, _ptr(out), ctypes.byref(w), ctypes.byref(h)), "rihvr_preprocess")
    return out


def params_from_config(cfg, **overrides) -> RihvrParams:
    """Parameters of a synthetic workload (``synth.HoloConfig``)."""
    p = default_params()
    for k in ("start_plane", "plane_stepsize", "num_planes", "wavelength", "resolution", "zero_padding",
              "num_inverse_iterations", "regularization_param", "regularization_TV_param", "num_tv_iterations"):
        setattr(p, k, getattr(cfg, k))
    for k, v in overrides.items():
        setattr(p, k, v)
    return p


def _ptr(a: np.ndarray):
    return ctypes.c_void_p(a.ctypes.data)


class SparseCompressiveHolo:
    """Mirror of ``umnholo::SparseCompressiveHolo`` (sparse_compressive_holo.h:30-96).

    ``SparseCompressiveHolo(params, width, height)`` allocates the solver for a
    padded ``height x width`` hologram; ``inverseReconstruct(b)`` runs the
    configured number of FISTA iterations from x = 0 and returns the objective
    at the final momentum point; ``getPlane(z)`` returns a plane of the volume.
    With ``z_first``/``z_count`` the solver holds only those planes of the
    plane list (a z-slab, rihvr_create_slab; whole solves of slabs run through
    ``slabs.slab_iterate``), and ``depth`` is ``z_count``.
    """

    def __init__(self, params: RihvrParams, width: int, height: int, z_first: int | None = None,
                 z_count: int | None = None):
        L = load_library()
        self._L = L
        self.params = params
        self.width, self.height = int(width), int(height)
        h = ctypes.c_void_p()
        if z_first is None and z_count is None:
            self.z_first, self.depth = 0, int(params.num_planes)
            _check(L.rihvr_create(ctypes.byref(params), self.width, self.height, ctypes.byref(h)), "rihvr_create")
        else:
            self.z_first = int(z_first or 0)
            self.depth = int(params.num_planes) - self.z_first if z_count is None else int(z_count)
            _check(L.rihvr_create_slab(ctypes.byref(params), self.width, self.height, self.z_first, self.depth,
                                       ctypes.byref(h)), "rihvr_create_slab")
        self._h = h

    # lifecycle ---------------------------------------------------------------
    def destroy(self):
        if getattr(self, "_h", None):
            self._L.rihvr_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.destroy()

    # operations --------------------------------------------------------------
    def setHologram(self, b: np.ndarray):
        b = np.ascontiguousarray(b, dtype=np.float32)
        if b.shape != (self.height, self.width):
            raise ValueError(f"hologram shape {b.shape} != {(self.height, self.width)}")
        _check(self._L.rihvr_set_hologram(self._h, _ptr(b), 0), "rihvr_set_hologram")

    def setHologramFrame(self, frame, background=None, files: FileParams | None = None):
        """The driver's preprocessing on the GPU (rihvr_set_hologram_frame):
        `frame` is the raw camera frame [H0, W0] (uint8, uint16 or float32
        samples; numpy or CUDA tensor), `background` one of the same kind;
        crop from `files`, padding from the parameters."""
        ptr, bits, dev, keep = _frames_arg(frame)
        bptr, bkeep = None, None
        if background is not None:
            bptr, bbits, bdev, bkeep = _frames_arg(background)
            if (bbits, bdev, bkeep.shape) != (bits, dev, keep.shape):
                raise ValueError("background must match the frame's type, place and shape")
            if files is None:
                files = FileParams()
                files.remove_background = 1
                files.roi_size = -1
                files.roi_x = files.roi_y = -1
        h0, w0 = keep.shape
        _check(self._L.rihvr_set_hologram_frame(self._h, ptr, bits, w0, h0, bptr,
                                                ctypes.byref(files) if files is not None else None, dev),
               "rihvr_set_hologram_frame")

    def getHologram(self) -> np.ndarray:
        out = np.empty((self.height, self.width), np.float32)
        _check(self._L.rihvr_get_hologram(self._h, _ptr(out), 0), "rihvr_get_hologram")
        return out

    def setInitialVolume(self, x0: np.ndarray):
        """Warm start (rihvr_set_initial_volume): continue FISTA from x0
        instead of 0; the hologram must be set."""
        x0 = np.ascontiguousarray(x0, dtype=np.complex64)
        if x0.shape != (self.depth, self.height, self.width):
            raise ValueError("volume shape mismatch")
        _check(self._L.rihvr_set_initial_volume(self._h, _ptr(x0), 0), "rihvr_set_initial_volume")

    def autotune(self) -> float:
        """Tune launch shapes on this context (rihvr_autotune); returns the
        chosen passes' total time in ms."""
        ms = ctypes.c_double()
        _check(self._L.rihvr_autotune(self._h, ctypes.byref(ms)), "rihvr_autotune")
        return ms.value

    def tuning(self) -> dict:
        """Launch shapes in use (rihvr_tuning); 0 = built-in choice."""
        v = [ctypes.c_int() for _ in range(6)]
        _check(self._L.rihvr_tuning(self._h, *[ctypes.byref(x) for x in v]), "rihvr_tuning")
        return dict(zip(("adj_chunks", "fwd_chunks", "tv_runs", "tv_kernel", "adj_recurrence", "fwd_horner"),
                        (x.value for x in v)))

    def inverseReconstruct(self, b: np.ndarray | None = None) -> float:
        if b is not None:
            self.setHologram(b)
        f = ctypes.c_double()
        _check(self._L.rihvr_reconstruct(self._h, ctypes.byref(f)), "rihvr_reconstruct")
        return f.value

    def reset(self):
        _check(self._L.rihvr_reset(self._h), "rihvr_reset")

    def iterate(self, n: int):
        _check(self._L.rihvr_iterate(self._h, int(n)), "rihvr_iterate")

    def iterate_timed(self, n: int) -> float:
        ms = ctypes.c_float()
        _check(self._L.rihvr_iterate_timed(self._h, int(n), ctypes.byref(ms)), "rihvr_iterate_timed")
        return ms.value

    def calcObjectiveFunction(self):
        f = ctypes.c_double()
        terms = (ctypes.c_double * 3)()
        _check(self._L.rihvr_objective(self._h, ctypes.byref(f), terms), "rihvr_objective")
        return f.value, np.array(terms[:])

    def iterations(self) -> np.ndarray:
        n = ctypes.c_int()
        _check(self._L.rihvr_get_iterations(self._h, None, 0, ctypes.byref(n)), "rihvr_get_iterations")
        out = np.zeros(n.value, ITER_DTYPE)
        if n.value:
            _check(self._L.rihvr_get_iterations(self._h, _ptr(out), n.value, ctypes.byref(n)), "rihvr_get_iterations")
        return out

    def getSparsity(self) -> float:
        v = ctypes.c_double()
        _check(self._L.rihvr_sparsity(self._h, ctypes.byref(v)), "rihvr_sparsity")
        return v.value

    def estimateLipschitz(self, iterations: int = 20, seed: int = 0):
        """FP64 power iteration for the largest eigenvalue of A^H A:
        (L, Rayleigh quotients of every step).  Resets the solve to x = 0."""
        L = ctypes.c_double()
        hist = np.zeros(int(iterations), np.float64)
        _check(self._L.rihvr_lipschitz(self._h, int(iterations), int(seed), ctypes.byref(L),
                                       hist.ctypes.data_as(ctypes.c_void_p)), "rihvr_lipschitz")
        return L.value, hist

    def initialEstimate(self) -> np.ndarray:
        out = np.empty((self.height, self.width), np.float32)
        _check(self._L.rihvr_initial_estimate(self._h, _ptr(out), 0), "rihvr_initial_estimate")
        return out

    def getPlane(self, z: int) -> np.ndarray:
        out = np.empty((self.height, self.width), np.complex64)
        _check(self._L.rihvr_get_plane(self._h, int(z), _ptr(out), 0), "rihvr_get_plane")
        return out

    def getVolume(self) -> np.ndarray:
        out = np.empty((self.depth, self.height, self.width), np.complex64)
        _check(self._L.rihvr_get_volume(self._h, _ptr(out), 0), "rihvr_get_volume")
        return out

    def saveState(self, path: str):
        """Checkpoint the solve between iterations (rihvr_save_state)."""
        _check(self._L.rihvr_save_state(self._h, os.fsencode(path)), "rihvr_save_state")

    def loadState(self, path: str):
        """Resume a checkpointed solve in this solver (rihvr_load_state): same
        sizes and parameters; later iterations continue it bit for bit."""
        _check(self._L.rihvr_load_state(self._h, os.fsencode(path)), "rihvr_load_state")

    def volume_device(self):
        """The momentum point volume in device memory, without a copy
        (rihvr_get_volume_ptr): a torch complex64 CUDA tensor of shape
        (depth, height, width) viewing the context's buffer, valid until the
        next call on this solver."""
        import torch

        ptr, dtype = ctypes.c_void_p(), ctypes.c_int()
        _check(self._L.rihvr_get_volume_ptr(self._h, ctypes.byref(ptr), ctypes.byref(dtype)), "rihvr_get_volume_ptr")
        if dtype.value != 0:
            raise RihvrError(ERR_UNSUPPORTED_SIZE, "unexpected volume type")

        class _DeviceView:  # the CUDA array interface torch reads (torch wants the read-only flag clear)
            __cuda_array_interface__ = {"shape": (self.depth, self.height, self.width), "typestr": "<c8",
                                        "data": (ptr.value, False), "version": 3}

        return torch.as_tensor(_DeviceView(), device="cuda")

    def getEstimate(self) -> np.ndarray:
        out = np.empty((self.height, self.width), np.float32)
        _check(self._L.rihvr_get_estimate(self._h, _ptr(out), 0), "rihvr_get_estimate")
        return out

    def getResidual(self) -> np.ndarray:
        out = np.empty((self.height, self.width), np.float32)
        _check(self._L.rihvr_get_residual(self._h, _ptr(out), 0), "rihvr_get_residual")
        return out

    def backpropagate(self) -> np.ndarray:
        """xbp = t A^H b of the hologram (t the initial step); resets the solve."""
        out = np.empty((self.depth, self.height, self.width), np.complex64)
        _check(self._L.rihvr_backpropagate(self._h, _ptr(out), 0), "rihvr_backpropagate")
        return out

    def warmStart(self, net: "UNet"):
        """Start the solve from the network's x0 (rihvr_warm_start)."""
        _check(self._L.rihvr_warm_start(self._h, net._h), "rihvr_warm_start")

    def segment(self, sp: SegmentParams | None = None, max_objects: int = 1 << 16):
        """SparseSegmentation on the current volume (binarize, close, label,
        extractObjects, blobSizeFilter): (objects, info), see segment_intensity."""
        sp = sp or segment_params()
        return _segment_call(lambda o, m, n, i: self._L.rihvr_segment(self._h, ctypes.byref(sp), o, m, n, i),
                             "rihvr_segment", max_objects)

    # operators ---------------------------------------------------------------
    def forward(self, vol: np.ndarray) -> np.ndarray:
        """backPropagate: d = Re(IFFT(sum_z H'_z FFT(x_z)))."""
        vol = np.ascontiguousarray(vol, dtype=np.complex64)
        if vol.shape != (self.depth, self.height, self.width):
            raise ValueError("volume shape mismatch")
        out = np.empty((self.height, self.width), np.float32)
        _check(self._L.rihvr_forward(self._h, _ptr(vol), _ptr(out), 0), "rihvr_forward")
        return out

    def adjoint(self, r: np.ndarray) -> np.ndarray:
        """SparseGradient: g_z = IFFT(conj(H'_z) FFT(r))."""
        r = np.ascontiguousarray(r, dtype=np.float32)
        out = np.empty((self.depth, self.height, self.width), np.complex64)
        _check(self._L.rihvr_adjoint(self._h, _ptr(r), _ptr(out), 0), "rihvr_adjoint")
        return out

    def prox_step(self, x: np.ndarray, r: np.ndarray, t: float):
        """denoise(): p = prox(x - t A^H r, t); returns (p, [lim1, lim2, restart])."""
        x = np.ascontiguousarray(x, dtype=np.complex64)
        r = np.ascontiguousarray(r, dtype=np.float32)
        out = np.empty_like(x)
        sums = (ctypes.c_double * 3)()
        _check(self._L.rihvr_prox_step(self._h, _ptr(x), _ptr(r), float(t), _ptr(out), sums, 0),
               "rihvr_prox_step")
        return out, np.array(sums[:])

    # profiling ---------------------------------------------------------------
    def set_profiling(self, on: bool):
        _check(self._L.rihvr_set_profiling(self._h, int(bool(on))), "rihvr_set_profiling")

    def kernel_times(self) -> dict:
        names = (ctypes.c_char_p * 16)()
        ms = (ctypes.c_double * 16)()
        cnt = (ctypes.c_int * 16)()
        n = ctypes.c_int()
        _check(self._L.rihvr_kernel_times(self._h, names, ms, cnt, 16, ctypes.byref(n)), "rihvr_kernel_times")
        return {names[i].decode(): (ms[i], cnt[i]) for i in range(n.value)}

    def stream(self) -> int:
        return int(self._L.rihvr_get_stream(self._h) or 0)

    def launch_count(self) -> int:
        return int(self._L.rihvr_launch_count(self._h))

    def device_bytes(self) -> int:
        return int(self._L.rihvr_device_bytes(self._h))
