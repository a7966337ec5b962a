"""ctypes front end of the FP64 CPU oracle (``rihvr_oracle.c``).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()``
and the ``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` as the
checker and the CPU baseline.  The product path never imports this module.

Parity status: pinned to the reference's own CUDA kernels, built unchanged by
``oracle/build_ref.py`` and driven by ``oracle/ref_harness.cu``
(``tests/test_gpu_ref_pin.py``); also checked against numpy.fft and
mathematical known answers in ``tests/test_oracle.py``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None


def build(force: bool = False) -> str:
    """Compile ``liboracle.so`` with the committed Makefile."""
    src = os.path.join(_HERE, "rihvr_oracle.c")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE, "liboracle.so"], check=True)
    return _LIB_PATH


class _Params(ctypes.Structure):
    _fields_ = [
        ("W", ctypes.c_int), ("H", ctypes.c_int), ("Nz", ctypes.c_int),
        ("dx", ctypes.c_double), ("lam", ctypes.c_double),
        ("z", ctypes.POINTER(ctypes.c_double)),
        ("l1", ctypes.c_double), ("tv", ctypes.c_double),
        ("n_tv", ctypes.c_int), ("mode", ctypes.c_int), ("faithful", ctypes.c_int),
        ("max_backtracks", ctypes.c_int), ("n_threads", ctypes.c_int), ("t0", ctypes.c_double),
    ]


ITER_DTYPE = np.dtype([
    ("f_prox", "f8"), ("f_resid_prox", "f8"), ("lim", "f8"), ("ratio", "f8"), ("t", "f8"),
    ("beta", "f8"), ("f_x", "f8"), ("f_resid_x", "f8"), ("l1_x", "f8"), ("tv_x", "f8"),
    ("restart_sum", "f8"), ("backtracks", "i4"), ("restarted", "i4"),
])


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        P = ctypes.POINTER
        dp = P(ctypes.c_double)
        L.orc_fft2.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int]
        L.orc_fft1.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int]
        L.orc_phase_table.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, dp]
        L.orc_forward.argtypes = [P(_Params), ctypes.c_void_p, dp]
        L.orc_adjoint.argtypes = [P(_Params), dp, ctypes.c_void_p]
        L.orc_prox_plane.argtypes = [P(_Params), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double,
                                     ctypes.c_void_p]
        L.orc_prox_from.argtypes = [P(_Params), ctypes.c_void_p, ctypes.c_void_p, dp, ctypes.c_double,
                                    ctypes.c_void_p, dp]
        L.orc_objective.argtypes = [P(_Params), dp, ctypes.c_void_p, dp]
        L.orc_objective.restype = ctypes.c_double
        L.orc_solve.argtypes = [P(_Params), dp, ctypes.c_int, P(ctypes.c_int), P(ctypes.c_int),
                                ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, dp, dp]
        L.orc_num_threads.restype = ctypes.c_int
        L.orc_segment.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                  ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                  ctypes.POINTER(ctypes.c_double)]
        _lib = L
    return _lib


@dataclass
class OracleParams:
    """Solver parameters in the reference's units (lengths in one unit)."""
    W: int
    H: int
    z: np.ndarray                 # plane positions, float64 (already float-rounded if faithful)
    dx: float
    lam: float
    l1: float = 0.01
    tv: float = 0.0
    n_tv: int = 5
    mode: int = 7
    faithful: int = 1
    max_backtracks: int = 2
    n_threads: int = 0
    t0: float = 0.0
    _z: np.ndarray = field(default=None, repr=False)

    @property
    def Nz(self) -> int:
        return int(len(self.z))

    def c(self) -> _Params:
        self._z = np.ascontiguousarray(self.z, dtype=np.float64)
        return _Params(self.W, self.H, self.Nz, self.dx, self.lam,
                       self._z.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                       self.l1, self.tv, self.n_tv, self.mode, self.faithful,
                       self.max_backtracks, self.n_threads, self.t0)


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def fft2(a: np.ndarray, inverse: bool = False) -> np.ndarray:
    out = np.ascontiguousarray(a, dtype=np.complex128).copy()
    lib().orc_fft2(out.shape[0], out.shape[1], out.ctypes.data, int(inverse))
    return out


def fft1(a: np.ndarray, inverse: bool = False) -> np.ndarray:
    out = np.ascontiguousarray(a, dtype=np.complex128).copy()
    lib().orc_fft1(out.shape[0], out.ctypes.data, int(inverse))
    return out


def phase_table(H: int, W: int, dx: float, lam: float) -> np.ndarray:
    c = np.empty((H, W), np.float64)
    lib().orc_phase_table(H, W, dx, lam, _dp(c))
    return c


def forward(p: OracleParams, vol: np.ndarray) -> np.ndarray:
    vol = np.ascontiguousarray(vol, dtype=np.complex128)
    assert vol.shape == (p.Nz, p.H, p.W)
    d = np.empty((p.H, p.W), np.float64)
    cp = p.c()
    lib().orc_forward(ctypes.byref(cp), vol.ctypes.data, _dp(d))
    return d


def adjoint(p: OracleParams, r: np.ndarray) -> np.ndarray:
    r = np.ascontiguousarray(r, dtype=np.float64)
    vol = np.empty((p.Nz, p.H, p.W), np.complex128)
    cp = p.c()
    lib().orc_adjoint(ctypes.byref(cp), _dp(r), vol.ctypes.data)
    return vol


def prox_plane(p: OracleParams, x0: np.ndarray, g: np.ndarray, t: float) -> np.ndarray:
    x0 = np.ascontiguousarray(x0, dtype=np.complex128)
    g = np.ascontiguousarray(g, dtype=np.complex128)
    out = np.empty_like(x0)
    cp = p.c()
    lib().orc_prox_plane(ctypes.byref(cp), x0.ctypes.data, g.ctypes.data, t, out.ctypes.data)
    return out


def prox_from(p: OracleParams, X: np.ndarray, Y0: np.ndarray, r: np.ndarray, t: float):
    X = np.ascontiguousarray(X, dtype=np.complex128)
    Y0 = np.ascontiguousarray(Y0, dtype=np.complex128)
    r = np.ascontiguousarray(r, dtype=np.float64)
    P = np.empty_like(X)
    sums = np.zeros(3, np.float64)
    cp = p.c()
    lib().orc_prox_from(ctypes.byref(cp), X.ctypes.data, Y0.ctypes.data, _dp(r), t, P.ctypes.data,
                        _dp(sums))
    return P, sums


def objective(p: OracleParams, r: np.ndarray, vol: np.ndarray):
    r = np.ascontiguousarray(r, dtype=np.float64)
    vol = np.ascontiguousarray(vol, dtype=np.complex128)
    terms = np.zeros(3, np.float64)
    cp = p.c()
    f = lib().orc_objective(ctypes.byref(cp), _dp(r), vol.ctypes.data, _dp(terms))
    return f, terms


def solve(p: OracleParams, b: np.ndarray, n_iter: int, forced_bt=None, forced_rs=None,
          want_volumes: bool = True):
    """Run ``n_iter`` FISTA iterations from x = 0.

    Returns (log, X, P, est, f0): the per-iteration records, the final momentum
    point, the final prox output, the estimated hologram at X and the initial
    objective.
    """
    b = np.ascontiguousarray(b, dtype=np.float64)
    assert b.shape == (p.H, p.W)
    log = np.zeros(n_iter, ITER_DTYPE)
    X = np.empty((p.Nz, p.H, p.W), np.complex128) if want_volumes else None
    P = np.empty((p.Nz, p.H, p.W), np.complex128) if want_volumes else None
    est = np.empty((p.H, p.W), np.float64)
    f0 = np.zeros(1, np.float64)
    ip = ctypes.POINTER(ctypes.c_int)
    fb = fr = None
    if forced_bt is not None:
        fb_arr = np.ascontiguousarray(forced_bt, dtype=np.int32)
        fb = fb_arr.ctypes.data_as(ip)
    if forced_rs is not None:
        fr_arr = np.ascontiguousarray(forced_rs, dtype=np.int32)
        fr = fr_arr.ctypes.data_as(ip)
    cp = p.c()
    rc = lib().orc_solve(ctypes.byref(cp), _dp(b), n_iter, fb, fr, log.ctypes.data,
                         X.ctypes.data if X is not None else None,
                         P.ctypes.data if P is not None else None, _dp(est), _dp(f0))
    if rc != 0:
        raise MemoryError("oracle could not allocate its volumes")
    return log, X, P, est, float(f0[0])


SEG_OBJECT_DTYPE = np.dtype([
    ("x", "f4"), ("y", "f4"), ("z", "f4"), ("wx", "f4"), ("wy", "f4"), ("wz", "f4"),
    ("num_voxels", "i4"), ("max_value", "f4"), ("mean_value", "f4"),
    ("xmin", "i4"), ("xmax", "i4"), ("ymin", "i4"), ("ymax", "i4"), ("zmin", "i4"), ("zmax", "i4"),
])


def segment(intensity: np.ndarray, min_intensity: float = 1.0, close_size: int = 3, min_area: int = 2,
            faithful: int = 1):
    """The reference's segmentation program on a (planes, height, width) stack of
    voxel intensities: (objects in the reference's order, (max intensity, threshold))."""
    I = np.ascontiguousarray(intensity, dtype=np.float32)
    nz, h, w = I.shape
    L = lib()
    cap = max(16, I.size // 2 + 1)
    out = np.zeros(cap, SEG_OBJECT_DTYPE)
    info = (ctypes.c_double * 2)()
    n = L.orc_segment(I.ctypes.data, w, h, nz, float(min_intensity), int(close_size), int(min_area),
                      int(faithful), out.ctypes.data, cap, info)
    if n < 0:
        raise RuntimeError("orc_segment: object buffer too small")
    return out[:n].copy(), (info[0], info[1])


def num_threads() -> int:
    return int(lib().orc_num_threads())
