"""ctypes front end of ``oracle/_ref/libref_kernels.so``: the reference's own
hot-path CUDA kernels (copied verbatim from the RIHVR sources at build time by
``build_ref.py``) driven with cuFFT in the reference's host order by
``ref_harness.cu``.

TEST INFRASTRUCTURE ONLY: the GPU pin of the FP64 oracle.  Tests load it to
check the oracle (and the product) against code the reference itself runs.
Needs a CUDA GPU; the library is prebuilt where the reference sources exist
and travels with the repository as a built file.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libref_kernels.so")
_lib = None

RECORD_FIELDS = ("f_x", "f_resid_x", "f_prox", "lim", "ratio", "t", "beta", "backtracks", "restarted",
                 "restart_sum")


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(f"{LIB_PATH} is not built (python oracle/build_ref.py)")
        L = ctypes.CDLL(LIB_PATH)
        vp, ip, fl, db = ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_double
        L.ref_last_error.restype = ctypes.c_char_p
        L.ref_forward.argtypes = [vp, ip, ip, ip, vp, fl, fl, vp]
        L.ref_adjoint.argtypes = [vp, ip, ip, ip, vp, fl, fl, vp]
        L.ref_prox.argtypes = [vp, vp, vp, ip, ip, ip, vp, fl, fl, ip, db, db, db, ip, vp, vp]
        L.ref_restart_sum.argtypes = [vp, vp, vp, ip, ip, ip, vp]
        L.ref_objective.argtypes = [vp, vp, ip, ip, ip, ip, db, db, vp, vp]
        L.ref_solve.argtypes = [vp, ip, ip, ip, vp, fl, fl, fl, fl, ip, ip, ip, vp, vp]
        assert L.ref_record_fields() == len(RECORD_FIELDS)
        _lib = L
    return _lib


def _check(rc: int, what: str):
    if rc != 0:
        raise RuntimeError(f"{what}: {lib().ref_last_error().decode(errors='replace')}")


def _c64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.complex64)


def _zl(z) -> np.ndarray:
    return np.ascontiguousarray(z, dtype=np.float32)


def forward(vol, z, lam: float, dx: float) -> np.ndarray:
    """backPropagate: the estimated hologram (complex, imaginary part 0) of a
    (Nz, H, W) complex volume."""
    v = _c64(vol)
    nz, h, w = v.shape
    out = np.empty((h, w), np.complex64)
    zl = _zl(z)
    _check(lib().ref_forward(v.ctypes.data, w, h, nz, zl.ctypes.data, lam, dx, out.ctypes.data), "ref_forward")
    return out


def adjoint(r, z, lam: float, dx: float) -> np.ndarray:
    """SparseGradient planes A^H r of a (H, W) residual (real or complex)."""
    rr = _c64(r)
    h, w = rr.shape
    zl = _zl(z)
    out = np.empty((len(zl), h, w), np.complex64)
    _check(lib().ref_adjoint(rr.ctypes.data, w, h, len(zl), zl.ctypes.data, lam, dx, out.ctypes.data), "ref_adjoint")
    return out


def prox(x0, r, z, lam: float, dx: float, mode: int, t: float, l1: float, tv: float, n_tv: int, y0=None):
    """denoise(mode): x1 = prox(x0 - t A^H r); returns (x1, sums) with sums =
    (line-search sum1, sum2, lim, restart sum against y0 (default x0))."""
    x = _c64(x0)
    nz, h, w = x.shape
    rr = _c64(r)
    zl = _zl(z)
    y = _c64(y0) if y0 is not None else None
    out = np.empty_like(x)
    sums = np.zeros(4, np.float64)
    _check(lib().ref_prox(x.ctypes.data, y.ctypes.data if y is not None else None, rr.ctypes.data, w, h, nz,
                          zl.ctypes.data, lam, dx, mode, t, l1, tv, n_tv, out.ctypes.data, sums.ctypes.data),
           "ref_prox")
    return out, sums


def restart_sum(x0, x1, y0) -> float:
    a, b, c = _c64(x0), _c64(x1), _c64(y0)
    nz, h, w = a.shape
    s = ctypes.c_double()
    _check(lib().ref_restart_sum(a.ctypes.data, b.ctypes.data, c.ctypes.data, w, h, nz, ctypes.byref(s)),
           "ref_restart_sum")
    return s.value


def objective(r, vol, mode: int, l1: float, tv: float):
    """calcObjectiveFunction: (f, (0.5|r|^2, L1, TV2d))."""
    rr = _c64(r)
    v = _c64(vol)
    nz, h, w = v.shape
    f = ctypes.c_double()
    terms = np.zeros(3, np.float64)
    _check(lib().ref_objective(rr.ctypes.data, v.ctypes.data, w, h, nz, mode, l1, tv, ctypes.byref(f),
                               terms.ctypes.data), "ref_objective")
    return f.value, terms


def solve(b, z, lam: float, dx: float, l1: float, tv: float, n_tv: int, mode: int, n_iter: int,
          want_volume: bool = False):
    """inverseReconstruct from x = 0: (records, final momentum point or None).
    records is a structured array with RECORD_FIELDS."""
    bb = np.ascontiguousarray(b, dtype=np.float32)
    h, w = bb.shape
    zl = _zl(z)
    rec = np.zeros((n_iter, len(RECORD_FIELDS)), np.float64)
    vol = np.empty((len(zl), h, w), np.complex64) if want_volume else None
    _check(lib().ref_solve(bb.ctypes.data, w, h, len(zl), zl.ctypes.data, lam, dx, l1, tv, n_tv, mode, n_iter,
                           rec.ctypes.data, vol.ctypes.data if vol is not None else None), "ref_solve")
    out = np.zeros(n_iter, [(k, "f8") for k in RECORD_FIELDS])
    for i, k in enumerate(RECORD_FIELDS):
        out[k] = rec[:, i]
    return out, vol
