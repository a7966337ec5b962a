"""Restatement of the reference's 8-bit volume images, for the output tests.

TEST INFRASTRUCTURE ONLY: imported by ``tests/`` to check the images that
``sparse-inverse-recon`` writes.  It follows

* ``SparseCompressiveHolo::savePlanes`` (``src/core/sparse_compressive_holo.cu:1039-1194``):
  magnitude over the global magnitude range, phase over 2 pi, real and
  imaginary parts over +-sqrt(global max) / 10;
* ``SparseVolume::saveProjections`` with ``MAX_CMB``
  (``src/core/sparse_volume.cu:684-813``): maxima of the scaled magnitude along
  x, y and z, the XY image starting from zeros and folding in planes z > 0 only.

Magnitude and phase come from OpenCV itself (``cv2.magnitude``,
``cv2.phase``), the functions the reference calls through
``CuMat::getMag``/``getPhase`` (``cumat.cu:1308-1336``).  The matrix expression
``(plane - lo) / (hi - lo)`` is evaluated as OpenCV evaluates it, one
``convertTo`` with alpha = 1 / (hi - lo) and beta = -lo * alpha in float, and
``convertTo(CV_8U, 255)`` multiplies by 255 in float and rounds half to even
with saturation.
"""
from __future__ import annotations

import numpy as np


def _cv2():
    import cv2

    return cv2


def _unit_map(v: np.ndarray, lo: float, hi: float) -> np.ndarray:
    a = 1.0 / (hi - lo)
    alpha, beta = np.float32(a), np.float32(-lo * a)
    return (v.astype(np.float32) * alpha + beta).astype(np.float32)


def to_u8(unit: np.ndarray) -> np.ndarray:
    """convertTo(CV_8U, 255): saturate_cast<uchar>(v * 255) with rounding half to even."""
    v = unit.astype(np.float32) * np.float32(255.0)
    return np.clip(np.rint(v), 0, 255).astype(np.uint8)


def magnitude(plane: np.ndarray) -> np.ndarray:
    re = np.ascontiguousarray(plane.real, np.float32)
    im = np.ascontiguousarray(plane.imag, np.float32)
    return _cv2().magnitude(re, im)


def phase(plane: np.ndarray) -> np.ndarray:
    re = np.ascontiguousarray(plane.real, np.float32)
    im = np.ascontiguousarray(plane.imag, np.float32)
    return _cv2().phase(re, im)


def global_range(volume: np.ndarray):
    lo = hi = 0.0
    for z in range(volume.shape[0]):
        m = magnitude(volume[z])
        a, b = float(m.min()), float(m.max())
        if z == 0:
            lo, hi = a, b
        lo, hi = min(lo, a), max(hi, b)
    return lo, hi


def save_planes(volume: np.ndarray) -> dict:
    """{'mag'|'phase'|'real'|'imag': uint8 array (Nz, H, W)} as savePlanes writes."""
    lo, hi = global_range(volume)
    rmax = np.sqrt(hi) / 10.0
    out = {k: np.empty(volume.shape, np.uint8) for k in ("mag", "phase", "real", "imag")}
    for z in range(volume.shape[0]):
        p = volume[z]
        out["mag"][z] = to_u8(_unit_map(magnitude(p), lo, hi))
        out["phase"][z] = to_u8(phase(p) * np.float32(1.0 / (2 * np.pi)))  # plane / (2 pi): convertTo(1 / 2 pi)
        out["real"][z] = to_u8(_unit_map(p.real, -rmax, rmax))
        out["imag"][z] = to_u8(_unit_map(p.imag, -rmax, rmax))
    return out


def save_projections(volume: np.ndarray) -> dict:
    """{'xy': (H, W), 'xz': (Nz, W), 'yz': (H, Nz)} uint8 images as saveProjections(MAX_CMB) writes."""
    lo, hi = global_range(volume)
    nz, h, w = volume.shape
    xy = np.zeros((h, w), np.float32)
    xz = np.zeros((nz, w), np.float32)
    yz = np.zeros((h, nz), np.float32)
    for z in range(nz):
        s = _unit_map(magnitude(volume[z]), lo, hi)
        xz[z] = s.max(axis=0)
        yz[:, z] = s.max(axis=1)
        if z > 0:
            xy = np.maximum(xy, s)
    return {"xy": to_u8(xy), "xz": to_u8(xz), "yz": to_u8(yz)}
