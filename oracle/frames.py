"""Restatement of the reference's frame preprocessing and background
generation, for the frame tests.

TEST INFRASTRUCTURE ONLY: imported by ``tests/`` to check
``rihvr_set_hologram_frame``, ``rihvr_preprocess``, ``rihvr_background_mean``,
``rihvr_background_median5`` and the ``create-background`` program.  It follows

* ``main_sparse_inverse.cu:106-124`` and ``Hologram`` (``src/core/hologram.cu``):
  ``rescale`` to [0, 1] (``:401-439``, fl(v / 255) in FP32), ``normalize``
  (``:332-358``, I / mean - 1 with the mean in FP64), background division
  (``:1365-1432``, (I - B) / max(sqrt(B), 0.1)), ``crop`` (``:768-887``) and
  ``zeroPad`` (``:889-945``);
* ``HoloSequence::useBackgroundSubtraction`` (``src/core/holo_sequence.cu:309-447``):
  the background is the FP32 sum of the frames in order (``cv::add``), then
  ``Mat /= n``, which OpenCV evaluates as ``convertTo`` with alpha = 1/n: an
  FP32 multiply by fl(1/n) (pinned against cv2 in the tests); per frame the
  FP64 mean and standard deviation of frame - background (``cv::meanStdDev``:
  sqrt(max(E[d^2] - E[d]^2, 0))); alpha, beta from their means (``:414-419``);
* ``median_background_calc`` (``src/core/main_create_background.cu:103-193``)
  with its five-frame stack: frames 0-4 give backgrounds 0-2, and frame i
  replaces slot (i - 3) mod 5 before background i (3 <= i < n - 2);
* the frame choice of ``HoloSequence::loadNextChunk`` (``holo_sequence.cu:127-229``)
  when every chosen frame fits in one chunk.

The mean of ``normalize`` is the correctly rounded sum (``math.fsum``) over
the count, which is what the library computes from its exact integer sum;
``cv::mean`` sums in FP64 in its own order, which can differ in the last bit
of the FP64 mean and, rarely, in the FP32 mean used.
"""
from __future__ import annotations

import math

import numpy as np

F32 = np.float32


def crop_rect(W0: int, H0: int, roi_x=-1, roi_y=-1, roi_size=-1, rect=(0, 0, 0, 0)):
    """Hologram::crop (hologram.cu:768-887): (x, y, w, h)."""
    rx, ry, rw, rh = rect
    if rw > 0 and rh > 0:
        return rx, ry, rw, rh
    if roi_size >= 1:
        s = roi_size
        x, y = roi_x - s // 2, roi_y - s // 2
        w = h = s
        x = max(x, 0)
        y = max(y, 0)
        if x + s > W0:
            x = W0 - s
        if y + s > H0:
            y = H0 - s
        if W0 < s:
            x, w = 0, W0
        if H0 < s:
            y, h = 0, H0
        return x, y, w, h
    return 0, 0, W0, H0


def unit(frame: np.ndarray) -> np.ndarray:
    """Hologram::rescale to [0, 1]: fl(v / 255) in FP32."""
    return (np.asarray(frame).astype(F32) / F32(255.0)).astype(F32)


def unit_mean(frame: np.ndarray) -> float:
    """FP64 mean of fl(v / 255): correctly rounded sum over the count."""
    f = unit(frame).astype(np.float64).ravel()
    return math.fsum(f) / f.size


def preprocess(frame: np.ndarray, background: np.ndarray | None = None, pad: int = 0, roi_x=-1, roi_y=-1,
               roi_size=-1, rect=(0, 0, 0, 0)) -> np.ndarray:
    """The driver's preprocessing of one raw frame to the hologram b (FP32)."""
    f = unit(frame)
    if background is not None:
        B = unit(background)
        sb = np.sqrt(B).astype(F32)
        sb = np.where(sb < F32(0.1), F32(0.1), sb).astype(F32)
        f = ((f - B).astype(F32) / sb).astype(F32)
    else:
        m = unit_mean(frame)
        if m == 0:
            raise ValueError("hologram mean is zero")
        f = ((f / F32(m)).astype(F32) - F32(1.0)).astype(F32)
    H0, W0 = f.shape
    x, y, w, h = crop_rect(W0, H0, roi_x, roi_y, roi_size, rect)
    out = np.zeros((h + 2 * pad, w + 2 * pad), F32)
    for r in range(h):
        sy = y + r
        if not 0 <= sy < H0:
            continue
        xs = np.arange(w) + x
        ok = (xs >= 0) & (xs < W0)
        out[pad + r, pad + np.arange(w)[ok]] = f[sy, xs[ok]]
    return out


def background_mean(frames: np.ndarray):
    """(background FP32 [H, W], (alpha, beta, minimum, average))."""
    frames = np.asarray(frames)
    acc = np.zeros(frames.shape[1:], F32)
    for k in range(frames.shape[0]):
        acc = (acc + frames[k].astype(F32)).astype(F32)
    n = frames.shape[0]
    bg = (acc * F32(1.0 / n)).astype(F32)
    average = math.fsum(bg.astype(np.float64).ravel()) / bg.size
    means, stds = [], []
    for k in range(n):
        d = (frames[k].astype(F32) - bg).astype(F32).astype(np.float64).ravel()
        m = math.fsum(d) / d.size
        sq = math.fsum(d * d) / d.size
        means.append(m)
        stds.append(math.sqrt(max(sq - m * m, 0.0)))
    mean_mean, mean_std = sum(means) / n, sum(stds) / n
    scale1 = 5.0  # bg_scale1 (holo_sequence.cu:22)
    return bg, (mean_mean - scale1 * mean_std, 255.0 / (2 * mean_std * scale1), 0.0, average)


def median5_frames(count: int) -> np.ndarray:
    """Frames in the five-frame stack behind each median background."""
    if count < 5:
        raise ValueError("needs at least 5 frames")
    stack = [0, 1, 2, 3, 4]
    rows = [list(stack) for _ in range(3)]
    for i in range(3, count - 2):
        stack[(i - 3) % 5] = i
        rows.append(list(stack))
    return np.array(rows, np.int32)


def background_median5(frames: np.ndarray) -> np.ndarray:
    frames = np.asarray(frames).astype(F32)
    sel = median5_frames(frames.shape[0])
    return np.stack([np.median(frames[s], axis=0).astype(F32) for s in sel])


def mean_frame_ids(start_image: int, image_count: int, background_start: int = -1, background_end: int = -1):
    """Frames useBackgroundSubtraction reads (one chunk)."""
    start, total = start_image, image_count
    if background_start >= 0 and background_end >= 0:
        start, total = background_start, background_end - background_start - 1
    step = total // 200 if total > 500 else 1
    return [start + k * step for k in range(total // step)]


def to_u8(v: np.ndarray) -> np.ndarray:
    """convertTo(CV_8U): round half to even, saturate."""
    return np.clip(np.rint(np.asarray(v, F32)), 0, 255).astype(np.uint8)
