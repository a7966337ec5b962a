"""Seeded synthetic holograms with the shapes and parameters of the reference's
datasets ("Dandelions" and "Rotating Rods", README.md:46-57 of the RIHVR tree),
which are not distributed with the reference.

A hologram is generated as ``I = |1 + F^-1 sum_z H'_z F(o_z)|^2`` where
``o_z = -mask_z`` marks opaque objects lying on the reconstruction planes and
``H'_z = exp(i z 2 pi/lambda (sqrt(1 - (lambda f)^2) - 1))`` is the carrier-free
Rayleigh-Sommerfeld transfer function the solver uses.  The camera records
``clip(I/2 + sigma n, 0, 1)`` quantised to uint8; the reference preprocessing
then applies: /255 (hologram.cu:401-439), ``I/mean - 1`` (hologram.cu:332-358),
whole-image crop and zero padding (hologram.cu:768-945).

This is input generation, not part of the measured path.
"""
from __future__ import annotations

import hashlib
import json
import os
from dataclasses import asdict, dataclass, field

import numpy as np

try:  # multithreaded FFT when available
    import scipy.fft as _sfft

    def _fft2(a):
        return _sfft.fft2(a, workers=os.cpu_count() or 1)

    def _ifft2(a):
        return _sfft.ifft2(a, workers=os.cpu_count() or 1)
except Exception:  # pragma: no cover
    _fft2, _ifft2 = np.fft.fft2, np.fft.ifft2


@dataclass
class HoloConfig:
    """Reconstruction parameters of one workload (reference .param names)."""
    name: str
    width: int                    # hologram width before padding
    height: int
    zero_padding: int
    num_planes: int
    start_plane: float            # z0
    plane_stepsize: float         # dz
    resolution: float             # dx
    wavelength: float             # lambda
    regularization_param: float   # sparsity (L1) weight
    regularization_TV_param: float
    num_inverse_iterations: int
    num_tv_iterations: int
    n_disks: int = 0
    disk_radius: tuple = (2.0, 6.0)
    n_rods: int = 0
    rod_length: tuple = (10.0, 60.0)
    rod_width: float = 2.0
    noise_sigma: float = 0.01
    seed: int = 0
    # frame of an advected tracer series (series_frames): when series_seed >= 0
    # the disks are the first n_disks tracers of that series at frame
    # series_frame, instead of independent random disks
    series_seed: int = -1
    series_frame: int = 0

    @property
    def W(self) -> int:
        return self.width + 2 * self.zero_padding

    @property
    def H(self) -> int:
        return self.height + 2 * self.zero_padding

    def plane_list(self) -> np.ndarray:
        """Plane positions as the reference computes them, in float32
        (holo_ui.cpp:478-483: float z = start_plane + i * plane_stepsize)."""
        z0 = np.float32(self.start_plane)
        dz = np.float32(self.plane_stepsize)
        return np.array([np.float32(z0 + np.float32(np.float32(i) * dz)) for i in range(self.num_planes)],
                        dtype=np.float32).astype(np.float64)

    def lam(self) -> float:
        return float(np.float32(self.wavelength))

    def dx(self) -> float:
        return float(np.float32(self.resolution))

    def l1(self) -> float:
        return float(np.float32(self.regularization_param))

    def tv(self) -> float:
        return float(np.float32(self.regularization_TV_param))

    def voxels(self) -> int:
        return self.W * self.H * self.num_planes

    def key(self) -> str:
        d = asdict(self)
        return hashlib.sha1(json.dumps(d, sort_keys=True).encode()).hexdigest()[:16]


def config1(**kw) -> HoloConfig:
    """Plain FISTA+TV, FP32 complex: 256x256 padded by 64 px per side, Nz=40."""
    c = HoloConfig(name="fista_tv_384x384x40", width=256, height=256, zero_padding=64, num_planes=40,
                   start_plane=0.0, plane_stepsize=2000.0, resolution=10.4, wavelength=0.633,
                   regularization_param=0.001, regularization_TV_param=0.01,
                   num_inverse_iterations=100, num_tv_iterations=5,
                   n_disks=50, disk_radius=(2.0, 6.0), noise_sigma=0.01)
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def config2(**kw) -> HoloConfig:
    """Precision study: 1024x1024, pad 0, Nz=1000, 1000 disks + 1000 rods."""
    c = HoloConfig(name="fista_tv_1024x1024x1000", width=1024, height=1024, zero_padding=0,
                   num_planes=1000, start_plane=2500.0, plane_stepsize=2.0, resolution=1.1,
                   wavelength=0.632, regularization_param=0.15, regularization_TV_param=0.1,
                   num_inverse_iterations=100, num_tv_iterations=5,
                   n_disks=1000, disk_radius=(1.0, 4.0), n_rods=1000, rod_length=(10.0, 60.0),
                   rod_width=2.0, noise_sigma=0.02)
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def config5(**kw) -> HoloConfig:
    """Large volume: 2048x2048 padded by 128 px per side (2304x2304), Nz=512,
    20000 tracer disks; run with FP16 volume storage."""
    c = HoloConfig(name="fista_tv_2304x2304x512", width=2048, height=2048, zero_padding=128, num_planes=512,
                   start_plane=1000.0, plane_stepsize=4.0, resolution=2.2, wavelength=0.532,
                   regularization_param=0.05, regularization_TV_param=0.05,
                   num_inverse_iterations=150, num_tv_iterations=10,
                   n_disks=20000, disk_radius=(1.0, 3.0), noise_sigma=0.02)
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def small_config(W=64, H=64, Nz=6, seed=0, **kw) -> HoloConfig:
    """Small case for parity tests (a few seconds in the oracle)."""
    c = HoloConfig(name=f"small_{W}x{H}x{Nz}", width=W, height=H, zero_padding=0, num_planes=Nz,
                   start_plane=100.0, plane_stepsize=40.0, resolution=2.0, wavelength=0.632,
                   regularization_param=0.01, regularization_TV_param=0.02,
                   num_inverse_iterations=10, num_tv_iterations=5,
                   n_disks=max(3, (W * H) // 600), disk_radius=(1.5, 3.5), noise_sigma=0.01, seed=seed)
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def _stamp_disk(plane: np.ndarray, cx: float, cy: float, r: float) -> None:
    H, W = plane.shape
    x0, x1 = int(np.floor(cx - r)), int(np.ceil(cx + r)) + 1
    y0, y1 = int(np.floor(cy - r)), int(np.ceil(cy + r)) + 1
    ys = np.arange(y0, y1)
    xs = np.arange(x0, x1)
    m = ((xs[None, :] - cx) ** 2 + (ys[:, None] - cy) ** 2) <= r * r
    yy = ys % H
    xx = xs % W
    sub = plane[np.ix_(yy, xx)]
    plane[np.ix_(yy, xx)] = np.maximum(sub, m.astype(plane.dtype))


# ---------------------------------------------------------------------------
# advected tracer series (the batched time-series workload)
# ---------------------------------------------------------------------------
SERIES_TRACERS = 3000   # tracers in the series; a frame images the first n_disks
SERIES_MODES = 8        # Fourier modes of the velocity field
SERIES_DT = 0.004       # time step between frames, in box lengths per unit velocity


def velocity_modes(series_seed: int, modes: int = SERIES_MODES):
    """A seeded random divergence-free velocity field on the periodic unit cube,
    u(x) = sum_m -sin(2 pi k_m . x + phi_m) (k_m x b_m) / |k_m|: the curl of the
    vector potential sum_m b_m cos(2 pi k_m . x + phi_m) / (2 pi |k_m|), so
    div u = 0 exactly.  Returns (k (m, 3) integer wave vectors, b (m, 3), phi (m,))."""
    rng = np.random.Generator(np.random.PCG64(1_000_003 + series_seed))
    k = rng.integers(-3, 4, size=(modes, 3))
    k[np.all(k == 0, axis=1)] = (1, 0, 0)
    b = rng.standard_normal((modes, 3))
    phi = rng.uniform(0, 2 * np.pi, modes)
    return k.astype(np.float64), b, phi


def velocity(pos: np.ndarray, field_) -> np.ndarray:
    """u at positions (n, 3) in the unit cube."""
    k, b, phi = field_
    kb = np.cross(k, b) / np.linalg.norm(k, axis=1)[:, None]  # (m, 3)
    arg = 2 * np.pi * pos @ k.T + phi[None, :]                 # (n, m)
    return -np.sin(arg) @ kb


def divergence(pos: np.ndarray, field_) -> np.ndarray:
    """div u at positions (analytic); zero up to rounding for every field here."""
    k, b, phi = field_
    kb = np.cross(k, b) / np.linalg.norm(k, axis=1)[:, None]
    arg = 2 * np.pi * pos @ k.T + phi[None, :]
    # d/dx_j of -sin(2 pi k.x + phi) kb_j = -2 pi cos(.) k_j kb_j, summed over j
    return -2 * np.pi * np.cos(arg) @ np.sum(k * kb, axis=1)


def tracer_positions(series_seed: int, frame: int, n: int = SERIES_TRACERS) -> np.ndarray:
    """Tracer positions (n, 3) in the periodic unit cube at `frame`: uniform at
    frame 0, then advected by velocity_modes(series_seed) with one midpoint
    (RK2) step of SERIES_DT per frame."""
    rng = np.random.Generator(np.random.PCG64(2_000_029 + series_seed))
    pos = rng.random((n, 3))
    f = velocity_modes(series_seed)
    for _ in range(frame):
        mid = pos + 0.5 * SERIES_DT * velocity(pos, f)
        pos = np.mod(pos + SERIES_DT * velocity(mid, f), 1.0)
    return pos


def series_frames(n_frames: int = 64, series_seed: int = 0, iterations: int = 100, sides=(512, 640, 768, 1024),
                  planes=(100, 400), tracers=(200, 3000)) -> list:
    """The uneven time series: frame i is a square hologram whose side is drawn
    from `sides`, with Nz from `planes` (inclusive), dz 2, dx 1.1, lambda 0.632
    (length units um); it images the first n_i (drawn from `tracers`) tracers
    of one advected population, each mapped from the unit cube to its own
    W x H x Nz box."""
    rng = np.random.Generator(np.random.PCG64(3_000_017 + series_seed))
    out = []
    for i in range(n_frames):
        h = w = int(rng.choice(sides))
        nz = int(rng.integers(planes[0], planes[1] + 1))
        nt = int(rng.integers(tracers[0], tracers[1] + 1))
        out.append(HoloConfig(name=f"series{series_seed}_frame{i:03d}_{w}x{h}x{nz}", width=w, height=h,
                              zero_padding=0, num_planes=nz, start_plane=2500.0, plane_stepsize=2.0,
                              resolution=1.1, wavelength=0.632, regularization_param=0.15,
                              regularization_TV_param=0.1, num_inverse_iterations=iterations, num_tv_iterations=5,
                              n_disks=nt, disk_radius=(1.0, 4.0), noise_sigma=0.02, seed=10_000 + i,
                              series_seed=series_seed, series_frame=i))
    return out


def object_masks(cfg: HoloConfig) -> dict:
    """Opaque-object masks per plane index: {z_index: mask (H, W) float64}."""
    rng = np.random.Generator(np.random.PCG64(cfg.seed))
    H, W, p = cfg.H, cfg.W, cfg.zero_padding
    masks: dict = {}

    def plane(k):
        if k not in masks:
            masks[k] = np.zeros((H, W), np.float64)
        return masks[k]

    if cfg.series_seed >= 0:
        pos = tracer_positions(cfg.series_seed, cfg.series_frame)[:cfg.n_disks]
        for x, y, z in pos:
            r = rng.uniform(*cfg.disk_radius)
            k = min(int(z * cfg.num_planes), cfg.num_planes - 1)
            _stamp_disk(plane(k), p + x * cfg.width, p + y * cfg.height, r)
        return masks

    for _ in range(cfg.n_disks):
        r = rng.uniform(*cfg.disk_radius)
        cx = p + rng.uniform(0, cfg.width)
        cy = p + rng.uniform(0, cfg.height)
        k = int(rng.integers(0, cfg.num_planes))
        _stamp_disk(plane(k), cx, cy, r)
    zscale = cfg.resolution / cfg.plane_stepsize  # rod z-extent in planes per pixel
    for _ in range(cfg.n_rods):
        L = rng.uniform(*cfg.rod_length)
        v = rng.standard_normal(3)
        v /= np.linalg.norm(v)
        cx = p + rng.uniform(0, cfg.width)
        cy = p + rng.uniform(0, cfg.height)
        cz = rng.uniform(0, cfg.num_planes - 1)
        n = max(2, int(np.ceil(L / 0.5)))
        for s in np.linspace(-L / 2, L / 2, n):
            k = int(round(cz + s * v[2] * zscale))
            if 0 <= k < cfg.num_planes:
                _stamp_disk(plane(k), cx + s * v[0], cy + s * v[1], cfg.rod_width / 2)
    return masks


def propagate_objects(cfg: HoloConfig, masks: dict) -> np.ndarray:
    """Field at the hologram plane, 1 + F^-1 sum_z H'_z F(-mask_z)."""
    H, W = cfg.H, cfg.W
    lam, dx = cfg.lam(), cfg.dx()
    zl = cfg.plane_list()
    fy = ((((np.arange(H) + H // 2) % H) - H // 2) / H)[:, None]
    fx = ((((np.arange(W) + W // 2) % W) - W // 2) / W)[None, :]
    a = (lam / dx) ** 2 * (fx ** 2 + fy ** 2)
    sm1 = np.where(a >= 1.0, -1.0, -a / (np.sqrt(np.maximum(1.0 - a, 0.0)) + 1.0))
    c = 2 * np.pi / lam * sm1
    S = np.zeros((H, W), np.complex128)
    for k in sorted(masks):
        S += np.exp(1j * zl[k] * c) * _fft2(-masks[k])
    return 1.0 + _ifft2(S)


def propagate_objects_torch(cfg: HoloConfig, masks: dict, device) -> np.ndarray:
    """propagate_objects in FP64 on a torch device (input generation only)."""
    import torch

    H, W = cfg.H, cfg.W
    lam, dx = cfg.lam(), cfg.dx()
    zl = cfg.plane_list()
    fy = ((((torch.arange(H, device=device, dtype=torch.float64) + H // 2) % H) - H // 2) / H)[:, None]
    fx = ((((torch.arange(W, device=device, dtype=torch.float64) + W // 2) % W) - W // 2) / W)[None, :]
    a = (lam / dx) ** 2 * (fx ** 2 + fy ** 2)
    sm1 = torch.where(a >= 1.0, torch.full_like(a, -1.0), -a / (torch.sqrt(torch.clamp(1.0 - a, min=0.0)) + 1.0))
    c = 2 * np.pi / lam * sm1
    S = torch.zeros((H, W), dtype=torch.complex128, device=device)
    for k in sorted(masks):
        m = torch.from_numpy(masks[k]).to(device)
        S += torch.polar(torch.ones_like(c), float(zl[k]) * c) * torch.fft.fft2(-m)
    return (1.0 + torch.fft.ifft2(S)).cpu().numpy()


def translated_frame(b: np.ndarray, k: int) -> np.ndarray:
    """Frame k of a series made by translating frame 0's particle field: the
    hologram of a translated field is the circularly shifted hologram (the
    transfer function is shift invariant and the planes are periodic)."""
    if k == 0:
        return b
    H, W = b.shape
    return np.roll(b, ((37 * k) % H, (53 * k) % W), axis=(0, 1)).copy()


def camera_image(cfg: HoloConfig, field_: np.ndarray) -> np.ndarray:
    """uint8 camera frame of the unpadded hologram area."""
    rng = np.random.Generator(np.random.PCG64(cfg.seed + 7919))
    p = cfg.zero_padding
    I = np.abs(field_[p:p + cfg.height, p:p + cfg.width]) ** 2
    I = 0.5 * I + cfg.noise_sigma * rng.standard_normal(I.shape)
    return np.round(np.clip(I, 0.0, 1.0) * 255.0).astype(np.uint8)


def preprocess(img: np.ndarray, zero_padding: int) -> np.ndarray:
    """Reference preprocessing without background: /255, I/mean - 1, zero pad
    (main_sparse_inverse.cu:115-124).  Returns float32 (H+2p, W+2p).  The
    reference allocates the padded image as (width+2p) rows x (height+2p)
    columns (hologram.cu:905), which only works for square inputs; rows and
    columns are kept apart here."""
    f = img.astype(np.float32) / np.float32(255.0)
    m = np.float64(f.astype(np.float64).mean())
    f = (f / np.float32(m) - np.float32(1.0)).astype(np.float32)
    h, w = f.shape
    out = np.zeros((h + 2 * zero_padding, w + 2 * zero_padding), np.float32)
    out[zero_padding:zero_padding + h, zero_padding:zero_padding + w] = f
    return out


def make_hologram(cfg: HoloConfig, cache_dir: str | None = None, device=None):
    """Return (uint8 camera image, preprocessed float32 hologram b).  With a
    torch `device` the propagation runs there in FP64 (faster for large
    frames; the result can differ from the CPU's in the last bits, so cached
    files record which was used)."""
    if cache_dir is None:
        cache_dir = os.environ.get("RIHVR_CACHE", "/tmp/rihvr_cache")
    tag = "" if device is None else "_dev"
    path = os.path.join(cache_dir, f"{cfg.name}_{cfg.key()}{tag}.npz")
    if os.path.exists(path):
        with np.load(path) as z:
            return z["img"], z["b"]
    masks = object_masks(cfg)
    U = propagate_objects(cfg, masks) if device is None else propagate_objects_torch(cfg, masks, device)
    img = camera_image(cfg, U)
    b = preprocess(img, cfg.zero_padding)
    try:
        os.makedirs(cache_dir, exist_ok=True)
        tmp = path + f".{os.getpid()}.tmp.npz"
        np.savez(tmp, img=img, b=b)
        os.replace(tmp, path)
    except OSError:
        pass
    return img, b
