"""Learned warm start: training data, training and evaluation of the 3-D U-Net
(``UNet``, ``rihvr_unet_*``).

Training holograms are synthesised by the project's forward model
(``synth.make_hologram``: opaque disks on the planes, Rayleigh-Sommerfeld
propagation, |1 + field|^2, camera noise, the reference's preprocessing).  For
each one the library computes the back-propagated volume xbp = t A^H b and
the plain-FISTA solution x* after the configured iterations; the network
learns x0 = g * alpha * xbp against x*.  Evaluation runs plain FISTA from zero
(the reference run) and FISTA from the network's x0 on held-out holograms and counts
the iterations each needs to come within 1e-3 (relative) of plain FISTA's
final objective.

    python warmstart.py train --out weights.npy [--samples 1024 --epochs 50]
    python warmstart.py train4 [--holograms 256 --crops 4 --epochs 8]   # 512x512x200, full-depth crops
    python warmstart.py evaluate --weights weights.npy [--samples 16]
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import sys
import time

import numpy as np

_PKG = __name__.rsplit(".", 1)[0] if "." in __name__ else None


def _pkg():
    if _PKG:
        return importlib.import_module(_PKG)
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    return importlib.import_module(os.path.basename(os.path.dirname(os.path.abspath(__file__))))


def _synth():
    return importlib.import_module(_pkg().__name__ + ".synth")


# The learned-warm-start workload at training size: the physics of the
# 512x512x200 configuration (dz 2 um, dx 1.1 um, lambda 0.632 um, 1000+ um
# from the hologram), at 128x128x32 voxels
SIZE, PLANES = 128, 32
WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), f"warmstart_unet_{PLANES}x{SIZE}x{SIZE}.npy")


def sample_config(seed: int, size: int = SIZE, planes: int = PLANES, iterations: int = 100):
    synth = _synth()
    rng = np.random.default_rng(seed + 1_000_003)
    return synth.HoloConfig(
        name=f"warmstart_{size}x{size}x{planes}_s{seed}", width=size, height=size, zero_padding=0,
        num_planes=planes, start_plane=1000.0, plane_stepsize=2.0, resolution=1.1, wavelength=0.632,
        regularization_param=0.15, regularization_TV_param=0.1, num_inverse_iterations=iterations,
        num_tv_iterations=5, n_disks=int(rng.integers(20, 121)), disk_radius=(1.0, 4.0),
        noise_sigma=float(rng.uniform(0.005, 0.03)), seed=seed)


# The configuration the warm start is specified on: 512 x 512 x 200 voxels
# with the same optics, 500-3000 particles (half disks of radius 1-4 px, half
# rods 10-60 px long), camera noise sigma 0.005-0.03.
C4_SIZE, C4_PLANES = 512, 200


def config4_sample(seed: int, size: int = C4_SIZE, planes: int = C4_PLANES, iterations: int = 100):
    synth = _synth()
    rng = np.random.default_rng(seed + 2_000_003)
    n = int(rng.integers(500, 3001))
    return synth.HoloConfig(
        name=f"warmstart_c4_{size}x{size}x{planes}_s{seed}", width=size, height=size, zero_padding=0,
        num_planes=planes, start_plane=1000.0, plane_stepsize=2.0, resolution=1.1, wavelength=0.632,
        regularization_param=0.15, regularization_TV_param=0.1, num_inverse_iterations=iterations,
        num_tv_iterations=5, n_disks=n // 2, disk_radius=(1.0, 4.0), n_rods=n - n // 2, rod_length=(10.0, 60.0),
        rod_width=2.0, noise_sigma=float(rng.uniform(0.005, 0.03)), seed=seed)


def make_set(seeds, size: int = SIZE, planes: int = PLANES, iterations: int = 100, log=None):
    """[(b, xbp, x*)] with xbp and x* as CUDA complex64 tensors."""
    import torch

    rihvr = _pkg()
    synth = _synth()
    out = []
    cfg0 = sample_config(int(seeds[0]), size, planes, iterations)
    p = rihvr.params_from_config(cfg0, record_objective=0)
    with rihvr.SparseCompressiveHolo(p, size, size) as s:
        for i, sd in enumerate(seeds):
            cfg = sample_config(int(sd), size, planes, iterations)
            _, b = synth.make_hologram(cfg)
            s.setHologram(b)
            xbp = torch.from_numpy(s.backpropagate()).cuda()
            s.iterate(iterations)
            xs = torch.from_numpy(s.getVolume()).cuda()
            out.append((b, xbp, xs))
            if log and (i + 1) % 32 == 0:
                log(f"  {i + 1}/{len(seeds)} samples")
    return out


# Training on the 512 x 512 x 200 configuration: full-depth crops of
# C4_CROP x C4_CROP pixels.  A crop keeps every plane, so its back-propagated
# field holds the same depth range and its RMS (by which the network divides
# its input) is close to the whole volume's.
C4_CROP = 128
C4_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)),
                          f"warmstart_unet_c4_{C4_PLANES}x{C4_CROP}x{C4_CROP}.npy")


def make_set_c4(seeds, crops: int = 4, iterations: int = 100, log=None, seed: int = 0):
    """[(None, xbp crop, x* crop)] from 512 x 512 x 200 holograms, `crops`
    random full-depth crops of each, as CUDA complex64 tensors; the volumes
    stay on the device."""
    import ctypes

    import torch

    rihvr = _pkg()
    synth = _synth()
    rng = np.random.default_rng(seed)
    S, Z, c = C4_SIZE, C4_PLANES, C4_CROP
    cfg0 = config4_sample(int(seeds[0]))
    p = rihvr.params_from_config(cfg0, record_objective=0)
    out = []
    xbp = torch.empty((Z, S, S), dtype=torch.complex64, device="cuda")
    xs = torch.empty_like(xbp)
    L = rihvr.load_library()
    with rihvr.SparseCompressiveHolo(p, S, S) as sol:
        for i, sd in enumerate(seeds):
            _, b = synth.make_hologram(config4_sample(int(sd), iterations=iterations), device="cuda")
            sol.setHologram(b)
            rihvr._check(L.rihvr_backpropagate(sol._h, ctypes.c_void_p(xbp.data_ptr()), 1), "rihvr_backpropagate")
            sol.iterate(iterations)
            rihvr._check(L.rihvr_get_volume(sol._h, ctypes.c_void_p(xs.data_ptr()), 1), "rihvr_get_volume")
            torch.cuda.synchronize()
            for _ in range(crops):
                y0, x0 = (int(v) for v in rng.integers(0, S - c + 1, 2))
                out.append((None, xbp[:, y0:y0 + c, x0:x0 + c].contiguous(), xs[:, y0:y0 + c, x0:x0 + c].contiguous()))
            if log and (i + 1) % 16 == 0:
                log(f"  {i + 1}/{len(seeds)} holograms")
    return out


def train(net, data, epochs: int = 20, lr: float = 1e-3, seed: int = 0, log=None):
    """Adam over shuffled samples, learning rate halved at 50 % and 75 % of the
    epochs.  Returns the mean loss of every epoch."""
    rng = np.random.default_rng(seed)
    hist = []
    for ep in range(epochs):
        f = 1.0 if ep < epochs // 2 else (0.5 if ep < 3 * epochs // 4 else 0.25)
        losses = [net.train_step(data[i][1], data[i][2], lr * f) for i in rng.permutation(len(data))]
        hist.append(float(np.mean(losses)))
        if log:
            log(f"  epoch {ep + 1}/{epochs}: loss {hist[-1]:.4f}")
    return hist


def _iters_to(f, target, tol=1e-3):
    hit = np.nonzero(np.abs(f - target) <= tol * abs(target))[0]
    return int(hit[0]) + 1 if len(hit) else None


def evaluate(net, seeds, size: int = SIZE, planes: int = PLANES, iterations: int = 100, tol: float = 1e-3,
             sampler=None, device=None):
    """Per held-out hologram: plain FISTA's final objective (the target), the
    iterations plain FISTA and the warm start need to come within tol of it,
    and the device time of both solves to that point (the warm start's
    including the network).  `sampler(seed, size, planes, iterations)` makes
    the holograms' configurations (sample_config by default); `device`
    synthesises them there."""
    import torch

    rihvr = _pkg()
    synth = _synth()
    sampler = sampler or sample_config
    cfg0 = sampler(int(seeds[0]), size, planes, iterations)
    rows = []
    rec = rihvr.params_from_config(cfg0, record_objective=1)
    fast = rihvr.params_from_config(cfg0, record_objective=0)
    with rihvr.SparseCompressiveHolo(rec, size, size) as s, rihvr.SparseCompressiveHolo(fast, size, size) as t:
        for sd in seeds:
            cfg = sampler(int(sd), size, planes, iterations)
            _, b = synth.make_hologram(cfg, device=device)
            s.setHologram(b)
            s.iterate(iterations)
            fp = s.iterations()["f_x"]
            target = float(fp[-1])
            s.setHologram(b)
            s.warmStart(net)
            s.iterate(iterations)
            fw = s.iterations()["f_x"]
            kp, kw = _iters_to(fp, target, tol), _iters_to(fw, target, tol)
            # device time to those points, without objective recording
            t.setHologram(b)
            t.iterate(1)  # warm (graphs, tables)
            stream = torch.cuda.ExternalStream(t.stream())
            e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
            t.setHologram(b)
            e[0].record(stream)
            t.iterate(kp or iterations)
            e[1].record(stream)
            t.setHologram(b)
            e[2].record(stream)
            t.warmStart(net)
            t.iterate(kw or iterations)
            e[3].record(stream)
            e[3].synchronize()
            rows.append({"seed": int(sd), "target": target, "iters_plain": kp, "iters_warm": kw,
                         "ms_plain": e[0].elapsed_time(e[1]), "ms_warm": e[2].elapsed_time(e[3]),
                         "f_warm_at_0": float(fw[0]), "f_plain_at_0": float(fp[0])})
    return rows


def summary(rows):
    kp = [r["iters_plain"] for r in rows if r["iters_plain"]]
    kw = [r["iters_warm"] if r["iters_warm"] else 101 for r in rows]
    mp = float(np.mean([r["ms_plain"] for r in rows]))
    mw = float(np.mean([r["ms_warm"] for r in rows]))
    return {"holograms": len(rows), "mean_iters_plain": float(np.mean(kp)), "mean_iters_warm": float(np.mean(kw)),
            "reached_warm": sum(1 for r in rows if r["iters_warm"]), "mean_ms_plain": mp, "mean_ms_warm": mw,
            "speedup_time": mp / mw if mw > 0 else None}


def main(argv=None):
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    tr = sub.add_parser("train")
    tr.add_argument("--out", default=WEIGHTS)
    tr.add_argument("--samples", type=int, default=1024)
    tr.add_argument("--epochs", type=int, default=50)
    tr.add_argument("--lr", type=float, default=1e-3)
    tr.add_argument("--eval", type=int, default=8)
    t4 = sub.add_parser("train4", help="train on full-depth crops of 512x512x200 holograms")
    t4.add_argument("--out", default=C4_WEIGHTS)
    t4.add_argument("--holograms", type=int, default=256)
    t4.add_argument("--crops", type=int, default=4)
    t4.add_argument("--epochs", type=int, default=8)
    t4.add_argument("--lr", type=float, default=1e-3)
    t4.add_argument("--init", default=WEIGHTS, help="starting weights ('' for a fresh network)")
    t4.add_argument("--eval", type=int, default=16)
    ev = sub.add_parser("evaluate")
    ev.add_argument("--weights", default=WEIGHTS)
    ev.add_argument("--samples", type=int, default=16)
    a = ap.parse_args(argv)
    rihvr = _pkg()
    log = lambda m: print(m, flush=True)
    if a.cmd == "train4":
        t0 = time.perf_counter()
        data = make_set_c4(np.arange(500_000, 500_000 + a.holograms), a.crops, log=log)
        t1 = time.perf_counter()
        log(f"training set: {len(data)} crops of {a.holograms} holograms in {t1 - t0:.1f} s")
        with rihvr.UNet(C4_PLANES, C4_CROP, C4_CROP, seed=0) as net:
            if a.init:
                net.load(a.init)
            hist = train(net, data, a.epochs, a.lr, log=log)
            net.save(a.out)
        t2 = time.perf_counter()
        del data
        with rihvr.UNet(C4_PLANES, C4_SIZE, C4_SIZE) as big:
            big.load(a.out)
            rows = evaluate(big, np.arange(400_000, 400_000 + a.eval), size=C4_SIZE, planes=C4_PLANES,
                            sampler=config4_sample, device="cuda")
        print(json.dumps({"train_s": t2 - t1, "data_s": t1 - t0, "losses": hist, "eval": summary(rows),
                          "rows": rows}), flush=True)
        return 0
    with rihvr.UNet(PLANES, SIZE, SIZE, seed=0) as net:
        if a.cmd == "train":
            t0 = time.perf_counter()
            data = make_set(np.arange(a.samples), log=log)
            t1 = time.perf_counter()
            log(f"training set: {a.samples} holograms in {t1 - t0:.1f} s")
            hist = train(net, data, a.epochs, a.lr, log=log)
            t2 = time.perf_counter()
            net.save(a.out)
            rows = evaluate(net, np.arange(100_000, 100_000 + a.eval))
            print(json.dumps({"train_s": t2 - t1, "data_s": t1 - t0, "losses": hist, "eval": summary(rows),
                              "rows": rows}), flush=True)
        else:
            net.load(a.weights)
            rows = evaluate(net, np.arange(100_000, 100_000 + a.samples))
            print(json.dumps({"eval": summary(rows), "rows": rows}), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
