"""FP64-oracle fixture for the 384x384x40 FISTA+TV workload (256x256 hologram
padded by 64 px per side, Nz=40, 100 FISTA / 5 TV iterations, faithful mode).

The full oracle run takes about a minute on 8 cores, so the GPU test compares
against this committed summary instead of re-running it: the objective and
decision history of every iteration, per-plane L1/L2 norms of the final
momentum point and a few 64x64 crops of it.

    python tests/golden/make_c1_golden.py
"""
import hashlib
import importlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402

S = importlib.import_module("rihvr---regularized-inverse-holographic-volume-reconstruction_b200.synth")
OUT = os.path.join(HERE, "oracle_c1_384x384x40.npz")
CROP_PLANES = (0, 13, 27, 39)


def crop(a):
    return a[..., 160:224, 160:224]


def main():
    cfg = S.config1()
    img, b = S.make_hologram(cfg)
    p = O.OracleParams(W=cfg.W, H=cfg.H, z=cfg.plane_list(), dx=cfg.dx(), lam=cfg.lam(), l1=cfg.l1(),
                       tv=cfg.tv(), n_tv=cfg.num_tv_iterations, mode=7, faithful=1)
    log, X, P, est, f0 = O.solve(p, b.astype(np.float64), cfg.num_inverse_iterations)
    np.savez_compressed(
        OUT,
        b_sha1=np.frombuffer(hashlib.sha1(b.tobytes()).digest(), np.uint8),
        f0=f0,
        f_x=log["f_x"], f_prox=log["f_prox"], f_resid_x=log["f_resid_x"], ratio=log["ratio"], t=log["t"],
        beta=log["beta"], backtracks=log["backtracks"], restarted=log["restarted"],
        restart_sum=log["restart_sum"], lim=log["lim"],
        plane_l1=np.abs(X).sum(axis=(1, 2)), plane_l2=np.sqrt((np.abs(X) ** 2).sum(axis=(1, 2))),
        crop_planes=np.array(CROP_PLANES), crops=crop(X[list(CROP_PLANES)]),
        est_crop=crop(est),
    )
    print(OUT, os.path.getsize(OUT), "bytes; final f_x", log["f_x"][-1])


if __name__ == "__main__":
    main()
