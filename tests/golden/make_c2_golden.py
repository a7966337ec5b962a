"""FP64-oracle objective history for the 1024x1024x1000 workload (100 FISTA /
5 TV iterations, faithful mode): the target of the time-to-objective metric.

The oracle needs three FP64 complex volumes (about 50 GB of host memory) and
roughly an hour on 8 cores, so the result is committed as a small JSON file:
the objective at every iteration, the backtracking/restart decisions and a
digest of the input hologram.

    python tests/golden/make_c2_golden.py [--threads N] [--iters K]
"""
import argparse
import hashlib
import importlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402

S = importlib.import_module("rihvr---regularized-inverse-holographic-volume-reconstruction_b200.synth")
OUT = os.path.join(HERE, "oracle_c2_1024x1024x1000.json")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--iters", type=int, default=0)
    a = ap.parse_args()
    cfg = S.config2()
    n = a.iters or cfg.num_inverse_iterations
    _, b = S.make_hologram(cfg)
    p = O.OracleParams(W=cfg.W, H=cfg.H, z=cfg.plane_list(), dx=cfg.dx(), lam=cfg.lam(), l1=cfg.l1(),
                       tv=cfg.tv(), n_tv=cfg.num_tv_iterations, mode=7, faithful=1, n_threads=a.threads)
    t0 = time.time()
    log, _, _, _, f0 = O.solve(p, b.astype(np.float64), n, want_volumes=False)
    dt = time.time() - t0
    out = {
        "workload": cfg.name, "iterations": n, "b_sha1": hashlib.sha1(b.tobytes()).hexdigest(),
        "f0": f0, "f_x": log["f_x"].tolist(), "f_prox": log["f_prox"].tolist(),
        "backtracks": log["backtracks"].tolist(), "restarted": log["restarted"].tolist(),
        "ratio": log["ratio"].tolist(), "t": log["t"].tolist(),
        "oracle_seconds": dt, "oracle_threads": a.threads or O.num_threads(),
    }
    with open(OUT, "w") as f:
        json.dump(out, f)
    print(OUT, "final f_x", out["f_x"][-1], f"{dt:.0f} s")


if __name__ == "__main__":
    main()
