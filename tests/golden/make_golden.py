"""Generate the golden fixtures that pin the C oracle.

The reference ships no golden data for this path (its Test/ suites are not
distributed), so the fixtures come from the independent numpy restatement in
``tests/numpy_ref.py`` (numpy.fft, vectorised stencils) on a small seeded case.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
import numpy_ref as R  # noqa: E402

OUT = os.path.join(HERE, "oracle_pin_16x24x3.npz")


def case():
    rng = np.random.Generator(np.random.PCG64(20240607))
    H, W, Nz = 16, 24, 3
    z = np.array([np.float32(150.0) + np.float32(i) * np.float32(35.0) for i in range(Nz)], np.float64)
    dx, lam = float(np.float32(2.0)), float(np.float32(0.632))
    # a sparse random object volume and a hologram made from it
    obj = np.zeros((Nz, H, W), np.complex128)
    for _ in range(6):
        k, y, x = rng.integers(0, Nz), rng.integers(0, H), rng.integers(0, W)
        obj[k, y, x] = -(0.5 + rng.random()) * np.exp(1j * rng.uniform(0, 2 * np.pi))
    c = R.phase_coeff(H, W, dx, lam)
    b = R.forward(obj, z, c) + 0.01 * rng.standard_normal((H, W))
    x = 0.1 * (rng.standard_normal((Nz, H, W)) + 1j * rng.standard_normal((Nz, H, W)))
    r = rng.standard_normal((H, W))
    return dict(H=H, W=W, Nz=Nz, z=z, dx=dx, lam=lam, b=b, x=x, r=r, c=c)


def main():
    d = case()
    z, c = d["z"], d["c"]
    out = dict(z=d["z"], dx=d["dx"], lam=d["lam"], b=d["b"], x=d["x"], r=d["r"], c=c)
    out["forward_x"] = R.forward(d["x"], z, c)
    out["adjoint_r"] = R.adjoint(d["r"], z, c)
    G = out["adjoint_r"]
    t = 0.3
    l1, tv = 0.02, 0.05
    for mode in (5, 6, 7):
        for faithful in (0, 1):
            out[f"prox_m{mode}_f{faithful}"] = R.prox(d["x"], G, t, l1, tv, 5, mode, faithful)
    for mode, t0 in ((7, 0.0), (7, 3.0 / d["Nz"]), (5, 3.0 / d["Nz"]), (6, 2.0 / d["Nz"])):
        log, X, P, dX = R.solve(d["b"], z, d["dx"], d["lam"], l1, tv, 5, mode, 1, 12, t0=t0)
        tag = f"solve_m{mode}_t{int(round(t0 * d['Nz']))}"
        out[tag + "_fx"] = np.array([e["f_x"] for e in log])
        out[tag + "_bt"] = np.array([e["backtracks"] for e in log])
        out[tag + "_rs"] = np.array([e["restarted"] for e in log])
        out[tag + "_X"] = X
    np.savez_compressed(OUT, **out)
    print(OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
