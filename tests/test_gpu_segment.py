"""GPU segmentation (rihvr_segment_intensity / rihvr_segment, through the C
ABI) against the oracle's orc_segment: every field of every object equal, the
floats bit for bit, and the objects in the same order.

Covers widths that are not multiples of the 32-voxel word, closing radii 0 to
3, both neighbourhoods (the reference's row-continuing one and the geometric
one), the size filter, device-resident input, the segmentation of a solved
volume, and a large volume of separated balls whose centroids are known.
"""
import numpy as np
import pytest

import oracle as O
from test_segment import as_rows, blob_stack, random_stack, same_bits

pytestmark = pytest.mark.gpu


CASES = [
    # seed, (nz, h, w), min_intensity, close_size, min_area, faithful, kind
    (0, (5, 12, 14), 1.0, 0, 1, 1, "random"),
    (1, (6, 20, 33), 1.0, 1, 1, 1, "random"),
    (2, (8, 31, 50), 30.0, 0, 2, 1, "random"),
    (3, (8, 31, 50), 30.0, 0, 2, 0, "random"),
    (4, (12, 40, 64), 20.0, 1, 2, 1, "blobs"),
    (5, (12, 40, 70), 20.0, 2, 1, 0, "blobs"),
    (6, (16, 48, 100), 10.0, 3, 2, 1, "blobs"),
    (7, (20, 64, 96), 5.0, 3, 2, 0, "blobs"),
    (8, (10, 33, 129), 2.0, 1, 3, 1, "blobs"),
]


@pytest.mark.parametrize("seed,shape,mi,cs,ma,faithful,kind", CASES)
def test_segment_matches_oracle(rihvr, seed, shape, mi, cs, ma, faithful, kind):
    nz, h, w = shape
    I = random_stack(seed, *shape, density=0.2) if kind == "random" else \
        blob_stack(seed, *shape, nblobs=max(4, nz * h * w // 3000))
    sp = rihvr.segment_params(min_intensity=mi, close_size=cs, min_area=ma, faithful=faithful)
    got, info = rihvr.segment_intensity(I, sp)
    ref, (rmax, rthr) = O.segment(I, mi, cs, ma, faithful)
    assert info["max_intensity"] == rmax and info["threshold"] == rthr
    assert len(ref) > 0
    same_bits(as_rows(got), as_rows(ref))


def test_row_continuing_neighbourhood(rihvr):
    I = np.zeros((3, 6, 40), np.float32)
    I[1, 2, 39] = 50.0
    I[1, 3, 0] = 60.0
    f, _ = rihvr.segment_intensity(I, rihvr.segment_params(close_size=0, min_area=1, faithful=1))
    g, _ = rihvr.segment_intensity(I, rihvr.segment_params(close_size=0, min_area=1, faithful=0))
    assert len(f) == 1 and f[0]["num_voxels"] == 2
    assert len(g) == 2


def test_device_input_equals_host_input(rihvr):
    import torch

    I = blob_stack(21, 16, 64, 80, nblobs=30)
    sp = rihvr.segment_params(min_intensity=5.0, close_size=2)
    a, _ = rihvr.segment_intensity(I, sp)
    b, _ = rihvr.segment_intensity(torch.from_numpy(I).cuda(), sp)
    same_bits(as_rows(a), as_rows(b))
    # two calls in a row give the same objects
    c, _ = rihvr.segment_intensity(I, sp)
    same_bits(as_rows(a), as_rows(c))


@pytest.mark.parametrize("storage", [0, 1, 2])
def test_segment_of_a_solved_volume(rihvr, synthmod, storage):
    """Reconstruct a small hologram (FP32, BF16 or FP16 volume storage), then
    segment the solver's volume in place: the oracle gets the voxel
    intensities |v|^2 (FP32, no contraction) of the volume the solver
    returns."""
    cfg = synthmod.config1()
    cfg.num_planes = 16
    _, b = synthmod.make_hologram(cfg)
    p = rihvr.params_from_config(cfg, storage=storage, faithful=int(storage != 1))  # BF16: faithful = 0
    with rihvr.SparseCompressiveHolo(p, cfg.W, cfg.H) as s:
        s.setHologram(b)
        s.iterate(15)
        vol = s.getVolume()
        sp = rihvr.segment_params(min_intensity=20.0, close_size=1)
        got, info = s.segment(sp)
    I = (vol.real * vol.real + vol.imag * vol.imag).astype(np.float32)
    ref, _ = O.segment(I, 20.0, 1, 2, 1)
    assert len(ref) > 0
    same_bits(as_rows(got), as_rows(ref))


def test_separated_balls_give_their_centres(rihvr):
    """1000 balls of radius 2 in a 512 x 512 x 200 volume, apart from each
    other and from the borders: one object each, centroids at the centres."""
    rng = np.random.default_rng(5)
    nz, h, w = 200, 512, 512
    I = np.zeros((nz, h, w), np.float32)
    centres = []
    occ = np.zeros((nz // 8, h // 8, w // 8), bool)
    while len(centres) < 1000:
        c = (rng.integers(1, nz // 8 - 1), rng.integers(1, h // 8 - 1), rng.integers(1, w // 8 - 1))
        if occ[c]:
            continue
        occ[c] = True
        centres.append((c[0] * 8 + 4, c[1] * 8 + 4, c[2] * 8 + 4))
    zz, yy, xx = np.mgrid[-2:3, -2:3, -2:3]
    ballm = zz * zz + yy * yy + xx * xx <= 4
    for cz, cy, cx in centres:
        I[cz - 2:cz + 3, cy - 2:cy + 3, cx - 2:cx + 3][ballm] = 36.0  # sqrt and square exact
    for faithful in (0, 1):
        got, info = rihvr.segment_intensity(I, rihvr.segment_params(close_size=0, min_area=1, faithful=faithful))
        assert len(got) == 1000
        # objects come in order of their smallest index (the ball's lowest voxel)
        first = sorted(centres, key=lambda c: ((c[0] - 2) * h + c[1]) * w + c[2])
        for o, (cz, cy, cx) in zip(got, first):
            assert (o["x"], o["y"], o["z"]) == (cx, cy, cz)
            assert (o["wx"], o["wy"], o["wz"]) == (cx, cy, cz)
            assert o["num_voxels"] == int(ballm.sum())
