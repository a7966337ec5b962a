"""Literal Python restatement of the reference's segmentation program, for
tiny volumes, used to pin the C oracle's ``orc_segment``.

Follows the reference's data structures: per-plane COO lists of (index,
value) as ``SparseVolume`` holds them, ``loadData`` turning each voxel-file
intensity I into the value (sqrt(I), 0) (src/core/sparse_volume.cu:562-665),
``calcMaxIntensity`` (:482-516), ``binarize`` with its mask
(src/core/sparse_segmentation.cu:39-112), ``simpleMorph`` counting ball
positions (:265-372), ``labelConnectedComponents`` with its sorted index
lists, binary search and repeated minimum sweeps (:374-555), then
``ObjectCloud``'s first-appearance objects, ``includeIntensity`` and
``blobSizeFilter`` (object_cloud.cu:127-328) and ``Blob3d``'s centroid,
weighted centroid, max, mean and bounds (blob3d.cu).  FP32 values are numpy
float32 scalars so each operation rounds as the reference's does.  Planes
outside the volume hold no voxels (the reference reads past its plane arrays
there).
"""
import bisect

import numpy as np

f32 = np.float32


def load(I):
    """SparseVolume::loadData: the voxel file's non-zero intensities."""
    nz, h, w = I.shape
    planes = []
    for z in range(nz):
        flat = I[z].ravel()
        idx = [int(i) for i in np.flatnonzero(flat != 0)]
        vals = [(f32(np.sqrt(f32(flat[i]))), f32(0)) for i in idx]
        planes.append((idx, vals))
    return planes


def intensity(v):
    return f32(f32(v[0] * v[0]) + f32(v[1] * v[1]))


def ball(cs):
    return [(sx, sy, sz) for sz in range(-cs, cs + 1) for sx in range(-cs, cs + 1) for sy in range(-cs, cs + 1)
            if sx * sx + sy * sy + sz * sz <= cs * cs]


def simple_morph(binary, w, h, cs, erode):
    """Count ball positions around every stored voxel; erosion keeps counts
    above (ball size - 0.1), dilation every non-zero count."""
    nz = len(binary)
    strel = ball(cs)
    out = []
    for z in range(nz):
        cnt = np.zeros(w * h, np.float32)
        for sx, sy, sz in strel:
            pz = z + sz
            if pz < 0 or pz >= nz:
                continue
            for index in binary[pz][0]:
                x, y = index % w, index // w
                tx, ty = x + sx, y + sy
                if 0 <= tx < w and 0 <= ty < h:
                    cnt[ty * w + tx] += 1
        if erode:
            thr = len(strel) - 0.1
            cnt = np.where(cnt > thr, cnt, 0)
        idx = [int(i) for i in np.flatnonzero(cnt != 0)]
        out.append((idx, [(f32(cnt[i]), f32(0)) for i in idx]))
    return out


def contains(arr, target):
    k = bisect.bisect_left(arr, target)
    return k if k < len(arr) and arr[k] == target else -1


def label(binary, w, h, faithful):
    nz = len(binary)
    idx = [sorted(p[0]) for p in binary]
    lab = [[z * w * h + i for i in idx[z]] for z in range(nz)]
    offsets = [ys * w + xs for xs in (-1, 0, 1) for ys in (-1, 0, 1)]
    nbrs = []
    for z in range(nz):
        pl = []
        for i in idx[z]:
            x, y = i % w, i // w
            lst = []
            for oid, o in enumerate(offsets):
                xs, ys = oid // 3 - 1, oid % 3 - 1
                for zs in (-1, 0, 1):
                    if z + zs < 0 or z + zs >= nz:
                        continue
                    t = i + o
                    if not faithful and not (0 <= x + xs < w and 0 <= y + ys < h):
                        continue
                    if t < 0:
                        continue
                    d = contains(idx[z + zs], t)
                    if d >= 0:
                        lst.append((z + zs, d))
            pl.append(lst)
        nbrs.append(pl)
    changed = True
    while changed:
        changed = False
        for z in range(nz):
            for k in range(len(idx[z])):
                v = lab[z][k]
                for zz, d in nbrs[z][k]:
                    if lab[zz][d] < v:
                        v = lab[zz][d]
                        changed = True
                lab[z][k] = v
    return idx, lab


def segment(I, min_intensity=1.0, close_size=3, min_area=2, faithful=1):
    nz, h, w = I.shape
    vol = load(I)
    max_int = 0.0
    for idx, vals in vol:
        for v in vals:
            t = float(intensity(v))
            if t > max_int:
                max_int = t
    thr = min_intensity * max_int / 256.0
    binary, masked = [], []
    for idx, vals in vol:
        b_idx, m_idx, m_val = [], [], []
        for i, v in zip(idx, vals):
            if float(intensity(v)) > thr:
                b_idx.append(i)
                m_idx.append(i)
                m_val.append(v)
        binary.append((b_idx, [(f32(1), f32(0))] * len(b_idx)))
        masked.append(dict(zip(m_idx, m_val)))
    if close_size > 0:
        binary = simple_morph(binary, w, h, close_size, erode=False)
        binary = simple_morph(binary, w, h, close_size, erode=True)
    idx, lab = label(binary, w, h, faithful)
    ids, voxels = [], []
    for z in range(nz):
        for k, i in enumerate(idx[z]):
            L = lab[z][k] & 0xffffffff
            if L not in ids:
                ids.append(L)
                voxels.append([])
            voxels[ids.index(L)].append((z, i))
    objs = []
    for vl in voxels:
        n = len(vl)
        sx = sy = sz = 0
        wsx = wsy = wsz = wsum = f32(0)
        vals = []
        xs, ys, zs = [], [], []
        for z, i in vl:
            x, y = i % w, i // w
            sx += x
            sy += y
            sz += z
            v = masked[z].get(i, (f32(0), f32(0)))
            q = intensity(v)
            vals.append(q)
            wsx = f32(wsx + f32(q * f32(x)))
            wsy = f32(wsy + f32(q * f32(y)))
            wsz = f32(wsz + f32(q * f32(z)))
            wsum = f32(wsum + q)
            xs.append(x)
            ys.append(y)
            zs.append(z)
        mean_sum = 0.0
        for q in vals:
            mean_sum += float(q)
        with np.errstate(divide="ignore", invalid="ignore"):
            objs.append((f32(f32(sx) / f32(n)), f32(f32(sy) / f32(n)), f32(f32(sz) / f32(n)),
                         f32(wsx / wsum), f32(wsy / wsum), f32(wsz / wsum), n, max(vals),
                         f32(f32(mean_sum) / f32(n)), min(xs), max(xs), min(ys), max(ys), min(zs), max(zs)))
    k = 0
    while k < len(objs):
        if objs[k][6] < min_area:
            objs[k] = objs[-1]
            objs.pop()
            continue
        k += 1
    return objs, (max_int, thr)
