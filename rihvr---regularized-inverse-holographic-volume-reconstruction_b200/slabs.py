"""Z-slab sharding of one hologram's volume.

The reference reconstructs a hologram's whole volume on one GPU
(src/core/sparse_compressive_holo.cu:173-633).  With a plane-separable prox
(modes 5 and 7) the volume splits along z: each slab holds a contiguous range
of planes, and one FISTA attempt needs only the sum of the slabs' partial
spectra (one H x W complex plane) and of eight FP64 sums (rihvr_slab_iterate
in include/rihvr.h).  Slabs either share one process (one context per slab,
on one device or on several with peer access) or sit one per process, e.g.
one process per GPU, summing over the processes through a reducer built on
torch.distributed here.
"""
from __future__ import annotations

import ctypes

import numpy as np

DTYPE_F32, DTYPE_F64 = 0, 1

SUM_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_longlong, ctypes.c_int,
                          ctypes.c_int)


class ReducerStruct(ctypes.Structure):
    """rihvr_slab_reducer (include/rihvr.h)."""
    _fields_ = [("sum", SUM_FN), ("user", ctypes.c_void_p), ("host_staged", ctypes.c_int)]


def slab_bounds(num_planes: int, n_slabs: int, index: int) -> tuple:
    """(z_first, z_count) of slab `index` of `n_slabs` contiguous slabs whose
    plane counts differ by at most one."""
    if n_slabs < 1 or not (0 <= index < n_slabs) or num_planes < n_slabs:
        raise ValueError("bad slab partition arguments")
    base, extra = divmod(int(num_planes), int(n_slabs))
    first = index * base + min(index, extra)
    return first, base + (1 if index < extra else 0)


class SlabReducer:
    """A rihvr_slab_reducer around a Python function sum_(array) that replaces
    the values of `array` (numpy on the host, a torch CUDA tensor on the
    device) by their sum over the processes.  Keep the object alive while the
    library may call it."""

    def __init__(self, sum_host, sum_device=None, host_staged: bool = False):
        self._sum_host = sum_host
        self._sum_device = sum_device
        self.errors = []

        def _call(user, data, count, dtype, on_device):
            try:
                if on_device:
                    if self._sum_device is None:
                        raise RuntimeError("device data given to a host-only reducer")
                    self._sum_device(_device_view(data, count, dtype))
                else:
                    ct = ctypes.c_float if dtype == DTYPE_F32 else ctypes.c_double
                    self._sum_host(np.ctypeslib.as_array((ct * int(count)).from_address(data)))
                return 0
            except Exception as e:  # reported to the library as a non-zero status
                self.errors.append(repr(e))
                return 1

        self._fn = SUM_FN(_call)
        self.struct = ReducerStruct(self._fn, None, 1 if (host_staged or sum_device is None) else 0)


def _device_view(ptr: int, count: int, dtype: int):
    import torch

    class _View:
        __cuda_array_interface__ = {"shape": (int(count),), "typestr": "<f4" if dtype == DTYPE_F32 else "<f8",
                                    "data": (int(ptr), False), "version": 3}

    return torch.as_tensor(_View(), device="cuda")


def torch_reducer(group=None, host_staged: bool | None = None) -> SlabReducer:
    """Sum over the ranks of a torch.distributed process group.  NCCL groups
    reduce the spectrum in device memory; gloo groups (host_staged by
    default) reduce host copies."""
    import torch
    import torch.distributed as dist

    nccl = dist.get_backend(group) == "nccl"
    if host_staged is None:
        host_staged = not nccl

    def sum_host(a: np.ndarray):
        t = torch.from_numpy(a)
        if nccl:
            d = t.cuda()
            dist.all_reduce(d, group=group)
            t.copy_(d.cpu())
        else:
            dist.all_reduce(t, group=group)

    def sum_device(t):
        dist.all_reduce(t, group=group)
        torch.cuda.synchronize()

    return SlabReducer(sum_host, sum_device if nccl else None, host_staged=host_staged)


def slab_iterate(solvers, iterations: int, reducer: SlabReducer | None = None):
    """rihvr_slab_iterate over SparseCompressiveHolo slab solvers (in plane
    order; one solver when `reducer` sums over other processes)."""
    from . import _check, load_library

    L = load_library()
    hs = (ctypes.c_void_p * len(solvers))(*[s._h.value for s in solvers])
    ref = ctypes.byref(reducer.struct) if reducer is not None else None
    rc = L.rihvr_slab_iterate(hs, len(solvers), int(iterations), ref)
    if rc != 0 and reducer is not None and reducer.errors:
        raise RuntimeError(f"slab reducer failed: {reducer.errors[-1]}")
    _check(rc, "rihvr_slab_iterate")


class SlabSolve:
    """One hologram's solve over `n_slabs` z-slabs in this process.
    `devices` (one per slab, default the current device for all) places each
    slab; devices other than the current one need peer access."""

    def __init__(self, params, width: int, height: int, n_slabs: int, devices=None):
        from . import SparseCompressiveHolo

        self.params = params
        self.solvers = []
        devs = list(devices) if devices is not None else [None] * n_slabs
        if len(devs) != n_slabs:
            raise ValueError("one device per slab")
        for i in range(n_slabs):
            z0, nz = slab_bounds(params.num_planes, n_slabs, i)
            if devs[i] is None:
                self.solvers.append(SparseCompressiveHolo(params, width, height, z_first=z0, z_count=nz))
            else:
                import torch

                with torch.cuda.device(devs[i]):
                    self.solvers.append(SparseCompressiveHolo(params, width, height, z_first=z0, z_count=nz))

    def setHologram(self, b):
        for s in self.solvers:
            s.setHologram(b)

    def reset(self):
        for s in self.solvers:
            s.reset()

    def iterate(self, n: int):
        slab_iterate(self.solvers, n)

    def inverseReconstruct(self, b=None) -> float:
        """num_inverse_iterations from x = 0; the objective at the final
        momentum point (the last record's f_x)."""
        if b is not None:
            self.setHologram(b)
        else:
            self.reset()
        self.iterate(self.params.num_inverse_iterations)
        rec = self.iterations()
        return float(rec["f_x"][-1]) if len(rec) else float("nan")

    def iterations(self):
        return self.solvers[0].iterations()

    def getVolume(self) -> np.ndarray:
        return np.concatenate([s.getVolume() for s in self.solvers], axis=0)

    def destroy(self):
        for s in self.solvers:
            s.destroy()
        self.solvers = []
