"""Benchmark of the FISTA + L1 + 2-D TV reconstruction on one B200 (or N
independent frames on N GPUs, one process per GPU).

A step is one FISTA iteration (prox sweep with its backtracking checks, the
forward operator, the momentum update and the adjoint) over the whole volume of
the 1024x1024x1000 workload (dz=2, dx=1.1, lambda=0.632, sparsity 0.15, TV 0.1,
5 TV iterations; 1000 synthetic disks + 1000 rods).  ``value`` is voxel
iterations per second over all ranks, timed on the device with CUDA events;
``e2e`` is the same metric through the C ABI from the host's raw 8-bit camera
frame (preprocessed on the GPU) to host results.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--config c2|c1|c5]
    python bench.py --config series    # uneven time series, batched vs frame by frame
    python bench.py --config segment   # particle segmentation of the reconstructed volume
    python bench.py --config warmstart --frames 16   # learned warm start against FISTA from zero
    python bench.py --config warmstart4              # the same at 512x512x200 on 256 held-out holograms
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = "rihvr---regularized-inverse-holographic-volume-reconstruction_b200"
sys.path.insert(0, ROOT)

METRIC = "s to FP64-oracle objective ±1e-3 at 1024²×1000 voxels; voxel-iters/s; % HBM roofline"
FALLBACK_HBM_GBS = 6650.0


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


FALLBACK_BF16_TFLOPS = 1590.0


def bf16_peak():
    """Dense BF16 tensor-core peak (burst) in TFLOP/s and where it came from."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["bf16_tflops"]), "measured (burst)"
    except Exception:
        return FALLBACK_BF16_TFLOPS, "fallback"


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader",
                                          "-lms", "200", "-i", str(self.idx)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1].split()[0]))
                smax = float(parts[2].split()[0])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


def workload(name: str):
    synth = importlib.import_module(PKG + ".synth")
    return {"c1": synth.config1, "c2": synth.config2, "c5": synth.config5}[name]()


# algorithmic bytes per voxel of each kernel class, s = bytes per stored voxel
def class_bytes(s: int) -> dict:
    return {
        "adj_col": 8,           # write the column-pass intermediate
        "adj_row": 16,          # read it, write the gradient volume
        "prox": 8 + 3 * s,      # read gradient, P_k, P_{k-1}; write P_{k+1}
        "fwd_row": s + 8,       # read P_{k+1}, write the row-pass intermediate
        "fwd_col": 8,           # read the intermediate (the z-sum stays on chip)
    }


# DRAM bytes per voxel that ncu measured for one launch of a kernel class
# (dram__bytes_read.sum + dram__bytes_write.sum of a 1024 x 1024 x 16-plane
# capture of `bench.py --nz 16 --no-autotune`, 64 planes for the adjoint column
# pass, divided by its voxels), keyed by (class, stored bytes per voxel).
# Scaled by the voxels of a launch, since traffic grows with the planes
# processed.  The prox figure is dram__bytes.sum.per_second x duration of the
# 2-warp-block kernel (2.754 TB/s x 201.98 us).
MEASURED_TRAFFIC_PER_VOXEL = {
    ("prox", 8): 2.753885e12 * 201.984e-6 / (1024 * 1024 * 16),
    ("fwd_col", 8): (145.2e6 + 19.8e6) / (1024 * 1024 * 16),
    ("fwd_row", 8): (134.3e6 + 85.1e6) / (1024 * 1024 * 16),
    ("adj_row", 8): (134.3e6 + 85.6e6) / (1024 * 1024 * 16),
    ("adj_col", 8): (79.2e6 + 483.9e6) / (1024 * 1024 * 64),
}


GOLDEN_C2 = os.path.join(ROOT, "tests", "golden", "oracle_c2_1024x1024x1000.json")


def time_to_objective(rihvr, cfg, b, s, storage, stream, hb, tol=1e-3):
    """Seconds until the solver holds an iterate whose objective is within
    `tol` (relative) of the FP64 oracle's objective after its 100 iterations
    (committed oracle run of the same hologram).  An untimed pass with the
    objective recorded at every iteration finds the first iteration k that is
    within the band; the timed pass is what a user runs: hologram in from
    pinned host memory, k iterations without per-iteration objective, the
    objective at the end.  The iterates of the two passes are identical."""
    import hashlib

    import torch

    if not os.path.exists(GOLDEN_C2):
        return None
    with open(GOLDEN_C2) as fh:
        g = json.load(fh)
    if g.get("workload") != cfg.name or hashlib.sha1(b.tobytes()).hexdigest() != g.get("b_sha1"):
        return None
    target = float(g["f_x"][-1])
    p = rihvr.params_from_config(cfg, record_objective=1, storage=storage, faithful=0 if storage == 1 else 1)
    with rihvr.SparseCompressiveHolo(p, cfg.W, cfg.H) as t:
        t.setHologram(b)
        t.iterate(1)  # first iteration runs eagerly (tables, graph capture)
        rec_ms = t.iterate_timed(len(g["f_x"]) - 1)  # the library default: objective at every iteration
        fx = np.asarray(t.iterations()["f_x"], np.float64)
    gx = np.asarray(g["f_x"], np.float64)
    band = tol * abs(target)
    hits = np.nonzero(np.abs(fx - target) <= band)[0]
    ohits = np.nonzero(np.abs(gx - target) <= band)[0]
    out = {"unit": "s", "target_objective": target, "tolerance": tol, "oracle_iterations": int(ohits[0]) + 1,
           "oracle_seconds_100_iterations": g.get("oracle_seconds"), "oracle_threads": g.get("oracle_threads"),
           "ms_per_iteration_recording_objective": rec_ms / (len(g["f_x"]) - 1),
           "max_rel_gap_to_oracle_trajectory": float(np.max(np.abs(fx - gx) / np.abs(gx))),
           "final_rel_gap": float((fx[-1] - target) / abs(target))}
    if not len(hits):
        out.update({"value": None, "reached": False})
        return out
    k = int(hits[0]) + 1
    L = rihvr.load_library()
    import ctypes

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    rihvr._check(L.rihvr_set_hologram(s._h, ctypes.c_void_p(hb.data_ptr()), 0), "set_hologram")
    s.iterate(k)
    f, _ = s.calcObjectiveFunction()
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    out.update({"value": ms / 1e3, "reached": True, "iterations": k, "objective": f,
                "rel_gap": (f - target) / abs(target)})
    return out


CPU_SAMPLE_PLANES = 192  # about 5 s of FP64 oracle work per FISTA iteration on a 16-core host


def cpu_sample(cfg, b, steps: int, warmup: int, planes: int = CPU_SAMPLE_PLANES):
    """Time the FP64 oracle on a bounded sample of the workload: the first
    `planes` planes of the volume, full plane size, one FISTA iteration per
    step.  Parameters come from the workload description alone (float plane
    list, lambda, dx and weights as the reference stores them), so this leg
    never loads the product library."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    nz = min(planes, cfg.num_planes)
    z = cfg.plane_list()[:nz]
    op = O.OracleParams(W=cfg.W, H=cfg.H, z=z, dx=cfg.dx(), lam=cfg.lam(), l1=cfg.l1(), tv=cfg.tv(),
                        n_tv=cfg.num_tv_iterations, mode=7, faithful=1)
    b64 = b.astype(np.float64)
    for _ in range(warmup):
        O.solve(op, b64, 1, want_volumes=False)
    t0 = time.perf_counter()
    for _ in range(steps):
        O.solve(op, b64, 1, want_volumes=False)
    dt = time.perf_counter() - t0
    vox = cfg.W * cfg.H * nz
    return {"value": vox * steps / dt, "unit": "voxel-iters/s", "cores": O.num_threads(), "kind": "port",
            "sample": f"FP64 oracle, {nz} of {cfg.num_planes} planes at {cfg.W}x{cfg.H}, 1 FISTA iteration "
                      f"per step, {steps} steps ({dt:.1f} s)"}


def cufft_comparator(cfg, ktimes, reps: int = 5):
    """cuFFT (torch.fft) on the same planes as the forward operator's FFT
    passes: a batched FP32 complex 2-D FFT of the Nz planes, out of place,
    timed with CUDA events.  Beside it the hand-written forward row and column
    passes per launch (which also apply the transfer function and sum over z)."""
    import torch

    dev = torch.device("cuda", torch.cuda.current_device())
    x = torch.randn((cfg.num_planes, cfg.H, cfg.W), dtype=torch.complex64, device=dev)
    y = torch.empty_like(x)
    torch.fft.fft2(x, out=y)  # plan creation
    torch.cuda.synchronize()
    st = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(reps):
        torch.fft.fft2(x, out=y)
    e1.record(st)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / reps
    del x, y
    torch.cuda.empty_cache()
    ours = None
    if "fwd_row" in ktimes and "fwd_col" in ktimes:
        ours = sum(ktimes[k][0] / max(ktimes[k][1], 1) for k in ("fwd_row", "fwd_col"))
    V = cfg.voxels()
    return {"what": "torch.fft.fft2 (cuFFT) of the Nz planes, complex64, out of place",
            "cufft_ms": ms, "cufft_voxels_per_s": V / (ms / 1e3),
            "ours_forward_row_plus_column_ms": ours,
            "ours_over_cufft": (ms / ours) if ours else None,
            "note": "the hand-written passes also multiply by the transfer function and sum over z"}


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    cfg = workload(args.config)
    synth = importlib.import_module(PKG + ".synth")
    _, b = synth.make_hologram(cfg)
    # the reference's own path is CUDA-only (it needs OpenCV C++, absent here);
    # its CPU stand-in is the FP64 oracle on the same sample as cpu_baseline
    cb = cpu_sample(cfg, b, args.steps, args.warmup)
    line = {"metric": METRIC, "value": cb["value"], "unit": "voxel-iters/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "impl": "reference",
            "dtype": "f64", "data": "synthetic", "config": {"workload": cfg.name, "sample": cb["sample"]},
            "cpu_baseline": cb, "e2e": {"value": cb["value"], "unit": "voxel-iters/s", "h2d_bytes_per_step": 0,
                                        "d2h_bytes_per_step": 0}, "vs_baseline": None}
    print(json.dumps(line), flush=True)
    return 0


def run_frames(args):
    """Batched time series (the uneven-series workload): `--frames` frames
    (default 64) of an advected tracer population (synth.series_frames: H and W
    from {512, 640, 768, 1024}, Nz 100-400, 200-3000 tracers, a seeded
    divergence-free velocity field between frames), `--steps` FISTA iterations
    each.  Frames run in waves whose contexts fit in device memory; each wave
    is reconstructed frame after frame and then all at once with
    rihvr_reconstruct_batch on the same contexts (graphs captured by an
    untimed warm-up call).  Prints one JSON line."""
    import torch

    torch.cuda.set_device(0)
    rihvr = importlib.import_module(PKG)
    synth = importlib.import_module(PKG + ".synth")
    n = args.frames if args.frames else 64
    cfgs = synth.series_frames(n, iterations=args.steps)
    t_gen = time.perf_counter()
    holos = [synth.make_hologram(c, device="cuda")[1] for c in cfgs]
    t_gen = time.perf_counter() - t_gen
    torch.cuda.empty_cache()
    budget = 0.75 * torch.cuda.mem_get_info()[0]
    vox = sum(c.voxels() for c in cfgs) * args.steps
    t_seq = t_bat = t_one = 0.0
    one_ok = True
    waves, seq_obj, bat_obj, one_obj = [], [], [], []
    i = 0
    while i < n:
        wave, bytes_ = [], 0
        while i < n:
            need = 44 * cfgs[i].voxels() + (256 << 20)  # FP32 volumes, gradient, intermediate, planes
            if wave and bytes_ + need > budget:
                break
            wave.append(i)
            bytes_ += need
            i += 1
        solvers = [rihvr.SparseCompressiveHolo(rihvr.params_from_config(cfgs[j], record_objective=0),
                                               cfgs[j].W, cfgs[j].H) for j in wave]
        hs = [holos[j] for j in wave]
        try:
            rihvr.reconstruct_batch(solvers, hs)  # warm-up: first launches and graph capture
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            seq = [s_.inverseReconstruct(b_) for s_, b_ in zip(solvers, hs)]
            torch.cuda.synchronize()
            t_seq += time.perf_counter() - t0
            t0 = time.perf_counter()
            bat = rihvr.reconstruct_batch(solvers, hs)
            torch.cuda.synchronize()
            t_bat += time.perf_counter() - t0
            # batch mode 2: the wave's whole solves as one graph launch (graph built inside the call)
            rihvr.set_batch_mode(2)
            try:
                rihvr.reconstruct_batch(solvers, hs)
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                one = rihvr.reconstruct_batch(solvers, hs)
                torch.cuda.synchronize()
                t_one += time.perf_counter() - t0
                one_ok = one_ok and rihvr.batch_last_combined() == 2
            finally:
                rihvr.set_batch_mode(0)
        finally:
            for s_ in solvers:
                s_.destroy()
        waves.append(len(wave))
        seq_obj += list(seq)
        bat_obj += list(bat)
        one_obj += list(one)
    line = {"metric": "frames reconstructed per second (uneven advected-tracer time series)", "value": n / t_bat,
            "unit": "frames/s", "higher_is_better": True, "n_gpus": 1, "steps": args.steps, "data": "synthetic",
            "config": {"workload": f"uneven_series_{n}_frames",
                       "frames": [[c.W, c.H, c.num_planes, c.n_disks] for c in cfgs],
                       "fista_iterations": args.steps, "tv_iterations": 5, "waves": waves},
            "batched_s": t_bat, "sequential_s": t_seq, "speedup": t_seq / t_bat,
            "voxel_iters_per_s_batched": vox / t_bat, "voxel_iters_per_s_sequential": vox / t_seq,
            "objectives_equal": bool(np.array_equal(np.asarray(seq_obj), np.asarray(bat_obj))),
            "one_graph": {"what": "batch mode 2: each wave's whole solves as one graph launch",
                          "s": t_one, "speedup_vs_sequential": t_seq / t_one, "ran_as_one_graph": one_ok,
                          "objectives_equal": bool(np.array_equal(np.asarray(seq_obj), np.asarray(one_obj)))},
            "hologram_generation_s": t_gen}
    print(json.dumps(line), flush=True)
    return 0


def run_segment(args):
    """Particle segmentation of the reconstructed 1024x1024x1000 volume (the
    reference's segmentation program with its default settings: threshold at
    max/256, closing with a ball of radius 3, 26-connected labels, centroids of
    objects of 2 voxels or more) on the volume in device memory.  A step is one
    rihvr_segment call, timed on the host around a device synchronisation (the
    call itself synchronises three times to size its buffers).  Prints one
    JSON line."""
    import torch

    torch.cuda.set_device(0)
    rihvr = importlib.import_module(PKG)
    synth = importlib.import_module(PKG + ".synth")
    cfg = workload("c2")
    if args.nz:
        cfg.num_planes = args.nz
        cfg.name = f"{cfg.name}_nz{args.nz}"
    _, b = synth.make_hologram(cfg)
    p = rihvr.params_from_config(cfg, record_objective=0)
    s = rihvr.SparseCompressiveHolo(p, cfg.W, cfg.H)
    s.setHologram(b)
    s.iterate(cfg.num_inverse_iterations)
    sp = rihvr.segment_params()
    for _ in range(args.warmup):
        objs, info = s.segment(sp)
    launches0 = s.launch_count()
    times = []
    with ClockSampler(0) as clk:
        time.sleep(0.3)
        for _ in range(args.steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            objs, info = s.segment(sp)
            torch.cuda.synchronize()
            times.append(time.perf_counter() - t0)
    launches = (s.launch_count() - launches0) // args.steps
    V = cfg.voxels()
    t = float(np.median(times))
    peak, peak_kind = peaks()
    # HBM bytes a voxel: P and P_prev read by the max pass and again by the
    # threshold pass (16 B each at FP32); the bit volumes are 1/8 B a voxel
    bpv = 32
    cpu = None
    if not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O

        nzs = min(16, cfg.num_planes)
        planes = np.stack([s.getPlane(z) for z in range(nzs)])
        I = (planes.real * planes.real + planes.imag * planes.imag).astype(np.float32)
        t0 = time.perf_counter()
        O.segment(I, sp.min_intensity, sp.close_size, sp.min_area, sp.faithful)
        dt = time.perf_counter() - t0
        cpu = {"value": I.size / dt, "unit": "voxels/s", "cores": 1, "kind": "port",
               "sample": f"oracle segmentation of the first {nzs} of {cfg.num_planes} planes ({dt:.2f} s)"}
    line = {"metric": "segmented voxels per second (1024x1024x1000 reconstructed volume)", "value": V / t,
            "unit": "voxels/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3,
            "higher_is_better": True, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "segment_" + cfg.name, "min_intensity": sp.min_intensity,
                       "close_size": sp.close_size, "min_area": sp.min_area, "faithful": sp.faithful,
                       "fista_iterations_before": cfg.num_inverse_iterations},
            "objects": int(len(objs)), "labelled_objects": int(info["labelled_objects"]),
            "closed_voxels": int(info["closed_voxels"]), "threshold": info["threshold"],
            "roofline": {"bound": "hbm", "bytes_per_voxel": bpv, "achieved": bpv * V / t / 1e9, "peak": peak,
                         "unit": "GB/s", "frac": bpv * V / t / 1e9 / peak, "peak_source": peak_kind},
            "cpu_baseline": cpu, "clocks": clk.summary(), "gpu_launches": launches,
            "step_ms_all": [x * 1e3 for x in times]}
    print(json.dumps(line), flush=True)
    s.destroy()
    return 0


def run_warmstart(args):
    """Learned warm start at 128x128x32 (the physics of the 512x512x200
    warm-start configuration): on held-out synthetic holograms, the iterations
    and the device time plain FISTA from zero and FISTA from the trained
    network's x0 need to reach plain FISTA's 100-iteration objective within
    1e-3, and the network's own inference time.  Prints one JSON line."""
    import torch

    torch.cuda.set_device(0)
    rihvr = importlib.import_module(PKG)
    ws = importlib.import_module(PKG + ".warmstart")
    seeds = np.arange(300_000, 300_000 + (args.frames if args.frames else 16))
    with rihvr.UNet(ws.PLANES, ws.SIZE, ws.SIZE) as net:
        net.load(ws.WEIGHTS)
        rows = ws.evaluate(net, seeds)
        # inference alone, on one held-out hologram
        data = ws.make_set(seeds[:1])
        xbp = data[0][1]
        for _ in range(3):
            net.predict(xbp)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            net.predict(xbp)
        torch.cuda.synchronize()
        infer_ms = (time.perf_counter() - t0) / args.steps * 1e3
    s = ws.summary(rows)
    vox = ws.PLANES * ws.SIZE * ws.SIZE
    flops = 0
    for cin, cout, lvl in [(16, 16, 0), (16, 16, 0), (16, 32, 1), (32, 32, 1), (32, 64, 2), (64, 64, 2),
                           (96, 32, 1), (32, 32, 1), (48, 16, 0), (16, 16, 0)]:
        flops += 2 * 27 * cin * cout * vox // (8 ** lvl)
    line = {"metric": "iterations and device ms to plain FISTA's 100-iteration objective (1e-3), warm start vs zero",
            "value": s["mean_iters_warm"], "unit": "iterations", "higher_is_better": False, "n_gpus": 1,
            "data": "synthetic", "config": {"workload": f"warmstart_{ws.SIZE}x{ws.SIZE}x{ws.PLANES}",
                                             "holograms": len(rows), "weights": os.path.basename(ws.WEIGHTS)},
            "summary": s, "inference_ms": infer_ms, "inference_tflops": flops / (infer_ms * 1e-3) / 1e12,
            "conv_flops": flops, "rows": rows}
    print(json.dumps(line), flush=True)
    return 0


def run_warmstart4(args):
    """The learned warm start on its specified configuration, 512x512x200
    (500-3000 disks and rods, noise 0.005-0.03): the network trained on
    full-depth crops of that configuration (or, without those weights, the
    one trained at 128x128x32; it is fully convolutional) applied to held-out
    holograms of that size; iterations and device time to plain FISTA's
    100-iteration objective within 1e-3, with and without it, and the
    network's inference time at that size.  Prints one JSON line."""
    import torch

    torch.cuda.set_device(0)
    rihvr = importlib.import_module(PKG)
    ws = importlib.import_module(PKG + ".warmstart")
    n = args.frames if args.frames else 256
    seeds = np.arange(400_000, 400_000 + n)
    S, Z = ws.C4_SIZE, ws.C4_PLANES
    weights = ws.C4_WEIGHTS if os.path.exists(ws.C4_WEIGHTS) else ws.WEIGHTS
    with rihvr.UNet(Z, S, S) as net:
        net.load(weights)
        t0 = time.perf_counter()
        rows = ws.evaluate(net, seeds, size=S, planes=Z, sampler=ws.config4_sample, device="cuda")
        eval_s = time.perf_counter() - t0
        cfg = ws.config4_sample(int(seeds[0]))
        synth = importlib.import_module(PKG + ".synth")
        _, b = synth.make_hologram(cfg, device="cuda")
        with rihvr.SparseCompressiveHolo(rihvr.params_from_config(cfg, record_objective=0), S, S) as s:
            s.setHologram(b)
            xbp = torch.from_numpy(s.backpropagate()).cuda()
        act_bits = net.activation_bits()
        for _ in range(3):
            net.predict(xbp)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            net.predict(xbp)
        e1.record()
        e1.synchronize()
        infer_ms = e0.elapsed_time(e1) / args.steps
    s_ = ws.summary(rows)
    vox = Z * S * S
    flops = 0
    for cin, cout, lvl in [(16, 16, 0), (16, 16, 0), (16, 32, 1), (32, 32, 1), (32, 64, 2), (64, 64, 2),
                           (96, 32, 1), (32, 32, 1), (48, 16, 0), (16, 16, 0)]:
        flops += 2 * 27 * cin * cout * vox // (8 ** lvl)
    line = {"metric": "iterations and device ms to plain FISTA's 100-iteration objective (1e-3), warm start vs zero",
            "value": s_["mean_iters_warm"], "unit": "iterations", "higher_is_better": False, "n_gpus": 1,
            "data": "synthetic", "config": {"workload": f"warmstart_{S}x{S}x{Z}", "holograms": len(rows),
                                             "weights": os.path.basename(weights),
                                             "activation_bits": act_bits},
            "summary": s_, "inference_ms": infer_ms, "inference_tflops": flops / (infer_ms * 1e-3) / 1e12,
            "conv_flops": flops, "eval_s": eval_s, "rows": rows}
    print(json.dumps(line), flush=True)
    return 0


UNET_LAYERS = [(16, 16, 0), (16, 16, 0), (16, 32, 1), (32, 32, 1), (32, 64, 2), (64, 64, 2), (96, 32, 1),
               (32, 32, 1), (48, 16, 0), (16, 16, 0)]  # (in, out channels, level) of the 3x3x3 convolutions


def run_unet(args):
    """The warm-start network's inference alone (rihvr_unet_predict: input
    normalisation, ten 3x3x3 convolutions on tcgen05 with BF16 activations,
    pooling, upsampling, the head fused into the last layer) on a
    `--nz` x 512 x 512 volume (default 200 planes, the warm start's
    configuration) of random complex values, with the weights trained there.
    A step is one inference; CUDA events on the network's stream.  Prints one
    JSON line with the tensor-core throughput of the convolutions."""
    import torch

    torch.cuda.set_device(0)
    rihvr = importlib.import_module(PKG)
    ws = importlib.import_module(PKG + ".warmstart")
    Z, S = (args.nz or ws.C4_PLANES), ws.C4_SIZE
    weights = ws.C4_WEIGHTS if os.path.exists(ws.C4_WEIGHTS) else ws.WEIGHTS
    g = torch.Generator(device="cuda").manual_seed(7)
    xbp = torch.complex(torch.randn((Z, S, S), device="cuda", generator=g),
                        torch.randn((Z, S, S), device="cuda", generator=g))
    with rihvr.UNet(Z, S, S) as net:
        net.load(weights)
        bits = net.activation_bits()
        for _ in range(max(3, args.warmup)):
            net.predict(xbp)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(0) as clk:
            e0.record()
            for _ in range(args.steps):
                net.predict(xbp)
            e1.record()
            e1.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
    vox = Z * S * S
    flops = sum(2 * 27 * ci * co * vox // (8 ** lv) for ci, co, lv in UNET_LAYERS)
    tf = flops / (ms * 1e-3) / 1e12
    peak, src = bf16_peak()
    line = {"metric": "warm-start network inference, TFLOP/s of the 3x3x3 convolutions", "value": tf,
            "unit": "TFLOP/s", "higher_is_better": True, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "dtype": "bf16", "data": "synthetic",
            "config": {"workload": f"unet_inference_{Z}x{S}x{S}", "weights": os.path.basename(weights),
                       "activation_bits": bits},
            "roofline": {"bound": "tensor", "achieved": tf, "peak": peak, "unit": "TFLOP/s",
                         "frac": tf / peak, "peak_source": src},
            "conv_flops": flops, "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    return 0


def run_slabs(args):
    """One hologram of the 1024 x 1024 x 1000 workload split into z-slabs
    (rihvr_slab_iterate).  On one GPU (`--slabs K` slabs in this process) the
    line compares the slab group's time per iteration with one context over
    all planes on the same hologram, i.e. the cost of the host-decided slab
    loop and its spectrum sums.  Under torchrun each rank holds one slab on
    its own GPU and the partial spectra are summed by NCCL all-reduce
    (strong scaling: the total work is one hologram at every N).  Timed with
    CUDA events on the slabs' streams; the solve is host-decided, so the time
    includes the host's part of every attempt."""
    ws, rank, local = dist_env()
    import torch

    torch.cuda.set_device(local)
    rihvr = importlib.import_module(PKG)
    synth = importlib.import_module(PKG + ".synth")
    frames = importlib.import_module(PKG + ".frames")
    slabs = importlib.import_module(PKG + ".slabs")
    pg = None
    if ws > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
        pg = dist
    cfg = workload("c2")
    if args.nz:
        cfg.num_planes = args.nz
        cfg.name = f"{cfg.name}_nz{args.nz}"
    _, b = synth.make_hologram(cfg)
    storage = {"f32": 0, "bf16": 1, "f16": 2}[args.storage]
    p = rihvr.params_from_config(cfg, record_objective=0, storage=storage, autotune=1 if args.autotune else 0,
                                 faithful=0 if storage == 1 else 1)
    V = cfg.voxels()
    single_ms = None
    if ws == 1:
        with rihvr.SparseCompressiveHolo(p, cfg.W, cfg.H) as s:
            s.setHologram(b)
            s.iterate(args.warmup)
            single_ms = s.iterate_timed(args.steps) / args.steps
            single_log = s.iterations()
        n_local = max(1, args.slabs)
        group = slabs.SlabSolve(p, cfg.W, cfg.H, n_local)
        solvers, reducer = group.solvers, None
    else:
        z0, nz = slabs.slab_bounds(cfg.num_planes, ws, rank)
        solvers = [rihvr.SparseCompressiveHolo(p, cfg.W, cfg.H, z_first=z0, z_count=nz)]
        reducer = slabs.torch_reducer()
    for s in solvers:
        s.setHologram(b)
    slabs.slab_iterate(solvers, args.warmup, reducer)
    streams = [torch.cuda.ExternalStream(s.stream()) for s in solvers]
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = [torch.cuda.Event(enable_timing=True) for _ in solvers]
    if pg is not None:
        pg.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        time.sleep(0.5)
        e0.record(streams[0])
        slabs.slab_iterate(solvers, args.steps, reducer)
        for e, st in zip(e1, streams):
            e.record(st)
        for e in e1:
            e.synchronize()
    ms = max(e0.elapsed_time(e) for e in e1)
    if pg is not None:
        pg.barrier()
    max_ms = frames.reduce_max(ms, device="cuda")
    log = solvers[0].iterations()
    line = None
    if rank == 0:
        line = {"metric": METRIC, "value": V * args.steps / (max_ms / 1e3), "unit": "voxel-iters/s", "n_gpus": ws,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": max_ms / args.steps,
                "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
                "dtype": "f32" if storage == 0 else args.storage, "data": "synthetic",
                "config": {"workload": cfg.name + "_zslabs", "W": cfg.W, "H": cfg.H, "Nz": cfg.num_planes,
                           "slabs": len(solvers) * ws, "slab_planes": [s.depth for s in solvers],
                           "parallelism": f"{ws} z-slabs, one per GPU, NCCL spectrum sums" if ws > 1 else
                           f"{len(solvers)} z-slabs on one GPU",
                           "l2": "inputs larger than L2", "storage": args.storage},
                "single_context_ms_per_step": single_ms,
                "slab_overhead": (max_ms / args.steps / single_ms) if single_ms else None,
                "same_decisions_as_single_context": (
                    bool(np.array_equal(log["backtracks"], single_log["backtracks"][:len(log)]) and
                         np.array_equal(log["restarted"], single_log["restarted"][:len(log)]))
                    if single_ms else None),
                "clocks": clk.summary()}
        print(json.dumps(line), flush=True)
    for s in solvers:
        s.destroy()
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()
    return 0


def run_ours(args):
    ws, rank, local = dist_env()
    import torch

    torch.cuda.set_device(local)
    pg = None
    if ws > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
        pg = dist
    rihvr = importlib.import_module(PKG)
    synth = importlib.import_module(PKG + ".synth")
    frames = importlib.import_module(PKG + ".frames")
    base = workload(args.config)
    # independent frames of a series: each rank reconstructs its own hologram
    (frame,) = frames.rank_frames(ws, ws, rank)
    cfg = base
    if args.nz:
        # smaller profiling case: same planes and physics, fewer of them
        cfg.num_planes = args.nz
        cfg.name = f"{cfg.name}_nz{args.nz}"
    img0, b0 = synth.make_hologram(cfg)
    b = synth.translated_frame(b0, frame)
    img = synth.translated_frame(img0, frame)  # the raw camera frame (uint8), for the end-to-end pass
    storage = {"f32": 0, "bf16": 1, "f16": 2}[args.storage]
    # BF16 storage is accepted only without the reference-faithful arithmetic
    p = rihvr.params_from_config(cfg, record_objective=0, storage=storage, autotune=1 if args.autotune else 0,
                                 faithful=0 if storage == 1 else 1)
    s = rihvr.SparseCompressiveHolo(p, cfg.W, cfg.H)
    V = cfg.voxels()
    s.setHologram(b)  # tunes launch shapes first with --autotune
    tuning = s.tuning()
    s.iterate(args.warmup)

    def barrier():
        if pg is not None:
            pg.barrier()
        torch.cuda.synchronize()

    # timed region: device time of K iterations on the solver stream (captured
    # graphs after the first iteration, no per-kernel events)
    launches0 = s.launch_count()
    barrier()
    with ClockSampler(local) as clk:
        time.sleep(0.5)  # let the sampler start before the timed region
        ms = s.iterate_timed(args.steps)
    barrier()
    launches = s.launch_count() - launches0
    log = s.iterations()
    # per-kernel split from a separate pass with CUDA events around each kernel class
    s.set_profiling(True)
    s.iterate(min(args.steps, 5))
    ktimes = s.kernel_times()
    s.set_profiling(False)
    max_ms = frames.reduce_max(ms, device="cuda")
    value = frames.weak_throughput(ws * V * args.steps, max_ms)

    # end to end through the C ABI: the raw 8-bit camera frame in (preprocessed
    # on the GPU, as the driver does it), host estimate + objective out
    stream = torch.cuda.ExternalStream(s.stream())
    hb = torch.from_numpy(b).pin_memory()
    himg = torch.from_numpy(np.ascontiguousarray(img)).pin_memory()
    hout = torch.empty((cfg.H, cfg.W), dtype=torch.float32).pin_memory()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    L = rihvr.load_library()
    import ctypes

    barrier()
    e0.record(stream)
    rihvr._check(L.rihvr_set_hologram_frame(s._h, ctypes.c_void_p(himg.data_ptr()), 8, img.shape[1], img.shape[0],
                                            None, None, 0), "set_hologram_frame")
    s.iterate(args.steps)
    rihvr._check(L.rihvr_get_estimate(s._h, ctypes.c_void_p(hout.data_ptr()), 0), "get_estimate")
    f_final, _ = s.calcObjectiveFunction()
    e1.record(stream)
    e1.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    barrier()
    e2e_ms = frames.reduce_max(e2e_ms, device="cuda")
    e2e = {"value": frames.weak_throughput(ws * V * args.steps, e2e_ms), "unit": "voxel-iters/s",
           "h2d_bytes_per_step": int(img.nbytes) / args.steps, "d2h_bytes_per_step": (int(hout.numel() * 4) + 8) / args.steps,
           "ms": e2e_ms, "what": "set_hologram_frame (8-bit camera frame H2D from pinned, preprocessed on the GPU) + "
                                 "K iterations + estimate and objective (D2H)"}

    cufft = cufft_comparator(cfg, ktimes) if ws == 1 else None

    tto = None
    if ws == 1 and not args.nz and args.config == "c2" and args.time_to_objective:
        tto = time_to_objective(rihvr, cfg, b, s, storage, stream, hb)

    # roofline of the dominant kernel class
    peak, peak_kind = peaks()
    sbytes = 8 if storage == 0 else 4
    cb = class_bytes(sbytes)
    dom = max((k for k in cb if k in ktimes and ktimes[k][1] > 0), key=lambda k: ktimes[k][0])
    tot_ms, nl = ktimes[dom]
    avg_ms = tot_ms / nl
    bytes_per_launch = cb[dom] * V
    achieved = bytes_per_launch / (avg_ms / 1e3) / 1e9
    tpv = MEASURED_TRAFFIC_PER_VOXEL.get((dom, sbytes))
    traffic = tpv * V if tpv is not None else None
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                "bytes_per_launch": bytes_per_launch, "avg_launch_ms": avg_ms}
    iter_bytes = (32 + 4 * sbytes) * V  # per voxel-iteration, minimal two-pass data flow
    kernels = {k: {"ms_total": v[0], "launches": v[1]} for k, v in ktimes.items()}

    if rank == 0:
        cpu = None
        if ws == 1 and not args.no_cpu_baseline:
            # the same sample as the reference arm: about 10 s of oracle work on a 16-core host
            cpu = cpu_sample(cfg, b, steps=2, warmup=1)
        line = {
            "metric": METRIC, "value": value, "unit": "voxel-iters/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if storage == 0 else args.storage, "data": "synthetic",
            "config": {"workload": cfg.name, "W": cfg.W, "H": cfg.H, "Nz": cfg.num_planes,
                       "tv_iterations": cfg.num_tv_iterations, "storage": args.storage,
                       "parallelism": f"{ws} independent frames" if ws > 1 else "single frame",
                       "l2": "inputs larger than L2 (volumes of %.1f GB each)" % (V * sbytes / 1e9),
                       "record_objective": False, "autotune": bool(args.autotune), "launch_shapes": tuning},
            "e2e": e2e, "time_to_objective": tto, "roofline": roofline, "cpu_baseline": cpu,
            "cufft_comparator": cufft,
            "iteration_roofline": {"bytes_per_voxel_iter": 32 + 4 * sbytes,
                                   "achieved": iter_bytes * args.steps / (max_ms / 1e3) / 1e9, "peak": peak,
                                   "frac": iter_bytes * args.steps / (max_ms / 1e3) / 1e9 / peak},
            "clocks": clk.summary(), "gpu_launches": launches, "kernels": kernels,
            "backtracks_in_timed_region": int(log["backtracks"][-args.steps:].sum()) if len(log) else 0,
            "final_objective_e2e": f_final, "device_bytes": s.device_bytes(),
        }
        print(json.dumps(line), flush=True)
    s.destroy()
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c2",
                    choices=["c2", "c1", "c5", "series", "segment", "warmstart", "warmstart4", "unet", "slabs"])
    ap.add_argument("--slabs", type=int, default=2,
                    help="z-slabs of the hologram on one GPU (--config slabs; one per rank under torchrun)")
    ap.add_argument("--frames", type=int, default=0,
                    help="frames of the uneven series (--config series, default 64) or of the warm-start set "
                         "(default 16; 256 for warmstart4)")
    ap.add_argument("--storage", default="f32", choices=["f32", "bf16", "f16"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--nz", type=int, default=0, help="override the plane count (profiling cases)")
    ap.add_argument("--no-time-to-objective", dest="time_to_objective", action="store_false",
                    help="skip the time-to-oracle-objective measurement (profiling runs)")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="keep the built-in launch shapes (by default they are tuned once before timing)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.config == "series":
        return run_frames(args)
    if args.config == "segment":
        return run_segment(args)
    if args.config == "warmstart":
        return run_warmstart(args)
    if args.config == "warmstart4":
        return run_warmstart4(args)
    if args.config == "unet":
        return run_unet(args)
    if args.config == "slabs":
        return run_slabs(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
