"""CPU checks of bench.py's contract pieces: the reference arm's JSON line (the
oracle on the host cores, small configuration), and the roofline inputs."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_contract_line():
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--config", "c1", "--steps", "1",
                          "--warmup", "3"], cwd=ROOT, capture_output=True, text=True, timeout=300, check=True)
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "voxel-iters/s" and d["value"] > 0
    assert d["steps"] == 1 and d["warmup"] == 3 and d["higher_is_better"] is True
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": "voxel-iters/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}


def test_warmup_below_three_is_raised_to_three():
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--config", "c1", "--steps", "1",
                          "--warmup", "1"], cwd=ROOT, capture_output=True, text=True, timeout=300, check=True)
    d = json.loads([ln for ln in out.stdout.splitlines() if ln.startswith("{")][0])
    assert d["warmup"] == 3


def test_roofline_inputs():
    sys.path.insert(0, ROOT)
    import bench

    # algorithmic bytes per voxel of each kernel class sum to the minimal two-pass flow
    for s in (8, 4):
        cb = bench.class_bytes(s)
        assert cb["prox"] == 8 + 3 * s and cb["fwd_row"] == s + 8 and cb["fwd_col"] == 8
        # as built: the minimal 32 + 4 s plus G written and read back (16 B)
        assert sum(cb.values()) == 48 + 4 * s
    # the prox's measured DRAM traffic (the roofline's `traffic`) is within 10 %
    # above its algorithmic bytes; the FFT passes' 16-plane captures leave part
    # of their writes in L2, so only the prox is held to this
    tpv = bench.MEASURED_TRAFFIC_PER_VOXEL[("prox", 8)]
    assert 32 * 0.98 <= tpv <= 32 * 1.10, tpv
    peak, kind = bench.peaks()
    assert peak > 1000 and kind in ("measured", "fallback")
