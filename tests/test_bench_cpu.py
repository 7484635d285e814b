"""bench.py pieces that run without a GPU: the reference arm on the 8^4 workload (one
JSON line with the contract's keys), the serve request streams, and the byte model of
the engine phases."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


@pytest.mark.timeout(600)
def test_reference_arm_cg8():
    env = dict(os.environ)
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        env.pop(k, None)
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--workload", "cg8", "--steps", "1",
                          "--warmup", "3"], cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "solves/s" and d["value"] > 0
    for key in ("metric", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling", "dtype",
                "config", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert "iterations to its stopping rule" in d["cpu_baseline"]["sample"]


def test_reference_arm_serve_unavailable():
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--workload", "serve32"], cwd=ROOT,
                         capture_output=True, text=True, timeout=120)
    assert out.returncode == 0
    d = json.loads(out.stdout.strip().splitlines()[-1])
    assert d["impl"] == "reference" and "unavailable" in d


def test_serve_streams():
    import bench
    for name in ("serve", "serve32"):
        w = bench.WORKLOADS[name]
        a, b = bench.serve_stream(w, seed=11), bench.serve_stream(w, seed=11)
        assert a == b and len(a) == w["requests"]
        pool = w.get("pool", bench.SERVE_POOL)
        lo, hi = w["nrhs_range"]
        times = [r[0] for r in a]
        assert times == sorted(times)
        for t, g, kappa, src in a:
            assert 0 <= g < len(w["lattices"]) and lo <= len(src) <= hi
            # consecutive sources of the pool, wrapping when a request has more than the pool
            assert all(0 <= k < pool for k in src) and len(set(src)) == min(len(src), pool)
            assert w["kappa_range"][0] <= kappa <= w["kappa_range"][1]


def test_engine_phase_bytes():
    import bench
    vh = 32 ** 4 // 2
    phases = ("P1", "P2", "P3", "P4", "R1", "R2", "R3", "R4", "R4L", "R5", "R5L", "P5")
    b16 = {p: bench.engine_phase_bytes(p, vh, 12, "f16", 12) for p in phases}
    b32 = {p: bench.engine_phase_bytes(p, vh, 12, "f32", 12) for p in phases}
    assert all(v > 0 for v in b16.values())
    # P1: 12 x (52 + 52) + 8 x 36 link bytes per site
    assert b16["P1"] == vh * (12 * 104 + 288)
    # FP32 storage moves more than FP16 in the low-precision phases
    assert all(b32[p] > b16[p] for p in ("P1", "P2", "P3", "P4", "P5"))
    # the FP64 phases do not depend on the inner precision's spinor size except through r
    assert b16["R2"] == b32["R2"]
