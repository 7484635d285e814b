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


# Arrays each engine phase reads or writes per slot and site, as the kernels in
# hila_b200/csrc/engine.cu touch them (epi_low, epi_f64, k_eng_vec): (array, kind, count)
# with kind "sp" a low-precision spinor, "f32" an FP32 spinor (96 B), "f64" an FP64 one.
PHASE_ARRAYS = {
    "P1": [("p", "sp", 1), ("t", "sp", 1)],
    "P2": [("t", "sp", 1), ("p", "sp", 1), ("Dp", "sp", 1)],
    "P3": [("Dp", "sp", 1), ("t", "sp", 1)],
    "P4": [("t", "sp", 1), ("Dp", "sp", 1), ("r read", "sp", 1), ("r write", "sp", 1), ("p", "sp", 1),
           ("y read", "f32", 1), ("y write", "f32", 1)],
    "R1": [("x read", "f64", 1), ("x write", "f64", 1), ("y read", "f32", 1)],
    "R2": [("x", "f64", 1), ("t64", "f64", 1)],
    "R3": [("t64", "f64", 1), ("x", "f64", 1), ("b", "f64", 1), ("s in y", "f32", 1)],
    "R4": [("s", "f64", 1), ("t64", "f64", 1)],
    "R4L": [("s in y", "f32", 1), ("t", "f32", 1)],
    "R5": [("t64", "f64", 1), ("s", "f64", 1), ("b", "f64", 1), ("r", "sp", 1)],
    "R5L": [("t", "f32", 1), ("y read", "f32", 1), ("y clear", "f32", 1), ("r", "sp", 1)],
    "P5": [("r", "sp", 1), ("p read", "sp", 1), ("p write", "sp", 1)],
}


def test_engine_phase_bytes():
    import bench
    for prec, sp in (("f16", 52), ("f32", 96)):
        size = {"sp": sp, "f32": 96, "f64": 192}
        for ph, arrays in PHASE_ARRAYS.items():
            main, alt, link, normal = bench.engine_unit_bytes(ph, prec, 12)
            assert main == sum(size[k] * n for _, k, n in arrays), (prec, ph)
            # links are read once per site by the hop phases, never by the vector phases
            assert (link > 0) == (ph not in ("R1", "P5")), ph
        # alternate forms: R1 of the normal system also clears y, R3 from x = 0 runs no hop,
        # P5 on a first iteration does not read p; R3 of the normal system stores s in FP64
        assert bench.engine_unit_bytes("R1", prec, 12)[1] == 2 * 192 + 2 * 96
        assert bench.engine_unit_bytes("R3", prec, 12)[1:] == (2 * 192 + 96, 8 * 96, 3 * 192)
        assert bench.engine_unit_bytes("P5", prec, 12)[1] == 2 * sp
    # links per site: FP16 inner phases 8 x 36 B (18 reals), FP32 8 x 48 B (12 reals), FP64 8 x 144 / 96 B
    assert bench.engine_unit_bytes("P1", "f16", 12)[2] == 288
    assert bench.engine_unit_bytes("P1", "f32", 12)[2] == 384
    assert bench.engine_unit_bytes("R2", "f16", 18)[2] == 1152
    # P4 of 12 FP16 sources at 32^4 (the headline kernel): 524,288 x (12 x 452 + 288) bytes
    vh = 32 ** 4 // 2
    assert bench.engine_phase_bytes("P4", (12 * vh, 0, vh, 0), "f16", 12) == vh * (12 * 452 + 288)


def test_phase_table_skips_idle_phases():
    import bench
    prof = {"P4": (2, 1.6, (24, 0, 2, 0)), "R4": (0, 0.0, (0, 0, 0, 0))}
    t = bench.phase_table(prof, "f16", 12, 6546.6)
    assert t["R4"]["gbs"] is None and t["R4"]["bytes_per_launch"] is None
    assert t["P4"]["bytes_per_launch"] == (24 * 452 + 2 * 288) // 2
    assert abs(t["P4"]["gbs"] - t["P4"]["bytes_per_launch"] / 0.8e-3 / 1e9) < 0.1
