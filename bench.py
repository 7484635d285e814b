#!/usr/bin/env python3
"""Benchmark of the Wilson even-odd solve path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl ours|reference]

Workloads (seeded synthetic inputs with the shapes of the reference's
benchmark configurations; no external data):
  cg      32^4, links exp(i 0.3 H), kappa = 0.124, Gaussian source;
          one step = one solve of M x = b to true residual |b - M x|/|b| <= 1e-10.
          metric: CG solves/s.
  dslash  32^4, the even-odd operator applied with its dagger; one step =
          100 x (apply + dagger).  metric: dslash HBM GB/s (algorithmic bytes).
  mrhs    (default) the cg workload with 12 Gaussian sources per step solved together
          by the batched mixed-precision engine (FP16 inner solve, FP64 reliable
          updates), next to the plain FP64 CG on the same workload in the same run.
          metric: CG solves/s (mixed), with fp64_solves_per_s and the speed-up.
  cg8     8^4, kappa = 0.12, plain FP64 CG (the CPU-runnable configuration).
  serve   Poisson stream of solve requests (default 2000 at 20 requests/s; --requests,
          --rate) over 8 device-resident gauge fields 8^4 .. 32^4, each request with
          1..12 sources, kappa in [0.115, 0.124], accuracy 1e-10, through the
          continuous-batching server; the same request sequence is also served by the
          plain FP64 CG one source at a time (FIFO).  metric: solves/s, p50/p99 latency.
  serve32 the mrhs workload served: 32 requests of 12 sources on the 32^4 lattice at
          kappa = 0.124, arriving at 10 requests/s (faster than they are served),
          against the FP64 CG serving the same stream (speedup_vs_fifo_f64_capacity).

Multi-GPU runs (torchrun) are replicas: every rank solves its own copy of the
workload; value = total solves over all ranks / max-over-ranks device time.
`--impl reference` times the CPU oracle in the reference's loop structure
(reference-structured even-odd operator + CG of conjugate_gradient.h) on the
host cores, on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import concurrent.futures
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "CG solves/s at 1e-10 residual (mixed vs FP64), dslash HBM GB/s, p50/p99 ms"

WORKLOADS = {
    "cg": dict(dims=(32, 32, 32, 32), eps=0.3, kappa=0.124, tol=1e-10, link_seed=100, src_seed=101),
    "mrhs": dict(dims=(32, 32, 32, 32), eps=0.3, kappa=0.124, tol=1e-10, link_seed=100, src_seed=101, nrhs=12),
    "cg8": dict(dims=(8, 8, 8, 8), eps=0.3, kappa=0.12, tol=1e-10, link_seed=1, src_seed=2),
    "dslash": dict(dims=(32, 32, 32, 32), eps=0.3, kappa=0.124, tol=None, link_seed=100, src_seed=101),
    "serve": dict(dims=(32, 32, 32, 32), eps=0.3, kappa=0.124, tol=1e-10, link_seed=100, src_seed=101,
                  lattices=[(8, 8, 8, 8), (12, 12, 12, 12), (16, 16, 16, 16), (16, 16, 16, 32), (20, 20, 20, 20),
                            (24, 24, 24, 24), (28, 28, 28, 28), (32, 32, 32, 32)],
                  requests=2000, rate=20.0, kappa_range=(0.115, 0.124), nrhs_range=(1, 12)),
    # the headline 32^4 kappa = 0.124 workload served: requests of 12 sources each arriving faster
    # than the GPU finishes them (saturating), against the FP64 CG serving the same stream
    "serve32": dict(dims=(32, 32, 32, 32), eps=0.3, kappa=0.124, tol=1e-10, link_seed=100, src_seed=101,
                    lattices=[(32, 32, 32, 32)], requests=32, rate=10.0, kappa_range=(0.124, 0.124),
                    nrhs_range=(12, 12), pool=12),
    # staggered fermions (dirac_staggered_evenodd) on the batched engine: 12 sources of M x = b
    # solved together with FP16 inner iterations, against the same batch in FP64; the mass sits
    # just above the hop's spectral radius (about 2.25 for these links), where M = m - D^dag D / m
    # is still positive and hardest to solve
    "stag": dict(dims=(32, 32, 32, 32), eps=0.3, mass=2.3, tol=1e-10, link_seed=100, src_seed=101, nrhs=12),
}
# CG iterations of one solve of each workload (FP64 CG on M^dag M, true residual 1e-10), used to turn the
# reference arm's per-iteration time into solves/s.  Measured by the FP64 GPU CG on exactly these seeded
# inputs; the CPU runs the same algorithm, so the count is the same.
ITERS_PER_SOLVE = {"cg": 59, "mrhs": 59, "cg8": None}

# DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum) of one k_eng_low<P4> launch per
# output site, 12 FP16 sources with 18-real FP16 links: 1027.8 MB over 165,888 sites in one ncu
# capture at 24^4; every array is read once, so it scales with the sites.
P4_TRAFFIC_PER_SITE_12 = 1027.8e6 / 165888

# DRAM traffic of the two k_hop launches of one even-odd apply (12-real FP64 links), per
# output site: 633.6 MB + 865.3 MB over 524,288 sites in one ncu capture at 32^4; every
# array is read once, so it scales with the sites.
HOP_F64_12_TRAFFIC_PER_SITE = (633.6e6 + 865.3e6) / 524288

MEASURED_PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0
NOMINAL_HBM_GBS = 8000.0  # B200 HBM3e, nominal; reported beside the measured peak


def hbm_peak():
    try:
        with open(MEASURED_PEAKS) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


# ------------------------------------------------------------------ distributed plumbing

class Dist:
    """Replica plumbing (hila_b200.replicas.ReplicaGroup), initialised by the arm that runs."""

    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.group = None

    def init(self, backend):
        from hila_b200.replicas import ReplicaGroup
        self.group = ReplicaGroup(backend)

    def barrier(self):
        if self.group:
            self.group.barrier()

    def max(self, v: float) -> float:
        return self.group.max(v) if self.group else v

    def sum(self, v: float) -> float:
        return self.group.sum(v) if self.group else v

    def close(self):
        if self.group:
            self.group.close()


# ------------------------------------------------------------------ clocks

class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ CPU baseline (oracle)

def cpu_sample(workload: str, seconds_budget: float = 20.0):
    """Reference-structured oracle on the host cores: time per CG iteration and per apply."""
    from oracle import oracle as o
    o.build()
    w = WORKLOADS[workload]
    dims = w["dims"]
    U = o.gen_links(dims, w["eps"], w["link_seed"])
    b = o.gen_spinor(dims, w["src_seed"], o.EVEN)
    R = o.RefStructured(dims)
    out = np.zeros_like(b)
    cores = o.num_threads()
    # one apply to estimate, then as many CG iterations as fit the budget (at least 2)
    t0 = time.perf_counter()
    R.eo_apply(U, w["kappa"], b, out, 1)
    t_apply = time.perf_counter() - t0
    n_it = max(2, min(50, int(seconds_budget / max(3 * t_apply, 1e-6))))
    x = np.zeros_like(b)
    t0 = time.perf_counter()
    it, _ = R.cg(U, w["kappa"], b, x, 1e-300, n_it)
    t_cg = time.perf_counter() - t0
    # context: one apply on one thread, and the oracle's fused operator (one pass over the
    # output sites, no temporaries) on all cores and on one thread
    applies = {"reference_structured": {str(cores): t_apply}, "fused": {}}
    t0 = time.perf_counter()
    o.eo_apply(dims, U, w["kappa"], b, 1)
    applies["fused"][str(cores)] = time.perf_counter() - t0
    o.set_num_threads(1)
    try:
        t0 = time.perf_counter()
        R.eo_apply(U, w["kappa"], b, out, 1)
        applies["reference_structured"]["1"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        o.eo_apply(dims, U, w["kappa"], b, 1)
        applies["fused"]["1"] = time.perf_counter() - t0
    finally:
        o.set_num_threads(cores)
    R.close()
    return dict(t_iter=t_cg / max(it, 1), iters=it, t_apply=t_apply, cores=cores, dims=dims,
                apply_seconds={k: {n: round(t, 4) for n, t in v.items()} for k, v in applies.items()})


# ------------------------------------------------------------------ our arm

def engine_unit_bytes(phase: str, prec: str, link_format: int) -> tuple:
    """Algorithmic bytes of one work unit of an engine phase (every array read or written once).

    Returns (main, alternate, link site, normal-system R3) bytes for the four counters of
    the engine profile (hw_engine_profile.work).  Low-precision spinor `sp`: FP16 48 B + 4 B
    norm, FP32 96 B; y and the FP32 s / t of the reliable update 96 B; FP64 spinor 192 B.
    Links: all 8 links of a site once per launch (inner phases FP16 18 reals = 36 B or FP32
    12 reals = 48 B; FP64 144 or 96 B in R2..R5).  Arrays per slot and site:
      P1  p (neighbours) read, t written                           2 sp
      P2  t (neighbours), p read; Dp written                       3 sp
      P3  Dp (neighbours) read, t written                          2 sp
      P4  t (neighbours), Dp, r, p read; r written; y read+written 5 sp + 2 x 96
      R1  x read+written, y read (alternate: y also cleared)       2 x 192 + 96 (+ 96)
      R2  x (neighbours) read, t64 written                         2 x 192
      R3  t64 (neighbours), x, b read; s written as FP32 in y      3 x 192 + 96
          alternate (x = 0 first update, no hop): x, b read, y     2 x 192 + 96
          normal system: t64, x read, s written in FP64            3 x 192
      R4  s (neighbours) read, t64 written                         2 x 192
      R4L y (= s, neighbours) read, t written (FP32)               2 x 96
      R5  t64 (neighbours), s, b read; r written                   3 x 192 + sp
      R5L t (neighbours), y read; y cleared; r written             3 x 96 + sp
      P5  r, p read; p written (alternate, first iteration: p = r) 3 sp (2 sp)"""
    sp = 52 if prec == "f16" else 96
    lk = 8 * (36 if prec == "f16" else 48)
    lk64 = 8 * (144 if link_format == 18 else 96)
    table = {"P1": (2 * sp, 0, lk, 0), "P2": (3 * sp, 0, lk, 0), "P3": (2 * sp, 0, lk, 0),
             "P4": (5 * sp + 2 * 96, 0, lk, 0), "R1": (2 * 192 + 96, 2 * 192 + 2 * 96, 0, 0),
             "R2": (2 * 192, 0, lk64, 0), "R3": (3 * 192 + 96, 2 * 192 + 96, lk64, 3 * 192),
             "R4": (2 * 192, 0, lk64, 0), "R4L": (2 * 96, 0, lk, 0), "R5": (3 * 192 + sp, 0, lk64, 0),
             "R5L": (3 * 96 + sp, 0, lk, 0), "P5": (3 * sp, 2 * sp, 0, 0)}
    return table[phase]


def engine_phase_bytes(phase: str, work, prec: str, link_format: int) -> int:
    """Algorithmic bytes of the work units `work` (the profile's four counters) of a phase."""
    unit = engine_unit_bytes(phase, prec, link_format)
    return int(sum(u * w for u, w in zip(unit, work)))


def phase_table(prof: dict, prec: str, link_format: int, peak: float) -> dict:
    """Per-phase launches, time and algorithmic bytes of the launches that did work."""
    out = {}
    for k, (n, ms, work) in prof.items():
        if not n:
            out[k] = {"launches": 0, "ms_per_launch": None, "bytes_per_launch": None, "gbs": None, "frac": None}
            continue
        byt = engine_phase_bytes(k, work, prec, link_format) / n
        gbs = byt / (ms / n * 1e-3) / 1e9 if ms > 0 else None
        out[k] = {"launches": n, "ms_per_launch": round(ms / n, 4), "bytes_per_launch": int(byt),
                  "gbs": round(gbs, 1) if gbs else None, "frac": round(gbs / peak, 4) if gbs else None,
                  "work_units": list(work)}
    return out


def workload_config(args, w, world: int) -> dict:
    """The `config` of a bench line; both arms print the same one for the same workload."""
    dims = w["dims"]
    V = int(np.prod(dims))
    link_bytes = 144 if args.link_format == 18 else 96
    cfg = {"workload": args.workload, "lattice": "x".join(map(str, dims)), "kappa": w["kappa"], "eps": w["eps"],
           "tol": w["tol"], "link_format": args.link_format, "parallelism": f"replicas{world}",
           "l2": "inputs larger than L2 (links %d MB)" % (4 * V * link_bytes // 2**20)}
    if "nrhs" in w:
        cfg["nrhs"] = w["nrhs"]
    return cfg


def run_ours(args, dist: Dist):
    import torch
    import hila_b200 as hw
    torch.cuda.set_device(dist.local_rank)
    dist.init("nccl")
    w = WORKLOADS[args.workload]
    dims = w["dims"]
    ctx = hw.Context(dist.local_rank)
    stream = torch.cuda.ExternalStream(ctx.stream())
    lat = hw.Lattice(ctx, dims, True)
    U = hw.generate_links(dims, w["eps"], w["link_seed"])
    G = hw.GaugeField(lat, U, args.link_format)
    b_host = hw.generate_spinor(dims, w["src_seed"], hw.EVEN)
    fb, fx = hw.Field(lat, b_host), hw.Field(lat)
    D = hw.Dirac_Wilson_evenodd(w["kappa"], G)
    V = int(np.prod(dims))
    Vh = V // 2
    peak, peak_kind = hbm_peak()
    link_bytes = 144 if args.link_format == 18 else 96
    # algorithmic bytes per hop launch (one output site): 8 links + neighbour spinors once + output
    hop_bytes = 8 * link_bytes + 192 + 192
    apply_bytes = (2 * hop_bytes + 2 * 192) * Vh  # second hop also reads in_e and clears out_o

    def dslash_time(nrep):
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        fy = hw.Field(lat)
        D.apply(fb, fy)
        D.dagger(fy, fx)
        ctx.synchronize()
        ev0.record(stream)
        for _ in range(nrep):
            D.apply(fb, fy)
            D.dagger(fy, fx)
        ev1.record(stream)
        ev1.synchronize()
        fy.close()
        return ev0.elapsed_time(ev1) / (2 * nrep)  # ms per eo apply

    result = {}
    clocks = ClockSampler(dist.local_rank)
    if args.workload == "dslash":
        nrep = 100
        for _ in range(args.warmup):
            dslash_time(10)
        dist.barrier()
        torch.cuda.synchronize()
        clocks.start()
        ms = [dslash_time(nrep) for _ in range(args.steps)]
        clk = clocks.stop()
        ms_apply = dist.max(statistics.mean(ms))
        gbs = apply_bytes / (ms_apply * 1e-3) / 1e9
        value = dist.sum(gbs)
        ms_per_step = ms_apply * 2 * nrep
        unit = "GB/s"
        launches = args.steps * nrep * 4
        result["flops_per_s"] = dist.sum(1320 * V / (ms_apply * 1e-3))
        result["ms_per_apply"] = ms_apply
        e2e = None
        dtype = "f64"
        roof_ms = ms_apply
    elif args.workload == "mrhs":
        nrhs = w["nrhs"]
        srcs = [b_host] + [hw.generate_spinor(dims, w["src_seed"] + k, hw.EVEN) for k in range(1, nrhs)]
        fbs = [hw.Field(lat, s_) for s_ in srcs]
        fxs = [hw.Field(lat) for _ in range(nrhs)]
        prec = args.precision if args.precision != "f64" else "f16"

        def batch_once():
            for f in fxs:
                f.zero()
            return hw.batch_solve(ctx, [(D, fbs[k], fxs[k], w["tol"]) for k in range(nrhs)], precision=prec,
                                  delta=args.delta)

        for _ in range(args.warmup):
            batch_once()
        dist.barrier()
        torch.cuda.synchronize()
        clocks.start()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        res = []
        for _ in range(args.steps):
            res += batch_once()
        ev1.record(stream)
        ev1.synchronize()
        clk = clocks.stop()
        t = dist.max(ev0.elapsed_time(ev1) * 1e-3)
        value = dist.world * args.steps * nrhs / t
        ms_per_step = t / args.steps * 1e3
        unit = "solves/s"
        launches = sum(r.kernel_launches for r in res) // nrhs
        lat_ms = sorted(1e3 * r.seconds for r in res)
        result.update(iterations=max(r.iterations for r in res), reliable_updates=max(r.reliable_updates for r in res),
                      true_residual=max(r.true_residual for r in res), all_converged=all(r.converged for r in res),
                      precision=prec, nrhs=nrhs, latency_ms_p50=lat_ms[len(lat_ms) // 2],
                      latency_ms_p99=lat_ms[min(len(lat_ms) - 1, int(0.99 * len(lat_ms)))])
        dtype = {"f32": "f32+f64", "f16": "f16+f64"}[prec]
        # e2e: host sources in, host solutions out, through the public API, with host arrays in
        # HILA's even-first site order (its Field storage order) in page-locked memory, so the
        # EVEN half of each source and of each solution crosses the bus in one copy each.
        # (a) through the server: a client with two steps in flight (each step one request of
        #     the 12 sources, solutions into one of two sets of arrays), so the copies of one
        #     step overlap the solve of the other -- the headline e2e;
        # (b) serially through the field API: upload, batch solve, download.
        order = hw.eo_order(dims)
        half = V // 2
        pins = [hw.PinnedArray((half, 4, 3, 2)) for _ in range(nrhs)]
        pouts = [hw.PinnedArray((half, 4, 3, 2)) for _ in range(2 * nrhs)]
        for k in range(nrhs):
            pins[k].array[:] = srcs[k][order[:half]]
        srv = hw.Server(ctx, precision=prec, delta=args.delta)
        gid = srv.add_gauge(G)

        def served_steps(nsteps):
            ids, res = [None] * nsteps, []
            for k in range(nsteps):
                if k >= 2:
                    res.append(srv.wait(ids[k - 2], nrhs, V, copy=False)[1])
                outs = [pouts[(k % 2) * nrhs + j].array for j in range(nrhs)]
                ids[k] = srv.submit_eo(gid, w["kappa"], [pa.array for pa in pins], outs, w["tol"])
            for k in range(max(0, nsteps - 2), nsteps):
                res.append(srv.wait(ids[k], nrhs, V, copy=False)[1])
            return res

        served_steps(2)  # graphs, staging ring
        dist.barrier()
        t0 = time.perf_counter()
        res_e2e = served_steps(args.steps)
        t_e2e = dist.max(time.perf_counter() - t0)
        srv.close()
        e2e = {"value": dist.world * args.steps * nrhs / t_e2e, "unit": "solves/s",
               "h2d_bytes_per_step": int(nrhs * pins[0].array.nbytes),
               "d2h_bytes_per_step": int(nrhs * pins[0].array.nbytes),
               "all_converged": all(r.converged for r in res_e2e),
               "max_true_residual": max(r.true_residual for r in res_e2e),
               "path": "hw_server_submit_eo, two steps in flight: page-locked host arrays in even-first "
                       "site order, the EVEN half copied each way every step"}
        dist.barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            for k in range(nrhs):
                fbs[k].upload_eo(pins[k].array, hw.EVEN)
            batch_once()
            for k in range(nrhs):
                fxs[k].download_eo(hw.EVEN, pouts[k].array)
        t_ser = dist.max(time.perf_counter() - t0)
        e2e["serial_api"] = {"value": round(dist.world * args.steps * nrhs / t_ser, 3),
                             "path": "hw_field_upload_eo, hw_batch_solve, hw_field_download_eo per step"}
        for pa in pins + pouts:
            pa.free()
        # the plain FP64 CG on the same workload, same run: the reference point of the speed-up
        for _ in range(2):
            fxs[0].zero()
            D.solve(fbs[0], fxs[0], accuracy=w["tol"])
        torch.cuda.synchronize()
        ev0.record(stream)
        r64 = []
        for k in range(args.steps):
            fxs[0].zero()
            r64.append(D.solve(fbs[k % nrhs], fxs[0], accuracy=w["tol"]))
        ev1.record(stream)
        ev1.synchronize()
        t64 = dist.max(ev0.elapsed_time(ev1) * 1e-3)
        fp64 = dist.world * args.steps / t64
        result.update(fp64_solves_per_s=round(fp64, 3), speedup_vs_fp64=round(value / fp64, 3),
                      fp64_iterations=r64[0].iterations, fp64_all_converged=all(r.converged for r in r64))
        roof_ms = dslash_time(50)
        result["dslash_ms_per_apply"] = roof_ms
        # per-phase device time of one more batch (events around every engine launch)
        ctx.engine_profile(True)
        batch_once()
        prof = ctx.engine_profile_get(prec)
        ctx.engine_profile(False)
        result["phases"] = phase_table(prof, prec, args.link_format, peak)
        engine_roof = result["phases"]["P4"]
        # the launch-shape tuner's entry for this batch (its work class: bit length of the
        # solves x 128-site tiles of the lattice), timed during the warm-up steps
        cls = (nrhs * -(-(V // 2) // 128)).bit_length()
        ent = next((t for t in ctx.engine_tuning(prec) if t["work_class"] == cls), None)
        if ent is not None:
            result["tuner"] = {
                "work_class": cls,
                "shapes": [{"variant": v, "dynamic_order": d, "ms_per_iteration": round(ms, 4), "samples": n}
                           for v, d, ms, n in ent["shapes"]],
                "chosen": ent["chosen"]}
        if not args.no_served and dist.world == 1:
            # the same 32^4 workload through the continuous-batching server (serve32: 32 requests of
            # 12 sources arriving faster than they are served), against the plain FP64 CG serving
            # the same stream
            m = serve_measure(ctx, WORKLOADS["serve32"], args)
            result["served_speedup_vs_fp64"] = m["speedup_vs_fifo_f64_capacity"]
            result["served"] = {k: m[k] for k in ("value", "requests", "solves", "latency_ms_p50", "latency_ms_p99",
                                                  "all_converged", "max_true_residual", "fifo_f64", "server_stats",
                                                  "wall_s")}
            result["served"]["workload"] = "serve32"
        for f in fbs + fxs:
            f.close()
    else:
        def solve_once():
            fx.zero()
            return D.solve(fb, fx, accuracy=w["tol"], precision=args.precision, use_graph=not args.no_graph,
                           delta=args.delta)

        for _ in range(args.warmup):
            r = solve_once()
        dist.barrier()
        torch.cuda.synchronize()
        clocks.start()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        res = [solve_once() for _ in range(args.steps)]
        ev1.record(stream)
        ev1.synchronize()
        clk = clocks.stop()
        t = dist.max(ev0.elapsed_time(ev1) * 1e-3)
        dist.barrier()
        value = dist.world * args.steps / t
        ms_per_step = t / args.steps * 1e3
        unit = "solves/s"
        launches = sum(r.kernel_launches for r in res)
        ok = all(r.converged for r in res)
        result.update(iterations=res[0].iterations, true_residual=max(r.true_residual for r in res),
                      all_converged=ok, restarts=res[0].restarts, precision=args.precision)
        dtype = {"f64": "f64", "f32": "f32+f64", "f16": "f16+f64"}[args.precision]
        # e2e: host arrays through the C ABI (H2D of b and D2H of x inside the timed region)
        pb = hw.PinnedArray((V, 4, 3, 2))
        px = hw.PinnedArray((V, 4, 3, 2))
        pb.array[:] = b_host
        D.solve_host(pb.array, px.array, accuracy=w["tol"], precision=args.precision)
        dist.barrier()
        t0 = time.perf_counter()
        re2e = [D.solve_host(pb.array, px.array, accuracy=w["tol"], precision=args.precision)
                for _ in range(args.steps)]
        t_e2e = dist.max(time.perf_counter() - t0)
        e2e = {"value": dist.world * args.steps / t_e2e, "unit": "solves/s",
               "h2d_bytes_per_step": int(pb.array.nbytes), "d2h_bytes_per_step": int(px.array.nbytes),
               "all_converged": all(r.converged for r in re2e)}
        pb.free()
        px.free()
        # dominant kernel: the hopping term; time it live on the library stream
        roof_ms = dslash_time(50)
        result["dslash_ms_per_apply"] = roof_ms
    hop_ms = roof_ms / 2
    achieved = (apply_bytes / 2) / (hop_ms * 1e-3) / 1e9
    hop_traffic = None
    if args.link_format == 12 and HOP_F64_12_TRAFFIC_PER_SITE:
        hop_traffic = {"bytes_per_launch": int(HOP_F64_12_TRAFFIC_PER_SITE * Vh / 2),
                       "source": "ncu capture at 32^4 (mean of the apply's two launches) scaled by sites"}
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
                "frac_of_nominal_8000": round(achieved / NOMINAL_HBM_GBS, 4),
                "traffic": hop_traffic, "kernel": "k_hop (FP64, %d-real links)" % args.link_format,
                "algorithmic_bytes_per_launch": apply_bytes / 2}
    if args.workload == "mrhs":
        # the dominant kernel of the batched solve: the engine's P4 phase
        result["roofline_fp64_hop"] = roofline
        a4 = engine_roof["bytes_per_launch"] / (engine_roof["ms_per_launch"] * 1e-3) / 1e9
        traffic = None
        if w["nrhs"] == 12 and prec == "f16":
            traffic = {"bytes_per_launch": int(P4_TRAFFIC_PER_SITE_12 * V // 2),
                       "source": "ncu capture at 24^4 scaled by sites"}
        roofline = {"bound": "hbm", "achieved": round(a4, 1), "peak": peak, "unit": "GB/s",
                    "frac": round(a4 / peak, 4), "peak_kind": peak_kind, "traffic": traffic,
                    "kernel": "k_eng_low<P4> (FP16 + norm, 18-real FP16 links, %d sources)" % w["nrhs"],
                    "algorithmic_bytes_per_launch": engine_roof["bytes_per_launch"],
                    "ms_per_launch": engine_roof["ms_per_launch"]}
    out = {
        "metric": METRIC, "value": round(value, 4), "unit": unit, "n_gpus": dist.world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": dtype, "data": "synthetic: seeded SU(3) links exp(i eps H), Gaussian sources",
        "config": workload_config(args, w, dist.world),
        "roofline": roofline, "e2e": e2e, "gpu_launches": int(launches), "clocks": clk, "impl": "ours",
        **result,
    }
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline and args.workload != "dslash":
        cs = cpu_sample(args.workload)
        iters = result.get("fp64_iterations") or result.get("iterations") or 1
        out["cpu_baseline"] = {"value": 1.0 / (cs["t_iter"] * iters), "unit": "solves/s", "cores": cs["cores"],
                               "kind": "port",
                               "sample": f"{cs['iters']} CG iterations of the reference-structured oracle at "
                                         f"{'x'.join(map(str, cs['dims']))} on {cs['cores']} threads "
                                         f"({cs['t_iter']:.3f} s/iteration), scaled by the {iters} iterations "
                                         f"of one solve",
                               "apply_seconds_by_threads": cs["apply_seconds"]}
    elif dist.rank == 0 and dist.world == 1 and args.workload == "dslash" and not args.no_cpu_baseline:
        cs = cpu_sample("cg", seconds_budget=5.0)
        out["cpu_baseline"] = {"value": apply_bytes / cs["t_apply"] / 1e9, "unit": "GB/s", "cores": cs["cores"],
                               "kind": "port", "sample": "one reference-structured even-odd apply at 32^4",
                               "apply_seconds_by_threads": cs["apply_seconds"]}
    if dist.rank == 0:
        print(json.dumps(out), flush=True)
    for f in (fb, fx):
        f.close()
    G.close()
    lat.close()
    ctx.close()
    dist.close()


# ------------------------------------------------------------------ serving

def serve_stream(w, seed=11):
    """The request stream: (arrival time s, lattice index, kappa, source indices)."""
    rng = np.random.default_rng(seed)
    t, reqs = 0.0, []
    lo, hi = w["nrhs_range"]
    pool = w.get("pool", SERVE_POOL)
    for n in range(w["requests"]):
        t += rng.exponential(1.0 / w["rate"])
        g = int(rng.integers(0, len(w["lattices"])))
        nrhs = int(rng.integers(lo, hi + 1))
        kappa = float(rng.uniform(*w["kappa_range"]))
        reqs.append((t, g, kappa, [(n + k) % pool for k in range(nrhs)]))
    return reqs


SERVE_POOL = 6  # distinct sources generated per lattice; a request takes consecutive ones


def pct(v, q):
    v = sorted(v)
    return v[min(len(v) - 1, int(q * len(v)))] if v else None


def serve_measure(ctx, w, args, rank: int = 0) -> dict:
    """Serve the Poisson request stream of workload `w` through the continuous-batching server,
    then the same stream through the plain FP64 CG (FIFO, one source at a time).  Returns the
    measured figures; the clocks are sampled while the server runs."""
    import torch
    import hila_b200 as hw
    reqs = serve_stream(w, seed=11 + rank)
    pool = w.get("pool", SERVE_POOL)
    # sources as a HILA application holds them on the host: even-first site order (its Field
    # storage order) in page-locked memory; only the EVEN half is a source, so the arrays hold
    # that half, and the server copies them by DMA with no host-side gather
    lats, gauges, pools, pinned = [], [], [], []
    for i, dims in enumerate(w["lattices"]):
        lat = hw.Lattice(ctx, dims, True)
        lats.append(lat)
        gauges.append(hw.GaugeField(lat, hw.generate_links(dims, w["eps"], w["link_seed"] + i), args.link_format))
        order = hw.eo_order(dims)[: lat.volume // 2]
        row = []
        for k in range(pool):
            pa = hw.PinnedArray((lat.volume // 2, 4, 3, 2))
            pa.array[:] = hw.generate_spinor(dims, w["src_seed"] + 100 * i + k, hw.EVEN)[order]
            pinned.append(pa)
            row.append(pa.array)
        pools.append(row)
    # solutions go by DMA into page-locked arrays of the caller as well: per lattice a ring of
    # arrays handed out in turn (only the spot check below reads a solution, so requests in
    # flight at the same time may share arrays)
    nmax = w["nrhs_range"][1]
    sol_rings = []
    for lat in lats:
        row = []
        for _ in range(2 * nmax):
            pa = hw.PinnedArray((lat.volume // 2, 4, 3, 2))
            pinned.append(pa)
            row.append(pa.array)
        sol_rings.append(row)
    cursor = [0] * len(lats)

    def sols_for(g, nrhs):
        ring = sol_rings[g]
        out = [ring[(cursor[g] + k) % len(ring)] for k in range(nrhs)]
        cursor[g] = (cursor[g] + nrhs) % len(ring)
        return out

    srv = hw.Server(ctx, precision=args.precision, delta=args.delta)
    gids = [srv.add_gauge(G) for G in gauges]
    # warm-up: two requests of the largest size per lattice, all at once, so that the graphs,
    # the engine's slot buffers (sized for the largest lattice first) and the staging rings
    # (made when a request has to wait) exist before the stream starts
    warm = []
    for g in sorted(range(len(lats)), key=lambda g: -lats[g].volume):
        for _ in range(2):
            warm.append((g, srv.submit_eo(gids[g], w["kappa"], [pools[g][k % pool] for k in range(nmax)],
                                          sols_for(g, nmax), w["tol"])))
    for g, rid in warm:
        srv.wait(rid, nmax, lats[g].volume, copy=False)
    st0 = srv.stats()
    torch.cuda.synchronize()
    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    ids, t_sub, t_call = [None] * len(reqs), [0.0] * len(reqs), [0.0] * len(reqs)
    submitted = [threading.Event() for _ in reqs]
    t0 = time.perf_counter()

    def submitter():
        for n, (ta, g, kappa, src) in enumerate(reqs):
            d = t0 + ta - time.perf_counter()
            if d > 0:
                time.sleep(d)
            t_sub[n] = time.perf_counter()
            ids[n] = srv.submit_eo(gids[g], kappa, [pools[g][k] for k in src], sols_for(g, len(src)), w["tol"])
            t_call[n] = time.perf_counter() - t_sub[n]
            submitted[n].set()

    # collect the results with a pool of waiting threads, each blocked in hw_server_wait (the
    # interpreter lock is released there), so the submitting thread keeps to its schedule and
    # a slow request holds one waiter, not the others
    results, t_done = [None] * len(reqs), [0.0] * len(reqs)

    def waiter(n):
        submitted[n].wait()
        res = srv.wait(ids[n], len(reqs[n][3]), lats[reqs[n][1]].volume, copy=False)[1]
        t_done[n] = t_sub[n] + res.latency_seconds
        results[n] = res

    th = threading.Thread(target=submitter)
    th.start()
    with concurrent.futures.ThreadPoolExecutor(max_workers=32) as ex:
        list(ex.map(waiter, range(len(reqs))))
    th.join()
    clk = clocks.stop()
    st = srv.stats()
    t_wall = max(t_done) - t0
    solves = sum(len(r[3]) for r in reqs)
    lat_ms = [1e3 * r.latency_seconds for r in results]
    # correctness spot check: a solution through the public API against the FP64 true residual
    g_chk = len(lats) - 1
    V_chk = lats[g_chk].volume
    sol = np.zeros((V_chk // 2, 4, 3, 2))
    rid = srv.submit_eo(gids[g_chk], w["kappa"], [pools[g_chk][0]], [sol], w["tol"])
    srv.wait(rid, 1, V_chk, copy=False)
    D_chk = hw.Dirac_Wilson_evenodd(w["kappa"], gauges[g_chk])
    srv.close()
    fx, fy = hw.Field(lats[g_chk]), hw.Field(lats[g_chk])
    fx.upload_eo(sol, hw.EVEN)
    D_chk.apply(fx, fy)
    mx = fy.download_eo(hw.EVEN)[: V_chk // 2]
    b0 = pools[g_chk][0]
    chk = float(np.linalg.norm(mx - b0) / np.linalg.norm(b0))
    fx.close()
    fy.close()
    # the same stream served by the plain FP64 CG, one source at a time, in arrival order, with
    # the same host arrays in and out (EVEN half by DMA each way): the service time of every
    # request is measured, the FIFO queue is then exact arithmetic
    fb64 = [hw.Field(lat) for lat in lats]
    fx64 = [hw.Field(lat) for lat in lats]
    outs = [hw.PinnedArray((lat.volume // 2, 4, 3, 2)) for lat in lats]

    def solve64(g, kappa, src):
        D = hw.Dirac_Wilson_evenodd(kappa, gauges[g])
        ok = True
        for k in src:
            fb64[g].upload_eo(pools[g][k], hw.EVEN)
            fx64[g].zero(hw.EVEN)
            ok &= D.solve(fb64[g], fx64[g], accuracy=w["tol"]).converged
            fx64[g].download_eo(hw.EVEN, outs[g].array)
        return ok

    for g in range(len(lats)):
        solve64(g, w["kappa"], [0])
    torch.cuda.synchronize()
    t_free, lat64, busy, ok64 = 0.0, [], 0.0, True
    for (ta, g, kappa, src) in reqs:
        s0 = time.perf_counter()
        ok64 &= solve64(g, kappa, src)
        dt = time.perf_counter() - s0
        busy += dt
        start = max(ta, t_free)
        t_free = start + dt
        lat64.append(1e3 * (t_free - ta))
    for f in fb64 + fx64:
        f.close()
    for pa in outs + pinned:
        pa.free()
    for G in gauges:
        G.close()
    for lat in lats:
        lat.close()
    fifo_capacity = solves / busy
    value = solves / t_wall
    k_lag = max(range(len(reqs)), key=lambda k: t_sub[k] - (t0 + reqs[k][0]))
    return {
        "value": value, "solves": solves, "requests": len(reqs), "wall_s": t_wall, "clocks": clk,
        "latency_ms_p50": pct(lat_ms, 0.5), "latency_ms_p99": pct(lat_ms, 0.99),
        "queue_ms_p50": pct([1e3 * r.queue_seconds for r in results], 0.5),
        "submit_lag_ms_max": round(1e3 * max(ts - (t0 + r[0]) for ts, r in zip(t_sub, reqs)), 3),
        "submit_call_ms_max": round(1e3 * max(t_call), 3),
        "submit_lag_worst": {"request": k_lag, "arrival_s": round(reqs[k_lag][0], 3),
                             "lattice": "x".join(map(str, w["lattices"][reqs[k_lag][1]])),
                             "call_ms": round(1e3 * t_call[k_lag], 3)},
        "all_converged": all(r.converged for r in results),
        "max_true_residual": max(r.true_residual for r in results), "spot_check_residual": chk,
        "speedup_vs_fifo_f64_capacity": round(value / fifo_capacity, 3),
        "fifo_f64": {"solves_per_s": round(solves / t_free, 3), "capacity_solves_per_s": round(fifo_capacity, 3),
                     "latency_ms_p50": pct(lat64, 0.5), "latency_ms_p99": pct(lat64, 0.99),
                     "all_converged": ok64},
        "server_stats": {k: (round(st[k] - st0[k], 3) if k.startswith("seconds") else st[k])
                         for k in ("completed", "solves_completed", "rejected", "cancelled", "seconds_admit",
                                   "seconds_run", "seconds_retire")},
        # longest single passes of the server thread's sections (warm-up included)
        "server_max_seconds": {k: round(st[k], 4) for k in ("max_admit_seconds", "max_launch_seconds",
                                                             "max_retire_seconds")},
        "gpu_launches": int(st["kernel_launches"] - st0["kernel_launches"]),
        "chunks": int(st["chunks"] - st0["chunks"]),
        "bytes_per_request": int(sum(len(r[3]) * lats[r[1]].volume * 96 for r in reqs) / len(reqs)),
        "host_arrays": "even-first site order (HILA Field storage), page-locked, EVEN half by DMA each way",
    }


def run_stag(args, dist: Dist):
    """The staggered workload: a batch of staggered solves of M x = b on the engine with FP16
    inner iterations and FP64 reliable updates (value), the same batch in FP64 on the engine,
    and the standalone FP64 CG (CG<dirac_staggered_evenodd>, normal equations) for context."""
    import torch
    import hila_b200 as hw
    torch.cuda.set_device(dist.local_rank)
    dist.init("nccl")
    w = WORKLOADS["stag"]
    dims, nrhs = w["dims"], w["nrhs"]
    ctx = hw.Context(dist.local_rank)
    stream = torch.cuda.ExternalStream(ctx.stream())
    lat = hw.Lattice(ctx, dims, True)
    G = hw.GaugeField(lat, hw.generate_links(dims, w["eps"], w["link_seed"]), args.link_format)
    D = hw.dirac_staggered_evenodd(w["mass"], G)
    # seeded Gaussian colour vectors on the EVEN sites (spin component 0 of the spinor generator)
    srcs = [np.ascontiguousarray(hw.generate_spinor(dims, w["src_seed"] + k, hw.EVEN)[:, 0]) for k in range(nrhs)]
    fbs = [hw.StaggeredField(lat, v) for v in srcs]
    fxs = [hw.StaggeredField(lat) for _ in srcs]

    def batch(prec):
        for f in fxs:
            f.zero()
        return hw.staggered_batch_solve(ctx, [(D, fb, fx, w["tol"]) for fb, fx in zip(fbs, fxs)], precision=prec,
                                        delta=args.delta)

    def timed(prec, steps):
        dist.barrier()
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        res = []
        for _ in range(steps):
            res += batch(prec)
        ev1.record(stream)
        ev1.synchronize()
        return dist.max(ev0.elapsed_time(ev1) * 1e-3), res

    for _ in range(args.warmup):
        batch("f16")
    batch("f64")
    clocks = ClockSampler(dist.local_rank)
    clocks.start()
    t, res = timed("f16", args.steps)
    clk = clocks.stop()
    value = dist.world * args.steps * nrhs / t
    t64, res64 = timed("f64", max(1, args.steps // 2))
    fp64 = dist.world * max(1, args.steps // 2) * nrhs / t64
    # the standalone FP64 CG on the normal equations of one source
    fy = hw.StaggeredField(lat)
    D.cg(fbs[0], fy, accuracy=w["tol"])
    fy.zero()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    rcg = D.cg(fbs[0], fy, accuracy=w["tol"])
    ev1.record(stream)
    ev1.synchronize()
    cfg = workload_config(args, dict(w, kappa=None), dist.world)
    cfg.pop("kappa", None)
    cfg["mass"] = w["mass"]
    out = {
        "metric": "staggered CG solves/s at 1e-10 residual (FP16 inner + FP64 reliable updates vs FP64)",
        "value": round(value, 4), "unit": "solves/s", "n_gpus": dist.world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(t / args.steps * 1e3, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f16+f64",
        "data": "synthetic: seeded SU(3) links exp(i eps H), Gaussian sources", "config": cfg,
        "iterations": max(r.iterations for r in res), "reliable_updates": max(r.reliable_updates for r in res),
        "true_residual": max(r.true_residual for r in res), "all_converged": all(r.converged for r in res),
        "fp64_engine_solves_per_s": round(fp64, 3), "fp64_engine_iterations": max(r.iterations for r in res64),
        "fp64_engine_all_converged": all(r.converged for r in res64), "speedup_vs_fp64_engine": round(value / fp64, 3),
        "fp64_cg_normal_equations": {"solves_per_s": round(1e3 / ev0.elapsed_time(ev1), 3),
                                     "iterations": rcg.iterations, "converged": rcg.converged},
        "clocks": clk, "impl": "ours"}
    if dist.rank == 0:
        print(json.dumps(out))
    dist.close()


def run_serve(args, dist: Dist):
    """Poisson request stream through the server, and the same stream through the FP64 CG (FIFO)."""
    import torch
    import hila_b200 as hw
    torch.cuda.set_device(dist.local_rank)
    dist.init("nccl")
    w = WORKLOADS[args.workload]
    ctx = hw.Context(dist.local_rank)
    dist.barrier()
    m = serve_measure(ctx, w, args, dist.rank)
    t_wall = dist.max(m["wall_s"])
    value = dist.sum(m["value"])
    out = {
        "metric": "served CG solves/s at 1e-10 residual (Poisson stream, %d lattices)" % len(w["lattices"]),
        "value": round(value, 4),
        "unit": "solves/s", "n_gpus": dist.world, "steps": m["requests"], "warmup": 2 * len(w["lattices"]),
        "ms_per_step": round(1e3 * t_wall / m["requests"], 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": {"f32": "f32+f64", "f16": "f16+f64"}[args.precision],
        "data": "synthetic: seeded SU(3) links exp(i eps H), Gaussian sources, Poisson arrivals",
        "config": {"workload": args.workload, "lattices": ["x".join(map(str, d)) for d in w["lattices"]],
                   "requests": m["requests"], "rate_per_s": w["rate"], "nrhs_range": w["nrhs_range"],
                   "kappa_range": w["kappa_range"], "tol": w["tol"], "link_format": args.link_format,
                   "precision": args.precision, "delta": args.delta, "parallelism": f"replicas{dist.world}",
                   "hbm_budget": "80% of free device memory"},
        "e2e": {"value": round(value, 4), "unit": "solves/s",
                "note": "host arrays in and out through the server (even-first order, EVEN half each way)",
                "h2d_bytes_per_step": m["bytes_per_request"], "d2h_bytes_per_step": m["bytes_per_request"]},
        "clocks": m["clocks"], "impl": "ours",
        **{k: v for k, v in m.items() if k not in ("value", "clocks", "bytes_per_request", "requests")},
    }
    if dist.rank == 0:
        print(json.dumps(out), flush=True)
    ctx.close()
    dist.close()


# ------------------------------------------------------------------ reference arm

def run_reference(args, dist: Dist):
    if dist.rank != 0:
        return
    w = WORKLOADS[args.workload]
    if args.workload.startswith("serve"):
        print(json.dumps({"impl": "reference", "unavailable": "the reference has no request server; its FP64 CG "
                          "is timed on the cg and mrhs workloads"}), flush=True)
        return
    if args.workload == "stag":
        print(json.dumps({"impl": "reference", "unavailable": "the stag workload compares the engine's FP16 and FP64 "
                          "staggered solves on the GPU; the reference's CPU CG is timed on the cg and mrhs "
                          "workloads"}), flush=True)
        return
    if args.workload == "dslash":
        samples = [cpu_sample("cg", seconds_budget=2.0) for _ in range(args.warmup + args.steps)][args.warmup:]
        t = statistics.mean(s["t_apply"] for s in samples)
        V = int(np.prod(w["dims"]))
        value = (2 * (8 * 144 + 384) + 192) * (V // 2) / t / 1e9
        unit, cs, sample = "GB/s", samples[0], "one reference-structured even-odd apply per step"
        ms_per_step = t * 1e3
    elif ITERS_PER_SOLVE.get(args.workload) is None:
        # small enough for whole solves: the reference-structured CG on M^dag M to its own
        # stopping rule (|r|^2 < acc^2 |b|^2, conjugate_gradient.h:63,91), one solve per step
        from oracle import oracle as o
        o.build()
        dims = w["dims"]
        U = o.gen_links(dims, w["eps"], w["link_seed"])
        b = o.gen_spinor(dims, w["src_seed"], o.EVEN)
        R = o.RefStructured(dims)
        times, its = [], []
        for k in range(args.warmup + args.steps):
            x = np.zeros_like(b)
            t0 = time.perf_counter()
            it, _ = R.cg(U, w["kappa"], b, x, w["tol"], 10000)
            if k >= args.warmup:
                times.append(time.perf_counter() - t0)
                its.append(it)
        R.close()
        t_solve = statistics.mean(times)
        value, unit = 1.0 / t_solve, "solves/s"
        cs = {"cores": o.num_threads()}
        sample = (f"whole solves of the reference-structured CG at {'x'.join(map(str, dims))} "
                  f"({its[0]} iterations to its stopping rule, {t_solve:.4f} s each)")
        ms_per_step = t_solve * 1e3
    else:
        iters = ITERS_PER_SOLVE.get(args.workload)
        samples = [cpu_sample(args.workload, seconds_budget=15.0) for _ in range(args.warmup + args.steps)]
        samples = samples[args.warmup:]
        t_iter = statistics.mean(s["t_iter"] for s in samples)
        value = 1.0 / (t_iter * iters)
        unit, cs = "solves/s", samples[0]
        sample = (f"{cs['iters']} CG iterations per step of the reference-structured oracle, scaled by the "
                  f"{iters} iterations one solve of this workload takes")
        ms_per_step = t_iter * iters * 1e3
    out = {"metric": METRIC, "value": value, "unit": unit, "n_gpus": dist.world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
           "config": workload_config(args, w, dist.world),
           "cpu_baseline": {"value": value, "unit": unit, "cores": cs["cores"], "kind": "port", "sample": sample},
           "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="mrhs", choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default=None, choices=["f64", "f32", "f16"],
                    help="default: f16 for mrhs/serve/serve32, f64 otherwise")
    ap.add_argument("--link-format", type=int, default=12, choices=[18, 12])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-graph", action="store_true", help="CG iterations from a host loop (for launch lists)")
    ap.add_argument("--no-served", action="store_true", help="mrhs: skip the served (serve32) comparison")
    ap.add_argument("--delta", type=float, default=None,
                    help="reliable-update factor of the mixed-precision solves (default 0.005 FP16, 1e-5 FP32)")
    ap.add_argument("--lattice", default=None, help="override the workload's lattice, e.g. 24x24x24x24")
    ap.add_argument("--nrhs", type=int, default=None, help="override the right-hand sides per step (mrhs)")
    ap.add_argument("--requests", type=int, default=None, help="serve: number of requests")
    ap.add_argument("--rate", type=float, default=None, help="serve: Poisson arrival rate (requests/s)")
    ap.add_argument("--mass", type=float, default=None, help="stag: staggered mass")
    args = ap.parse_args()
    if args.precision is None:
        args.precision = "f16" if args.workload in ("mrhs", "serve", "serve32") else "f64"
    if args.delta is None:
        args.delta = 1e-5 if args.precision == "f32" else (0.05 if args.workload == "stag" else 0.005)
    if args.requests and args.workload.startswith("serve"):
        WORKLOADS[args.workload]["requests"] = args.requests
    if args.rate and args.workload.startswith("serve"):
        WORKLOADS[args.workload]["rate"] = args.rate
    if args.lattice:
        WORKLOADS[args.workload]["dims"] = tuple(int(v) for v in args.lattice.split("x"))
    if args.nrhs:
        WORKLOADS[args.workload]["nrhs"] = args.nrhs
    if args.mass and args.workload == "stag":
        WORKLOADS["stag"]["mass"] = args.mass
    if args.no_graph:
        os.environ["HW_USE_GRAPH"] = "0"
    if args.warmup < 3:
        args.warmup = 3
    dist = Dist()
    if args.impl == "reference":
        run_reference(args, dist)
    elif args.workload.startswith("serve"):
        run_serve(args, dist)
    elif args.workload == "stag":
        run_stag(args, dist)
    else:
        run_ours(args, dist)


if __name__ == "__main__":
    main()
