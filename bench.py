#!/usr/bin/env python
"""PME particle-kicks/s on B200 (tigerpm_b200) -- one JSON line on rank 0.

A step is one whole PME kick of every particle of a box, as the reference's
kick_pme_test runs it (src/test.cpp:182-234): restore the box's particles,
chain-mesh sort, deposit, r2c FFT, Green's function, c2r FFT, interpolation +
short-range PP + rung kick.  `value` times the step with the inputs already
resident in HBM; `e2e` times the same step through the C ABI from pinned host
buffers (H2D of the particles, D2H of the kicked particles) every step, with
tpm_pme_steps_host (the served stream: the copies of neighbouring steps
overlap each step's kernels); `e2e.serial` is set_particles + pme_step +
get_particles one after the other.

Workloads (synthetic, seeded Philox; see tigerpm_b200/workloads.py):
  c2-accurate  (default) 256^3 Zel'dovich particles (P(k) ~ k^-2 cut at
               k_Nyq/2, rms displacement 0.3 particle spacings), the
               reference's cloud4 deposit on a 768^3 mesh (3x the lattice),
               r_s = 2 mesh cells, cutoff 6 r_s: the form of the 256^3
               configuration that meets rms force error <= 1e-4 at the lowest
               measured step time (TSC and the literal r_s / mesh do not).
  c2-accurate-128  the same form at 128^3 particles / 384^3 mesh: the same
               chain-cell occupancy (64 per cell) and kernel shapes, an eighth of
               the work; the small case the ncu captures run on.
  c2           the same particles with the configuration's literal mesh
               parameters: 256^3 mesh, TSC, r_s = 1.25 cells, cutoff 4.5 r_s.
  c1           64^3 uniform particles, 64^3 mesh, CIC, r_s 1.25, 4.5 r_s.
Every run also reports the rms force error of the kick against the FP64
Ewald sum on 4,096 sampled particles.

--impl reference times the oracle (oracle/, the CPU restatement of the
reference path; the reference itself cannot be built here) on the host
cores on the same workload; rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CONFIGS = {
    "c2-accurate": dict(kind="zeldovich", n_side=256, grid=768, assign="cloud4", rs_cells=2.0, rcut_over_rs=6.0,
                        ewald_samples=4096),
    "c2-accurate-128": dict(kind="zeldovich", n_side=128, grid=384, assign="cloud4", rs_cells=2.0, rcut_over_rs=6.0,
                            ewald_samples=4096),
    "c2": dict(kind="zeldovich", n_side=256, grid=256, assign="tsc", rs_cells=1.25, rcut_over_rs=4.5,
               ewald_samples=4096),
    "c1": dict(kind="uniform", n_side=64, grid=64, assign="cic", rs_cells=1.25, rcut_over_rs=4.5,
               ewald_samples=1000),
}
METRIC = "PME particle-kicks/s at rms force err<=1e-4 vs FP64 Ewald"
FLOPS_PER_PAIR = 44.0      # in-cutoff pair, FMA = 2, MUFU = 1 (the reference's inner loop)
FLOPS_PER_CULLED = 8.0     # candidate pair rejected by the r^2 test
REF_BUDGET_S = 150.0       # CPU seconds the reference arm spends on timed whole kicks


def max_over_ranks(ms, dist, device=None):
    """Largest per-rank time (every rank calls it; dist None: one process)."""
    if dist is None:
        return ms
    import torch
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(n_per_rank, world, steps, ms):
    """Whole-job particle-kicks/s: every rank's particles over the slowest rank's time."""
    return n_per_rank * world * steps / (ms * 1e-3)


def hbm_peak_gbs():
    """Measured copy bandwidth of this pool's B200s (MEASURED_PEAKS.json), or
    the pool's earlier measurement when the file is absent."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs, copy)"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback (6.65 TB/s, an earlier measurement on this pool)"


def stage_hbm(grid, n, stages):
    """HBM fractions of the long-range stages: algorithmic bytes per step
    (each array read or written once: packed positions 16 B per particle,
    the real mesh 4 N^3 B, the half spectrum 8 N^2 (N/2+1) B, results 16 B
    and rung 1 B per particle) over the event-timed stage, against the
    measured copy bandwidth."""
    mesh = 4 * grid ** 3
    spec = 8 * grid * grid * (grid // 2 + 1)
    algo = {"deposit_ms": 16 * n + mesh,                      # positions in, density out
            "fft_forward_ms": (mesh + spec) + 2 * spec,       # z (real -> half spectrum), y
            "green_ms": 2 * spec,                             # x forward + Green + x inverse
            "fft_inverse_ms": 2 * spec + (spec + mesh),       # y, z (half spectrum -> real)
            "interp_ms": mesh + 16 * n + n + 16 * n}          # phi, positions, rung in; g, pot out
    peak, source = hbm_peak_gbs()
    out = {"peak_gbs": peak, "peak_source": source}
    for k, b in algo.items():
        ms = stages.get(k)
        if ms:
            gbs = b / (ms * 1e-3) / 1e9
            out[k[:-3]] = {"bytes": int(b), "gbs": round(gbs, 1), "frac": round(gbs / peak, 3)}
    return out


def make_particles(cfg, seed):
    from tigerpm_b200 import workloads as W
    if cfg["kind"] == "uniform":
        return W.uniform(cfg["n_side"] ** 3, seed)
    return W.zeldovich(cfg["n_side"], seed, rms_cells=0.3, grid=cfg["n_side"])


def make_opts(cfg):
    from tigerpm_b200.api import make_options
    return make_options(cfg["n_side"], cfg["grid"], rs_cells=cfg["rs_cells"], rcut_over_rs=cfg["rcut_over_rs"],
                        assign=cfg["assign"])


def host_opts(cfg):
    """The same option values make_opts derives, computed without the CUDA
    library (the reference arm must not load it)."""
    from types import SimpleNamespace
    grid = cfg["grid"]
    width = cfg["rcut_over_rs"] * cfg["rs_cells"]
    return SimpleNamespace(four_dim=grid, chain_dim=max(3, int(grid / width)), rs=cfg["rs_cells"] / grid,
                           hsoft=2.0 / 25.0 / cfg["n_side"], eta=0.2 / math.sqrt(2.0), GM=1.0,
                           rcut_over_rs=cfg["rcut_over_rs"])


def workload_desc(name, cfg, opts):
    return {
        "workload": f"{name}: {cfg['n_side']}^3 {cfg['kind']} particles, {cfg['grid']}^3 mesh {cfg['assign'].upper()}, "
                    f"r_s={cfg['rs_cells']} cells, cutoff={cfg['rcut_over_rs']} r_s, chain mesh {opts.chain_dim}^3",
        "particles": cfg["n_side"] ** 3, "grid": cfg["grid"], "assign": cfg["assign"], "rs_cells": cfg["rs_cells"],
        "rcut_over_rs": cfg["rcut_over_rs"], "chain_dim": opts.chain_dim, "sort": "parity",
        "precision": "fp32 pair terms, Kahan-compensated per-target sums",
        "l2": ("inputs larger than L2 (particles + mesh > 126 MB)"
               if 25 * cfg["n_side"] ** 3 + 12 * cfg["grid"] ** 3 > 126e6 else
               "inputs smaller than L2; no flush (secondary, launch-bound entry)"),
    }


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# -------------------------------------------------------------- GPU arm
def gpu_arm(args, cfg, name, rank, world, dist):
    import torch
    from tigerpm_b200 import _lib
    from tigerpm_b200.api import TigerPM, fp32_peak_probe

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    ps = make_particles(cfg, args.seed + rank)
    n = ps.n
    opts = make_opts(cfg)
    ctx = TigerPM(opts, n)
    ext = torch.cuda.ExternalStream(ctx.stream(), device=dev)
    # resident inputs (pristine copy in HBM) and pinned host buffers for e2e
    dev_in = [torch.from_numpy(a).to(dev) for a in ps.arrays()]
    pinned_in = [torch.from_numpy(a).pin_memory() for a in ps.arrays()]
    pinned_out = [torch.empty_like(t).pin_memory() for t in pinned_in]
    ptr_in = [t.data_ptr() for t in dev_in]
    lib = _lib.load()
    import ctypes as C

    def step_resident():
        ctx.set_particles_device(n, ptr_in)
        ctx.pme_step(0, 1.0, 1.0, True)

    h_in = [C.c_void_p(t.data_ptr()) for t in pinned_in]
    h_out = [C.c_void_p(t.data_ptr()) for t in pinned_out]

    def step_e2e():
        _lib.check(lib.tpm_set_particles(ctx.h, n, *h_in), "set_particles")
        ctx.pme_step(0, 1.0, 1.0, True)
        _lib.check(lib.tpm_get_particles(ctx.h, *h_out), "get_particles")

    def barrier():
        torch.cuda.synchronize(dev)
        if dist is not None:
            dist.barrier()

    def timed(fn, steps):
        barrier()
        ctx.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(ext)
        for _ in range(steps):
            fn()
        e1.record(ext)
        e1.synchronize()
        return max_over_ranks(e0.elapsed_time(e1), dist, dev)

    for _ in range(args.warmup):
        step_resident()
    ctx.check_errors()
    ctx.reset_stage_times()
    l0 = ctx.launch_count()
    with ClockSampler(dev.index) as clk:
        ms = timed(step_resident, args.steps)
    launches = (ctx.launch_count() - l0) // args.steps * args.steps
    ctx.check_errors()
    stages = ctx.stage_times()
    for _ in range(max(1, args.warmup // 2)):
        step_e2e()
    ms_serial = timed(step_e2e, args.steps)

    # e2e headline: the served stream (tpm_pme_steps_host) -- every step
    # uploads its particles from pinned host memory and downloads the kicked
    # particles, overlapped with the neighbouring steps' kernels; host clock
    # around the call, which returns after the last download
    from tigerpm_b200 import workloads as W
    host_in = W.ParticleSet(*(t.numpy() for t in pinned_in))
    host_out = W.ParticleSet(*(t.numpy() for t in pinned_out))
    ctx.pme_steps_host([host_in] * 2, [host_out] * 2)
    barrier()
    t_host = time.perf_counter()
    ctx.pme_steps_host([host_in] * args.steps, [host_out] * args.steps)
    ms_e2e = max_over_ranks((time.perf_counter() - t_host) * 1e3, dist, dev)

    total = n * world * args.steps
    out = {
        "value": replica_rate(n, world, args.steps, ms), "ms_per_step": ms / args.steps,
        "e2e": {"value": replica_rate(n, world, args.steps, ms_e2e), "unit": "particle-kicks/s",
                "h2d_bytes_per_step": int(sum(t.numel() * t.element_size() for t in pinned_in)),
                "d2h_bytes_per_step": int(sum(t.numel() * t.element_size() for t in pinned_out)),
                "ms_per_step": ms_e2e / args.steps, "api": "tpm_pme_steps_host (served stream)",
                "serial": {"value": total / (ms_serial * 1e-3), "ms_per_step": ms_serial / args.steps,
                           "api": "tpm_set_particles + tpm_pme_step + tpm_get_particles"}},
        "stages_ms": {k: round(v, 4) for k, v in stages.items() if v > 0},
        "stages_hbm": stage_hbm(cfg["grid"], n, stages),
        "gpu_launches": int(launches), "clocks": clk.summary(),
    }
    # roofline of the dominant kernel (PP: FP32-bound)
    cand, inside = ctx.count_pairs(0)
    flops = FLOPS_PER_PAIR * inside + FLOPS_PER_CULLED * (cand - inside)
    kick_ms = stages["kick_ms"]
    # the FP32 peak: the FMA-chain probe repeated for ~1 s with the SM clock
    # sampled meanwhile (the median probe value, and the clock it ran at)
    probes = []
    with ClockSampler(dev.index) as pclk:
        t_probe = time.perf_counter()
        while len(probes) < 3 or time.perf_counter() - t_probe < 1.0:
            probes.append(fp32_peak_probe())
    peak = statistics.median(probes)
    achieved = flops / (kick_ms * 1e-3) / 1e12
    out["roofline"] = {"bound": "fp32", "kernel": "k_kick_pme", "achieved": round(achieved, 3),
                       "peak": round(peak, 2), "unit": "TFLOP/s", "frac": round(achieved / peak, 4),
                       "traffic": read_traffic(name),
                       "peak_source": "measured FP32 FMA probe on this GPU (tpm_fp32_peak_probe, median of "
                                      f"{len(probes)})",
                       "peak_clocks": pclk.summary(),
                       # the same kernel credited with the in-cutoff pairs' flops only
                       "frac_in_cutoff_only": round(FLOPS_PER_PAIR * inside / (kick_ms * 1e-3) / 1e12 / peak, 4),
                       "pairs_in_cutoff": inside, "pairs_candidate": cand,
                       "flops_per_launch": flops, "kick_ms": round(kick_ms, 4)}
    # accuracy of this kick vs the FP64 Ewald sum
    if args.ewald_samples:
        step_resident()
        ctx.check_errors()
        err = ctx.gravity_short_ewald_compare(min(args.ewald_samples, cfg["ewald_samples"]), seed=args.seed + 7)
        out["accuracy"] = {k: (float(f"{v:.4e}") if isinstance(v, float) else v) for k, v in err.items()}
    ctx.close()
    return out


def ensemble_opts(sides):
    from tigerpm_b200 import workloads as W
    from tigerpm_b200.api import make_options
    out = []
    for n in sides:
        p = W.accurate_box_params(int(n))
        out.append(make_options(p["n_side"], p["grid"], rs_cells=p["rs_cells"], rcut_over_rs=p["rcut_over_rs"],
                                assign=p["assign"]))
    return out


def ensemble_accuracy(boxes, sets, samples_per_box, seed):
    """Vector rms force error over a few boxes of an ensemble, each against
    its own FP64 Ewald sum, pooled as one sum of squares."""
    from tigerpm_b200 import workloads as W
    num = den = 0.0
    count = 0
    for j, t in boxes:
        idx = W.sample_indices(sets[j].n, samples_per_box, seed + j)
        gx, gy, gz, _ = t.get_forces()
        _, g = t.ewald_samples(idx, 1)
        gk = np.stack([gx[idx], gy[idx], gz[idx]], axis=1).astype(np.float64)
        num += float(np.sum((gk - g) ** 2))
        den += float(np.sum(g * g))
        count += idx.size
    return {"force_rms_vector": float(f"{math.sqrt(num / den):.4e}"), "samples": count, "boxes": len(boxes)}


def batch_arm(args, rank, world, dist, n_boxes=64, lo=32, hi=128):
    """Config 4: n_boxes independent Zel'dovich boxes, sides log-uniform in
    [lo, hi], each on its own mesh; one batch step (graph replay: every box's
    sort + long-range solve concurrently, one interpolation launch, one
    persistent PP + kick launch, kick shape autotuned) against the same boxes
    through the plain single-box path one after another."""
    import torch
    from tigerpm_b200 import workloads as W
    from tigerpm_b200.api import Batch
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    sides, sets = W.ensemble(n_boxes, lo, hi, seed=args.seed + 40 + rank)
    opts = ensemble_opts(sides)
    total = int(sum(s.n for s in sets))
    b = Batch(opts, [s.n for s in sets])
    for i, ps in enumerate(sets):
        b.set_input(i, ps)
    ext = torch.cuda.ExternalStream(b.stream(), device=dev)

    def timed(fn, steps):
        torch.cuda.synchronize(dev)
        if dist is not None:
            dist.barrier()
        b.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(ext)
        for _ in range(steps):
            fn()
        e1.record(ext)
        e1.synchronize()
        return max_over_ranks(e0.elapsed_time(e1), dist, dev)

    b.step(restore=True, graph=False)
    b.synchronize()
    shape = b.autotune(repeats=2)
    for _ in range(args.warmup):
        b.step(restore=True, graph=True)
    l0 = b.launch_count()
    ms = timed(lambda: b.step(restore=True, graph=True), args.steps)
    launches = (b.launch_count() - l0) // args.steps
    phases = b.phase_times()
    for _ in range(max(1, args.warmup // 2)):
        b.steps_sequential(restore=True)
    ms_seq = timed(lambda: b.steps_sequential(restore=True), args.steps)
    b.step(restore=True, graph=True)
    b.synchronize()
    acc = None
    if args.ewald_samples:
        picks = sorted(set([0, n_boxes // 3, 2 * n_boxes // 3, n_boxes - 1]))
        acc = ensemble_accuracy([(j, b.box(j)) for j in picks], sets, 256, args.seed + 11)
    b.close()
    v = total * world * args.steps / (ms * 1e-3)
    v_seq = total * world * args.steps / (ms_seq * 1e-3)
    return {"config": f"{n_boxes} Zel'dovich boxes, sides log-uniform in [{lo}, {hi}] (seeded), "
                      f"each on its own cloud4 mesh >= 3 points per particle spacing, r_s = 2/3 spacing, "
                      f"cutoff 6 r_s; {total} particles in all",
            "sides": [int(s) for s in sides], "meshes": [int(o.four_dim) for o in opts], "particles": total,
            "value": v, "ms_per_step": ms / args.steps, "gpu_launches_per_step": int(launches),
            "api": "tpm_batch_step (restore + CUDA graph replay)", "phases_ms": {k: round(x, 4) for k, x in phases.items()},
            "kick_shape": shape,
            "sequential": {"value": v_seq, "ms_per_step": ms_seq / args.steps,
                           "api": "tpm_batch_steps_sequential (plain single-box path, box after box)"},
            "speedup_vs_sequential": round(ms_seq / ms, 3), "accuracy": acc}


def serve_arm(args, rank, world, dist, pool=256, lo=32, hi=192, rate=200.0, seconds=12.0, slots=32):
    """Config 5: a resident pool of `pool` Zel'dovich boxes (sides
    log-uniform in [lo, hi], generated on the device, each on its own mesh),
    kick + drift requests arriving as a Poisson process at `rate` per second
    for `seconds`, admitted by the HBM budget into up to `slots` concurrent
    steps.  Latency = submission to completion (host clock).  The offered
    load (~2.7e8 particle-kicks/s) is close to what the slots sustain: with
    8 slots a 12 s replay could fall behind it (p50 1 s), with 16 or 32 it
    keeps up (p50 13 ms)."""
    from tigerpm_b200 import workloads as W
    from tigerpm_b200.api import Server, TigerPM, ic_zeldovich
    g = W.rng(args.seed + 90 + rank)
    sides = W.log_uniform_sides(pool, lo, hi, args.seed + 70 + rank)
    opts = ensemble_opts(sides)
    t_gen = time.perf_counter()
    srv = Server(budget_bytes=0, max_slots=slots)
    ids = [srv.add_box_ic(o, int(n), seed=args.seed * 1000 + 7 * i + 3) for i, (o, n) in enumerate(zip(opts, sides))]
    t_gen = time.perf_counter() - t_gen
    dt = 1e-4
    # warm-up: every slot and the working-set pool see a few steps
    warm = [srv.submit(ids[int(j)], dt) for j in g.integers(0, pool, 4 * slots)]
    for r in warm:
        srv.wait(r)
    nreq = int(rate * seconds)
    arrivals = np.cumsum(g.exponential(1.0 / rate, nreq))
    which = g.integers(0, pool, nreq)
    if dist is not None:
        dist.barrier()
    t0 = time.perf_counter()
    res = srv.replay([ids[int(j)] for j in which], arrivals, dt)
    wall = time.perf_counter() - t0
    st = srv.stats()
    lat = np.array([r["latency_ms"] for r in res])
    qms = np.array([r["queue_ms"] for r in res])
    dev = np.array([r["device_ms"] for r in res])
    parts = float(sum(r["particles"] for r in res))
    srv.close()
    # accuracy of the served step form: the same step (sort + PME + kick) on
    # two pool boxes through a context, against FP64 Ewald
    acc = None
    if args.ewald_samples:
        num = den = 0.0
        cnt = 0
        for j in (int(np.argmin(np.abs(sides - np.median(sides)))), int(np.argmax(sides))):
            n = int(sides[j])
            with TigerPM(opts[j], n ** 3) as t:
                ic_zeldovich(t, n, args.seed * 1000 + 7 * j + 3, rms_disp=0.3)
                t.pme_step(0, 1.0, 1.0, True)
                idx = W.sample_indices(n ** 3, 512, args.seed + j)
                gx, gy, gz, _ = t.get_forces()
                _, gref = t.ewald_samples(idx, 1)
                gk = np.stack([gx[idx], gy[idx], gz[idx]], 1).astype(np.float64)
                num += float(np.sum((gk - gref) ** 2))
                den += float(np.sum(gref * gref))
                cnt += idx.size
        acc = {"force_rms_vector": float(f"{math.sqrt(num / den):.4e}"), "samples": cnt, "boxes": 2}
    return {"config": f"{pool} resident Zel'dovich boxes, sides log-uniform in [{lo}, {hi}] (seeded, generated on "
                      f"the device), each on its own cloud4 mesh >= 3 points per spacing; kick + drift requests, "
                      f"Poisson arrivals at {rate:g}/s for {seconds:g} s; up to {slots} steps in flight",
            "requests": nreq, "particles_pool": int(sum(int(n) ** 3 for n in sides)),
            "value": parts / wall, "unit": "particle-kicks/s",
            "latency_ms": {"p50": round(float(np.percentile(lat, 50)), 3), "p99": round(float(np.percentile(lat, 99)), 3),
                           "mean": round(float(lat.mean()), 3), "max": round(float(lat.max()), 3)},
            "queue_ms": {"p50": round(float(np.percentile(qms, 50)), 3), "p99": round(float(np.percentile(qms, 99)), 3)},
            "device_ms": {"p50": round(float(np.percentile(dev, 50)), 3), "p99": round(float(np.percentile(dev, 99)), 3)},
            "wall_s": round(wall, 3), "offered_s": round(float(arrivals[-1]), 3),
            "device_busy_frac_sum": round(float(dev.sum() / 1e3 / wall), 3),
            "stats": st, "generation_s": round(t_gen, 2), "accuracy": acc,
            "api": "tpm_serve_replay (submit at arrival, dispatcher admits by HBM budget)"}


def clustered_arm(args, rank, world, dist, n_side=256, steps=2):
    """Config 3 form: 70 % of the particles in 2,000 NFW halos (masses
    log-uniform over 3 decades, c in [5, 15]), 30 % uniform; the accurate
    mesh form (cloud4, mesh 3x the lattice, r_s = 2 cells, cutoff 6 r_s).
    The step with the default persistent (cell, sink pass) queue and with the
    per-cell launch, and the error against FP64 Ewald."""
    import torch
    from tigerpm_b200 import workloads as W
    from tigerpm_b200.api import TigerPM
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    t_gen = time.perf_counter()
    ps = W.nfw_halos(n_side, args.seed + 30 + rank, n_halo=2000, halo_frac=0.7)
    t_gen = time.perf_counter() - t_gen
    opts = ensemble_opts([n_side])[0]
    out = {"config": f"{n_side}^3 particles, 70% in 2000 NFW halos (c 5-15, masses log-uniform over 3 decades), "
                     f"30% uniform; {opts.four_dim}^3 cloud4 mesh, r_s = 2 cells, cutoff 6 r_s, chain mesh "
                     f"{opts.chain_dim}^3", "particles": ps.n, "generation_s": round(t_gen, 1)}
    for mode in (0, 1):
        opts.kick_grid = mode
        with TigerPM(opts, ps.n) as t:
            ext = torch.cuda.ExternalStream(t.stream(), device=dev)
            t.set_particles(ps)
            t.pme_step(0, 1.0, 1.0, True)
            t.synchronize()
            if mode == 0:
                offs = t.chainmesh_offsets()
                cnt = np.diff(offs)
                out["occupancy"] = {"max": int(cnt.max()), "mean": float(cnt.mean()),
                                    "max_over_mean": round(float(cnt.max() / cnt.mean()), 1)}
            t.reset_stage_times()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(ext)
            for _ in range(steps):
                t.set_particles(ps)
                t.pme_step(0, 1.0, 1.0, True)
            e1.record(ext)
            e1.synchronize()
            ms = max_over_ranks(e0.elapsed_time(e1), dist, dev) / steps
            st = t.stage_times()
            key = "queue" if mode == 0 else "per_cell_launch"
            out[key] = {"ms_per_step": round(ms, 3), "value": ps.n * world / (ms * 1e-3),
                        "kick_ms": round(st["kick_ms"], 3), "interp_ms": round(st["interp_ms"], 3),
                        "sort_ms": round(st["sort_ms"], 3)}
            if mode == 0:
                cand, inside = t.count_pairs(0)
                out["pairs_in_cutoff"] = inside
                out["pairs_candidate"] = cand
                if args.ewald_samples:
                    t.check_errors()
                    err = t.gravity_short_ewald_compare(1024, seed=args.seed + 9)
                    out["accuracy"] = {k: (float(f"{v:.4e}") if isinstance(v, float) else v) for k, v in err.items()}
    out["value"] = out["queue"]["value"]
    out["speedup_queue_vs_per_cell"] = round(out["per_cell_launch"]["ms_per_step"] / out["queue"]["ms_per_step"], 3)
    return out


def read_traffic(name):
    """DRAM bytes per kick launch from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", f"kick_pme_{name}.md")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.strip().startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1])
            except ValueError:
                return None
    return None


# ---------------------------------------------------------- CPU (oracle) arm
def cpu_full_kick(cfg, opts, ps, threads):
    """Seconds for one whole kick of the workload on the host cores with the
    oracle (the CPU restatement of the reference path): chain-mesh sort,
    deposit + FFT + Green + inverse FFT, and interpolation + PP + rung kick of
    every particle, each timed as it runs (nothing extrapolated)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    p = O.Particles(*(np.array(a, copy=True) for a in ps.arrays()))
    C_, N = opts.chain_dim, opts.four_dim
    t = time.perf_counter()
    pb, pe = O.chainmesh_sort(C_, p, nthreads=threads)
    t_sort = time.perf_counter() - t
    t = time.perf_counter()
    phi = O.gravity_long(N, cfg["rs_cells"], {"cloud4": 0, "cic": 1, "tsc": 2}[cfg["assign"]], p.x, p.y, p.z,
                         nthreads=threads)
    t_long = time.perf_counter() - t
    kp = O.KickParams(N=N, C=C_, rs=opts.rs, GM=opts.GM, eta=opts.eta, hsoft=opts.hsoft,
                      rcut=opts.rcut_over_rs * opts.rs, min_rung=0, scale=1.0, t0=1.0, first_call=1, precision=0)
    phi32 = phi.astype(np.float32)
    t = time.perf_counter()
    _, _, _, _, cnt, _ = O.kick_pme(kp, p, pb, pe, phi32, nthreads=threads)
    t_kick = time.perf_counter() - t
    total = t_sort + t_long + t_kick
    return total, {"sort_s": round(t_sort, 3), "long_range_s": round(t_long, 3), "kick_s": round(t_kick, 3),
                   "pairs_candidate": int(cnt[0]), "pairs_in_cutoff": int(cnt[1])}


def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


# --------------------------------------------------------------------- main
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c2-accurate", choices=sorted(CONFIGS))
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--ewald-samples", type=int, default=4096)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-named", action="store_true", help="skip the literal c2 secondary measurement")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-ensemble secondary measurement")
    ap.add_argument("--no-serve", action="store_true", help="skip the served-stream secondary measurement")
    ap.add_argument("--no-clustered", action="store_true", help="skip the NFW-halo secondary measurement")
    ap.add_argument("--clustered-side", type=int, default=256,
                    help="particles per side of the NFW-halo box (512 = the full configuration)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    cfg = CONFIGS[args.config]

    if args.impl == "reference":
        if rank != 0:
            return
        opts = host_opts(cfg)
        ps = make_particles(cfg, args.seed)
        th = cpu_threads()
        # Whole kicks, each timed in full.  A CPU kick of the headline box
        # takes tens of seconds, so at most one warm-up kick runs and the
        # timed kicks stop once ~REF_BUDGET_S is spent; `steps` is the number
        # actually timed (steps_requested keeps what was asked).
        for _ in range(min(args.warmup, 1)):
            cpu_full_kick(cfg, opts, ps, th)
        times, parts = [], None
        t_all = time.perf_counter()
        while len(times) < args.steps:
            tt, parts = cpu_full_kick(cfg, opts, ps, th)
            times.append(tt)
            if time.perf_counter() - t_all + tt > REF_BUDGET_S:
                break
        sec = statistics.mean(times)
        v = ps.n / sec
        sample = f"{len(times)} whole kicks of all {ps.n} particles, each timed in full"
        line = {"metric": METRIC, "value": v, "unit": "particle-kicks/s", "impl": "reference",
                "n_gpus": args.gpus, "steps": len(times), "steps_requested": args.steps,
                "warmup": min(args.warmup, 1), "ms_per_step": sec * 1e3,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic", "config": workload_desc(args.config, cfg, opts),
                "cpu_baseline": {"value": v, "unit": "particle-kicks/s", "cores": th, "kind": "port",
                                 "sample": sample, "stages_s": parts},
                "e2e": {"value": v, "unit": "particle-kicks/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    dist = None
    if world > 1:
        import torch.distributed as dist_mod
        import datetime
        dist_mod.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = dist_mod
    res = gpu_arm(args, cfg, args.config, rank, world, dist)
    batch = None
    if args.config == "c2-accurate" and not args.no_batch:
        batch = batch_arm(args, rank, world, dist)
    serve = None
    if args.config == "c2-accurate" and not args.no_serve:
        serve = serve_arm(args, rank, world, dist)
    clustered = None
    if args.config == "c2-accurate" and not args.no_clustered:
        clustered = clustered_arm(args, rank, world, dist, n_side=args.clustered_side)
    named = {}
    if args.config == "c2-accurate" and not args.no_named:
        # the configurations' literal forms, measured in the same run: the
        # 256^3 Zel'dovich box on its own 256^3 TSC mesh, and the 64^3 box
        for nm in ("c2", "c1"):
            named[nm] = gpu_arm(args, CONFIGS[nm], nm, rank, world, dist)
    if rank == 0:
        opts = make_opts(cfg)
        line = {"metric": METRIC, "value": res["value"], "unit": "particle-kicks/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["ms_per_step"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded Philox; Zel'dovich / uniform as configured)",
                "config": dict(workload_desc(args.config, cfg, opts), parallelism=f"replicas x{world}"),
                "e2e": res["e2e"], "roofline": res["roofline"], "gpu_launches": res["gpu_launches"],
                "clocks": res["clocks"], "stages_ms": res["stages_ms"], "stages_hbm": res["stages_hbm"],
                "accuracy": res.get("accuracy")}
        if batch is not None:
            batch["vs_plain_single_box"] = round(batch["value"] / res["value"], 4)
            line["batch"] = batch
        if serve is not None:
            line["serve"] = serve
        if clustered is not None:
            line["named_config_c3"] = clustered
        for nm, r in named.items():
            entry = {"config": workload_desc(nm, CONFIGS[nm], make_opts(CONFIGS[nm])),
                     "value": r["value"], "ms_per_step": r["ms_per_step"], "e2e": r["e2e"]["value"],
                     "accuracy": r.get("accuracy"), "stages_ms": r["stages_ms"],
                     "roofline_frac": r["roofline"]["frac"]}
            line["named_config" if nm == "c2" else f"named_config_{nm}"] = entry
        if world == 1 and not args.no_cpu_baseline:
            ps = make_particles(cfg, args.seed)
            th = cpu_threads()
            sec, parts = cpu_full_kick(cfg, opts, ps, th)
            line["cpu_baseline"] = {"value": ps.n / sec, "unit": "particle-kicks/s", "cores": th, "kind": "port",
                                    "sample": f"one whole kick of all {ps.n} particles, timed in full",
                                    "stages_s": parts}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
