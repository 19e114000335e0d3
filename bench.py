#!/usr/bin/env python
"""Benchmark of the fused uniform-grid hydro step: zone-updates/s and the HBM roofline fraction.

Workload: the 3D Taylor-Green vortex at 512^3 (periodic [0, 2 pi]^3, rho = 1, p0 = 100,
gamma = 5/3), PPM + HLLC, float32 state, CFL 0.4 — the configuration the headline metric
(512^3 HLLC FP32) is quoted on. Synthetic data: the analytic initial condition, generated on the
host in float64 and rounded once to float32.

  value   zone-updates/s of `--steps` steps with the state resident in HBM, timed with CUDA events
          on the library's stream. With N > 1 ranks (torchrun), weak scaling: one periodic grid of
          512 x 512 x 512N cells split into z-slabs of 512^3, one per GPU, with NCCL halo exchange
          and a max all-reduce of the rate before every step (shaderous_b200.dist); the time is the
          slowest rank's.
  e2e     the same metric through the C ABI with host buffers: upload of the state from pinned
          host memory, the configuration's full run of 200 steps with the clock read back between
          batches (shz_run), download of the final state.
  roofline  the sweep kernel: 64 algorithmic bytes per zone-update (read the float32 state once,
          write it once) / its mean CUDA-event duration, against the measured HBM copy bandwidth.
  cpu_baseline  the float64 oracle (a C++ port of the reference's CPU scheme) on a bounded sample
          of the same workload, on the host's cores.

`--impl reference` times that CPU oracle alone (the reference's own CPU path is TypeScript and has
no runtime here) and prints its line with "impl": "reference".
"""
from __future__ import annotations

import argparse
import json
import math
import os
import re
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "zone-updates/s (512^3 HLLC FP32)"
UNIT = "zone-updates/s"
BYTES_PER_ZU = 64  # read u1, u2 (32 B) + write u1', u2' (32 B) per cell per step
L2_BYTES = 126 * 2**20


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=512, help="cells per side")
    ap.add_argument("--recon", default="ppm")
    ap.add_argument("--e2e-steps", type=int, default=200)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-amr", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--no-comparable", action="store_true",
                    help="skip the configurations the reference publishes throughputs for")
    ap.add_argument("--serve-requests", type=int, default=100)
    ap.add_argument("--serve-sizes", choices=["config", "small"], default="config",
                    help="the serving stream's size and step distributions")
    ap.add_argument("--section", choices=["all", "amr", "serving", "comparable"], default="all",
                    help="amr / serving: only that measurement, printed as its own JSON line")
    ap.add_argument("--amr-variant", choices=["both", "spec", "developed", "bins", "spread"], default="both",
                    help="spread: a mesh of the developed run's size at once, for profiling")
    ap.add_argument("--amr-cap", type=int, default=26000, help="block slots of the AMR runs")
    ap.add_argument("--amr-levels", type=int, default=4,
                    help="levels above the roots of the spread mesh (3: a quarter of the leaves, for full captures)")
    ap.add_argument("--profile-window", action="store_true",
                    help="AMR section: bracket one step after the warm-up with cudaProfilerStart/Stop")
    ap.add_argument("--pin-assemble", type=int, default=None, metavar="V",
                    help="AMR section: fix the assemble's launch shape to variant V (0-2 one pass, 3-4 split, "
                         "5-6 split side by side) instead of the tuned one, e.g. to profile one form")
    ap.add_argument("--slabs", action="store_true",
                    help="the z-slab driver also at N = 1 (one periodic slab exchanging with itself)")
    return ap.parse_args()


def _amr_cfg(levels, nr, cap, time_bins=0, two_pass=False):
    from shaderous_b200 import Config
    from shaderous_b200.amr import AmrConfig

    hyd = Config(gamma=5 / 3, bc_lo=(1, 1, 1), bc_hi=(1, 1, 1), recon="koren", isentropic=True, cfl=0.5, p_floor=1e-12)
    return AmrConfig(hydro=hyd, ndim=3, nr=nr, max_level=levels, cap=cap, refine_hi=0.1, refine_lo=0.05,
                     regrid_every=8, two_pass=two_pass, time_bins=time_bins, time_bins_always=time_bins > 0)


def _time_amr(a, steps, time_bins=0, profile_window=False):
    """Warm-up (one refinement check; with bins the run's first single steps), then `steps` steps
    timed by CUDA events on the handle's stream. Zone-updates are leaf cells x steps, the leaves
    counted at the start and end of the timed run; with per-block timesteps a step is a substep
    of the cycles (the fastest block's step), so the same figure counts the single-step work the
    cycles stand for."""
    a.profile(8 if not time_bins else 16 + (1 << time_bins))
    if profile_window:
        # one graph-replayed step between cudaProfilerStart/Stop, for `ncu --profile-from-start off`
        import torch

        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        a.step(1)
        a.diagnostics()
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
    n0 = len(a.leaves()[0])
    l0 = a.kernel_launches
    prof = a.profile(steps)
    steps = prof["steps"]
    _, lv, _ = a.leaves()
    n1 = len(lv)
    work = a.bin_work() if time_bins else None
    leaf_cells = 0.5 * (n0 + n1) * 4096
    extra = {"time_bins": time_bins, "block_update_share": work["updates"] / max(work["single"], 1)} if work else {}
    return {"value": leaf_cells * steps / (prof["total_ms"] / 1000.0), "unit": UNIT, "steps": steps, **extra,
            "ms_per_step": prof["total_ms"] / steps, "leaf_blocks": [n0, n1], "levels": int(lv.max()) + 1,
            "gpu_launches": a.kernel_launches - l0,
            "note": "time includes the refinement checks (flag, host adapt, regrid) every 8 steps"}


def amr_sedov(levels=4, nr=8, radius_cells=3.5, steps=24, cap=26000, profile_window=False, time_bins=0,
              two_pass=False):
    """3D Sedov blast on the block grid as configured: 16^3-cell blocks, levels 0-levels above nr^3
    roots (finest nr * 16 << levels cells per side), E = 1 spread over the finest cells within
    radius_cells of the centre, Löhner refinement above 0.1 (below 0.05 merges), a refinement
    check every 8 steps; timed on its initial mesh."""
    from shaderous_b200 import Problem
    from shaderous_b200.amr import AmrSim

    t0 = time.perf_counter()
    with AmrSim(_amr_cfg(levels, nr, cap, time_bins, two_pass)) as a:
        a.reset(Problem("sedov", a=(1.0, 1e-5, 1.0, radius_cells)))
        t_init = time.perf_counter() - t0
        out = _time_amr(a, steps, time_bins, profile_window)
    out.update({"finest_cells_per_side": nr * 16 << levels, "radius_finest_cells": radius_cells, "init_s": t_init})
    return out


def amr_sedov_spread(levels=4, nr=8, steps=16, cap=30000, profile_window=False):
    """A profiling mesh of the developed run's size at once: the same energy (E = 1, gamma = 5/3)
    as a uniform hot sphere of radius 0.16 of the box, whose refined shell holds 22,520 leaves
    (25,664 blocks) from the start; the configured run reaches 20k only after some 34,000 steps."""
    from shaderous_b200 import Problem
    from shaderous_b200.amr import AmrSim

    r = 0.16
    with AmrSim(_amr_cfg(levels, nr, cap)) as a:
        a.reset(Problem("blast", a=(1.0, (2.0 / 3.0) / (4.0 / 3.0 * math.pi * r ** 3), 1.0, 1e-5, r)))
        out = _time_amr(a, steps, 0, profile_window)
    out["note"] += "; a profiling mesh: the blast's energy spread within 0.16 of the box"
    return out


def amr_sedov_developed(levels=4, nr=8, radius_cells=3.5, steps=16, bins_steps=64, cap=26000, target_leaves=20000,
                        advance_s=330.0, profile_window=False, bins=True):
    """The same configured Sedov run advanced (untimed) until its mesh holds about `target_leaves`
    leaves (the blast's shell, refined to the finest level, grows with its radius; about 34,000
    steps), then timed with one timestep for every block and, restarted on the same mesh, state
    and clock (shz_amr_reset_mesh), with per-block timesteps (5 bins)."""
    import numpy as np

    from shaderous_b200 import Problem
    from shaderous_b200.amr import AmrSim

    out = {}
    with AmrSim(_amr_cfg(levels, nr, cap)) as a:
        a.reset(Problem("sedov", a=(1.0, 1e-5, 1.0, radius_cells)))
        t1 = time.perf_counter()
        taken = 0
        while len(a.leaves()[0]) < target_leaves and time.perf_counter() - t1 < advance_s:
            taken += a.run(steps=256).taken
        t_sim, _, st = a.clock()
        advanced = {"steps": taken, "t": t_sim, "leaves": int(len(a.leaves()[0])), "target_leaves": target_leaves,
                    "seconds": time.perf_counter() - t1}
        slots, levels_l, coords = a.leaves()
        u1, u2 = a.leaves_state()
        t_sim, _, st = a.clock()
        out["developed"] = _time_amr(a, steps, 0, profile_window)
        out["developed"]["advanced_before_timing"] = advanced
    if bins:
        with AmrSim(_amr_cfg(levels, nr, cap, time_bins=5)) as b:
            n = nr * 16
            b.reset_mesh(levels_l, coords, (n, n, n), (16, 16, 16), (-0.5,) * 3, (0.5,) * 3, 0)
            _, lv2, co2 = b.leaves()
            where = {(int(l), *map(int, c)): i for i, (l, c) in enumerate(zip(levels_l, coords))}
            order = np.array([where[(int(l), *map(int, c))] for l, c in zip(lv2, co2)])
            b.set_leaves_state(u1[order], u2[order])
            b.set_clock(t_sim, st)
            out["developed_time_bins"] = _time_amr(b, bins_steps, 5)
            out["developed_time_bins"]["advanced_before_timing"] = dict(advanced, restarted=True)
    return out


# The reference's published throughputs (WebGPU in Chrome, zone-updates/s) for the same
# configurations, for context: other hardware and another implementation.
PUBLISHED = {
    "kh_2d_1024": {"H200 NVL": 2.339e9, "RTX 3080": 1.633e9},
    "kh_2d_2048": {"H200 NVL": 2.743e9, "H100": 2.602e9, "A100": 1.736e9, "RTX 3080": 1.849e9},
    "sedov_3d_256": {"H200 NVL": 1.670e9, "H100": 1.571e9, "A100": 1.196e9, "RTX 3080": 1.386e9},
}


def comparable(steps=40):
    """The configurations the reference publishes throughputs for, with its default scheme
    (koren + isentropic density + HLLC, CFL 0.8 unless stated): 2D Kelvin-Helmholtz at 1024^2 and
    2048^2 and the 3D Sedov blast on a uniform 256^3 grid. Device time of `steps` steps after a
    warm-up, CUDA events on the library's stream."""
    from shaderous_b200 import Config, Problem, Sim

    out = {}
    cases = [
        ("kh_2d_1024", Config(n=(1024, 1024, 1), gamma=1.4, recon="koren"), Problem("kh", a=(2, 1, 0.5, 2.5, 0.01, 1e-3), seed=1)),
        ("kh_2d_2048", Config(n=(2048, 2048, 1), gamma=1.4, recon="koren"), Problem("kh", a=(2, 1, 0.5, 2.5, 0.01, 1e-3), seed=1)),
        ("sedov_3d_256", Config(n=(256, 256, 256), gamma=5 / 3, recon="koren", bc_lo=(1, 1, 1), bc_hi=(1, 1, 1),
                                p_floor=1e-12), Problem("sedov", a=(1.0, 1e-5, 1.0, 3.5))),
    ]
    for name, cfg, prob in cases:
        with Sim(cfg) as s:
            s.reset(prob)
            s.profile(5)  # warm-up (tunes)
            prof = s.profile(steps)
        v = cfg.ncell * steps / (prof["total_ms"] / 1000.0)
        out[name] = {"value": v, "unit": UNIT, "ms_per_step": prof["total_ms"] / steps, "steps": steps,
                     "scheme": "koren+isentropic+hllc, cfl 0.8", "published_reference": PUBLISHED[name]}
    # the second configuration as stated: Kelvin-Helmholtz 1024^2, MC + HLLC, CFL 0.4, its 1000
    # steps timed whole (the run the parity tests hold to the oracle)
    cfg = Config(n=(1024, 1024, 1), dx=1.0 / 1024, gamma=1.4, cfl=0.4, recon="mc", riemann="hllc", isentropic=False)
    prob = Problem("kh", a=(2, 1, 0.5, 2.5, 0.01, 1e-3), seed=20240601)
    with Sim(cfg) as s:
        s.reset(prob)
        s.profile(5)  # warm-up (tunes)
        s.reset(prob)
        prof = s.profile(1000)
    out["kh_2d_1024_1000"] = {"value": cfg.ncell * 1000 / (prof["total_ms"] / 1000.0), "unit": UNIT,
                              "ms_per_step": prof["total_ms"] / 1000, "steps": 1000,
                              "scheme": "mc+hllc, cfl 0.4 (the configuration as stated)"}
    return out


SERVE_SIZES = {
    # the configuration's stream: 64^2-1024^2 (2D) and 32^3-256^3 (3D), 100-2000 steps
    "config": {"sizes2": (64, 1024), "sizes3": (32, 256), "steps": (100, 2000)},
    # a reduced stream of small grids, where the plain loop is launch-bound
    "small": {"sizes2": (64, 512), "sizes3": (32, 128), "steps": (100, 500)},
}


def serving(n_requests=100, seed=2024, budget=150e9, sizes="config"):
    """A seeded stream of Sod / Kelvin-Helmholtz / blast requests with Poisson arrivals, served with
    continuous batching, and the same stream run one request after another through the plain
    uniform-grid step. Each arm's GPU-busy share (CUDA-event spans over the makespan) says how
    much of its time the device was working."""
    from dataclasses import replace

    from shaderous_b200.serve import Server, ServerConfig, plain_run_stream, request_stream

    sz = SERVE_SIZES[sizes]
    reqs = request_stream(n_requests, seed=seed, rate=100.0, **sz)
    cfg = ServerConfig(budget_bytes=budget, max_grids=512, round_steps=8)
    try:
        srv = Server(cfg)
    except Exception:
        cfg.budget_bytes = budget / 3
        srv = Server(cfg)
    # warm-up: one untimed pass of the same requests, 16 steps each, on this server, which fills
    # the launch-shape tuner's process-wide table for the work-list sizes the stream reaches (a
    # running server tunes once, not per stream); the timed pass runs on a fresh server
    with srv:
        srv.run_stream([replace(r, steps=16) for r in reqs])
    with Server(cfg) as srv:
        batched = srv.run_stream(reqs)
    plain = plain_run_stream(cfg, reqs)
    keep = ["completed", "makespan_s", "p50_s", "p99_s", "mean_s", "zone_updates", "zu_per_s", "max_concurrent",
            "kernel_launches", "busy_s"]
    out = {"requests": n_requests,
           "stream": f"seeded (seed {seed}) Poisson arrivals at 100/s; Sod, KH or blast; 2D {sz['sizes2'][0]}^2-"
                     f"{sz['sizes2'][1]}^2 and 3D {sz['sizes3'][0]}^3-{sz['sizes3'][1]}^3 log-uniform; "
                     f"{sz['steps'][0]}-{sz['steps'][1]} steps; rho ratio U[1,10], p ratio log-U[1,1000], gamma "
                     f"1.4 or 5/3; koren+HLLC; budget {cfg.budget_bytes / 1e9:.0f} GB",
           "sizes": sizes,
           "warmup": "one untimed pass of the same requests at 16 steps each on another server (the tuner's table)",
           "batched": {k: batched[k] for k in keep}, "plain": {k: plain[k] for k in keep},
           "aggregate_speedup": batched["zu_per_s"] / plain["zu_per_s"] if plain["zu_per_s"] else None}
    for arm in ("batched", "plain"):
        out[arm]["gpu_busy_share"] = out[arm]["busy_s"] / out[arm]["makespan_s"] if out[arm]["makespan_s"] else None
    return out


def workload(n: int, recon: str):
    from shaderous_b200 import Config, Problem

    cfg = Config(n=(n, n, n), dx=2 * math.pi / n, gamma=5 / 3, cfl=0.4, recon=recon, riemann="hllc",
                 isentropic=(recon != "ppm"))
    prob = Problem("tgv", a=(1.0, 100.0, 1.0))
    return cfg, prob


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_figure(recon: str, key: str):
    """A per-cell figure of the sweep kernel from the committed ncu summary, if present."""
    f = ROOT / "profiles" / f"sweep_3d_{recon}.md"
    if not f.exists():
        return None
    m = re.search(key + r":\s*([0-9.]+)", f.read_text())
    return float(m.group(1)) if m else None


def profile_traffic(recon: str):
    return profile_figure(recon, "dram_bytes_per_cell")


# The B200's issue and FP32 ceilings at its maximum SM clock (148 SMs x 4 schedulers, one warp
# instruction each per cycle; 128 FP32 lanes per SM, an FMA counting 2): no measured figure exists
# for these, so they are the nominal ones.
SM_COUNT, SM_MHZ = 148, 1965.0
ISSUE_PEAK = SM_COUNT * 4 * SM_MHZ * 1e6          # warp instructions / s
FP32_PEAK = SM_COUNT * 128 * 2 * SM_MHZ * 1e6     # FLOP / s


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 200 ms while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = Path(os.environ.get("TMPDIR", "/tmp")) / f"shz_clocks_{os.getpid()}.csv"

    def __enter__(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.gpu)], stdout=self.fh, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        if self.proc is None or not self.path.exists():
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        try:
            self.path.unlink()
        except OSError:
            pass
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons), "samples": len(sm)}


def cpu_sample(recon: str, min_seconds: float = 10.0, max_steps: int = 40):
    """The float64 oracle on a bounded sample of the workload: TGV at 128^3 (the oracle resolution of
    the configuration), as many steps as fill ~10 s, all host threads."""
    from oracle.oracle import RefHydro
    from shaderous_b200 import problem_prims

    n = 128
    cfg, prob = workload(n, recon)
    prims = problem_prims(cfg, prob)
    threads = os.cpu_count() or 1
    h = RefHydro(n=cfg.n, dx=cfg.dx, gamma=cfg.gamma, bc_lo=(0, 0, 0), bc_hi=(0, 0, 0), cfl=cfg.cfl, limiter=recon,
                 isentropic=cfg.isentropic and recon != "ppm", threads=threads)
    h.init_prims(prims)
    h.step()  # untimed first step (allocations)
    t0 = time.perf_counter()
    steps = 0
    while steps < max_steps and (steps < 2 or time.perf_counter() - t0 < min_seconds):
        h.step()
        steps += 1
    dt = time.perf_counter() - t0
    return {"value": n ** 3 * steps / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"TGV {n}^3 {recon.upper()}+HLLC, {steps} float64 steps of the C++ oracle (a port of "
                      f"src/reference/hydro.ts), {threads} threads, {dt:.1f} s"}


def cpu_extra() -> list:
    """Short samples of the oracle on the reference's own CPU test cases and on one thread: Sod 512
    to t = 0.2, KH 256^2, Sedov 64^3 (all host threads) and TGV 128^3 PPM on one thread."""
    from oracle.oracle import RefHydro
    from shaderous_b200 import Config, Problem, problem_prims

    threads = os.cpu_count() or 1
    out = []

    def sample(name, cfg, prob, limiter, nthreads, steps=None, t_end=None):
        h = RefHydro(n=cfg.n, dx=cfg.dx, gamma=cfg.gamma, bc_lo=cfg.bc_lo, bc_hi=cfg.bc_hi, cfl=cfg.cfl,
                     limiter=limiter, isentropic=cfg.isentropic and limiter != "ppm", threads=nthreads)
        h.init_prims(problem_prims(cfg, prob))
        t0 = time.perf_counter()
        if t_end is not None:
            h.run(t_end)
        else:
            for _ in range(steps):
                h.step()
        dt = time.perf_counter() - t0
        out.append({"case": name, "value": cfg.ncell * h.steps / dt, "unit": UNIT, "cores": nthreads, "steps": h.steps,
                    "seconds": dt})

    sample("sod 512 minmod+hllc to t=0.2", Config(n=(512, 1, 1), gamma=1.4, bc_lo=(1, 0, 0), bc_hi=(1, 0, 0), cfl=0.4,
                                                   recon="minmod", p_floor=1e-12),
           Problem("sod", a=(1, 0, 1, 0.125, 0, 0.1)), "minmod", 1, t_end=0.2)
    sample("kh 256^2 mc+hllc, 20 steps", Config(n=(256, 256, 1), gamma=1.4, cfl=0.4, recon="mc"),
           Problem("kh", a=(2.0, 1.0, 0.5, 2.5, 0.01, 1e-3), seed=7), "mc", threads, steps=20)
    sample("sedov 64^3 koren+hllc, 10 steps", Config(n=(64, 64, 64), gamma=5 / 3, cfl=0.5, recon="koren",
                                                      bc_lo=(1, 1, 1), bc_hi=(1, 1, 1), p_floor=1e-12),
           Problem("sedov", a=(1.0, 1e-5, 1.0, 3.5)), "koren", threads, steps=10)
    cfg, prob = workload(128, "ppm")
    sample("tgv 128^3 ppm+hllc, 2 steps, one thread", cfg, prob, "ppm", 1, steps=2)
    return out


def tgv_prims(n: int) -> np.ndarray:
    """The Taylor-Green initial primitives (rho, vx, vy, vz, p, s) at the cell centres of an n^3
    grid on [0, 2 pi]^3, x fastest: rho = 1, p = 100, u = sin x cos y cos z, v = -cos x sin y cos z,
    w = 0. Built here with numpy alone (cell centres at (i + 1/2) 2 pi / n, the reference's
    cell-centre rule, src/reference/hydro.ts:195-214), so the reference arm loads no product code."""
    c = (np.arange(n) + 0.5) * (2 * math.pi / n)
    sx, cx = np.sin(c), np.cos(c)
    w = np.zeros((n, n, n, 6))  # [z][y][x]
    w[..., 0] = 1.0
    w[..., 1] = sx[None, None, :] * cx[None, :, None] * cx[:, None, None]
    w[..., 2] = -cx[None, None, :] * sx[None, :, None] * cx[:, None, None]
    w[..., 4] = 100.0
    return w.reshape(-1, 6)


def run_reference(args, rank, world):
    """The reference arm: the CPU oracle on the host's cores, one bounded sample step per bench
    step. It imports only the oracle and numpy (no product library is loaded in this process)."""
    if rank != 0:
        return
    from oracle.oracle import RefHydro

    n = 128
    threads = os.cpu_count() or 1
    recon = args.recon
    h = RefHydro(n=(n, n, n), dx=2 * math.pi / n, gamma=5 / 3, bc_lo=(0, 0, 0), bc_hi=(0, 0, 0), cfl=0.4,
                 limiter=recon, isentropic=recon != "ppm", threads=threads)
    h.init_prims(tgv_prims(n))
    for _ in range(args.warmup):
        h.step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        h.step()
    dt = time.perf_counter() - t0
    v = n ** 3 * args.steps / dt
    sample = (f"TGV {n}^3 {recon.upper()}+HLLC per step (bounded sample of the {args.n}^3 workload), float64 "
              f"C++ oracle ported from src/reference/hydro.ts (the TypeScript original has no runtime here), "
              f"{threads} threads")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000 * dt / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"taylor-green {n}^3 periodic (a bounded sample of the {args.n}^3 workload: the "
                                   f"float64 oracle at {args.n}^3 needs tens of GB), {recon}+hllc, cfl 0.4",
                       "sample_cells": n ** 3, "workload_cells": args.n ** 3},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def headline(args, world, value, total_ms, sweep_ms, ncell, launches, clocks, e2e_value, e2e_s, config):
    """The JSON line: the metric, the sweep's roofline (ncell cells per GPU), e2e, launches, clocks."""
    sweep_avg_s = sweep_ms / args.steps / 1000.0
    peak, peak_kind = measured_peaks()
    achieved = BYTES_PER_ZU * ncell / sweep_avg_s / 1e9
    tr = profile_traffic(args.recon)
    state_bytes = 2 * ncell * 16
    e2e_steps = args.e2e_steps
    return {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic", "config": config,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": (tr * ncell) if tr else None, "kernel": "sweep_kernel",
                     "algorithmic_bytes_per_zu": BYTES_PER_ZU, "peak_source": f"{peak_kind} hbm_gbs",
                     "sweep_ms_per_step": sweep_ms / args.steps},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": state_bytes / e2e_steps,
                "d2h_bytes_per_step": (state_bytes + 64 * math.ceil(math.log2(e2e_steps + 1))) / e2e_steps,
                "steps": e2e_steps, "seconds": e2e_s},
        "gpu_launches": launches,
        "clocks": clocks,
        **extra_rooflines(args, ncell * args.steps / (sweep_ms / 1000.0)),
    }


def extra_rooflines(args, zu_per_s_gpu: float) -> dict:
    """The sweep's issue and FP32 rooflines: warp instructions and executed FP32 FLOP per cell from
    the committed ncu capture, times this run's zone-updates/s of the sweep on one GPU, against the
    nominal ceilings."""
    out = {}
    inst = profile_figure(args.recon, "warp_inst_per_cell")
    flop = profile_figure(args.recon, "fp32_flop_per_cell")
    if inst:
        a = inst * zu_per_s_gpu
        out["roofline_issue"] = {"bound": "issue", "achieved": a, "peak": ISSUE_PEAK, "unit": "warp instructions/s",
                                 "frac": a / ISSUE_PEAK, "per_zu": inst, "peak_source": "nominal (148 SMs x 4 x 1965 MHz)"}
    if flop:
        a = flop * zu_per_s_gpu
        out["roofline_fp32"] = {"bound": "fp32", "achieved": a / 1e12, "peak": FP32_PEAK / 1e12, "unit": "TFLOP/s",
                                "frac": a / FP32_PEAK, "per_zu": flop,
                                "peak_source": "nominal (148 SMs x 128 lanes x 2 x 1965 MHz); executed FADD + FMUL + 2 FFMA"}
    return out


def run_slabs(args, rank, world, local):
    """N GPUs, weak scaling: one periodic Taylor-Green grid of n x n x (n N) cells on
    [0,2pi]^2 x [0,2pi N] (the vortex repeated N times along z), split into N z-slabs of n^3, one
    per rank (shaderous_b200.dist.SlabSim): before every step NCCL send/recv fills each slab's halo
    planes and a max all-reduce of the rate gives every slab the same dt."""
    import torch
    import torch.distributed as dist

    from shaderous_b200.dist import SlabSim, max_over_ranks

    cfg, prob = workload(args.n, args.recon)
    cfg.n = (args.n, args.n, args.n * world)
    cfg.device = local
    dev = f"cuda:{local}"
    sl = SlabSim(cfg, device=local)
    sl.reset(prob)
    ncell_local = sl.sim.ncell
    total_cells = ncell_local * world

    sl.step(max(args.warmup, 1))  # warm-up (the first step tunes the sweep's launch shape)
    sl.sync()
    dist.barrier()
    launches0 = sl.sim.kernel_launches
    visible = [v for v in os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",") if v.strip()]
    gpu_index = visible[local] if local < len(visible) else local
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(gpu_index) as clocks:
        torch.cuda.synchronize()
        e0.record(sl.stream)
        sl.step(args.steps)
        e1.record(sl.stream)
        e1.synchronize()
    step_ms = max_over_ranks(e0.elapsed_time(e1), device=dev)
    launches = sl.sim.kernel_launches - launches0
    value = total_cells * args.steps / (step_ms / 1000.0)
    # the sweep alone (clock + sweep launches, no exchange) for the kernel's roofline
    prof = sl.sim.profile(args.steps)
    sweep_ms = max_over_ranks(prof["sweep_ms"], device=dev)

    # end to end: each rank's slab from pinned host memory, steps with exchanges, back to the host
    u1_0, u2_0 = sl.read_state()
    h_in1 = torch.from_numpy(u1_0).pin_memory()
    h_in2 = torch.from_numpy(u2_0).pin_memory()
    h_out1 = torch.empty_like(h_in1).pin_memory()
    h_out2 = torch.empty_like(h_in2).pin_memory()
    del u1_0, u2_0
    lib = sl.sim._lib
    dist.barrier()
    t0 = time.perf_counter()
    sl.sim._ok(lib.shz_set_state(sl.sim._h, h_in1.data_ptr(), h_in2.data_ptr(), ncell_local))
    sl.step(args.e2e_steps)
    sl.sim._ok(lib.shz_get_state(sl.sim._h, h_out1.data_ptr(), h_out2.data_ptr(), ncell_local))
    e2e_s = max_over_ranks(time.perf_counter() - t0, device=dev)
    if not np.isfinite(h_out1[:: max(1, ncell_local // 4096)].numpy()).all():
        raise RuntimeError("non-finite state after the end-to-end run")
    sl.destroy()
    return {"value": value, "total_ms": step_ms, "sweep_ms": sweep_ms, "launches": launches, "clocks": clocks.summary(),
            "ncell": ncell_local, "total_cells": total_cells,
            "e2e_value": total_cells * args.e2e_steps / e2e_s, "e2e_s": e2e_s,
            "config": {"workload": f"taylor-green {args.n}x{args.n}x{args.n * world} periodic [0,2pi]^2 x [0,2pi*{world}]"
                                   f" (the vortex repeated along z), rho 1, p0 100, gamma 5/3, {args.recon}+hllc, cfl 0.4",
                       "cells": total_cells, "cells_per_gpu": ncell_local,
                       "parallelism": f"z-slabs x{world}: NCCL send/recv halo planes + max all-reduce of the rate per step",
                       "l2": f"inputs larger than L2 ({2 * ncell_local * 16 / 1e9:.2f} GB state per GPU vs "
                             f"{L2_BYTES / 1e6:.0f} MB L2)"}}


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.section != "all":
        out = {}
        if args.section == "amr" and args.pin_assemble is not None:
            from shaderous_b200 import tune

            tune.pin("amr_assemble", args.pin_assemble, 2)
        if args.section == "amr":
            if args.amr_variant in ("both", "spec"):
                out["spec"] = amr_sedov(steps=max(args.steps, 8), cap=args.amr_cap, profile_window=args.profile_window)
            if args.amr_variant == "spread":
                out["spread"] = amr_sedov_spread(levels=args.amr_levels, steps=max(args.steps, 8),
                                                 cap=max(args.amr_cap, 30000), profile_window=args.profile_window)
            if args.amr_variant in ("both", "developed", "bins"):
                out.update(amr_sedov_developed(steps=max(args.steps, 8), cap=args.amr_cap,
                                               profile_window=args.profile_window, bins=args.amr_variant != "developed"))
        elif args.section == "comparable":
            out = comparable()
        else:
            out = serving(args.serve_requests, sizes=args.serve_sizes)
        print(json.dumps({"section": args.section, "result": out}), flush=True)
        return

    import torch

    dist = None
    if world > 1 or args.slabs:
        import datetime

        import torch.distributed as dist

        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        os.environ.setdefault("MASTER_PORT", "29511")
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    if world > 1 or args.slabs:
        r = run_slabs(args, rank, world, local)
        dist.barrier()
        dist.destroy_process_group()
        if rank == 0:
            print(json.dumps(headline(args, world, r["value"], r["total_ms"], r["sweep_ms"], r["ncell"], r["launches"],
                                      r["clocks"], r["e2e_value"], r["e2e_s"], r["config"])), flush=True)
        return

    from shaderous_b200 import Sim, problem_prims, prims_to_state

    cfg, prob = workload(args.n, args.recon)
    cfg.device = local
    ncell = cfg.ncell
    sim = Sim(cfg)
    sim.reset(prob)
    lib = sim._lib

    # warm-up: W untimed steps
    sim.profile(max(args.warmup, 1))
    sim.sync()
    if dist:
        dist.barrier()
    launches0 = sim.kernel_launches
    visible = [v for v in os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",") if v.strip()]
    gpu_index = visible[local] if local < len(visible) else local
    with ClockSampler(gpu_index) as clocks:
        prof = sim.profile(args.steps)  # synchronizes on the last event
    launches = sim.kernel_launches - launches0
    total_ms = prof["total_ms"]
    sweep_ms = prof["sweep_ms"]
    if dist:
        t = torch.tensor([total_ms, sweep_ms], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms, sweep_ms = float(t[0]), float(t[1])
    value = ncell * args.steps * world / (total_ms / 1000.0)

    # end to end through the C ABI with pinned host buffers
    u1_0, u2_0 = prims_to_state(problem_prims(cfg, prob), cfg.gamma)
    h_in1 = torch.from_numpy(u1_0).pin_memory()
    h_in2 = torch.from_numpy(u2_0).pin_memory()
    h_out1 = torch.empty_like(h_in1).pin_memory()
    h_out2 = torch.empty_like(h_in2).pin_memory()
    del u1_0, u2_0
    e2e_steps = args.e2e_steps
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    sim._ok(lib.shz_set_state(sim._h, h_in1.data_ptr(), h_in2.data_ptr(), ncell))
    sim.set_clock(0.0, 0)
    res = sim.run(steps=e2e_steps)
    sim._ok(lib.shz_get_state(sim._h, h_out1.data_ptr(), h_out2.data_ptr(), ncell))
    e2e_s = time.perf_counter() - t0
    assert res.taken == e2e_steps, res
    if dist:
        t = torch.tensor([e2e_s], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t[0])
    e2e_value = ncell * e2e_steps * world / e2e_s
    if not np.isfinite(h_out1[:: max(1, ncell // 4096)].numpy()).all():
        raise RuntimeError("non-finite state after the end-to-end run")

    sim.destroy()
    del h_in1, h_in2, h_out1, h_out2
    amr = serve = None
    if rank == 0 and not args.no_amr:
        amr = {"spec": amr_sedov()}
        # the same run advanced to about 20k leaves; then per-block timesteps (cycles of 32
        # substeps) on that mesh, zone-updates counted as single steps would make them
        amr.update(amr_sedov_developed(steps=16, bins_steps=64))
    if rank == 0 and not args.no_serving:
        serve = serving(args.serve_requests, sizes=args.serve_sizes)
    comp = comparable() if rank == 0 and not args.no_comparable else None
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu = cpu_sample(args.recon)
        cpu["extra"] = cpu_extra()
        cpu["reference_js"] = ("src/reference/hydro.ts itself: unavailable on this box (no JavaScript runtime); "
                               "these are its C++ float64 restatement")
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    config = {"workload": f"taylor-green {args.n}^3 periodic [0,2pi]^3, rho 1, p0 100, gamma 5/3, "
                          f"{args.recon}+hllc, cfl 0.4",
              "cells": ncell, "parallelism": "single grid",
              "l2": f"inputs larger than L2 ({2 * ncell * 16 / 1e9:.2f} GB state vs {L2_BYTES / 1e6:.0f} MB L2)"}
    line = headline(args, world, value, total_ms, sweep_ms, ncell, launches, clocks.summary(), e2e_value, e2e_s, config)
    if cpu:
        line["cpu_baseline"] = cpu
    if amr:
        line["amr_sedov"] = amr
    if serve:
        line["serving"] = serve
    if comp:
        line["comparable"] = comp
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
