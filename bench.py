#!/usr/bin/env python
"""Benchmark of the SPH cutting step (leap_frog::step of iwf_mfree_gpu_3d) on B200.

Workload (one "step" = one full time step of one scene): orthogonal cutting of
a steel block, 200 x 100 x 50 = 1,000,000 particles, CSPM correction,
artificial stress and PSE conduction on, Johnson-Cook plasticity, rigid-wedge
contact, FP32 (the configuration the headline metric is quoted on).  Data is
synthetic: a seeded jittered lattice and a generated wedge mesh (the reference
ships no dataset).  The particle state (~0.5 GB) is larger than the 126 MB L2,
so no L2 flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (torchrun, one process per GPU) every rank steps its own
independent scene (the reference is single-GPU; scenes shard with no
collective): weak scaling, value = all ranks' particle-steps / max rank time.

--impl reference times the reference's CPU algorithm -- the FP64 oracle
restatement, OpenMP on every host core -- on the same scene (a bounded
sub-block of it per step when the full scene would not finish in minutes).

At N = 1 the line also carries the two systems forms, measured live:
  * "batched": 256 independent cutting scenes of log-uniform size in
    [5k, 200k] particles (seed 1; speed, depth, rake and Johnson-Cook A, B, n
    drawn per scene; compensated positions) stepped together -- one launch per
    kernel, one captured graph per step, autotuned tiling -- against the plain
    path run scene by scene with the same tiling;
  * "serving": a Poisson request stream admitted into one resident batch by a
    150 GB budget, with p50/p99 latency (arrival to result) and throughput;
    rate, duration, sizes and step counts are scaled down so the run takes
    seconds (the scaling is stated in the line).
  * "precision_form" (1M workload): the same step in the precision form;
  * "small": the 8,000-particle configuration as stated, 1,000 steps;
  * "grain": the single-grain configuration (400 x 160 x 64 block plus the
    grain's tool particles, ~4.1M, compensated positions): particle-steps/s and
    HBM GB/s.
--no-extras skips these.

Beside the main line (and the grain leg), "reference_gpu" times the
reference's own GPU step -- leap_frog::step built for sm_100a from its
sources by baseline/build_ref_gpu.sh -- on the same scene and GPU.
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

# ---- algorithmic FLOPs of the pair kernel (counted from the reference's pair
# formulas, interactions_gpu.cu:152-471 and kernels.cuh:26-92; add/mul = 1,
# FMA = 2, div/sqrt/exp = 1; the artificial-viscosity branch counted for half
# of the pairs) ----
F_CANDIDATE = 8            # distance test of every stencil candidate
F_CANDIDATE_PSE = 6        # PSE term of every stencil candidate
F_PAIR = 16 + 24 + 15 + 30 + 15 + 7    # spline, grad v, art. stress, stress divergence, AV, XSPH
F_PAIR_CSPM = 44 + 15      # CSPM matrix term (with its spline) + corrected gradient
F_PAIR_BROOKSHAW = 10
F_PARTICLE_EPILOGUE = 150  # Jaumann, continuity, momentum, corrector, yield check

CLOCK_QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
               "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
               "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["1m", "8k", "grain"], default="1m")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--lpp", type=int, default=0, help="lanes per particle (0 = default)")
    ap.add_argument("--no-extras", action="store_true", help="skip the batched and serving measurements")
    ap.add_argument("--batch-scenes", type=int, default=256)
    ap.add_argument("--batch-steps", type=int, default=20)
    ap.add_argument("--serve-rate", type=float, default=20.0, help="requests per second")
    ap.add_argument("--serve-seconds", type=float, default=30.0, help="arrival window")
    ap.add_argument("--serve-nmax", type=int, default=500000, help="largest request (particles)")
    ap.add_argument("--serve-step-scale", type=float, default=0.1,
                    help="factor on every request's U[500, 5000] step count")
    ap.add_argument("--serve-chunk", type=int, default=25, help="steps between admissions")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip the reference's own GPU step (baseline/_ref) on the same scene")
    ap.add_argument("--no-grain", action="store_true", help="skip the single-grain leg")
    return ap.parse_args()


def make_scene(workload: str, seed: int = 0, precision: int = 0):
    from iwf_mfree_gpu_3d_b200 import scenes
    if workload == "8k":
        return scenes.small_scene(seed=seed, precision=precision)
    if workload == "grain":
        return scenes.single_grain(seed=seed)  # compensated positions, as the configuration asks
    return scenes.million_scene(seed=seed, precision=precision)


def workload_config(workload: str, sc) -> dict:
    names = {"1m": "orthogonal cutting 200x100x50 steel block (1,000,000 particles), CSPM + artificial "
                   "stress + PSE, Johnson-Cook, wedge contact",
             "8k": "orthogonal cutting 40x20x10 steel block (8,000 particles), Brookshaw, artificial "
                   "stress, Johnson-Cook, wedge contact",
             "grain": "single-grain cutting, 400x160x64 steel block (4,096,000 particles) + the grain volume "
                      "as diamond tool particles, 1,280-triangle truncated icosphere (radius 20 dx, -10 deg rake) "
                      "at 30 m/s, depth 8 dx, Brookshaw, compensated positions"}
    return {"workload": names[workload],
            "particles": sc.n, "dx_cm": 1e-3, "h_over_dx": 1.3, "dt_us": sc.dt,
            "cspm": bool(sc.options["cspm"]), "conduction": ["none", "brookshaw", "pse"][sc.options["conduction"]],
            "l2": {"1m": "inputs larger than L2 (particle state ~0.5 GB)",
                   "grain": "inputs larger than L2 (particle state ~2.9 GB)"}.get(
                       workload, "inputs smaller than L2 (8k particles)"),
            "parallelism": "one independent scene per GPU"}


# ------------------------------------------------------------ clocks ----
class ClockSampler:
    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={CLOCK_QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
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
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------- algorithmic counts ----
def stencil_counts(sim) -> tuple[float, float]:
    """(candidates, in-support pairs) summed over the active particles of the
    last step: candidates from the cell ranges of each particle's 5x5x5
    stencil, pairs from the kernel's own neighbour counts."""
    (nx, ny, nz), _, _ = sim.grid()
    cs, ce = sim.cells()
    n_act, _ = sim.counts()
    cnt = np.where(cs >= 0, ce - cs, 0).astype(np.int64)
    first = np.concatenate([[0], np.cumsum(cnt)])
    key = sim.get("HASH")[:n_act].astype(np.int64)
    gi = key // (ny * nz)
    gj = (key - gi * ny * nz) // nz
    gk = key % nz
    z0 = np.maximum(gk - 2, 0)
    z1 = np.minimum(gk + 2, nz - 1)
    cand = np.zeros(n_act, np.int64)
    for dxi in range(-2, 3):
        for dyi in range(-2, 3):
            cx, cy = gi + dxi, gj + dyi
            ok = (cx >= 0) & (cx < nx) & (cy >= 0) & (cy < ny)
            cb = (np.clip(cx, 0, nx - 1) * ny + np.clip(cy, 0, ny - 1)) * nz
            cand += np.where(ok, first[cb + z1 + 1] - first[cb + z0], 0)
    pairs = sim.get("NUM_NBH")[:n_act].astype(np.int64)
    return float(cand.sum()), float(pairs.sum())


def interact_flops(sc, cand: float, pairs: float, n_act: int, pse_share: float = 1.0) -> float:
    """Algorithmic FLOPs of one pair-kernel launch.  pse_share: the share of
    targets whose PSE sum must be evaluated; where every temperature a tile's
    stencils reach is equal, the sum is exactly zero and is not work (the
    kernel skips it, mfree_counters.pse_zero_targets)."""
    fp = F_PAIR + (F_PAIR_CSPM if sc.options["cspm"] else 0) + (
        F_PAIR_BROOKSHAW if sc.options["conduction"] == 1 else 0)
    fc = F_CANDIDATE + (F_CANDIDATE_PSE * pse_share if sc.options["conduction"] == 2 else 0)
    return cand * fc + pairs * fp + n_act * F_PARTICLE_EPILOGUE


def read_traffic() -> float | None:
    """DRAM bytes per launch of the pair kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "roofline_traffic.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith("interact_dram_bytes_per_launch_1m:"):
            try:
                return float(line.split(":", 1)[1].strip().split()[0])
            except ValueError:
                return None
    return None


def hbm_roofline(rate: float, sc) -> dict:
    """Whole-step HBM roofline: the compulsory particle state crossing HBM once
    per step (152 B read + 144 B written + 8 B sort key; the precision form adds
    24 + 24 B of low parts) times the rate, against the measured copy bandwidth."""
    b_alg = 352 if sc.options.get("precision") else 304
    peak, src = 6650.0, "fallback 6.65 TB/s (no MEASURED_PEAKS.json)"
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peak, src = float(json.load(f)["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except (OSError, KeyError, ValueError):
        pass
    gbs = rate * b_alg / 1e9
    return {"algorithmic_bytes_per_particle_step": b_alg, "achieved_gbs": gbs, "peak_gbs": peak,
            "frac": gbs / peak, "peak_source": src,
            "note": "the step is bound by the pair kernel's FP32 pipe, not by HBM"}


def kernel_hbm(sc, n_act: int, step_ms: dict) -> dict:
    """HBM roofline of the memory-bound kernels of the step, from their
    CUDA-event times: algorithmic bytes per launch (each array element the
    kernel must read or write, once) / time, against the measured copy
    bandwidth."""
    prec = 32 if sc.options.get("precision") else 0
    blank = sc.blank_vmax > 0
    # kb_gather_predict: perm 4 + state 176 (+ low parts) + key 4 read; state 176 (+ low parts)
    # + sorted key 4 + neighbour records 96 written
    gather = 4 + 176 + prec + 4 + 176 + prec + 4 + 96
    # kb_hash: pos + blank flag 32 (+ vel 16 with blanking) read, key 4 written; the rates
    # are read only for blanked particles, which the box and speed tests may unblank
    hsh = 32 + (16 if blank else 0) + 4
    peak = 6650.0
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peak = float(json.load(f)["hbm_gbs"])
    except (OSError, KeyError, ValueError):
        pass
    out = {}
    for k, b in (("gather_predict", gather), ("hash", hsh)):
        ms = step_ms.get(k, 0.0)
        if ms > 0:
            gbs = sc.n * b / (ms * 1e-3) / 1e9
            out[k] = {"bytes_per_particle": b, "ms": ms, "achieved_gbs": gbs, "frac": gbs / peak}
    return out


# -------------------------------------------------------------- oracle ----
def cpu_model() -> str:
    """The host CPU's model name (/proc/cpuinfo), for the baseline's record."""
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_baseline(workload: str, budget_s: float = 20.0) -> dict:
    """FP64 oracle (OpenMP, every host core) on a bounded sample of the workload."""
    import oracle
    oracle.build()
    cores = os.cpu_count() or 1
    sc = make_scene(workload)
    orc = oracle.Oracle(sc, prec=64, threads=cores)
    t0 = time.perf_counter()
    orc.step()  # warm-up step
    t_one = time.perf_counter() - t0
    nsteps = max(1, min(5, int(budget_s / max(t_one, 1e-3))))
    t0 = time.perf_counter()
    for _ in range(nsteps):
        orc.step()
    t = time.perf_counter() - t0
    return {"value": sc.n * nsteps / t, "unit": "particle-steps/s", "cores": cores, "cpu": cpu_model(), "kind": "port",
            "sample": f"{nsteps} FP64 oracle step(s) of the full {sc.n}-particle scene after 1 warm-up step"}


def run_reference(args, rank: int, world: int):
    if rank != 0:
        return
    import oracle
    oracle.build()
    cores = os.cpu_count() or 1
    sc = make_scene(args.workload)
    orc = oracle.Oracle(sc, prec=64, threads=cores)
    t0 = time.perf_counter()
    orc.step()
    t_full = time.perf_counter() - t0
    budget = 150.0
    total = args.steps + args.warmup
    if t_full * total <= budget:
        sample, n_sample = orc, sc.n
        desc = f"full {sc.n}-particle scene per step"
    else:
        # a sub-block of the same lattice (same z depth) sized to the budget
        from iwf_mfree_gpu_3d_b200 import scenes
        frac = budget / (t_full * total)
        nx = max(8, int(200 * math.sqrt(frac)))
        ny = max(4, int(100 * math.sqrt(frac)))
        sub = scenes.orthogonal_cutting(nx, ny, 50, cspm=True, conduction=2)
        sample, n_sample = oracle.Oracle(sub, prec=64, threads=cores), sub.n
        desc = f"{nx}x{ny}x50 sub-block ({sub.n} particles) of the same scene per step"
    for _ in range(args.warmup):
        sample.step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        sample.step()
    t = time.perf_counter() - t0
    v = n_sample * args.steps / t
    line = {"metric": "particle-steps/s", "value": v, "unit": "particle-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference", "config": workload_config(args.workload, sc),
            "cpu_baseline": {"value": v, "unit": "particle-steps/s", "cores": cores, "cpu": cpu_model(), "kind": "port",
                             "sample": "FP64 oracle restatement of leap_frog::step, " + desc},
            "e2e": {"value": v, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------- multi-process ----
def reduce_max(dist, x: float, device: str) -> float:
    """Max over ranks (the slowest rank's time), or x itself without a process group."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate(n_particles: int, steps: int, world: int, max_seconds: float) -> float:
    """Whole-job particle-steps/s: every rank steps its own scene of the same size."""
    return n_particles * steps * world / max_seconds


# ---------------------------------------------------------------- ours ----
def run_ours(args, rank: int, world: int, local_rank: int, dist):
    from iwf_mfree_gpu_3d_b200 import api
    api.set_device(local_rank)
    sc = make_scene(args.workload, seed=rank)
    opts = {"lanes_per_particle": args.lpp} if args.lpp else {}

    # --- algorithmic counts of one step (outside the timed region)
    probe = api.Simulation.from_scene(sc, diagnostics=1, **opts)
    probe.step()
    cand, pairs = stencil_counts(probe)
    n_act = probe.counts()[0]
    flops_launch = interact_flops(sc, cand, pairs, n_act)
    probe.close()
    peak_fp32 = api.fp32_peak_tflops()

    # --- device-resident throughput: K replays of the captured step (CUDA graph)
    sim = api.Simulation.from_scene(sc, **opts)
    sim.advance(max(args.warmup, 3), use_graph=True)  # warm-up (and the capture)
    sim.sync()
    if dist:
        dist.barrier()
    with ClockSampler(local_rank) as clk:
        sim.sync()
        sim.timer_start()
        sim.advance(args.steps, use_graph=True)
        ms = sim.timer_stop()
    # --- per-kernel device times (eager steps, CUDA events around every kernel)
    eager = min(args.steps, 20)
    sim.set_kernel_timing(True)
    sim.kernel_times()  # reset
    pz0 = sim.counters()["pse_zero_targets"]
    for _ in range(eager):
        sim.step()
    ktimes = sim.kernel_times()
    counters = sim.counters()
    pse_zero_share = (counters["pse_zero_targets"] - pz0) / float(eager * sim.counts()[0])
    sim.close()
    ms = reduce_max(dist, ms, f"cuda:{local_rank}")
    if dist:
        dist.barrier()

    # --- end to end through the C ABI with host buffers
    e2e = run_e2e(sc, args, opts, dist, local_rank)

    if rank != 0:
        return
    value = aggregate(sc.n, args.steps, world, ms * 1e-3)
    ik_ms, ik_n = ktimes["interact"]
    ik_avg = ik_ms / max(ik_n, 1)
    # the PSE terms of targets whose PSE sum is exactly zero are not work
    flops_launch = interact_flops(sc, cand, pairs, n_act, pse_share=1.0 - pse_zero_share)
    achieved = flops_launch / (ik_avg * 1e-3) / 1e12
    traffic = read_traffic() if args.workload == "1m" else None  # the ncu capture is of the 1M scene
    roofline = {"bound": "fp32", "achieved": achieved, "peak": peak_fp32, "unit": "TFLOP/s",
                "frac": achieved / peak_fp32,
                "traffic": traffic,
                "kernel": "kb_interact (pair loop + fused per-particle rest of the step)",
                "peak_source": "measured: FP32 FMA-throughput probe on this GPU (mfree_probe_fp32_peak); "
                               "MEASURED_PEAKS.json holds HBM and bf16 tensor peaks only",
                "algorithmic_flops_per_launch": flops_launch,
                "candidates_per_particle": cand / n_act, "pairs_per_particle": pairs / n_act,
                "pse_zero_share": pse_zero_share if sc.options["conduction"] == 2 else None}
    step_ms_dev = {k: (v[0] / max(v[1], 1)) for k, v in ktimes.items()}
    line = {"metric": "particle-steps/s", "value": value, "unit": "particle-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded jittered lattice, generated " +
                    ("truncated-icosphere grain)" if args.workload == "grain" else "wedge tool)"),
            "config": workload_config(args.workload, sc),
            "roofline": roofline,
            "e2e": e2e,
            "gpu_launches": int(round(sum(v[1] for v in ktimes.values()) / eager * args.steps)),
            "timing": "CUDA events around K graph replays of the step on the context's stream; the per-kernel "
                      "times (roofline) from separate eager steps with events around every kernel",
            "kernel_ms_per_step": step_ms_dev,
            "clocks": clk.summary(),
            "counters": counters,
            "hbm": hbm_roofline(value, sc),
            "hbm_kernels": kernel_hbm(sc, n_act, step_ms_dev)}
    if world == 1 and not args.no_reference_gpu:
        line["reference_gpu"] = run_reference_gpu(sc, ms / args.steps, e2e)
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args.workload)
    if world == 1 and not args.no_extras and not args.no_grain and args.workload != "grain":
        line["grain"] = run_grain(args, opts)
    if world == 1 and not args.no_extras and args.workload == "1m":
        line["precision_form"] = run_precision_form(sc, args, opts)
        line["small"] = run_small(args, opts)
    if world == 1 and not args.no_extras:
        line["batched"] = run_batched(args)
        line["serving"] = run_serve(args, tuple(line["batched"]["tiling"]))
    print(json.dumps(line), flush=True)


# ------------------------------------------- the reference's own GPU step -----
def run_reference_gpu(sc, ours_ms_per_step: float, e2e: dict | None = None, steps: int = 10,
                      warmup: int = 3, repeats: int = 3) -> dict:
    """Baseline (a): the reference's leap_frog::step (src/leap_frog.cu:121-195)
    built for sm_100a from its own sources (baseline/build_ref_gpu.sh), on the
    same scene and GPU, timed with CUDA events around its step loop (its step
    synchronises the device after its launches; setup and read-back excluded).

    The reference's step allocates and frees thrust's temporary storage in
    every sort and reduction and synchronises the host several times a step
    (grid_gpu_green.cu:270-305, grid_gpu_base.cu:137-198), so its time varies
    from run to run with the allocator's latency (22-110 ms per step measured
    on the 1M scene, the same steps and results).  The line takes the fastest
    of `repeats` runs, each a fresh process on the same scene, and lists all."""
    from baseline import refgpu
    variant = refgpu.variant_of(sc)
    if variant is None or not refgpu.available(variant):
        return {"unavailable": "the reference's GPU build (baseline/_ref) is not built here"}
    runs = [refgpu.run(sc, warmup, steps)["ms_per_step"] for _ in range(max(1, repeats))]
    ms = min(runs)
    out = {"metric": "particle-steps/s", "value": sc.n / (ms * 1e-3), "unit": "particle-steps/s",
           "ms_per_step": ms, "ms_per_step_runs": runs, "steps": steps, "warmup": warmup, "variant": variant,
           "ours_over_reference_device": ms / ours_ms_per_step,
           "build": "the reference's sources, -O3 -rdc=true for sm_100a, texture references read through __ldg "
                    "and a project-written GLM-compatible header (baseline/build_ref_gpu.sh)",
           "timing": "CUDA events around the reference's step loop, after warm-up; the fastest of the runs "
                     "(the reference allocates thrust temporaries and synchronises the host within every step)"}
    if e2e and e2e.get("value"):
        out["ours_e2e_over_reference_device"] = e2e["value"] / out["value"]
    return out


def run_grain(args, opts) -> dict:
    """The single-grain configuration (4.1M particles, compensated positions):
    particle-steps/s and HBM GB/s, timed like the main line, with the
    reference's own GPU step on the same scene beside it."""
    from iwf_mfree_gpu_3d_b200 import api
    sc = make_scene("grain")
    sim = api.Simulation.from_scene(sc, **opts)
    sim.advance(max(args.warmup, 3), use_graph=True)
    sim.sync()
    steps = min(args.steps, 20)
    sim.timer_start()
    sim.advance(steps, use_graph=True)
    ms = sim.timer_stop()
    sim.close()
    value = sc.n * steps / (ms * 1e-3)
    out = {"metric": "particle-steps/s", "value": value, "ms_per_step": ms / steps, "steps": steps,
           "config": workload_config("grain", sc), "hbm": hbm_roofline(value, sc),
           "timing": "CUDA events around K graph replays, as the main line"}
    if not args.no_reference_gpu:
        out["reference_gpu"] = run_reference_gpu(sc, ms / steps, steps=5, warmup=2)
    return out


def run_small(args, opts) -> dict:
    """The small configuration as stated: the 8,000-particle scene for 1,000
    steps (graph replays), with the reference's own GPU step beside it (its
    1,000-step parity is a test: tests/test_gpu_parity.py
    test_1000_steps_small_configuration)."""
    from iwf_mfree_gpu_3d_b200 import api
    sc = make_scene("8k")
    sim = api.Simulation.from_scene(sc, **opts)
    sim.advance(max(args.warmup, 3), use_graph=True)
    sim.sync()
    steps = 1000
    sim.timer_start()
    sim.advance(steps, use_graph=True)
    ms = sim.timer_stop()
    sim.close()
    value = sc.n * steps / (ms * 1e-3)
    out = {"metric": "particle-steps/s", "value": value, "ms_per_step": ms / steps, "steps": steps,
           "config": workload_config("8k", sc), "timing": "CUDA events around K graph replays, as the main line"}
    if not args.no_reference_gpu:
        out["reference_gpu"] = run_reference_gpu(sc, ms / steps, steps=100, warmup=3)
    return out


# ------------------------------------------------------ systems forms -----
def run_precision_form(sc, args, opts) -> dict:
    """The 1M configuration's second run: the precision form (FP32 bulk,
    compensated hi/lo positions and velocities), timed like the main line."""
    from iwf_mfree_gpu_3d_b200 import api
    sim = api.Simulation.from_scene(sc, precision=1, **opts)
    sim.advance(max(args.warmup, 3), use_graph=True)
    sim.sync()
    sim.timer_start()
    sim.advance(args.steps, use_graph=True)
    ms = sim.timer_stop()
    sim.close()
    return {"metric": "particle-steps/s", "value": sc.n * args.steps / (ms * 1e-3), "ms_per_step": ms / args.steps,
            "dtype": "f32 + compensated hi/lo positions and velocities",
            "timing": "CUDA events around K graph replays, as the main line",
            "error_vs_fp64": "per-field relative L2 at step 100: tests/test_gpu_parity.py "
                             "test_100_steps_against_fp64_oracle_full_size_1m_plain_and_precision"}

def run_batched(args) -> dict:
    """Mixed-size scenes stepped together against the plain path scene by scene."""
    from iwf_mfree_gpu_3d_b200 import api, scenes
    specs = scenes.mixed_specs(args.batch_scenes, seed=1)
    n_total = sum(sp.n for sp in specs)
    K = args.batch_steps
    b = api.Batch()
    t0 = time.perf_counter()
    for sp in specs:
        b.admit(api.Simulation.from_scene(scenes.mixed_scene(sp)))
    setup_s = time.perf_counter() - t0
    lpp, depth, _ = b.autotune(trial_steps=2)
    b.step(max(args.warmup, 3), use_graph=True)
    b.sync()
    b.timer_start()
    b.step(K, use_graph=True)
    ms = b.timer_stop()
    mem = b.info()["bytes"]
    b.close()
    # the plain path, one scene after the other, same tiling, same steps
    plain_ms = 0.0
    for sp in specs:
        sim = api.Simulation.from_scene(scenes.mixed_scene(sp), lanes_per_particle=lpp, tile_depth=depth)
        sim.advance(max(args.warmup, 3), use_graph=True)
        sim.sync()
        sim.timer_start()
        sim.advance(K, use_graph=True)
        plain_ms += sim.timer_stop()
        sim.close()
    batched = n_total * K / (ms * 1e-3)
    plain = n_total * K / (plain_ms * 1e-3)
    return {"metric": "particle-steps/s", "value": batched, "plain_scene_by_scene": plain,
            "batched_over_plain": batched / plain, "ms_per_step": ms / K, "plain_ms_per_step": plain_ms / K,
            "scenes": len(specs), "particles": n_total, "steps": K, "tiling": [lpp, depth],
            "device_bytes": mem, "setup_s": setup_s, "dtype": "f32 (compensated positions)",
            "timing": "CUDA events on the batch's stream (batched) and per scene on its stream, summed (plain)",
            "config": "256 cutting scenes, n log-uniform [5k, 200k] (nx=4nz, ny=2nz), v U[1e-4, 5e-3] cm/us, "
                      "depth U[2, 10] dx, rake U[-20, 10] deg, Johnson-Cook A, B, n x U[0.9, 1.1], seed 1"}


def run_serve(args, tiling) -> dict:
    """Poisson request stream into one resident batch (continuous batching):
    the serving configuration's arrival process (20 requests/s, scenes
    log-uniform in [10k, 500k] particles), over a shorter arrival window and
    with every request's step count scaled (both stated in the line)."""
    from iwf_mfree_gpu_3d_b200 import serve
    lo, hi = int(round(500 * args.serve_step_scale)), int(round(5000 * args.serve_step_scale))
    reqs = serve.poisson_requests(rate=args.serve_rate, duration=args.serve_seconds, seed=2, n_lo=10000,
                                  n_hi=args.serve_nmax, steps_lo=lo, steps_hi=hi)
    srv = serve.Server(hbm_budget=150 * 10**9, chunk_steps=args.serve_chunk, tiling=tiling)
    horizon = 4 * args.serve_seconds
    out = srv.run(reqs, horizon=horizon)
    srv.close()
    offered = sum(r.spec.n * r.spec.steps for r in reqs) / args.serve_seconds
    trace, last = [], -1e9
    for t, waiting, running, parts in out["queue_trace"]:  # about one sample per 2 s
        if t - last >= 2.0:
            trace.append([round(t, 2), waiting, running, parts])
            last = t
    return {"metric": "p50/p99 solve latency (s)", "p50_s": out["p50_s"], "p99_s": out["p99_s"],
            "p50_with_censored_s": out["p50_censored_s"], "p99_with_censored_s": out["p99_censored_s"],
            "particle_steps_per_s": out["particle_steps_per_s"], "offered_particle_steps_per_s": offered,
            "requests": out["offered"], "completed": out["completed"], "unfinished": out["unfinished"],
            "censored": out["censored"], "rejected": out["rejected"],
            "elapsed_s": out["elapsed_s"], "horizon_s": horizon, "chunk_steps": args.serve_chunk,
            "budget_bytes": 150 * 10**9,
            "queue_trace": {"columns": ["t_s", "waiting", "running", "running_particles"], "rows": trace},
            "timing": "wall clock on the host, arrival to result read-back; requests unfinished at the horizon "
                      "enter the *_with_censored_s percentiles at the time they have waited (lower bounds)",
            "config": f"Poisson {args.serve_rate}/s for {args.serve_seconds} s (seed 2), n log-uniform "
                      f"[10k, {args.serve_nmax}], steps U[{lo}, {hi}]: the serving configuration (20/s for "
                      f"600 s, [10k, 500k], U[500, 5000]) with the arrival window shortened to "
                      f"{args.serve_seconds:g} s and each request's step count scaled by {args.serve_step_scale:g}"}


def run_e2e(sc, args, opts, dist, local_rank) -> dict:
    """The same metric through the C ABI from pinned host buffers: the particle
    arrays are uploaded (mfree_create, as the reference's particle_gpu
    constructor), every step (one replay of the captured step) records and
    reads back the tool force (as the reference's driver does on its output
    steps), and the state the user reads (position, velocity, stress,
    temperature, plastic strain) is copied back at the end; wall clock around
    all of it."""
    from iwf_mfree_gpu_3d_b200 import api
    import torch
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    host = {k: pin(getattr(sc, k)) for k in ("pos", "vel", "rho", "T", "h", "fixed", "tool_p")}
    h2d = sum(v.nbytes for v in host.values())
    names = ("POS", "VEL", "S", "T", "EPS_PL")
    widths = {"POS": 4, "VEL": 4, "S": 9, "T": 1, "EPS_PL": 1}
    res = {k: pin(np.empty(sc.n * widths[k], np.float32)) for k in names}  # page-locked result buffers
    # warm the path once (module load, allocator)
    w = api.Simulation(host["pos"], host["vel"], host["rho"], host["h"], T=host["T"], fixed=host["fixed"],
                       tool_p=host["tool_p"])
    w.close()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    s = api.Simulation(host["pos"], host["vel"], host["rho"], host["h"], T=host["T"], fixed=host["fixed"],
                       tool_p=host["tool_p"])
    t_create = time.perf_counter()
    s.set_physics(**sc.phys)
    s.set_correctors(**sc.corr)
    if sc.joco:
        s.set_johnson_cook(**sc.joco)
    s.set_thermal_workpiece(**sc.trml_wp)
    s.set_thermal_tool(**sc.trml_tool)
    o = dict(sc.options)
    o.update(opts)
    s.set_options(**o)
    s.set_grid(sc.grid_bbmin, sc.grid_bbmax, sc.grid_h)
    s.set_blanking(sc.blank_bbmin, sc.blank_bbmax, sc.blank_vmax)
    for t in sc.tools:
        s.add_tool(t.verts, t.tris, t.vel, t.contact_alpha, t.mu, t.algorithm)
    dt = np.float32(sc.dt)
    s.set_time(float(dt), float(dt))
    d2h = 0
    t_setup = time.perf_counter()
    marks = []
    for _ in range(args.steps):
        s.advance(1, record_every=1, use_graph=True)  # one replay of the captured step, forces recorded
        f = s.tool_forces()  # the step's result, read back every step
        d2h += f.nbytes
        if len(marks) < 1:
            marks.append(time.perf_counter())
    t_steps = time.perf_counter()
    if not marks:
        marks.append(t_steps)
    out = [s.get(n, out=res[n]) for n in names]
    d2h += sum(a.nbytes for a in out)
    t_end = time.perf_counter()
    t = t_end - t0
    phases = {"create": t_create - t0, "setup": t_setup - t_create, "first_step": marks[0] - t_setup,
              "other_steps": t_steps - marks[0], "read_back": t_end - t_steps}
    s.close()
    t = reduce_max(dist, t, f"cuda:{local_rank}")
    world = dist.get_world_size() if dist else 1
    return {"value": aggregate(sc.n, args.steps, world, t), "unit": "particle-steps/s",
            "h2d_bytes_per_step": int(h2d / args.steps), "d2h_bytes_per_step": int(d2h / args.steps),
            "phases_ms": {k: round(v * 1e3, 2) for k, v in phases.items()},
            "note": "wall clock: context creation from pinned host arrays, setup, steps with a per-step tool-force "
                    "read-back, final read-back of POS/VEL/S/T/EPS_PL into pinned host arrays; state bytes amortised "
                    "over the steps"}


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1 and args.impl == "ours":  # the reference arm runs on rank 0 alone
        import datetime
        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(local_rank)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = tdist
    try:
        if args.impl == "reference":
            run_reference(args, rank, world)
        else:
            run_ours(args, rank, world, local_rank, dist)
    finally:
        if dist:
            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
