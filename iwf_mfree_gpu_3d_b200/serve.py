"""Serving loop: cutting-scene requests admitted into one resident batch.

The reference runs one scene per process to completion (main(),
src/mfree_gpu_3d.cpp:75-218); this module has no counterpart there.  Requests
(a scene plus a number of steps) arrive over time.  The loop keeps a single
``api.Batch`` on the GPU and, between chunks of steps:

  * admits waiting requests in arrival order while their device memory fits
    the budget (continuous batching: a request joins while others run); a
    request that would not fit even an empty batch is rejected;
  * enqueues a chunk of steps of every running scene (the call returns once
    the work is queued, so the host builds the next scenes while the GPU
    computes);
  * retires finished requests, reading their result back, and records the
    latency from arrival to the result on the host.

``run`` returns per-request records and the aggregate numbers (p50/p99
latency, particle-steps/s).  All state stays on the device between steps.
"""
from __future__ import annotations

import collections
import dataclasses
import math
import time
from typing import Callable, Dict, List, Optional

import numpy as np

from . import api, scenes


@dataclasses.dataclass
class Request:
    rid: int
    arrival: float          # seconds after the start of the run
    spec: scenes.MixedSpec  # the scene; spec.steps = steps asked for


@dataclasses.dataclass
class Result:
    rid: int
    n: int
    steps: int
    arrival: float
    admitted: float
    finished: float
    state: Optional[Dict[str, np.ndarray]] = None  # fields by particle id, when kept

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def poisson_requests(rate: float, duration: float, seed: int = 2, n_lo: int = 10000, n_hi: int = 500000,
                     steps_lo: int = 500, steps_hi: int = 5000) -> List[Request]:
    """Poisson arrivals at `rate` per second over `duration` seconds; scenes of
    log-uniform size in [n_lo, n_hi] asking for U[steps_lo, steps_hi] steps."""
    rng = np.random.Generator(np.random.PCG64(seed))
    t, times = 0.0, []
    while True:
        t += float(rng.exponential(1.0 / rate))
        if t > duration:
            break
        times.append(t)
    specs = scenes.mixed_specs(len(times), seed=seed + 1, n_lo=n_lo, n_hi=n_hi, steps_lo=steps_lo,
                               steps_hi=steps_hi)
    return [Request(rid=k, arrival=times[k], spec=specs[k]) for k in range(len(times))]


def grid_cells(scene) -> int:
    """Cell count mfree_set_grid derives from the scene's grid box (float32, as the library)."""
    lo = np.float32(np.asarray(scene.grid_bbmin, np.float64) - 1e-6)
    hi = np.float32(np.asarray(scene.grid_bbmax, np.float64) + 1e-6)
    dx = np.float32(scene.grid_h)
    n = [int(math.ceil(np.float32(hi[d] - lo[d]) / dx)) for d in range(3)]
    return n[0] * n[1] * n[2]


def scene_state(sim: api.Simulation, names=("POS", "VEL", "S", "T", "EPS_PL", "RHO")) -> Dict[str, np.ndarray]:
    ids = sim.get("ID").astype(np.int64)
    out = {}
    for name in names:
        a = sim.get(name)
        b = np.empty_like(a)
        b[ids] = a
        out[name] = b
    return out


class Server:
    """Continuous-batching request loop over one api.Batch."""

    def __init__(self, hbm_budget: int, chunk_steps: int = 50, use_graph: bool = True,
                 tiling: Optional[tuple] = None, keep_state: Callable[[Request], bool] = lambda r: False,
                 tool_bytes: int = 1 << 20, precision: int = 1):
        self.batch = api.Batch(hbm_budget=hbm_budget)
        self.budget = hbm_budget
        self.chunk = chunk_steps
        self.use_graph = use_graph
        self.keep_state = keep_state
        self.tool_bytes = tool_bytes
        self.precision = precision
        if tiling:
            self.batch.set_tiling(*tiling)

    def _fits(self, scene) -> bool:
        if not self.budget:
            return True
        need = api.scene_bytes(scene.pos.shape[0], grid_cells(scene)) + self.tool_bytes
        return self.batch.info()["bytes"] + need <= self.budget

    def run(self, requests: List[Request], clock: Callable[[], float] = time.perf_counter,
            horizon: Optional[float] = None) -> dict:
        pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
        waiting: collections.deque = collections.deque()
        active: Dict[int, tuple] = {}
        results: List[Result] = []
        rejected: List[Request] = []
        t0 = clock()
        psteps = 0
        chunks = 0
        queue_trace = []  # (time, requests arrived and waiting, requests running, running particles)
        while pending or waiting or active:
            now = clock() - t0
            if horizon is not None and now > horizon:
                break
            while pending and pending[0].arrival <= now:
                waiting.append(pending.popleft())
            # admission, in arrival order, while the budget allows
            while waiting:
                req = waiting[0]
                scene = scenes.mixed_scene(req.spec, precision=self.precision)
                if not self._fits(scene):
                    if self.batch.info()["scenes"] == 0:  # larger than the whole budget
                        rejected.append(waiting.popleft())
                        continue
                    break
                sim = api.Simulation.from_scene(scene)
                slot = self.batch.admit(sim, req.spec.steps)
                if slot is None:
                    sim.close()
                    if self.batch.info()["scenes"] == 0:
                        rejected.append(waiting.popleft())
                        continue
                    break
                waiting.popleft()
                active[slot] = (req, clock() - t0, sim)
            if not active:
                if pending:
                    time.sleep(max(0.0, min(0.05, pending[0].arrival - (clock() - t0))))
                continue
            queue_trace.append((clock() - t0, len(waiting), len(active),
                                sum(v[2].n_init for v in active.values())))
            # a chunk of steps (the batch stops each scene at its own count)
            before = {s: self.batch.query(s)[0] for s in active}
            self.batch.step(self.chunk, record_every=0, use_graph=self.use_graph)
            chunks += 1
            for slot in list(active):
                done, target, status = self.batch.query(slot)
                psteps += (done - before[slot]) * active[slot][2].n_init
                if status == api.Batch.RUNNING:
                    continue
                req, t_adm, sim = active.pop(slot)
                if status < 0:
                    raise api.MfreeError(status, f"request {req.rid} failed")
                state = scene_state(sim) if self.keep_state(req) else None
                sim.get("POS")  # the result read-back completes the request
                finished = clock() - t0
                self.batch.retire(slot)
                results.append(Result(rid=req.rid, n=sim.n_init, steps=int(done), arrival=req.arrival,
                                      admitted=t_adm, finished=finished, state=state))
        elapsed = clock() - t0
        lat = np.array([r.latency for r in results]) if results else np.zeros(0)
        # requests still queued or running when the loop stops are censored: their
        # latency is at least the time they have waited so far
        unfinished = [v[0] for v in active.values()] + list(waiting) + [r for r in pending if r.arrival <= elapsed]
        cens = np.array([elapsed - r.arrival for r in unfinished]) if unfinished else np.zeros(0)
        both = np.concatenate([lat, cens])
        return dict(
            results=results,
            completed=len(results),
            offered=len(requests),
            rejected=len(rejected),
            unfinished=len(active) + len(waiting) + len(pending),
            elapsed_s=elapsed,
            particle_steps=psteps,
            particle_steps_per_s=psteps / elapsed if elapsed > 0 else 0.0,
            p50_s=float(np.percentile(lat, 50)) if lat.size else None,
            p99_s=float(np.percentile(lat, 99)) if lat.size else None,
            # p50/p99 over completed and censored requests, the censored ones at
            # their lower bound (a lower bound of the true percentiles)
            p50_censored_s=float(np.percentile(both, 50)) if both.size else None,
            p99_censored_s=float(np.percentile(both, 99)) if both.size else None,
            censored=int(cens.size),
            queue_trace=queue_trace,
            chunks=chunks,
        )

    def close(self):
        self.batch.close()
