"""Continuous-batching server for scene-step requests.

A request is a new scene plus a number of steps K.  The server keeps every admitted scene
resident on the device and, every tick:

  1. admits waiting requests in arrival order while their footprint fits the HBM budget
     (``ar_scene_footprint``, which counts the scene's state and its share of the step
     workspace) -- admission is never blocked by a request that arrived later;
  2. advances all resident scenes together as one batch (``ar_batch_step``: one launch per
     stage, CUDA graph) by ``min(tick_steps, smallest remaining K)`` steps, so no scene is
     stepped past its K;
  3. retires finished scenes (their device memory is freed and reused by the next admissions)
     and records completion times.

Batching is continuous: a request arriving while others run joins the next tick without
waiting for the batch to drain.  Because every scene occupies its own key range in the
batch's sort, a scene's result does not depend on which other scenes shared its batches.

Latency = completion - arrival (queueing + service).  Times are wall-clock on the host;
arrivals are scheduled against the same clock.
"""
from __future__ import annotations

import heapq
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import api
from ._lib import lib
from .scenes import Scene


@dataclass(order=True)
class Request:
    arrival: float
    rid: int
    scene: Scene = field(compare=False)
    steps: int = field(compare=False)
    # filled in by the server
    admitted: float = field(default=-1.0, compare=False)
    done: float = field(default=-1.0, compare=False)
    result: dict | None = field(default=None, compare=False)


@dataclass
class ServerStats:
    completed: int
    offered: int
    wall_s: float
    scene_steps: int
    particle_steps: int
    latencies: np.ndarray
    peak_resident: int
    peak_bytes: int
    ticks: int

    def summary(self) -> dict:
        lat = self.latencies
        return {
            "completed": self.completed, "offered": self.offered, "wall_s": self.wall_s,
            "scene_steps_per_s": self.scene_steps / self.wall_s if self.wall_s else 0.0,
            "mparticle_steps_per_s": self.particle_steps / self.wall_s / 1e6 if self.wall_s else 0.0,
            "p50_latency_s": float(np.percentile(lat, 50)) if len(lat) else None,
            "p99_latency_s": float(np.percentile(lat, 99)) if len(lat) else None,
            "peak_resident_scenes": self.peak_resident, "peak_resident_bytes": self.peak_bytes,
            "ticks": self.ticks,
        }


class Server:
    def __init__(self, ctx: api.Context, hbm_budget_bytes: float, tick_steps: int = 10,
                 keep_results: bool = False):
        self.ctx = ctx
        self.budget = float(hbm_budget_bytes)
        self.tick_steps = int(tick_steps)
        self.keep_results = keep_results
        self.batch = api.Batch(ctx)
        self.stream = torch.cuda.Stream()

    @staticmethod
    def footprint(scene: Scene) -> int:
        import ctypes as C
        d = api.make_desc(scene)
        return int(lib.ar_scene_footprint(C.byref(d)))

    def run(self, requests: list[Request], time_limit: float | None = None) -> ServerStats:
        pending = list(requests)
        heapq.heapify(pending)
        waiting: list[Request] = []
        active: list[tuple[Request, api.GpuScene, int, int]] = []  # req, scene, remaining, bytes
        used = 0
        done: list[Request] = []
        scene_steps = particle_steps = 0
        peak_res = peak_bytes = ticks = 0
        t0 = time.perf_counter()
        with torch.cuda.stream(self.stream):
            while pending or waiting or active:
                now = time.perf_counter() - t0
                if time_limit is not None and now > time_limit and not active:
                    break
                while pending and pending[0].arrival <= now:
                    waiting.append(heapq.heappop(pending))
                changed = False
                while waiting and (time_limit is None or now <= time_limit):
                    need = self.footprint(waiting[0].scene)
                    if used + need > self.budget and active:
                        break  # wait for memory to free up
                    req = waiting.pop(0)
                    gs = api.GpuScene(self.ctx, req.scene)
                    req.admitted = time.perf_counter() - t0
                    active.append((req, gs, req.steps, need))
                    used += need
                    changed = True
                if not active:
                    if pending:  # idle until the next arrival
                        time.sleep(max(0.0, min(0.001, pending[0].arrival - now)))
                    continue
                if changed or ticks == 0:
                    self.batch.set_scenes([a[1] for a in active])
                k = min(self.tick_steps, min(a[2] for a in active))
                self.batch.step(k, use_graph=True, stream=self.stream)
                ticks += 1
                peak_res = max(peak_res, len(active))
                peak_bytes = max(peak_bytes, used)
                still = []
                finished = []
                for req, gs, rem, nbytes in active:
                    scene_steps += k
                    particle_steps += k * gs.num_particles
                    if rem - k <= 0:
                        finished.append((req, gs, nbytes))
                    else:
                        still.append((req, gs, rem - k, nbytes))
                if finished:
                    self.stream.synchronize()
                    tdone = time.perf_counter() - t0
                    for req, gs, nbytes in finished:
                        req.done = tdone
                        if self.keep_results:
                            req.result = gs.download()
                        gs.close()
                        used -= nbytes
                        done.append(req)
                    active = still
                    self.batch.set_scenes([a[1] for a in active])
                else:
                    active = still
            self.stream.synchronize()
        wall = time.perf_counter() - t0
        self.ctx.check(self.stream)
        lat = np.array([r.done - r.arrival for r in done])
        return ServerStats(len(done), len(requests), wall, scene_steps, particle_steps, lat,
                           peak_res, peak_bytes, ticks)

    def close(self) -> None:
        self.batch.close()


def poisson_requests(rate_per_s: float, duration_s: float, make, seed: int = 0) -> list[Request]:
    """Poisson arrivals over [0, duration); make(rng) -> (Scene, K)."""
    rng = np.random.default_rng(seed)
    t, out, rid = 0.0, [], 0
    while True:
        t += rng.exponential(1.0 / rate_per_s)
        if t >= duration_s:
            break
        scene, k = make(rng)
        out.append(Request(t, rid, scene, k))
        rid += 1
    return out
