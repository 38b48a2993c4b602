"""Continuous-batching server for scene-step requests.

A request is a new scene plus a number of steps K.  The server keeps every admitted scene
resident on the device and, every tick:

  1. admits waiting requests in arrival order while their footprint fits the HBM budget
     (``ar_scene_footprint``, which counts the scene's state and its share of the step
     workspace) and the batch stays within its particle and cell limits -- admission is
     never blocked by a request that arrived later;
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

import contextlib
import ctypes as C
import heapq
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import api
from ._lib import AR_MAX_BATCH_CELLS, AR_MAX_BATCH_PARTICLES, lib
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
    host_s: dict = field(default_factory=dict)  # host seconds per loop phase

    def summary(self) -> dict:
        lat = self.latencies
        return {
            "completed": self.completed, "offered": self.offered, "wall_s": self.wall_s,
            "scene_steps_per_s": self.scene_steps / self.wall_s if self.wall_s else 0.0,
            "mparticle_steps_per_s": self.particle_steps / self.wall_s / 1e6 if self.wall_s else 0.0,
            "p50_latency_s": float(np.percentile(lat, 50)) if len(lat) else None,
            "p99_latency_s": float(np.percentile(lat, 99)) if len(lat) else None,
            "peak_resident_scenes": self.peak_resident, "peak_resident_bytes": self.peak_bytes,
            "ticks": self.ticks, "host_s": self.host_s,
        }


class Server:
    """Continuous-batching request loop.

    Admission needs the request's footprint to fit the HBM budget and the resident batch to
    stay within the library's batch limits (AR_MAX_BATCH_PARTICLES particles and
    AR_MAX_BATCH_CELLS grid cells) and the optional ``max_batch_particles`` cap.
    ``scene_factory(ctx, scene)`` and ``batch`` default to the device classes; they are
    parameters so that the admission and tick logic can be driven by host-only stand-ins."""

    def __init__(self, ctx, hbm_budget_bytes: float, tick_steps: int = 10,
                 keep_results: bool = False, max_batch_particles: int | None = None,
                 broadphase: str = "grid", scene_factory=None, batch=None, stream=None):
        self.ctx = ctx
        self.budget = float(hbm_budget_bytes)
        self.tick_steps = int(tick_steps)
        self.keep_results = keep_results
        self.max_particles = min(int(max_batch_particles or AR_MAX_BATCH_PARTICLES),
                                 AR_MAX_BATCH_PARTICLES)
        self.broadphase = broadphase
        self.scene_factory = scene_factory or (
            lambda c, sc: api.GpuScene(c, sc, broadphase=self.broadphase))
        self.batch = batch if batch is not None else api.Batch(ctx)
        self.stream = stream if stream is not None else torch.cuda.Stream()

    def cost(self, scene: Scene) -> tuple[int, int]:
        """(device bytes, grid cells) a scene holds while resident."""
        d = api.make_desc(scene, api.broadphase_code(self.broadphase))
        return int(lib.ar_scene_footprint(C.byref(d))), int(lib.ar_scene_cells(C.byref(d)))

    def _fits(self, used, need) -> bool:
        return (used[0] + need[0] <= self.budget and used[1] + need[1] <= AR_MAX_BATCH_CELLS
                and used[2] + need[2] <= self.max_particles)

    def run(self, requests: list[Request], time_limit: float | None = None) -> ServerStats:
        pending = list(requests)
        heapq.heapify(pending)
        waiting: list[Request] = []
        active: list[list] = []  # [req, scene, remaining, (bytes, cells, particles)]
        used = [0, 0, 0]
        done: list[Request] = []
        scene_steps = particle_steps = 0
        peak_res = peak_bytes = ticks = 0
        phase = {"admit": 0.0, "set_scenes": 0.0, "step": 0.0, "retire": 0.0}
        t0 = time.perf_counter()
        stream_ctx = torch.cuda.stream(self.stream) if isinstance(self.stream, torch.cuda.Stream) \
            else contextlib.nullcontext()
        with stream_ctx:
            while pending or waiting or active:
                now = time.perf_counter() - t0
                if time_limit is not None and now > time_limit and not active:
                    break
                while pending and pending[0].arrival <= now:
                    waiting.append(heapq.heappop(pending))
                changed = False
                while waiting and (time_limit is None or now <= time_limit):
                    nbytes, cells = self.cost(waiting[0].scene)
                    need = (nbytes, cells, waiting[0].scene.num_particles)
                    if not self._fits(used, need):
                        if active:
                            break  # wait for resident scenes to retire
                        if need[1] > AR_MAX_BATCH_CELLS or need[2] > self.max_particles:
                            raise ValueError(f"request {waiting[0].rid} can never be admitted")
                    req = waiting.pop(0)
                    ta = time.perf_counter()
                    gs = self.scene_factory(self.ctx, req.scene)
                    phase["admit"] += time.perf_counter() - ta
                    req.admitted = time.perf_counter() - t0
                    active.append([req, gs, req.steps, need])
                    used = [u + x for u, x in zip(used, need)]
                    changed = True
                if not active:
                    if pending:  # idle until the next arrival
                        time.sleep(max(0.0, min(0.001, pending[0].arrival - now)))
                    continue
                tb = time.perf_counter()
                if changed or ticks == 0:
                    self.batch.set_scenes([a[1] for a in active])
                k = min(self.tick_steps, min(a[2] for a in active))
                tc = time.perf_counter()
                self.batch.step(k, use_graph=True, stream=self.stream)
                td = time.perf_counter()
                phase["set_scenes"] += tc - tb
                phase["step"] += td - tc
                ticks += 1
                peak_res = max(peak_res, len(active))
                peak_bytes = max(peak_bytes, used[0])
                finished = []
                for a in active:
                    scene_steps += k
                    particle_steps += k * a[0].scene.num_particles
                    a[2] -= k
                    if a[2] <= 0:
                        finished.append(a)
                if finished:
                    tr = time.perf_counter()
                    self.stream.synchronize()
                    tdone = time.perf_counter() - t0
                    for req, gs, _, need in finished:
                        req.done = tdone
                        if self.keep_results:
                            req.result = gs.download()
                        gs.close()
                        used = [u - x for u, x in zip(used, need)]
                        done.append(req)
                    active = [a for a in active if a[2] > 0]
                    self.batch.set_scenes([a[1] for a in active])
                    phase["retire"] += time.perf_counter() - tr
            self.stream.synchronize()
        wall = time.perf_counter() - t0
        self.ctx.check(self.stream)
        lat = np.array([r.done - r.arrival for r in done])
        return ServerStats(len(done), len(requests), wall, scene_steps, particle_steps, lat,
                           peak_res, peak_bytes, ticks, phase)

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
