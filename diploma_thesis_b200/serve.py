"""Continuous-batching server for scene-step requests.

``NativeServer`` runs the request loop in C++ (``ar_server_run``, csrc/ar_serve.cu): request
templates stay resident on the device and an admission is a device-side clone.  ``Server`` is
the same policy written over the Python binding; its scene, batch and stream objects are
parameters, so its admission and tick logic is tested on the CPU with host-only stand-ins.

A request is a new scene plus a number of steps K.  The server keeps every admitted scene
resident on the device and runs fixed-size ticks of ``tick_steps`` batch steps:

  1. admits waiting requests in arrival order while their footprint fits the HBM budget
     (``ar_scene_footprint``, which counts the scene's state and its share of the step
     workspace) and the batch stays within its particle and cell limits -- admission is
     never blocked by a request that arrived later.  New scenes are uploaded on a separate
     admission stream; the compute stream waits for the upload before the next tick;
  2. advances all resident scenes together as one batch (``ar_batch_step``: one launch per
     stage, CUDA graph) with a step budget per scene (``ar_batch_set_scenes_limited``): a
     scene whose K runs out inside a tick is frozen on the device after exactly K steps;
  3. queues, on the compute stream behind the tick, the copy of each finished scene's state
     into pinned host memory; at the next member change the finished scenes leave the batch
     and their memory is released in stream order (``ar_scene_destroy_async``) for the next
     admissions.  A request completes when the host sees its copy done.

The host never waits for the tick it has just queued: it runs at most ``max_inflight`` ticks
ahead of the device, so admission (scene building and upload) overlaps device work.
Because every scene occupies its own key range in the batch's sort and frozen scenes do not
change, a scene's result does not depend on which other scenes shared its batches.

Latency = completion - arrival (queueing + service).  Times are wall-clock on the host;
arrivals are scheduled against the same clock.
"""
from __future__ import annotations

import ctypes as C
import heapq
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import api
from ._lib import AR_MAX_BATCH_CELLS, AR_MAX_BATCH_PARTICLES, ServerStatsC, call, lib
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
    ``scene_factory(ctx, scene, stream)``, ``batch`` and the streams default to the device
    classes; they are parameters so that the admission and tick logic can be driven by
    host-only stand-ins (objects with the same methods)."""

    def __init__(self, ctx, hbm_budget_bytes: float, tick_steps: int = 10,
                 keep_results: bool = False, max_batch_particles: int | None = None,
                 broadphase: str = "grid", scene_factory=None, batch=None, stream=None,
                 admission_stream=None, max_inflight: int = 2):
        self.ctx = ctx
        self.budget = float(hbm_budget_bytes)
        self.tick_steps = int(tick_steps)
        self.keep_results = keep_results
        self.max_particles = min(int(max_batch_particles or AR_MAX_BATCH_PARTICLES),
                                 AR_MAX_BATCH_PARTICLES)
        self.broadphase = broadphase
        self.max_inflight = max(1, int(max_inflight))
        self.scene_factory = scene_factory or (
            lambda c, sc, st: api.GpuScene(c, sc, broadphase=self.broadphase, stream=st))
        self.batch = batch if batch is not None else api.Batch(ctx)
        self.stream = stream if stream is not None else torch.cuda.Stream()
        self.adm_stream = admission_stream if admission_stream is not None else (
            torch.cuda.Stream() if isinstance(self.stream, torch.cuda.Stream) else self.stream)

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
        active: list[list] = []    # [req, scene, steps left, (bytes, cells, particles)]
        retiring: list[list] = []  # [req, scene, need, host copy, copy-done event]
        leaving: list = []         # finished scenes still members of the batch
        inflight: list = []        # events of queued ticks, oldest first
        used = [0, 0, 0]
        done: list[Request] = []
        scene_steps = particle_steps = 0
        peak_res = peak_bytes = ticks = 0
        changed = False
        phase = {"admit": 0.0, "set_scenes": 0.0, "step": 0.0, "retire": 0.0, "wait": 0.0}
        t0 = time.perf_counter()
        while pending or waiting or active or retiring:
            now = time.perf_counter() - t0
            while pending and pending[0].arrival <= now:
                waiting.append(heapq.heappop(pending))
            # ---- admission (overlaps the ticks in flight) ----
            ta = time.perf_counter()
            admitted = False
            while waiting and (time_limit is None or now <= time_limit):
                nbytes, cells = self.cost(waiting[0].scene)
                need = (nbytes, cells, waiting[0].scene.num_particles)
                if not self._fits(used, need):
                    if active or retiring:
                        break  # wait for resident scenes to retire
                    if need[1] > AR_MAX_BATCH_CELLS or need[2] > self.max_particles:
                        raise ValueError(f"request {waiting[0].rid} can never be admitted")
                req = waiting.pop(0)
                gs = self.scene_factory(self.ctx, req.scene, self.adm_stream)
                req.admitted = time.perf_counter() - t0
                active.append([req, gs, req.steps, need])
                used = [u + x for u, x in zip(used, need)]
                admitted = changed = True
            if admitted and self.adm_stream is not self.stream:
                self.stream.wait_event(self.adm_stream.record_event())
            phase["admit"] += time.perf_counter() - ta
            # ---- retire: finished copies the host can see ----
            tr = time.perf_counter()
            still = []
            for item in retiring:
                req, gs, need, host, ev = item
                if ev.query():
                    req.done = time.perf_counter() - t0
                    if self.keep_results:
                        req.result = {k: v.copy() for k, v in host.items() if k != "_pinned"}
                    used = [u - x for u, x in zip(used, need)]
                    done.append(req)
                else:
                    still.append(item)
            retiring = still
            phase["retire"] += time.perf_counter() - tr
            if not active:
                if retiring:  # nothing to step: wait for the oldest copy
                    tw = time.perf_counter()
                    retiring[0][4].synchronize()
                    phase["wait"] += time.perf_counter() - tw
                elif pending:  # idle until the next arrival
                    time.sleep(max(0.0, min(0.001, pending[0].arrival - now)))
                elif time_limit is not None and now > time_limit:
                    break
                if leaving and not active:
                    self.batch.set_scenes([])
                    for gs in leaving:
                        gs.close_async(self.stream)
                    leaving = []
                continue
            # ---- queue one tick ----
            tb = time.perf_counter()
            if changed or ticks == 0:
                self.batch.set_scenes([a[1] for a in active], [a[2] for a in active])
                changed = False
                for gs in leaving:  # no longer members: free behind the ticks that used them
                    gs.close_async(self.stream)
                leaving = []
            phase["set_scenes"] += time.perf_counter() - tb
            tw = time.perf_counter()
            while len(inflight) >= self.max_inflight:
                inflight.pop(0).synchronize()
            phase["wait"] += time.perf_counter() - tw
            tc = time.perf_counter()
            k = self.tick_steps
            self.batch.step(k, use_graph=True, stream=self.stream)
            ticks += 1
            peak_res = max(peak_res, len(active))
            peak_bytes = max(peak_bytes, used[0])
            finished = []
            for a in active:
                n = min(k, a[2])
                scene_steps += n
                particle_steps += n * a[0].scene.num_particles
                a[2] -= k
                if a[2] <= 0:
                    finished.append(a)
            for req, gs, _, need in finished:  # frozen on the device after exactly K steps
                host = gs.download_async(self.stream)
                retiring.append([req, gs, need, host, self.stream.record_event()])
                leaving.append(gs)
            if finished:
                active = [a for a in active if a[2] > 0]
                changed = True
            inflight.append(self.stream.record_event())
            phase["step"] += time.perf_counter() - tc
        if leaving:
            self.batch.set_scenes([])
            for gs in leaving:
                gs.close_async(self.stream)
        self.stream.synchronize()
        wall = time.perf_counter() - t0
        self.ctx.check(self.stream)
        lat = np.array([r.done - r.arrival for r in done])
        return ServerStats(len(done), len(requests), wall, scene_steps, particle_steps, lat,
                           peak_res, peak_bytes, ticks, phase)

    def close(self) -> None:
        self.batch.close()


class NativeServer:
    """The continuous-batching loop in C++ (ar_server_create / ar_server_add_template /
    ar_server_run): the same policy as ``Server`` -- admission in arrival order by HBM budget
    and batch limits, ticks of ``tick_steps`` batch steps with a step budget per scene, state
    copies behind the tick, at most ``max_inflight`` ticks queued ahead -- with no Python in the
    loop.  Each distinct scene of the requests becomes a resident template once; admitting a
    request clones its template on the device."""

    def __init__(self, ctx, hbm_budget_bytes: float, tick_steps: int = 10,
                 max_batch_particles: int | None = None, max_inflight: int = 2,
                 broadphase: str = "grid"):
        self.ctx = ctx
        self.broadphase = api.broadphase_code(broadphase)
        self.handle = C.c_void_p()
        call("ar_server_create", ctx.handle, C.c_double(hbm_budget_bytes), int(tick_steps),
             C.c_longlong(int(max_batch_particles or 0)), int(max_inflight),
             C.byref(self.handle))
        self._templates: dict[int, int] = {}  # id(Scene) -> template index
        self._keep: list = []

    def template(self, scene: Scene) -> int:
        key = id(scene)
        if key not in self._templates:
            desc = api.make_desc(scene, self.broadphase)
            arrays = [np.ascontiguousarray(a) for a in (
                scene.body_pos, scene.body_quat, scene.body_vel, scene.body_angvel,
                scene.body_mass.astype(np.float32), scene.body_inv_inertia.astype(np.float32),
                scene.body_offsets.astype(np.int32), scene.particle_rel)]
            init = api.SceneInit(*[C.c_void_p(a.ctypes.data) for a in arrays])
            tid = C.c_int()
            call("ar_server_add_template", self.handle, C.byref(desc), C.byref(init),
                 C.byref(tid))
            self._templates[key] = tid.value
            self._keep.append(scene)  # the id stays unique while the scene lives
        return self._templates[key]

    def run(self, requests: list[Request], time_limit: float | None = None,
            keep_results: bool = False) -> ServerStats:
        n = len(requests)
        tids = np.array([self.template(r.scene) for r in requests], np.int32)
        steps = np.array([r.steps for r in requests], np.int32)
        arrival = np.array([r.arrival for r in requests], np.float64)
        latency = np.full(n, -1.0)
        results = None
        pinned = []
        if keep_results:
            ptrs = []
            for r in requests:
                t = torch.empty((4, r.scene.num_bodies, 4), dtype=torch.float32, pin_memory=True)
                pinned.append(t)
                ptrs.append(t.data_ptr())
            results = (C.c_void_p * max(1, n))(*ptrs)
        st = ServerStatsC()
        call("ar_server_run", self.handle, n, C.c_void_p(tids.ctypes.data),
             C.c_void_p(steps.ctypes.data), C.c_void_p(arrival.ctypes.data),
             C.c_double(-1.0 if time_limit is None else float(time_limit)), results,
             C.c_void_p(latency.ctypes.data), C.byref(st))
        done = []
        for i, r in enumerate(requests):
            if latency[i] >= 0:
                r.done = r.arrival + latency[i]
                done.append(latency[i])
                if keep_results:
                    packed = pinned[i].numpy()  # [4, B, 4]: pos, quat, vel, angvel
                    r.result = {k: packed[j].copy() for j, k in
                                enumerate(("pos", "quat", "vel", "angvel"))}
        host = {"admit": st.host_admit_s, "set_scenes": st.host_set_s, "step": st.host_step_s,
                "retire": st.host_retire_s, "wait": st.host_wait_s}
        return ServerStats(st.completed, st.offered, st.wall_s, st.scene_steps,
                           st.particle_steps, np.array(done), st.peak_resident, st.peak_bytes,
                           st.ticks, host)

    def close(self) -> None:
        if self.handle:
            call("ar_server_destroy", self.handle)
            self.handle = C.c_void_p()


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
