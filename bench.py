"""Benchmark of the fused rigid-body step (one JSON line on stdout).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload pile|plain]

Workload (default "pile"): the plain large pile -- 2,097,152 particles, 32,768 bodies of 64
(cubes, rods, padded spheres), r = 1/512, 1 x 3 x 1 box, dt = 1e-4, k = 5e4, damping 0.02,
shear 0.1, grid broad phase (256 x 512 x 256 wrapped cells of 2r).  "plain" is the 110,592-particle
single scene (4,096 cubes, 128^3 grid); "sis" the reference's sequential-impulse update path
(REFERENCE semantics) on 4,096 packed cubes.  Seeded synthetic scenes; no dataset exists.

Metric: Mparticle-steps/s (whole job).  A step is one pass of the fused pipeline over the
scene.  value: device-timed throughput with the scene resident in HBM (K graph replays
between CUDA events, barrier + synchronise on both sides, max over ranks); e2e: the same
metric through the public API with the body state uploaded from pinned host memory and
downloaded back every step.  N > 1 runs independent replicas, one per GPU (weak scaling).

The reference arm (--impl reference) times the reference's own kernel bodies on the host
cores (oracle/_ref/libref_cpu.so, OpenMP) on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

PEAKS = ROOT / "MEASURED_PEAKS.json"
FALLBACK_HBM_GBS = 6650.0

# Algorithmic bytes per particle and per body for each stage of the fused step (compulsory
# traffic of this design: every array element read or written once; neighbour reads that hit
# in L2 are not counted).  P = sort passes, ppb = particles per body.  A step runs: clear |
# keys | sort | scatter + cell table | collide | body (sums, integration).
STAGES = ["clear", "keys", "sort", "scatter", "collide", "body"]
# Steps each configuration runs (c2 pile: 500; c0 plain scene: 1,000).
CONFIG_STEPS = {"pile": 500, "plain": 1000}
BODY_STATE = 16 * 4  # pos, quat, vel, angvel (float4 each)


def _body_bytes(nb: int) -> int:
    # state + mass + inverse inertia in, state + force / torque sums out
    return nb * (BODY_STATE + 4 + 36 + BODY_STATE + 32)


def sort_passes(bits: int) -> int:
    """Digit passes of the radix sort over `bits` key bits (8-bit digits, 9 where that saves
    a pass: 24 bits -> 3, 25 -> 3, 30 -> 4, 63 -> 7)."""
    return (bits + 8) // 9 if bits > 0 else 0


def stage_bytes(n: int, nb: int, passes: int, occupied_cells: int,
                cells: int = 0) -> dict[str, float]:
    """Algorithmic bytes of one grid step that re-sorts from the previous order (every step
    but the first after a change of the member list).  The movers' own bytes (about 1 % of the
    particles, 8-16 bytes each per kernel) are left out."""
    tiles = (n + 2047) // 2048
    return {
        # re-sort counters and bucket counts; one 255th of the 8-byte cell table
        "clear": 4 * (4 + 2 * 4096) + 8 * cells // 255,
        # rel in, key out; body pose (32) per body
        "keys": n * (16 + 4) + nb * 32,
        # movers: previous keys + indices in, new key gathered, mover bits out; placement:
        # previous keys + indices and mover bits in, keys + indices out; tile counts/headers
        "sort": n * (8 + 4 + 0.125) + n * (8 + 0.125 + 8) + tiles * 40,
        # sorted key + index and rel in, sorted position + velocity and the order kept for the
        # next step out; body state per body; one 8-byte cell entry per occupied cell
        "scatter": n * (8 + 16 + 32 + 8) + nb * BODY_STATE + occupied_cells * 8,
        # own key, index, position, velocity in; force out
        "collide": n * (4 + 4 + 32 + 16),
        # force + rel in; body state
        "body": n * (16 + 16) + _body_bytes(nb),
    }


BVH_STAGES = ["clear", "keys", "sort", "tree", "collide", "body"]


def stage_bytes_bvh(n: int, nb: int, passes: int, key_bits: int = 64) -> dict[str, float]:
    """The same accounting for the BVH broad phase (64-byte wide nodes).  Keys of up to 32 bits
    (up to four scenes) are re-sorted from the previous step's order after the first step
    (movers' own bytes left out); wider keys are radix-sorted as 64-bit keys."""
    tiles = (n + 8191) // 8192
    k32 = key_bits <= 32
    return {
        "clear": 4 * n + (4 * (4 + 2 * 4096) if k32 else 0),  # refit arrival counters
        # rel in, key out; body pose per body
        "keys": n * (16 + (4 if k32 else 8)) + nb * 32,
        # re-sort: previous keys + indices in, new key gathered, mover bits; placement: previous
        # keys + indices and bits in, keys + indices out.  Radix: histogram pass reads the keys;
        # first pass reads keys, every pass writes key + index, later passes read both
        "sort": (n * (8 + 4 + 0.125) + n * (8 + 0.125 + 8) + (n // 2048) * 40) if k32 else
                n * 8 + n * (8 + 12) + (passes - 1) * n * 24 + passes * 4 * 512 * tiles,
        # nodes: keys in, flags, children, parent, ranges and wide-node ids out; leaves: index,
        # rel in, sorted pos + vel and the leaf box out (and the order kept, 32-bit keys), body
        # state per body; refit: links and the node's two child boxes in, its box out
        "tree": n * ((4 if k32 else 8) + 21 + 8 + 8) + n * (4 + 16 + 32 + 24 + 9) +
                (n * 8 if k32 else 0) + nb * BODY_STATE + n * (8 + 64 + 24),
        # own index, position + velocity in; force out
        "collide": n * (4 + 32 + 16),
        "body": n * (16 + 16) + _body_bytes(nb),
    }


TRAFFIC = ROOT / "profiles" / "traffic.json"


def measured_traffic(workload: str, broadphase: str, kernel: str):
    """DRAM bytes (read + write) per launch of `kernel` from the committed ncu capture of this
    workload (profiles/traffic.json), with the capture it came from; None when there is none."""
    try:
        t = json.loads(TRAFFIC.read_text())[f"{workload}/{broadphase}/{kernel}"]
        return t["bytes_per_launch"], t["source"]
    except Exception:
        return None, None


def peaks() -> tuple[float, str]:
    if PEAKS.exists():
        try:
            return float(json.loads(PEAKS.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []
        self.first = 0           # index of the first sample at or after mark_start()
        self.last = None         # one past the last sample before mark_end()

    def mark_start(self):
        self.first = len(self.lines)

    def mark_end(self):
        self.last = len(self.lines)

    def samples_since_start(self) -> int:
        return len(self.lines) - self.first

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "20"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines[self.first:self.last]:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(max(mx)) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_scene(workload: str):
    from diploma_thesis_b200 import scenes
    if workload == "pile":
        return scenes.config2(0), ("plain large pile: 2,097,152 particles, 32,768 bodies x 64 "
                                   "(cubes/rods/spheres), r=1/512, box 1x3x1, grid 256x512x256 "
                                   "wrapped, dt=1e-4, k=5e4")
    if workload == "plain":
        return scenes.config0(0), ("plain single scene: 110,592 particles, 4,096 cubes x 27, "
                                   "r=1/256, unit box, grid 128^3, dt=1e-4, k=5e4")
    raise SystemExit(f"unknown workload {workload}")


def dist_setup(ngpus: int, backend: str = "nccl"):
    """Replicas: one process per GPU (RANK / LOCAL_RANK / WORLD_SIZE from torchrun); the
    process group only carries the barrier and the max-over-ranks timing, never data."""
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        from datetime import timedelta
        if backend == "nccl":
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                    device_id=torch.device(f"cuda:{local}"))
        else:
            dist.init_process_group(backend, timeout=timedelta(seconds=60))
    return world, rank, local


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(world: int, units_per_rank: int, steps: int, ms: float) -> float:
    """Whole-job throughput in millions of units per second: every rank processes
    units_per_rank per step, the time is the slowest rank's."""
    return world * units_per_rank * steps / (ms / 1e3) / 1e6


# ---- CPU legs (oracle) ---------------------------------------------------------------------
def cpu_reference_rate(scene, grid, target_s: float, broadphase: str = "grid",
                       warmup: int = 1, steps: int | None = None):
    """Particle-steps/s of the reference CPU step on the whole workload (every body of the
    scene): `warmup` untimed steps, then steps until `target_s` seconds have passed (or exactly
    `steps`).  Returns (rate, cores, kind, sample description, steps run, seconds)."""
    from oracle import ref
    from oracle.ref_step import ReferenceCPUStep, ReferenceCPUStepBVH
    if not ref.available():
        return None
    runner = (ReferenceCPUStepBVH if broadphase == "bvh" else ReferenceCPUStep)(scene, grid)
    cores = ref.max_threads()
    for _ in range(warmup):
        runner.step()
    t0 = time.perf_counter()
    k = 0
    while True:
        runner.step()
        k += 1
        el = time.perf_counter() - t0
        if (steps is not None and k >= steps) or (steps is None and el >= target_s):
            break
    rate = scene.num_particles * k / el
    where = "BVH" if broadphase == "bvh" else "grid"
    desc = (f"the whole workload ({scene.num_bodies} bodies, {scene.num_particles} particles), "
            f"{where} path, {k} timed steps after {warmup} untimed, {el:.1f} s")
    return rate, cores, "reference", desc, k, el


# ---- the reference arm -----------------------------------------------------------------------
def run_reference(args):
    """The reference's own kernel bodies (oracle/_ref/libref_cpu.so, OpenMP over all host
    cores) stepping the same scene as our arm.  Imports nothing from diploma_thesis_b200 but
    the pure-numpy scene generator."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import cpu, ref
    from oracle.ref_step import REFERENCE_SEMANTICS
    scene, desc = make_scene(args.workload)
    if args.broadphase == "bvh":
        desc = desc.replace("grid 256x512x256 wrapped", "BVH").replace("grid 128^3", "BVH")
    grid = cpu.scene_grid(scene)
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable":
                          "the reference CPU build (oracle/_ref/libref_cpu.so) is not present"}))
        return 0
    r = cpu_reference_rate(scene, grid, 0.0, args.broadphase, warmup=args.warmup,
                           steps=args.steps)
    rate, cores, kind, sample, k, el = r
    rate /= 1e6
    line = {"metric": "Mparticle-steps/s", "value": rate, "unit": "Mparticle-steps/s",
            "impl": "reference", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * el / k, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": desc, "broadphase": args.broadphase,
                       "particles": scene.num_particles, "bodies": scene.num_bodies,
                       "parallelism": f"host CPU, {cores} threads",
                       "semantics": REFERENCE_SEMANTICS},
            "cpu_baseline": {"value": rate, "unit": "Mparticle-steps/s", "cores": cores,
                             "kind": kind, "sample": sample},
            "e2e": {"value": rate, "unit": "Mparticle-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ---- our arm -----------------------------------------------------------------------------------
def run_ours(args):
    import torch
    world, rank, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    from diploma_thesis_b200 import api

    scene, desc = make_scene(args.workload)
    if args.broadphase == "bvh":
        desc = desc.replace("grid 256x512x256 wrapped", "BVH").replace("grid 128^3", "BVH")
    ctx = api.Context(local)
    gs = api.GpuScene(ctx, scene, broadphase=args.broadphase)
    n, nb = scene.num_particles, scene.num_bodies
    # the timed window sits in the middle of the configuration's run (contacts build up as the
    # bodies drift together), unless --start-step says otherwise
    run_len = CONFIG_STEPS.get(args.workload, args.steps)
    start_step = (args.start_step if args.start_step is not None
                  else max(0, (run_len - args.steps) // 2 - args.warmup))
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream), ClockSampler(local) as clocks:
        if start_step:
            gs.step(start_step, use_graph=True, stream=stream)
        gs.step(args.warmup, use_graph=True, stream=stream)
        stream.synchronize()
        ctx.check(stream)
        # ---- device-timed region: K graph replays ----
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier(world)
        torch.cuda.synchronize()
        clocks.mark_start()
        start.record(stream)
        gs.step(args.steps, use_graph=True, stream=stream)
        end.record(stream)
        end.synchronize()
        torch.cuda.synchronize()
        barrier(world)
        ms = start.elapsed_time(end)
        ctx.check(stream)
        # a timed region shorter than the sampling period gets no sample of its own: keep the
        # same step loop running (untimed, on a copy of the scene, so that the measured scene
        # is not advanced further) until the sampler has seen the GPU under this load
        if clocks.samples_since_start() < 5:
            twin = api.GpuScene(ctx, scene, broadphase=args.broadphase)
            twin.upload_state(gs.download_state(stream=stream), stream=stream)
            t_end = time.perf_counter() + 2.0
            while clocks.samples_since_start() < 5 and time.perf_counter() < t_end:
                twin.step(50, use_graph=True, stream=stream)
                stream.synchronize()
            twin.close()
        clocks.mark_end()
    ms = max_over_ranks(ms, world)
    ms_per_step = ms / args.steps
    value = job_rate(world, n, args.steps, ms)

    # ---- stage profile (event-bracketed eager steps right after the timed region) ----
    with torch.cuda.stream(stream):
        prof_steps = max(5, min(args.steps, 50))
        stage_ms = gs.profile(prof_steps, stream=stream)
    sv = gs.step_view()
    passes = sort_passes(sv.key_bits)
    if args.broadphase == "bvh":
        names = BVH_STAGES
        sbytes = stage_bytes_bvh(n, nb, passes, int(sv.key_bits))
    else:
        names = STAGES
        keys = api.device_view(sv.sorted_keys, n, torch.int32)
        occupied = int((keys[1:] != keys[:-1]).sum().item()) + 1
        sbytes = stage_bytes(n, nb, passes, occupied, int(sv.num_cells))
    hbm, peak_kind = peaks()
    dom = max(range(len(names)), key=lambda i: stage_ms[i])
    dom_name = names[dom]
    traffic, traffic_src = measured_traffic(args.workload, args.broadphase, dom_name)
    achieved = sbytes[dom_name] / (stage_ms[dom] / 1e3) / 1e9
    step_bytes = sum(sbytes.values())
    step_ms_prof = sum(stage_ms)

    # ---- end to end: host state in, step, host state out, every step ----
    e2e_steps = max(3, min(args.steps, 100))
    # body state (pos, quat, vel, angvel) in one pinned host array; each step uploads it,
    # steps, and returns only once the new state is back on the host
    pinned = torch.empty((4, nb, 4), dtype=torch.float32).pin_memory()
    host = pinned.numpy()
    gs.download_state(host, stream=stream)
    with torch.cuda.stream(stream):
        barrier(world)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):  # upload, one graph step, download: one library call
            gs.step_io(host, 1, host, stream=stream)
        torch.cuda.synchronize()
        e2e_s = time.perf_counter() - t0
        barrier(world)
    e2e_s = max_over_ranks(e2e_s, world)
    e2e_value = world * n * e2e_steps / e2e_s / 1e6

    # ---- CPU baseline (rank 0, N = 1) ----
    cpu_baseline = None
    if rank == 0 and world == 1 and not args.no_cpu:
        from oracle import cpu
        from oracle.ref_step import REFERENCE_SEMANTICS
        r = cpu_reference_rate(scene, cpu.scene_grid(scene), target_s=15.0,
                               broadphase=args.broadphase)
        if r is not None:
            rate, cores, kind, sample, k, el = r
            cpu_baseline = {"value": rate / 1e6, "unit": "Mparticle-steps/s", "cores": cores,
                            "kind": kind, "sample": sample, "semantics": REFERENCE_SEMANTICS}

    # memset nodes are not kernels: the BVH step has two (refit counters, sort head), the grid
    # step none (its clears are a kernel)
    memsets = 2 if args.broadphase == "bvh" else 0
    launches = args.steps * (gs.launches_per_step() - memsets)
    if rank == 0:
        line = {
            "metric": "Mparticle-steps/s", "value": value, "unit": "Mparticle-steps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": desc, "broadphase": args.broadphase, "particles": n,
                       "bodies": nb,
                       "timed_window": f"steps {start_step + args.warmup} to "
                                       f"{start_step + args.warmup + args.steps} of the "
                                       f"{run_len}-step run",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "l2": "per-step working set > 126 MB L2 (inputs larger than L2)",
                       "timed": "CUDA graph replays, events on the launching stream"},
            "roofline": {"bound": "hbm", "kernel": dom_name, "achieved": achieved,
                         "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                         "peak_kind": f"{peak_kind} hbm_gbs", "traffic": traffic,
                         "traffic_source": traffic_src,
                         "algorithmic_bytes_per_launch": sbytes[dom_name],
                         "launch_ms": stage_ms[dom]},
            "step_roofline": {"achieved": step_bytes / (ms_per_step / 1e3) / 1e9, "peak": hbm,
                              "unit": "GB/s", "frac": step_bytes / (ms_per_step / 1e3) / 1e9 / hbm,
                              "bytes_per_particle_step": step_bytes / n},
            "stages_ms": dict(zip(names, stage_ms)), "stage_profile_ms_per_step": step_ms_prof,
            "cpu_baseline": cpu_baseline,
            "e2e": {"value": e2e_value, "unit": "Mparticle-steps/s",
                    "h2d_bytes_per_step": 4 * 16 * nb, "d2h_bytes_per_step": 4 * 16 * nb,
                    "steps": e2e_steps},
            "gpu_launches": launches,
            "clocks": clocks.summary(),
        }
        print(json.dumps(line))
    gs.close()
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def _event_time(stream, fn) -> float:
    import torch
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record(stream)
    fn()
    b.record(stream)
    b.synchronize()
    return a.elapsed_time(b)


def run_batched(args):
    """Config 3: 256 independent scenes (log-uniform 2k-200k particles), batched (one launch
    per stage, CUDA graph) against the plain one-scene-at-a-time form on the same GPU."""
    import torch
    from diploma_thesis_b200 import api, autotune, scenes
    torch.cuda.set_device(0)
    ctx = api.Context(0)
    scs = scenes.config3(0)
    tuner = autotune.Tuner(ctx, args.tune_cache) if args.tune else None
    kws = [tuner.scene_kwargs(s) if tuner else {} for s in scs]
    groups = autotune.group(kws)
    if tuner:  # one launch per stage: a group uses the block size tuned for its median scene
        for idx in groups.values():
            med = sorted(scs[i].num_particles for i in idx)[len(idx) // 2]
            bs = tuner.choice(med).block_size
            for i in idx:
                kws[i]["block_size"] = bs
    n_total = sum(s.num_particles for s in scs)
    stream = torch.cuda.Stream()
    plain = [api.GpuScene(ctx, s, **kw) for s, kw in zip(scs, kws)]
    batch_scenes = [api.GpuScene(ctx, s, **kw) for s, kw in zip(scs, kws)]
    batches = [api.Batch(ctx, [batch_scenes[i] for i in idx]) for idx in groups.values()]
    k = args.steps
    with torch.cuda.stream(stream):
        for g in plain:
            g.step(args.warmup, use_graph=True, stream=stream)
        for b in batches:
            b.step(args.warmup, use_graph=True, stream=stream)
        stream.synchronize()

        def plain_steps():
            for _ in range(k):
                for g in plain:
                    g.step(1, use_graph=True, stream=stream)

        def batch_steps():
            for _ in range(k):
                for b in batches:
                    b.step(1, use_graph=True, stream=stream)

        ms_plain = _event_time(stream, plain_steps)
        ms_batch = _event_time(stream, batch_steps)
        ctx.check(stream)
    # same states after the same number of steps: batched == solo, bit for bit
    same = all(np.array_equal(a.download()["pos"], b.download()["pos"])
               for a, b in zip(plain[::32], batch_scenes[::32]))
    ss = len(scs) * k
    line = {"metric": "scene-steps/s (batched)", "value": ss / (ms_batch / 1e3),
            "unit": "scene-steps/s", "n_gpus": 1, "steps": k, "warmup": args.warmup,
            "ms_per_step": ms_batch / k, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "batched: 256 scenes, particle counts log-uniform in "
                                   "2k-200k (27-particle cubes), box side U[0.5,2]",
                       "particles": n_total, "autotuned": bool(tuner),
                       "broadphase_groups": {k2: len(v) for k2, v in groups.items()}},
            "plain": {"value": ss / (ms_plain / 1e3), "unit": "scene-steps/s",
                      "ms_per_step": ms_plain / k},
            "batched_over_plain": ms_plain / ms_batch,
            "mparticle_steps_per_s": {"batched": n_total * k / ms_batch / 1e3,
                                      "plain": n_total * k / ms_plain / 1e3},
            "batched_equals_plain": bool(same),
            "gpu_launches": {"batched_per_step": sum(b.launches_per_step() for b in batches),
                             "plain_per_step": sum(g.launches_per_step() for g in plain)}}
    print(json.dumps(line))
    for g in plain + batch_scenes:
        g.close()
    for b in batches:
        b.close()
    return 0


def lbvh_bytes(kb: int, passes: int) -> dict[str, float]:
    """Algorithmic bytes per point of the LBVH stages (kb = key bytes, 4 or 8)."""
    return {
        # AABB reads the points once; encoding reads them again and writes the key
        "encode": 16 + 16 + kb,
        # histogram pass reads the keys; first pass reads keys, every pass writes key + index,
        # later passes read both
        "sort": kb + kb + (kb + 4) + (passes - 1) * 2 * (kb + 4),
        # own and neighbour keys (L2 reuse not counted); per internal node: flag, children,
        # ranges, and the two children's parent links
        "build": kb + 1 + 16 + 8,
        # leaves: index and point in; centre, box, radius, flag and range out; refit per
        # internal node: links and both child boxes in, own box out
        "refit": (4 + 16 + 16 + 32 + 4 + 9) + (8 + 4 + 64 + 32),
    }


def run_lbvh(args):
    """Config 1: LBVH microbenchmark.  N = 2^20, 2^22, 2^24 points, uniform or a 16-component
    Gaussian mixture with 5 % exact duplicates, 30- and 63-bit Morton codes; encode (AABB +
    codes), sort, build and leaves + refit timed separately with CUDA events (median of the
    repetitions), each against the HBM roofline."""
    import torch
    from diploma_thesis_b200 import api, scenes
    from diploma_thesis_b200._lib import call
    torch.cuda.set_device(0)
    ctx = api.Context(0)
    P, S = api.ptr, api.stream_handle
    stream = torch.cuda.Stream()
    hbm, peak_kind = peaks()
    sizes = [1 << 20, 1 << 22, 1 << 24] if not args.lbvh_sizes else \
        [int(x) for x in args.lbvh_sizes.split(",")]
    rows = []
    for n in sizes:
        for dist in ("uniform", "gmm"):
            pts = torch.from_numpy(scenes.lbvh_points(n, dist, seed=1)).cuda()
            for wide in (False, True):
                kdt = torch.int64 if wide else torch.int32
                kb, bits = (8, 63) if wide else (4, 30)
                mn = torch.empty(4, device="cuda")
                mx = torch.empty(4, device="cuda")
                codes = torch.empty(n, dtype=kdt, device="cuda")
                skeys = torch.empty(n, dtype=kdt, device="cuda")
                svals = torch.empty(n, dtype=torch.int32, device="cuda")
                m = 2 * n - 1
                t = {k: torch.empty(m, dtype=torch.int32, device="cuda")
                     for k in ("left", "right", "parent", "min_r", "max_r")}
                leaf = torch.empty(m, dtype=torch.uint8, device="cuda")
                cms = torch.empty((n, 4), device="cuda")
                bounds = torch.empty((m, 8), device="cuda")
                radii = torch.empty(n, device="cuda")
                st = S(stream)

                def encode():
                    call("ar_scene_aabb", ctx.handle, P(pts), n, P(mn), P(mx), st)
                    call("ar_morton63" if wide else "ar_morton30", ctx.handle, P(pts), n, P(mn),
                         P(mx), P(codes), None, st)

                def sort():
                    call("ar_radix_sort_pairs_u64" if wide else "ar_radix_sort_pairs_u32",
                         ctx.handle, P(codes), None, P(skeys), P(svals), n, 0, bits, st)

                def build():
                    call("ar_lbvh_build64" if wide else "ar_lbvh_build", ctx.handle, P(skeys), n,
                         P(leaf), P(t["left"]), P(t["right"]), P(t["parent"]), P(t["min_r"]),
                         P(t["max_r"]), st)

                def refit():
                    call("ar_lbvh_leaves", ctx.handle, n, P(svals), P(pts), 1e-3, P(leaf),
                         P(t["min_r"]), P(t["max_r"]), P(cms), P(bounds), P(radii), st)
                    call("ar_lbvh_refit", ctx.handle, n, P(t["left"]), P(t["right"]),
                         P(t["parent"]), P(bounds), st)

                stages = {"encode": encode, "sort": sort, "build": build, "refit": refit}
                times = {k: [] for k in stages}
                with torch.cuda.stream(stream):
                    for rep in range(args.warmup + args.lbvh_reps):
                        for name, fn in stages.items():
                            ms = _event_time(stream, fn)
                            if rep >= args.warmup:
                                times[name].append(ms)
                    ctx.check(stream)
                    ok = bool((skeys[1:] >= skeys[:-1]).all().item())
                med = {k: float(np.median(v)) for k, v in times.items()}
                total = sum(med.values())
                by = lbvh_bytes(kb, sort_passes(bits))
                rows.append({
                    "n": n, "dist": dist, "bits": bits, "ms": med, "total_ms": total,
                    "mpoints_per_s": n / total / 1e3,
                    "roofline_frac": {k: by[k] * n / (med[k] / 1e3) / 1e9 / hbm for k in med},
                    "sorted": ok})
                del codes, skeys, svals, t, leaf, cms, bounds, radii
            del pts
            torch.cuda.empty_cache()
    big = [r for r in rows if r["n"] == max(sizes)]
    head = max(big, key=lambda r: r["mpoints_per_s"])
    # reference kernel bodies on the host cores: findAABBCub, generateMortonCodes, the CUB-order
    # stable sort, kernelConstructRadixTreeSoA, leaf and internal nodes (2^20 uniform points)
    cpu_baseline = None
    if not args.no_cpu:
        from oracle import ref
        if ref.available():
            pts = scenes.lbvh_points(1 << 20, "uniform", seed=1)
            k, t0 = 0, time.perf_counter()
            while time.perf_counter() - t0 < 10.0 or k == 0:
                mn, mx = ref.aabb(pts)
                codes, idx = ref.morton30(pts, mn, mx)
                sk, si = ref.sort_pairs_u32(codes, idx)
                tree = ref.radix_tree(sk)
                ref.leaves_and_refit(tree, si, pts, 1e-3)
                k += 1
            el = time.perf_counter() - t0
            cpu_baseline = {"value": k * len(pts) / el / 1e6, "unit": "Mpoints/s",
                            "cores": ref.max_threads(), "kind": "reference",
                            "sample": f"2^20 uniform points, 30-bit, {k} builds in {el:.1f} s"}
    line = {"metric": "Mpoints/s (LBVH encode+sort+build+refit)", "value": head["mpoints_per_s"],
            "unit": "Mpoints/s", "n_gpus": 1, "higher_is_better": True, "dtype": "f32",
            "data": "synthetic", "warmup": args.warmup, "reps": args.lbvh_reps,
            "config": {"workload": "LBVH microbenchmark: uniform / 16-component Gaussian mixture "
                                   "with 5% duplicates, 30/63-bit Morton",
                       "headline": {k: head[k] for k in ("n", "dist", "bits")}},
            "peak_gbs": hbm, "peak_kind": f"{peak_kind} hbm_gbs",
            "bytes_per_point": {"30": lbvh_bytes(4, sort_passes(30)),
                                "63": lbvh_bytes(8, sort_passes(63))},
            "cpu_baseline": cpu_baseline, "rows": rows}
    print(json.dumps(line))
    return 0


def run_sis(args):
    """The reference's default update path (updateUniformGridSIS) in REFERENCE semantics: a
    packed 16^3 block of 4,096 cubes x 27 (110,592 particles, r = 1/256, 128^3 grid), every
    cube in contact with its neighbours; per step the integration, the contact search, the
    gather and 18 sequential-impulse sweeps, all on the device.  The CPU baseline is the
    reference's own code for the same step on the host (kind "reference"): its kernel bodies
    for the contact search, its gather and solver host loops."""
    import torch
    from diploma_thesis_b200 import api, scenes
    from diploma_thesis_b200.sis import SISScene, ITERATIONS
    torch.cuda.set_device(0)
    ctx = api.Context(0)
    sc = scenes.small_scene(4, nb_side=16, packed=True, r=1 / 256)
    g = SISScene(ctx, sc, dt=1e-4, grid_log2=(7, 7, 7))
    steps = max(1, min(args.steps, 20))
    g.step(args.warmup)
    torch.cuda.synchronize()
    with ClockSampler(0) as clocks:
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        g.step(steps)
        b.record()
        b.synchronize()
    ms = a.elapsed_time(b) / steps
    st = g.state()
    ctx.check()
    n = sc.num_particles
    cpu = None
    if not args.no_cpu:
        # the second half of the same step (after the integration) by the reference's own code
        # on the host: its hash / sort / reorder / contact-search kernel bodies (OpenMP), then
        # GatherRigidBodyCollisions + SequentialImpulseSolver and the re-posing tail, its host
        # loops (Particles/updateFunctions.cpp:1431-1874, one thread, as in the reference)
        import ctypes as C
        from oracle import ref
        if ref.available():
            prm = ref.SimParams()
            C.memmove(C.byref(prm), C.byref(g.params), C.sizeof(prm))
            rb = sc.body_index().astype(np.int32)
            t0 = time.perf_counter()
            h, idx = ref.calc_hash(prm, st["pos"])
            sh, si = ref.sort_pairs_u32(h, idx)
            cs, ce, sp, _ = ref.reorder(sh, si, st["pos"], st["pvel"], 128 ** 3)
            cd, cb, cp = ref.find_rb_collisions_grid(prm, rb, sp, si, cs, ce,
                                                     np.zeros(n, np.float32))
            res = ref.sis_step(prm, rb, sc.body_offsets, st["cms"], st["vel"], st["ang"],
                               st["cur"], sc.body_mass.astype(np.float32), st["rel"], cd, cb,
                               cp)
            cpu_s = time.perf_counter() - t0
            cpu = {"value": n / cpu_s / 1e6, "unit": "Mparticle-steps/s",
                   "cores": ref.max_threads(), "kind": "reference",
                   "sample": f"one step's hash, sort, reorder and contact search (the "
                             f"reference's kernel bodies, OpenMP) and its gather, "
                             f"{res['count']} contacts' sequential-impulse sweeps and particle "
                             f"update (the reference's host loops, one thread) on the same "
                             f"scene state"}
    print(json.dumps({
        "metric": "Mparticle-steps/s (sequential-impulse path)", "value": n / ms / 1e3,
        "unit": "Mparticle-steps/s", "n_gpus": 1, "steps": steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": "sequential-impulse path: 4,096 packed cubes x 27 (110,592 "
                               "particles), r=1/256, grid 128^3, dt=1e-4, 18 sweeps, "
                               "REFERENCE semantics",
                   "contacts_per_step": st["contacts"], "timed": "eager stage calls, events"},
        "cpu_baseline": cpu, "clocks": clocks.summary()}))
    return 0


def run_served(args):
    """Config 4: Poisson request stream (scenes of 1k-500k particles, cubes and rods, K in
    10..500) served with continuous batching under an HBM budget; the plain form serves the
    same requests one at a time."""
    import torch
    from diploma_thesis_b200 import api, scenes, serve
    torch.cuda.set_device(0)
    ctx = api.Context(0)
    rng = np.random.default_rng(1)
    pool = [scenes.config4_request(rng) for _ in range(args.pool)]  # distinct scenes, reused

    def make(r):
        sc, _ = pool[int(r.integers(len(pool)))]
        return sc, int(r.integers(10, 501))

    reqs = serve.poisson_requests(args.rate, args.duration, make, seed=2)
    # the request loop in C++ (ar_server_run); the pool's scenes become resident templates
    server = serve.NativeServer(ctx, args.hbm_budget_gb * 1e9, tick_steps=10)
    stats = server.run(reqs, time_limit=args.duration)
    s = stats.summary()
    # plain: a sample of the same requests, one at a time (create, K steps, download)
    sample = reqs[: min(len(reqs), args.plain_sample)]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    steps = parts = 0
    for r in sample:
        g = api.GpuScene(ctx, r.scene)
        g.step(r.steps, use_graph=True)
        g.download()
        g.close()
        steps += r.steps
        parts += r.steps * r.scene.num_particles
    plain_s = time.perf_counter() - t0
    offered = sum(r.steps * r.scene.num_particles for r in reqs) / args.duration / 1e6
    line = {"metric": "scene-steps/s (served)", "value": s["scene_steps_per_s"],
            "unit": "scene-steps/s", "n_gpus": 1, "higher_is_better": True,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"served: Poisson {args.rate}/s for {args.duration} s, "
                                   "scenes 1k-500k particles (cubes/rods 50/50), K in 10..500, "
                                   f"HBM budget {args.hbm_budget_gb} GB",
                       "scene_pool": args.pool, "loop": "C++ (ar_server_run)"},
            "p50_latency_s": s["p50_latency_s"], "p99_latency_s": s["p99_latency_s"],
            "completed": s["completed"], "offered_requests": s["offered"],
            "mparticle_steps_per_s": s["mparticle_steps_per_s"],
            "offered_mparticle_steps_per_s": offered,
            "plain": {"scene_steps_per_s": steps / plain_s,
                      "mparticle_steps_per_s": parts / plain_s / 1e6,
                      "sample_requests": len(sample)},
            "served_over_plain": s["scene_steps_per_s"] / (steps / plain_s),
            "peak_resident_scenes": s["peak_resident_scenes"],
            "peak_resident_gb": s["peak_resident_bytes"] / 1e9, "ticks": s["ticks"],
            "host_s": s["host_s"]}
    print(json.dumps(line))
    server.close()
    return 0


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["pile", "plain", "batched", "served", "lbvh", "sis"],
                    default="pile")
    ap.add_argument("--lbvh-sizes", default="", help="lbvh: comma-separated point counts")
    ap.add_argument("--lbvh-reps", type=int, default=10, help="lbvh: timed repetitions")
    ap.add_argument("--broadphase", choices=["grid", "bvh"], default="grid",
                    help="pile / plain: broad phase of the fused step")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--start-step", type=int, default=None,
                    help="pile / plain: untimed steps run before the warm-up (default: centre "
                         "the timed window in the configuration's run, 500 steps for the pile, "
                         "1,000 for the plain scene)")
    ap.add_argument("--tune", action="store_true", help="batched: autotune per size bucket")
    ap.add_argument("--tune-cache", default=str(ROOT / "diploma_thesis_b200" / "autotune_b200.json"))
    ap.add_argument("--rate", type=float, default=2000.0, help="served: requests per second")
    ap.add_argument("--duration", type=float, default=60.0, help="served: seconds of arrivals")
    ap.add_argument("--pool", type=int, default=64, help="served: distinct scenes drawn from")
    ap.add_argument("--plain-sample", type=int, default=200,
                    help="served: requests timed one at a time for the plain form")
    ap.add_argument("--hbm-budget-gb", type=float, default=150.0)
    args = ap.parse_args(argv)
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batched":
        return run_batched(args)
    if args.workload == "served":
        return run_served(args)
    if args.workload == "lbvh":
        return run_lbvh(args)
    if args.workload == "sis":
        return run_sis(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
