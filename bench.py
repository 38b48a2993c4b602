"""Benchmark of the fused rigid-body step (one JSON line on stdout).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload pile|plain]

Workload (default "pile"): the plain large pile -- 2,097,152 particles, 32,768 bodies of 64
(cubes, rods, padded spheres), r = 1/512, 1 x 3 x 1 box, dt = 1e-4, k = 5e4, damping 0.02,
shear 0.1, grid broad phase (256^3 wrapped cells of 2r).  "plain" is the 110,592-particle
single scene (4,096 cubes, 128^3 grid).  Seeded synthetic scenes; no dataset exists.

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
# in L2 are not counted).  P = sort passes, ppb = particles per body.
STAGES = ["clear", "repose_hash", "sort", "scatter", "collide", "reduce_integrate"]


def stage_bytes(n: int, nb: int, passes: int, occupied_cells: int) -> dict[str, float]:
    body_state = 16 * 4  # pos, quat, vel, angvel (float4 each)
    return {
        # sort workspace head (histograms + look-back status), written once
        "clear": 4 * 256 * 8 + passes * 4 * 256 * ((n + 4095) // 4096),
        # read rel (16) + previous sorted key (4), write key (4); body pose (32) per body;
        # reset of the previous step's occupied cells (4 each)
        "repose_hash": n * (16 + 4 + 4) + nb * 32 + occupied_cells * 4,
        # first pass reads the key only; every pass writes key + index; later passes read both
        "sort": n * (4 + 8) + (passes - 1) * n * 16 + passes * 4 * 256 * ((n + 4095) // 4096),
        # read sorted key + index (8) and rel (16); write sorted pos + vel (32); body state per
        # body; cell (start, end) per occupied cell
        "scatter": n * (8 + 16 + 32) + nb * body_state + occupied_cells * 8,
        # own index (4), position + velocity (32); force (16) out
        "collide": n * (4 + 32 + 16),
        # force + rel (32) in; body state + mass + inverse inertia in, body state + sums out
        "reduce_integrate": n * 32 + nb * (body_state + 4 + 36 + body_state + 32),
    }


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

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
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
        for ln in self.lines:
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
                                   "(cubes/rods/spheres), r=1/512, box 1x3x1, grid 256^3 "
                                   "wrapped, dt=1e-4, k=5e4")
    if workload == "plain":
        return scenes.config0(0), ("plain single scene: 110,592 particles, 4,096 cubes x 27, "
                                   "r=1/256, unit box, grid 128^3, dt=1e-4, k=5e4")
    raise SystemExit(f"unknown workload {workload}")


def dist_setup(ngpus: int):
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=torch.device(f"cuda:{local}"))
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
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---- CPU legs (oracle) ---------------------------------------------------------------------
def reference_sample(scene, bodies: int):
    """The first `bodies` bodies of the scene as its own scene (bounded CPU sample)."""
    from diploma_thesis_b200.scenes import Scene
    off = scene.body_offsets
    n = int(off[bodies])
    return Scene(radius=scene.radius, box_min=scene.box_min, box_max=scene.box_max,
                 body_pos=scene.body_pos[:bodies].copy(), body_quat=scene.body_quat[:bodies].copy(),
                 body_vel=scene.body_vel[:bodies].copy(), body_angvel=scene.body_angvel[:bodies].copy(),
                 body_mass=scene.body_mass[:bodies].copy(),
                 body_inv_inertia=scene.body_inv_inertia[:bodies].copy(),
                 body_offsets=off[: bodies + 1].copy(), particle_rel=scene.particle_rel[:n].copy(),
                 gravity=scene.gravity, dt=scene.dt, spring=scene.spring, damping=scene.damping,
                 shear=scene.shear, grid_log2=scene.grid_log2, cell_size=scene.cell_size)


class ReferenceCPUStep:
    """One updateUniformGridDEM step (RigidBodies/UniformGridUpdate.cpp:939-999) made of the
    reference's own kernel bodies run on the host cores: GPUintegratorKernel,
    computeGlobalAttributes, calcHashD, the CUB-order stable sort, reorder (with its
    full-grid clear), FindAndHandleRigidBodyCollisionsUniformGridKernel and
    ReducePerParticleImpulses.  Physical constants are given the reference's per-step form
    (impulse = force * dt, velocity increment g * dt)."""

    def __init__(self, scene, grid):
        from diploma_thesis_b200.api import sim_params
        from oracle import ref
        self.ref = ref
        self.s = scene
        origin, cell, dims = grid
        dt = scene.dt
        self.prm = sim_params(scene.radius, origin, cell[0], dims, scene.spring * dt,
                              scene.damping * dt, scene.shear * dt, scene.attraction * dt,
                              gravity=tuple(g * dt for g in scene.gravity), w_damping=1.0)
        self.ncell = int(np.prod(dims))
        n, nb = scene.num_particles, scene.num_bodies
        self.rb = scene.body_index()
        self.counts = np.diff(scene.body_offsets).astype(np.int32)
        self.st = {"cms": scene.body_pos.copy(), "vel": scene.body_vel.copy(),
                   "ang": scene.body_angvel.copy(), "quat": np.tile([0, 0, 0, 1.0], (nb, 1)).astype(np.float32),
                   "ib": scene.body_inv_inertia.copy(), "cur": np.zeros((nb, 9), np.float32),
                   "model": np.zeros((nb, 16), np.float32), "cum": scene.body_quat.copy()}
        # world-frame relative positions, as the reference keeps them
        from diploma_thesis_b200.scenes import quat_to_matrix
        R = quat_to_matrix(scene.body_quat.astype(np.float64))[self.rb]
        self.rel = np.zeros((n, 4), np.float32)
        self.rel[:, :3] = np.einsum("nij,nj->ni", R, scene.particle_rel[:, :3])

    def step(self):
        ref, s = self.ref, self.s
        self.st = ref.gpu_integrator(self.prm, s.dt, self.st)
        self.rel, pos, vel, q = ref.global_attributes(self.st["cms"], self.st["vel"],
                                                      self.st["ang"], self.st["quat"], self.rb,
                                                      self.rel)
        self.st["quat"] = q
        h, idx = ref.calc_hash(self.prm, pos)
        sh, si = ref.sort_pairs_u32(h, idx)
        cs, ce, sp, sv = ref.reorder(sh, si, pos, vel, self.ncell)
        pf, pt = ref.collide_grid_dem(self.prm, self.rb, sp, sv, self.rel, si, cs, ce)
        self.st["vel"], self.st["ang"] = ref.reduce_impulses(
            pf, pt, self.st["vel"], self.st["ang"], s.body_mass, s.body_inv_inertia, self.counts)


def cpu_reference_rate(scene, grid, target_s: float, steps: int | None = None):
    """Particle-steps/s of the reference CPU step on a bounded sample; returns
    (rate, cores, kind, sample description, steps run, seconds)."""
    from oracle import ref
    if not ref.available():
        return None
    bodies = min(scene.num_bodies, 4096)
    sample = reference_sample(scene, bodies)
    runner = ReferenceCPUStep(sample, grid)
    cores = ref.max_threads()
    runner.step()  # warm caches / page in
    t0 = time.perf_counter()
    k = 0
    while True:
        runner.step()
        k += 1
        el = time.perf_counter() - t0
        if (steps is not None and k >= steps) or (steps is None and el >= target_s):
            break
    rate = sample.num_particles * k / el
    desc = (f"first {bodies} bodies ({sample.num_particles} particles) of the workload on the "
            f"same grid, {k} reference steps in {el:.1f} s")
    return rate, cores, "reference", desc, k, el


# ---- the reference arm -----------------------------------------------------------------------
def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import cpu, ref
    scene, desc = make_scene(args.workload)
    grid = cpu.scene_grid(scene)
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable":
                          "the reference CPU build (oracle/_ref/libref_cpu.so) is not present"}))
        return 0
    bodies = min(scene.num_bodies, 2048 if args.workload == "pile" else 4096)
    sample = reference_sample(scene, bodies)
    runner = ReferenceCPUStep(sample, grid)
    for _ in range(args.warmup):
        runner.step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        runner.step()
    el = time.perf_counter() - t0
    rate = sample.num_particles * args.steps / el / 1e6
    cores = ref.max_threads()
    line = {"metric": "Mparticle-steps/s", "value": rate, "unit": "Mparticle-steps/s",
            "impl": "reference", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * el / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": desc, "sample": f"first {bodies} bodies "
                       f"({sample.num_particles} particles)", "broadphase": "grid"},
            "cpu_baseline": {"value": rate, "unit": "Mparticle-steps/s", "cores": cores,
                             "kind": "reference",
                             "sample": f"first {bodies} bodies ({sample.num_particles} particles) "
                                       f"of the workload, {args.steps} steps"},
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
    ctx = api.Context(local)
    gs = api.GpuScene(ctx, scene)
    n, nb = scene.num_particles, scene.num_bodies
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        gs.step(args.warmup, use_graph=True, stream=stream)
        stream.synchronize()
        ctx.check(stream)
        # ---- device-timed region: K graph replays ----
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier(world)
        torch.cuda.synchronize()
        with ClockSampler(local) as clocks:
            start.record(stream)
            gs.step(args.steps, use_graph=True, stream=stream)
            end.record(stream)
            end.synchronize()
        torch.cuda.synchronize()
        barrier(world)
        ms = start.elapsed_time(end)
        ctx.check(stream)
    ms = max_over_ranks(ms, world)
    ms_per_step = ms / args.steps
    value = world * n * args.steps / (ms / 1e3) / 1e6

    # ---- stage profile (event-bracketed eager steps right after the timed region) ----
    with torch.cuda.stream(stream):
        prof_steps = max(5, min(args.steps, 50))
        stage_ms = gs.profile(prof_steps, stream=stream)
    sv = gs.step_view()
    keys = api.device_view(sv.sorted_keys, n, torch.int32)
    occupied = int((keys[1:] != keys[:-1]).sum().item()) + 1
    passes = (sv.key_bits + 7) // 8
    sbytes = stage_bytes(n, nb, passes, occupied)
    hbm, peak_kind = peaks()
    dom = max(range(len(STAGES)), key=lambda i: stage_ms[i])
    dom_name = STAGES[dom]
    achieved = sbytes[dom_name] / (stage_ms[dom] / 1e3) / 1e9
    step_bytes = sum(sbytes.values())
    step_ms_prof = sum(stage_ms)

    # ---- end to end: host state in, step, host state out, every step ----
    e2e_steps = max(3, min(args.steps, 100))
    pinned = {k: torch.empty((nb, 4), dtype=torch.float32).pin_memory() for k in
              ("pos", "quat", "vel", "angvel")}
    host = {k: v.numpy() for k, v in pinned.items()}
    gs.download_into(host["pos"], host["quat"], host["vel"], host["angvel"], stream=stream)
    with torch.cuda.stream(stream):
        barrier(world)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            gs.upload(host["pos"], host["quat"], host["vel"], host["angvel"], stream=stream)
            gs.step(1, use_graph=True, stream=stream)
            gs.download_into(host["pos"], host["quat"], host["vel"], host["angvel"], stream=stream)
        torch.cuda.synchronize()
        e2e_s = time.perf_counter() - t0
        barrier(world)
    e2e_s = max_over_ranks(e2e_s, world)
    e2e_value = world * n * e2e_steps / e2e_s / 1e6

    # ---- CPU baseline (rank 0, N = 1) ----
    cpu_baseline = None
    if rank == 0 and world == 1 and not args.no_cpu:
        from oracle import cpu
        r = cpu_reference_rate(scene, cpu.scene_grid(scene), target_s=15.0)
        if r is not None:
            rate, cores, kind, sample, k, el = r
            cpu_baseline = {"value": rate / 1e6, "unit": "Mparticle-steps/s", "cores": cores,
                            "kind": kind, "sample": sample}

    launches = args.steps * (gs.launches_per_step() - 1)  # minus the memset node
    if rank == 0:
        line = {
            "metric": "Mparticle-steps/s", "value": value, "unit": "Mparticle-steps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": desc, "broadphase": "grid", "particles": n, "bodies": nb,
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "l2": "per-step working set > 126 MB L2 (inputs larger than L2)",
                       "timed": "CUDA graph replays, events on the launching stream"},
            "roofline": {"bound": "hbm", "kernel": dom_name, "achieved": achieved,
                         "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                         "peak_kind": f"{peak_kind} hbm_gbs", "traffic": None,
                         "algorithmic_bytes_per_launch": sbytes[dom_name],
                         "launch_ms": stage_ms[dom]},
            "step_roofline": {"achieved": step_bytes / (ms_per_step / 1e3) / 1e9, "peak": hbm,
                              "unit": "GB/s", "frac": step_bytes / (ms_per_step / 1e3) / 1e9 / hbm,
                              "bytes_per_particle_step": step_bytes / n},
            "stages_ms": dict(zip(STAGES, stage_ms)), "stage_profile_ms_per_step": step_ms_prof,
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


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["pile", "plain"], default="pile")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    args = ap.parse_args(argv)
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
