"""The reference's own GPU step beside this repository's fused step, stage by stage.

BASELINE INFRASTRUCTURE ONLY (oracle).  Runs the reference's updateUniformGridDEM
(oracle/_ref/libref_gpu.so: its CUDA sources compiled for sm_100a, its wrappers with their
allocations and synchronisations; built by oracle/ref_gpu_build.py, checked against the
reference's CPU build by tests/test_gpu_ref_gpu.py) and the fused grid step on the same scene
and GPU, and prints one JSON line:

    python -m oracle.ref_gpu_bench [--scene pile|plain] [--steps K] [--warmup W]

Both start from the scene's initial state; W untimed steps, then K timed steps each (the
reference's stages by CUDA events on its legacy stream, host time included where the GPU waits
for it; ours by graph replays between events and the event-bracketed stage profile).  The
reference runs REFERENCE semantics (impulses as velocity increments), ours PHYSICAL: the same
broad phase, contact law and summation order over the same particles and cells.
"""
from __future__ import annotations

import argparse
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

# stages of the fused step's profile (ar_step_profile)
OURS = ["clear", "keys", "sort", "scatter", "collide", "body"]
SCENES = {
    "pile": "plain large pile: 2,097,152 particles, 32,768 bodies x 64 (cubes/rods/spheres), "
            "r=1/512, box 1x3x1, grid 256x512x256 wrapped, dt=1e-4, k=5e4",
    "plain": "plain single scene: 110,592 particles, 4,096 cubes x 27, r=1/256, unit box, "
             "grid 128^3, dt=1e-4, k=5e4",
}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--scene", choices=sorted(SCENES), default="pile")
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    args = ap.parse_args(argv)
    import torch
    from diploma_thesis_b200 import api, scenes
    from oracle import cpu, ref_gpu
    if not ref_gpu.available():
        print(json.dumps({"unavailable": "the reference GPU build (oracle/_ref/libref_gpu.so) "
                                         "is not present"}))
        return 0
    torch.cuda.set_device(0)
    scene = scenes.config2(0) if args.scene == "pile" else scenes.config0(0)
    n = scene.num_particles
    # the reference's step
    rg = ref_gpu.RefGpuStep(scene, cpu.scene_grid(scene))
    for _ in range(args.warmup):
        rg.step()
    acc = np.zeros(len(ref_gpu.STAGES))
    host = 0.0
    for _ in range(args.steps):
        ms, wall = rg.step()
        acc += ms
        host += wall
    rg.close()
    ref_stage = acc / args.steps
    ref_ms = float(ref_stage.sum())
    # ours, same scene and step window
    ctx = api.Context(0)
    gs = api.GpuScene(ctx, scene)
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        gs.step(args.warmup, use_graph=True, stream=stream)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        stream.synchronize()
        a.record(stream)
        gs.step(args.steps, use_graph=True, stream=stream)
        b.record(stream)
        b.synchronize()
        ours_ms = a.elapsed_time(b) / args.steps
        ours_stage = gs.profile(min(args.steps, 50), stream=stream)
    ctx.check(stream)
    gs.close()
    ctx.close()
    print(json.dumps({
        "metric": "ms per step", "scene": SCENES[args.scene], "particles": n,
        "steps": args.steps, "warmup": args.warmup,
        "reference_gpu": {"ms_per_step": ref_ms, "host_ms_per_step": host / args.steps,
                          "mparticle_steps_per_s": n / ref_ms / 1e3,
                          "stages_ms": dict(zip(ref_gpu.STAGES, ref_stage.tolist())),
                          "semantics": "REFERENCE"},
        "ours": {"ms_per_step": ours_ms, "mparticle_steps_per_s": n / ours_ms / 1e3,
                 "stages_ms": dict(zip(OURS, [float(x) for x in ours_stage])),
                 "semantics": "PHYSICAL"},
        "speedup": ref_ms / ours_ms}))
    return 0


if __name__ == "__main__":
    sys.exit(main())
