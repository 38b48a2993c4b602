"""Autotuner: per scene-size bucket, the broad phase (uniform grid or BVH), and for the grid the
cell size and wrapped grid size, and the block size of the DEM gather, that give the fastest
fused step on this GPU.

Buckets are powers of two of the particle count.  For each bucket a representative scene
(27-particle cubes, config-0 distributions) is stepped under every candidate and timed with
CUDA events over CUDA-graph replays by the library's C++ loop (ar_tune_candidates); the
fastest candidate is kept.  Results are cached in a
JSON file keyed by GPU name, so a deployment tunes once.

Candidates: grid with cell = f * 2r for f in CELL_FACTORS and cells per axis wrapped so that
the grid holds at most next_pow2(m * N) cells for m in GRID_MULTS, or the BVH; block size in
BLOCK_SIZES.  Every candidate gives the same contacts (the cell is never smaller than the contact distance and the
wrap only aliases distant cells, which the distance test rejects), so the choice changes speed,
not results -- except for the summation order of a particle's contacts, which follows the cell
order (grid) or the tree's visit order (BVH).  Scenes of one batch share a broad phase, so a
mixed table is stepped as one batch per broad phase (``group``).
"""
from __future__ import annotations

import ctypes as C
import json
import math
from dataclasses import asdict, dataclass
from pathlib import Path

import numpy as np
import torch

from . import api, scenes
from ._lib import call

CELL_FACTORS = (1.0, 1.25, 1.5)
GRID_MULTS = (2, 8, 32)
BLOCK_SIZES = (64, 128, 256)


@dataclass
class Choice:
    cell_factor: float
    grid_mult: int
    block_size: int
    ms_per_step: float
    broadphase: str = "grid"


def bucket_of(num_particles: int) -> int:
    return max(10, int(math.ceil(math.log2(max(num_particles, 2)))))


def grid_for(scene: scenes.Scene, cell: float, mult: int) -> tuple[int, int, int]:
    """log2 cells per axis: cover the box, then halve the largest axis while the grid holds
    more than next_pow2(mult * N) cells."""
    dims = []
    for a in range(3):
        ext = float(scene.box_max[a]) - float(scene.box_min[a])
        cells = max(1, int(math.ceil(ext / cell)))
        dims.append(max(2, int(math.ceil(math.log2(cells)))))
    cap = max(12, int(math.ceil(math.log2(mult * max(scene.num_particles, 1)))))
    while sum(dims) > cap:
        a = int(np.argmax(dims))
        if dims[a] <= 2:
            break
        dims[a] -= 1
    return tuple(dims)


def apply(scene: scenes.Scene, choice: Choice) -> dict:
    """Keyword arguments for api.GpuScene that realise a choice for this scene."""
    if choice.broadphase == "bvh":
        return {"broadphase": "bvh", "block_size": choice.block_size}
    cell = float(np.float32(choice.cell_factor * 2 * scene.radius))
    return {"cell_size": cell, "grid_log2": grid_for(scene, cell, choice.grid_mult),
            "block_size": choice.block_size}


def _init_of(scene: scenes.Scene):
    """ar_scene_init of a scene (the arrays kept alive by the returned list)."""
    keep = [np.ascontiguousarray(a) for a in (
        scene.body_pos, scene.body_quat, scene.body_vel, scene.body_angvel,
        scene.body_mass.astype(np.float32), scene.body_inv_inertia.astype(np.float32),
        scene.body_offsets.astype(np.int32), scene.particle_rel)]
    return api.SceneInit(*[C.c_void_p(a.ctypes.data) for a in keep]), keep


def time_candidates(ctx: api.Context, scene: scenes.Scene, choices: list[Choice],
                    steps: int = 20, warmup: int = 3) -> list[float]:
    """Milliseconds per graph-replayed step of the scene under each choice, timed by the
    library's C++ loop (ar_tune_candidates)."""
    descs = (api.SceneDesc * len(choices))()
    for i, c in enumerate(choices):
        kw = apply(scene, c)
        descs[i] = api.make_desc(scene, api.broadphase_code(kw.get("broadphase", "grid")),
                                 kw.get("block_size", 0), kw.get("cell_size"),
                                 kw.get("grid_log2"))
    init, _keep = _init_of(scene)
    ms = np.zeros(len(choices), np.float32)
    call("ar_tune_candidates", ctx.handle, descs, len(choices), C.byref(init), int(warmup),
         int(steps), C.c_void_p(ms.ctypes.data))
    return [float(x) for x in ms]


def tune_bucket(ctx: api.Context, bucket: int, steps: int = 20, seed: int = 0) -> Choice:
    n = 1 << bucket
    side = float(np.clip((n / 27 * 0.035 ** 3 * 4) ** (1 / 3), 0.5, 2.0))
    scene = scenes.cube_scene(seed + bucket, n // 27 * 27, side)
    cands = [Choice(f, m, bs, 0.0) for f in CELL_FACTORS for m in GRID_MULTS for bs in BLOCK_SIZES]
    cands += [Choice(1.0, 0, bs, 0.0, "bvh") for bs in BLOCK_SIZES]
    for c, ms in zip(cands, time_candidates(ctx, scene, cands, steps)):
        c.ms_per_step = ms
    return min(cands, key=lambda c: c.ms_per_step)  # the first of equal times


def group(kwargs: list[dict]) -> dict[str, list[int]]:
    """Indices of the scenes per broad phase (each group is stepped as one batch)."""
    out: dict[str, list[int]] = {}
    for i, kw in enumerate(kwargs):
        out.setdefault(kw.get("broadphase", "grid"), []).append(i)
    return out


class Tuner:
    """Per-bucket choices, tuned on first use and cached per GPU name."""

    def __init__(self, ctx: api.Context, cache: str | Path | None = None,
                 gpu_name: str | None = None):
        self.ctx = ctx
        self.cache = Path(cache) if cache else None
        self.table: dict[int, Choice] = {}
        self.gpu = gpu_name or torch.cuda.get_device_name()
        if self.cache and self.cache.exists():
            data = json.loads(self.cache.read_text())
            for k, v in data.get(self.gpu, {}).items():
                self.table[int(k)] = Choice(**v)

    def choice(self, num_particles: int) -> Choice:
        b = bucket_of(num_particles)
        if b not in self.table:
            self.table[b] = tune_bucket(self.ctx, b)
            self.save()
        return self.table[b]

    def save(self) -> None:
        if not self.cache:
            return
        data = json.loads(self.cache.read_text()) if self.cache.exists() else {}
        data[self.gpu] = {str(k): asdict(v) for k, v in sorted(self.table.items())}
        self.cache.write_text(json.dumps(data, indent=1))

    def scene_kwargs(self, scene: scenes.Scene) -> dict:
        return apply(scene, self.choice(scene.num_particles))
