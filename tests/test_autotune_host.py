"""Autotuner host logic (no GPU): size buckets, the wrapped grid a choice gives, the keyword
arguments per broad phase, grouping by broad phase, and the per-GPU JSON cache."""
import json
import math

import numpy as np

from diploma_thesis_b200 import autotune, scenes


def test_buckets_are_powers_of_two():
    assert autotune.bucket_of(1) == 10
    assert autotune.bucket_of(1024) == 10
    assert autotune.bucket_of(1025) == 11
    assert autotune.bucket_of(200_000) == 18


def test_grid_covers_box_within_cell_cap():
    sc = scenes.cube_scene(3, 27 * 500, 1.5)
    for f in autotune.CELL_FACTORS:
        cell = f * 2 * sc.radius
        for m in autotune.GRID_MULTS:
            dims = autotune.grid_for(sc, cell, m)
            cap = max(12, math.ceil(math.log2(m * sc.num_particles)))
            assert sum(dims) <= cap or all(d <= 2 for d in dims)
            for a in range(3):
                ext = float(sc.box_max[a] - sc.box_min[a])
                need = max(2, math.ceil(math.log2(max(1, math.ceil(ext / cell)))))
                assert 2 <= dims[a] <= need


def test_apply_per_broadphase_and_group():
    sc = scenes.cube_scene(4, 27 * 100, 1.0)
    g = autotune.apply(sc, autotune.Choice(1.25, 8, 64, 0.1))
    assert set(g) == {"cell_size", "grid_log2", "block_size"}
    assert g["cell_size"] == float(np.float32(1.25 * 2 * sc.radius))
    b = autotune.apply(sc, autotune.Choice(1.0, 0, 128, 0.1, "bvh"))
    assert b == {"broadphase": "bvh", "block_size": 128}
    assert autotune.group([g, b, g, {}]) == {"grid": [0, 2, 3], "bvh": [1]}


def test_cache_round_trip(tmp_path):
    path = tmp_path / "tune.json"
    t = autotune.Tuner(None, path, gpu_name="GPU-A")
    t.table[12] = autotune.Choice(1.5, 32, 256, 0.25, "grid")
    t.table[17] = autotune.Choice(1.0, 0, 64, 0.5, "bvh")
    t.save()
    u = autotune.Tuner(None, path, gpu_name="GPU-A")
    assert u.table == t.table
    assert u.choice(3000) == t.table[12]  # cached: no tuning run
    assert autotune.Tuner(None, path, gpu_name="GPU-B").table == {}
    # entries written before the broad-phase field existed read as grid
    data = json.loads(path.read_text())
    del data["GPU-A"]["12"]["broadphase"]
    path.write_text(json.dumps(data))
    assert autotune.Tuner(None, path, gpu_name="GPU-A").table[12].broadphase == "grid"
