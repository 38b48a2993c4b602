"""Particle-body files (the reference's Data/OBJparticles format): reading, centring,
inertia, the scale -> file mapping, the hand-set inertia table, and scenes built from files.
Synthetic files in the same format are written here; set AR_SIM_DATA to a Data/OBJparticles
directory to also read the shipped models."""
import os
from pathlib import Path

import numpy as np
import pytest

from diploma_thesis_b200 import bodies, scenes
from oracle import cpu, ref


def _write_cube(root: Path, k: int = 4, spacing: float = 2 / 64, suffix: str = "1_0"):
    d = root / "cube"
    d.mkdir(parents=True, exist_ok=True)
    g = (np.arange(k) - (k - 1) / 2) * spacing - 0.0  # centred lattice
    pts = np.array([[x, y, z] for x in g for y in g for z in g], np.float32) + 0.01
    lines = [str(len(pts))] + [f"{x:.6f} {y:.6f} {z:.6f}" for x, y, z in pts]
    (d / f"cube_{suffix}.txt").write_text("\n".join(lines) + "\n")
    return pts


def test_scale_selects_the_file_like_the_reference():
    cases = {0.5: "1_0", 1.0: "1_0", 1.2: "1_5", 1.5: "1_5", 1.7: "2_0", 2.0: "2_0",
             2.3: "2_5", 2.5: "2_5", 3.0: "1_5"}
    for scale, suffix in cases.items():
        assert bodies.file_suffix(scale) == suffix, scale
    assert bodies.body_file("D", "teapot", 2.0).as_posix() == "D/teapot/teapot_2_0.txt"


def test_read_centre_and_inertia(tmp_path):
    pts = _write_cube(tmp_path)
    got = bodies.read_points(bodies.body_file(tmp_path, "cube", 1.0))
    assert got.shape == (64, 3) and np.allclose(got, pts, atol=1e-6)
    rel = bodies.centre(got, "cube", 1 / 64)
    assert np.abs(rel.mean(0)).max() < 1e-6
    inv = bodies.inverse_inertia(rel)
    assert np.allclose(inv, scenes.inverse_inertia(rel), rtol=1e-5, atol=1e-6)
    # per-model shift of the centre (teapot: 2r along y)
    shifted = bodies.centre(got, "teapot", 1 / 64)
    assert np.allclose(rel - shifted, [0, 2 / 64, 0], atol=1e-6)


def test_header_count_is_checked(tmp_path):
    f = tmp_path / "bad.txt"
    f.write_text("3\n0 0 0\n1 1 1\n")
    with pytest.raises(ValueError):
        bodies.read_points(f)


def test_hand_set_inertia_table():
    rel = np.zeros((8, 3), np.float32)
    inv = bodies.inverse_inertia(rel, "cube", 1.0, reference_inertia=True).reshape(3, 3)
    assert np.allclose(np.diag(inv), 600.0)
    inv = bodies.inverse_inertia(rel, "banana", 2.0, reference_inertia=True).reshape(3, 3)
    assert np.allclose(np.diag(inv), 1 / np.array([0.0140314, 0.0218576, 0.0309458]))


def test_scene_from_files_steps_on_the_oracle(tmp_path):
    _write_cube(tmp_path)
    r = 1 / 64
    placements = [("cube", 1.0)] * 3
    centres = [[0.3, 0.12, 0.3], [0.3, 0.2, 0.3], [0.6, 0.5, 0.5]]
    quats = scenes.random_quaternions(np.random.default_rng(0), 3)
    sc = bodies.scene_from_files(tmp_path, placements, centres, quats, r, [0, 0, 0], [1, 1, 1])
    assert sc.num_particles == 192 and sc.num_bodies == 3
    assert np.allclose(sc.body_mass, 64.0)
    out = cpu.step(sc, 20)
    assert out["finite"]
    assert (np.abs(out["pforce"]).sum(1) > 0).sum() > 0  # the first two cubes touch


REF_ROOT = Path(os.environ.get("AR_REFERENCE_ROOT", "/root/reference"))
DATA = REF_ROOT / "AR_Sim" / "Data" / "OBJparticles"


@pytest.mark.skipif(not DATA.is_dir(), reason="the reference checkout's particle-body files are absent")
def test_shipped_models_read_and_centre():
    """Every shipped model and scale (the reference's own Data/OBJparticles files) loads, with
    the counts the files declare, centred offsets whose mean is the model's shift, and a finite
    physical inverse inertia."""
    r = 1 / 64
    for model in ("cube", "bunny", "banana", "teapot"):
        for scale in (1.0, 1.5, 2.0, 2.5):
            path = bodies.body_file(DATA, model, scale)
            n = int(path.read_text().split()[0])
            rel, inv, m = bodies.load_body(DATA, model, scale, r)
            assert rel.shape == (n, 3) and m == n and np.isfinite(inv).all()
            shift = np.asarray(bodies._CM_SHIFT.get(model, (0, 0, 0))) * r
            assert np.allclose(rel.astype(np.float64).mean(0), -shift, atol=1e-5)
    assert len(bodies.read_points(bodies.body_file(DATA, "cube", 1.0))) == 64


@pytest.mark.skipif(not DATA.is_dir() or not ref.available(),
                    reason="needs the reference checkout and its host build (oracle/_ref)")
def test_shipped_models_equal_the_reference_init_object():
    """bodies.load_body(..., reference_inertia=True) against the reference's own initObject body
    set-up (RigidBodyAddition.cpp:1576-1756, built for the host by oracle/ref_build.py) on every
    shipped model and scale: the centred offsets and the inverse inertia bit for bit.  That
    includes the reference's quirks: the inertia sum starts from the identity (a
    default-constructed glm::mat3), the hand-set tensors (banana, bunny 1.5, teapot) and hand-set
    inverse tensors (cube 1.0, 1.5, 2.0)."""
    r = 1 / 64
    for model in ("cube", "bunny", "banana", "teapot"):
        for scale in (1.0, 1.5, 2.0, 2.5):
            rel, inv, m = bodies.load_body(DATA, model, scale, r, reference_inertia=True)
            want_rel, want_inv = ref.init_object(bodies.body_file(DATA, model, scale), model,
                                                 scale, r)
            assert np.array_equal(rel, want_rel), (model, scale)
            assert np.array_equal(inv, want_inv), (model, scale)
            assert m == 1.0
