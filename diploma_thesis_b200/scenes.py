"""Seeded synthetic scenes with the shapes, sizes and distributions of the benchmark configs.

A scene is a set of rigid bodies, each a cloud of equal spheres ("particles") of radius r
at lattice spacing 2r, as in AR_Sim's OBJparticles bodies (AR_Sim/Data/OBJparticles/*).
Every body has unit particle mass; its inverse inertia is the inverse of the particle sum
sum_i (|r_i|^2 E - r_i r_i^T) about the centre of mass, the construction of initObject
(RigidBodies/RigidBodyAddition.cpp:1598-1735).  Gravity points along -y.

There is no dataset: these generators are the whole workload.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class Scene:
    """Host-side scene state (float32 arrays, AR_Sim layouts)."""
    radius: float
    box_min: np.ndarray
    box_max: np.ndarray
    body_pos: np.ndarray        # [B,4]
    body_quat: np.ndarray       # [B,4] (x, y, z, w)
    body_vel: np.ndarray        # [B,4]
    body_angvel: np.ndarray     # [B,4]
    body_mass: np.ndarray       # [B]
    body_inv_inertia: np.ndarray  # [B,9] glm::mat3 (column-major), body frame
    body_offsets: np.ndarray    # [B+1] int32
    particle_rel: np.ndarray    # [N,4] body-frame offsets (w unused)
    gravity: tuple = (0.0, -9.81, 0.0)
    dt: float = 1e-4
    spring: float = 5e4
    damping: float = 0.02
    shear: float = 0.1
    attraction: float = 0.0
    grid_log2: tuple = (0, 0, 0)
    cell_size: float = 0.0
    name: str = ""
    extra: dict = field(default_factory=dict)

    @property
    def num_bodies(self) -> int:
        return int(self.body_pos.shape[0])

    @property
    def num_particles(self) -> int:
        return int(self.particle_rel.shape[0])

    def body_index(self) -> np.ndarray:
        counts = np.diff(self.body_offsets)
        return np.repeat(np.arange(self.num_bodies, dtype=np.int32), counts)

    def world_positions(self) -> np.ndarray:
        """Particle world positions [N,4] (float64 rotation, for scene building only)."""
        b = self.body_index()
        rot = quat_to_matrix(self.body_quat.astype(np.float64))[b]
        p = np.einsum("nij,nj->ni", rot, self.particle_rel[:, :3].astype(np.float64))
        p += self.body_pos[b, :3]
        out = np.zeros((self.num_particles, 4), np.float32)
        out[:, :3] = p
        return out


# ---- bodies --------------------------------------------------------------------------------
def _centred(points: np.ndarray) -> np.ndarray:
    return points - points.mean(axis=0)


def cube_body(k: int, spacing: float) -> np.ndarray:
    g = np.arange(k, dtype=np.float64) * spacing
    pts = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    return _centred(pts)


def rod_body(length: int, spacing: float) -> np.ndarray:
    pts = np.zeros((length, 3))
    pts[:, 0] = np.arange(length) * spacing
    return _centred(pts)


def sphere_body(count: int, spacing: float) -> np.ndarray:
    """`count` lattice points closest to the centre (a voxelised sphere padded to `count`)."""
    m = int(np.ceil(count ** (1 / 3))) + 3
    g = np.arange(-m, m + 1, dtype=np.float64)
    pts = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    d = np.linalg.norm(pts + 0.25, axis=1)  # off-centre so the padding is deterministic
    order = np.lexsort((np.arange(len(d)), d))
    return _centred(pts[order[:count]] * spacing)


def inverse_inertia(rel: np.ndarray, mass: float = 1.0) -> np.ndarray:
    """glm::mat3 (column-major; symmetric anyway) of the inverse particle-sum inertia."""
    r2 = np.einsum("ni,ni->n", rel, rel)
    inertia = mass * (r2.sum() * np.eye(3) - rel.T @ rel)
    if abs(np.linalg.det(inertia)) < 1e-30:  # rods: regularise the axial moment
        inertia = inertia + np.eye(3) * (1e-3 * np.trace(inertia) + 1e-12)
    return np.linalg.inv(inertia).T.reshape(9)


# ---- orientation helpers -------------------------------------------------------------------
def random_quaternions(rng: np.random.Generator, n: int) -> np.ndarray:
    """Uniform random unit quaternions (Shoemake), layout (x, y, z, w)."""
    u1, u2, u3 = rng.random(n), rng.random(n), rng.random(n)
    a, b = np.sqrt(1 - u1), np.sqrt(u1)
    q = np.stack([a * np.sin(2 * np.pi * u2), a * np.cos(2 * np.pi * u2),
                  b * np.sin(2 * np.pi * u3), b * np.cos(2 * np.pi * u3)], -1)
    return q


def quat_to_matrix(q: np.ndarray) -> np.ndarray:
    x, y, z, w = q[..., 0], q[..., 1], q[..., 2], q[..., 3]
    return np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)], -1),
        np.stack([2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)], -1),
        np.stack([2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)], -1),
    ], -2)


def _assemble(shapes: list[np.ndarray], centres: np.ndarray, quats: np.ndarray,
              vels: np.ndarray, radius: float, box_min, box_max, **kw) -> Scene:
    nb = len(shapes)
    counts = np.array([len(s) for s in shapes], np.int64)
    offsets = np.zeros(nb + 1, np.int32)
    offsets[1:] = np.cumsum(counts)
    rel = np.zeros((int(offsets[-1]), 4), np.float32)
    rel[:, :3] = np.concatenate(shapes).astype(np.float32)
    # inverse inertia per distinct shape (shapes are shared objects)
    inv = np.zeros((nb, 9), np.float32)
    cache: dict[int, np.ndarray] = {}
    for b, s in enumerate(shapes):
        if id(s) not in cache:
            cache[id(s)] = inverse_inertia(s.astype(np.float32).astype(np.float64))
        inv[b] = cache[id(s)]
    pos = np.zeros((nb, 4), np.float32)
    pos[:, :3] = centres
    vel = np.zeros((nb, 4), np.float32)
    vel[:, :3] = vels
    return Scene(radius=float(radius), box_min=np.asarray(box_min, np.float32),
                 box_max=np.asarray(box_max, np.float32), body_pos=pos,
                 body_quat=quats.astype(np.float32), body_vel=vel,
                 body_angvel=np.zeros((nb, 4), np.float32),
                 body_mass=counts.astype(np.float32), body_inv_inertia=inv,
                 body_offsets=offsets, particle_rel=rel, **kw)


# ---- config 0: plain single scene ----------------------------------------------------------
def config0(seed: int = 0, lattice: int = 16) -> Scene:
    """4,096 3x3x3 cubes (r = 1/256, spacing 2r) on a jittered 16^3 lattice in the unit box,
    uniform random orientations, v ~ N(0, 0.1); grid 128^3 at cell 2r."""
    rng = np.random.default_rng(seed)
    r = 1.0 / 256
    pitch = 1.0 / lattice
    idx = np.stack(np.meshgrid(*[np.arange(lattice)] * 3, indexing="ij"), -1).reshape(-1, 3)
    centres = (idx + 0.5) * pitch + rng.uniform(-0.2, 0.2, idx.shape) * pitch
    nb = len(centres)
    shape = cube_body(3, 2 * r)
    scene = _assemble([shape] * nb, centres, random_quaternions(rng, nb),
                      rng.normal(0.0, 0.1, (nb, 3)), r, (0, 0, 0), (1, 1, 1),
                      grid_log2=(7, 7, 7), name="plain single scene: 4096 cubes x 27")
    return scene


def small_scene(seed: int, nb_side: int = 4, k: int = 3, r: float = 1.0 / 64,
                box: float = 1.0, v_sigma: float = 0.3, packed: bool = False) -> Scene:
    """A small scene for parity tests: nb_side^3 cubes of k^3 particles in a box of side
    `box`; `packed` places neighbours close enough to be in contact from the first step."""
    rng = np.random.default_rng(seed)
    shape = cube_body(k, 2 * r)
    ext = (k - 1) * 2 * r + 2 * r
    pitch = ext * (0.98 if packed else 1.6)
    idx = np.stack(np.meshgrid(*[np.arange(nb_side)] * 3, indexing="ij"), -1).reshape(-1, 3)
    centres = 0.5 * box + (idx - (nb_side - 1) / 2) * pitch
    centres += rng.uniform(-0.05, 0.05, centres.shape) * pitch
    nb = len(centres)
    return _assemble([shape] * nb, centres, random_quaternions(rng, nb),
                     rng.normal(0.0, v_sigma, (nb, 3)), r, (0, 0, 0), (box, box, box),
                     name=f"small {nb} cubes")


# ---- config 2: plain large pile -------------------------------------------------------------
def config2(seed: int = 0, num_bodies: int = 32768) -> Scene:
    """2,097,152 particles: 32,768 bodies of 64 (equal thirds of 4x4x4 cubes, 1x1x64 rods and
    voxelised spheres padded to 64), r = 1/512, dropped from heights in [0.5, 2] into the box
    [0,1] x [0,3] x [0,1] (y up).  Bodies are laid out in horizontal layers: rod layers (rods
    along x or z, alternating) and block layers (cubes and spheres, random orientations),
    interleaved from y = 0.5 upward, each body jittered inside its slot.  Grid: cell 2r,
    256 x 512 x 256 wrapped cells (25-bit keys), so y in [0, 2) -- the whole pile -- maps to
    distinct cells; a 256^3 grid would fold y = 1 .. 1.8 onto y = 0 .. 0.8 and make the
    gather visit the folded occupants."""
    rng = np.random.default_rng(seed)
    r = 1.0 / 512
    sp = 2 * r
    cube, rod, sph = cube_body(4, sp), rod_body(64, sp), sphere_body(64, sp)
    kinds = np.arange(num_bodies) % 3  # 0 cube, 1 rod, 2 sphere
    rng.shuffle(kinds)
    n_rod = int((kinds == 1).sum())
    n_blk = num_bodies - n_rod
    # block layers: pitch 0.034 on a 28 x 28 lattice; rod layers: 3 rods per row, rows 0.0105 apart
    blk_pitch, blk_side = 0.034, 28
    rod_rows, rods_per_row, rod_pitch_y = 90, 3, 0.0085
    blk_layers = -(-n_blk // (blk_side * blk_side))
    rod_layers = -(-n_rod // (rod_rows * rods_per_row))
    layer_kind = np.array([0] * blk_layers + [1] * rod_layers)
    rng.shuffle(layer_kind)
    centres, quats, shapes = [], [], []
    y = 0.5
    blk_iter = iter(np.flatnonzero(kinds != 1))
    rod_iter = iter(np.flatnonzero(kinds == 1))
    slots = {}
    rod_layer_no = 0
    for lk in layer_kind:
        if lk == 0:
            y += blk_pitch / 2
            for i in range(blk_side):
                for j in range(blk_side):
                    b = next(blk_iter, None)
                    if b is None:
                        break
                    c = np.array([(i + 0.5) / blk_side, y, (j + 0.5) / blk_side])
                    c += rng.uniform(-0.1, 0.1, 3) * np.array([blk_pitch * 0.5, blk_pitch, blk_pitch * 0.5])
                    slots[b] = (c, random_quaternions(rng, 1)[0])
            y += blk_pitch / 2
        else:
            y += rod_pitch_y / 2
            along_x = rod_layer_no % 2 == 0
            rod_layer_no += 1
            for row in range(rod_rows):
                for k in range(rods_per_row):
                    b = next(rod_iter, None)
                    if b is None:
                        break
                    u = (k + 0.5) / rods_per_row
                    v = (row + 0.5) / rod_rows
                    c = np.array([u, y, v] if along_x else [v, y, u])
                    c[1] += rng.uniform(-0.1, 0.1) * rod_pitch_y
                    # rods lie along x; a 90-degree turn about y puts them along z
                    q = np.array([0, 0, 0, 1.0]) if along_x else np.array([0, np.sin(np.pi / 4), 0, np.cos(np.pi / 4)])
                    slots[b] = (c, q)
            y += rod_pitch_y / 2
    for b in range(num_bodies):
        c, q = slots[b]
        centres.append(c)
        quats.append(q)
        shapes.append([cube, rod, sph][kinds[b]])
    scene = _assemble(shapes, np.array(centres), np.array(quats),
                      rng.normal(0.0, 0.1, (num_bodies, 3)), r, (0, 0, 0), (1, 3, 1),
                      grid_log2=(8, 9, 8), name="plain large pile: 32768 bodies x 64")
    scene.extra["top"] = float(y)
    return scene


# ---- configs 3 / 4: many independent scenes ---------------------------------------------------
def cube_scene(seed: int, num_particles: int, box_side: float, r: float = 1.0 / 256,
               body: str = "cube", mix_rods: bool = False) -> Scene:
    """A scene of 27-particle bodies (3x3x3 cubes; with mix_rods half are 1x1x27 rods) on a
    jittered lattice in a box of the given side (the box is made taller when the bodies need
    more room), config-0 initial distributions."""
    rng = np.random.default_rng(seed)
    nb = max(1, num_particles // 27)
    cube, rod = cube_body(3, 2 * r), rod_body(27, 2 * r)
    kinds = (rng.random(nb) < 0.5) if mix_rods else np.zeros(nb, bool)
    slot = 2 * (27 * r) if mix_rods else 0.035 * (r * 256)
    slot = max(slot, 0.035 * (r * 256))
    side = max(box_side, 4 * slot)
    per_axis = max(1, int(side / slot))
    layers = -(-nb // (per_axis * per_axis))
    height = max(side, (layers + 1) * slot)
    b = np.arange(nb)
    layer, rem = np.divmod(b, per_axis * per_axis)
    i, j = np.divmod(rem, per_axis)
    centres = np.stack([(i + 0.5) * side / per_axis, (layer + 0.5) * slot,
                        (j + 0.5) * side / per_axis], -1)
    centres = centres + rng.uniform(-0.1, 0.1, (nb, 3)) * slot
    quats = random_quaternions(rng, nb)
    if mix_rods:  # rods stay horizontal so neighbouring slots never overlap
        yaw = rng.uniform(0, 2 * np.pi, nb)
        rq = np.stack([np.zeros(nb), np.sin(yaw / 2), np.zeros(nb), np.cos(yaw / 2)], -1)
        quats = np.where(kinds[:, None], rq, quats)
    shapes = [rod if k else cube for k in kinds]
    return _assemble(shapes, centres, quats, rng.normal(0.0, 0.1, (nb, 3)), r,
                     (0, 0, 0), (side, height, side), name=f"{nb} bodies x 27")


def config3(seed: int = 0, num_scenes: int = 256) -> list[Scene]:
    """256 scenes, particle counts log-uniform in [2k, 200k] (multiples of 27), box side
    U[0.5, 2]."""
    rng = np.random.default_rng(seed)
    counts = np.exp(rng.uniform(np.log(2000), np.log(200000), num_scenes))
    sides = rng.uniform(0.5, 2.0, num_scenes)
    return [cube_scene(int(rng.integers(1 << 31)), int(c) // 27 * 27, float(s))
            for c, s in zip(counts, sides)]


def config4_request(rng: np.random.Generator) -> tuple[Scene, int]:
    """One served request: a scene of 1k-500k particles (log-uniform), cubes and rods 50/50,
    asking for K ~ U{10..500} steps."""
    n = int(np.exp(rng.uniform(np.log(1000), np.log(500000))))
    side = float(rng.uniform(0.5, 2.0))
    k = int(rng.integers(10, 501))
    return cube_scene(int(rng.integers(1 << 31)), n, side, mix_rods=True), k


# ---- LBVH point sets ------------------------------------------------------------------------
def lbvh_points(n: int, dist: str, seed: int = 0) -> np.ndarray:
    """[n,4] float32 points (w = 0) for the LBVH microbenchmark: 'uniform' in [0,1]^3, or
    'gmm', a 16-component Gaussian mixture (sigma 0.02, means uniform in [0.1,0.9]^3, clipped
    to [0,1]^3) in which 5 % of the points are replaced by exact copies of other points, so
    that equal Morton codes exercise the index tie-break."""
    rng = np.random.default_rng(seed)
    out = np.zeros((n, 4), np.float32)
    if dist == "uniform":
        out[:, :3] = rng.random((n, 3), dtype=np.float32)
    elif dist == "gmm":
        means = rng.uniform(0.1, 0.9, (16, 3))
        comp = rng.integers(0, 16, n)
        p = means[comp] + rng.normal(0.0, 0.02, (n, 3))
        out[:, :3] = np.clip(p, 0.0, 1.0)
        dup = rng.choice(n, n // 20, replace=False)
        out[dup] = out[rng.integers(0, n, len(dup))]
    else:
        raise ValueError(f"unknown point distribution {dist!r}")
    return out
