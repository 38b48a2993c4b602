"""Rigid bodies from AR_Sim's particle-body files (Data/OBJparticles/<model>/<model>_<scale>.txt).

File format (read by initObject, RigidBodies/RigidBodyAddition.cpp:1486-1580): the first line
is the particle count N, then N lines of "x y z" -- particle centres of a voxelised model at
the file's scale (the shipped files use particle radius 1/64 at scale 1.0, e.g. cube_1_0 is a
4 x 4 x 4 lattice at spacing 2/64).

A body built from a file is centred the way the reference centres it
(RigidBodyAddition.cpp:1579-1624): the mean of the points (summed in file order in float) is
subtracted, plus a per-model shift of a few particle radii (bunny: (-r, r, -r); banana:
(0, 3r, 0); teapot: (0, 2r, 0)).  Its inertia is the particle sum sum_i (|r_i|^2 E - r_i r_i^T)
for unit particle mass.  With ``reference_inertia=True`` the inverse inertia is the one the
reference computes (RigidBodyAddition.cpp:1625-1756): the sum accumulated in float onto a
default-constructed glm::mat3 -- which glm 0.9.7 initialises to the identity, so the tensor is
E + sum -- then the hand-set tensors for some model / scale pairs, glm::inverse, and hand-set
inverse tensors for the cube; the body mass is 1 as the reference keeps it (rbMass,
RigidBodyAddition.cpp:1873).
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

from .scenes import Scene

# per-model shift added to the centre of mass, in particle radii (RigidBodyAddition.cpp:1607-1619)
_CM_SHIFT = {"bunny": (-1.0, 1.0, -1.0), "banana": (0.0, 3.0, 0.0), "teapot": (0.0, 2.0, 0.0)}

# hand-set inertia tensors (diagonal) that replace the particle sum before inversion, and
# hand-set inverse tensors for the cube (RigidBodyAddition.cpp:1683-1756)
_INERTIA_DIAG = {
    ("banana", 2.0): (0.0140314, 0.0218576, 0.0309458),
    ("banana", 1.5): (0.00596544, 0.00895867, 0.0125508),
    ("banana", 1.0): (0.00321249, 0.00464048, 0.00641495),
    ("bunny", 1.5): (0.00989096, 0.00979847, 0.0119784),
    ("teapot", 2.0): (0.0122465, 0.0232885, 0.0208828),
    ("teapot", 1.5): (0.0075797, 0.0140341, 0.012614),
}
_INVERSE_INERTIA_DIAG = {
    ("cube", 1.0): 6.0 / (0.1 * 0.1),
    ("cube", 2.0): 6.0 / (0.2 * 0.2),
    ("cube", 1.5): 6.0 / (0.15 * 0.15),
}


def file_suffix(scale: float) -> str:
    """The file a scale selects.  The reference's comparisons are written
    ``abs(scale - 1.0 < 0.01)``, i.e. ``scale < 1.01``, so in effect: below 1.01 -> 1_0,
    below 1.51 -> 1_5, below 2.01 -> 2_0, below 2.51 -> 2_5, else 1_5
    (RigidBodyAddition.cpp:1493-1503)."""
    for limit, suffix in ((1.01, "1_0"), (1.51, "1_5"), (2.01, "2_0"), (2.51, "2_5")):
        if scale < limit:
            return suffix
    return "1_5"


def body_file(root: str | Path, model: str, scale: float) -> Path:
    """<root>/<model>/<model>_<suffix>.txt, root being a Data/OBJparticles directory."""
    return Path(root) / model / f"{model}_{file_suffix(scale)}.txt"


def read_points(path: str | Path) -> np.ndarray:
    """[N, 3] float32 particle centres from a particle-body file."""
    lines = Path(path).read_text().split("\n")
    n = int(lines[0].split()[0])
    pts = np.array([[float(v) for v in ln.split()[:3]] for ln in lines[1:] if ln.strip()],
                   dtype=np.float32)
    if pts.shape != (n, 3):
        raise ValueError(f"{path}: header says {n} particles, found {len(pts)}")
    return pts


def centre(points: np.ndarray, model: str, radius: float) -> np.ndarray:
    """Body-frame offsets: points minus their mean (a float sum in file order, then divided by
    the count), minus the model's shift."""
    p = np.asarray(points, np.float32)
    cm = np.add.accumulate(p, axis=0, dtype=np.float32)[-1] / np.float32(len(p))
    shift = np.asarray(_CM_SHIFT.get(model, (0.0, 0.0, 0.0)), np.float32) * np.float32(radius)
    return p - (cm + shift)


def _glm_inverse3(m):
    """glm 0.9.7 compute_inverse for tmat3x3<float> (glm/detail/type_mat3x3.inl:37-56), in float;
    m[c][r] is column c, row r."""
    f = np.float32
    det = (f(m[0][0] * (m[1][1] * m[2][2] - m[2][1] * m[1][2]))
           - f(m[1][0] * (m[0][1] * m[2][2] - m[2][1] * m[0][2]))
           + f(m[2][0] * (m[0][1] * m[1][2] - m[1][1] * m[0][2])))
    one = f(1) / f(det)
    inv = [[f(0)] * 3 for _ in range(3)]
    inv[0][0] = (m[1][1] * m[2][2] - m[2][1] * m[1][2]) * one
    inv[1][0] = -(m[1][0] * m[2][2] - m[2][0] * m[1][2]) * one
    inv[2][0] = (m[1][0] * m[2][1] - m[2][0] * m[1][1]) * one
    inv[0][1] = -(m[0][1] * m[2][2] - m[2][1] * m[0][2]) * one
    inv[1][1] = (m[0][0] * m[2][2] - m[2][0] * m[0][2]) * one
    inv[2][1] = -(m[0][0] * m[2][1] - m[2][0] * m[0][1]) * one
    inv[0][2] = (m[0][1] * m[1][2] - m[1][1] * m[0][2]) * one
    inv[1][2] = -(m[0][0] * m[1][2] - m[1][0] * m[0][2]) * one
    inv[2][2] = (m[0][0] * m[1][1] - m[1][0] * m[0][1]) * one
    return inv


def _reference_inverse_inertia(rel: np.ndarray, model: str, scale: float) -> np.ndarray:
    """The inverse inertia initObject computes (RigidBodyAddition.cpp:1625-1756), operation for
    operation in float: E + sum over particles, the hand-set tensors, glm::inverse, the cube's
    hand-set inverse tensors."""
    f = np.float32
    t = [[f(1) if c == r else f(0) for r in range(3)] for c in range(3)]
    for x, y, z in np.asarray(rel, np.float32):
        t[0][0] = t[0][0] + (y * y + z * z)
        t[0][1] = t[0][1] - x * y
        t[0][2] = t[0][2] - x * z
        t[1][0] = t[1][0] - x * y
        t[1][1] = t[1][1] + (x * x + z * z)
        t[1][2] = t[1][2] - y * z
        t[2][0] = t[2][0] - x * z
        t[2][1] = t[2][1] - y * z
        t[2][2] = t[2][2] + (x * x + y * y)
    sf = f(scale)

    def near_f(v):  # abs(scale - v.f) < 0.0001, the difference taken in float
        return abs(float(sf - f(v))) < 0.0001

    def diag(d):
        return [[f(d[c]) if c == r else f(0) for r in range(3)] for c in range(3)]

    for m_, chain in (("banana", (2.0, 1.5, 1.0)), ("bunny", (1.5,)), ("teapot", (2.0, 1.5))):
        if model == m_:
            for v in chain:  # an if / else-if chain: the first match wins
                if near_f(v):
                    t = diag(_INERTIA_DIAG[(model, v)])
                    break
    t = _glm_inverse3(t)
    if model == "cube":
        if near_f(1.0):
            t = diag([_INVERSE_INERTIA_DIAG[("cube", 1.0)]] * 3)
        elif near_f(2.0):
            t = diag([_INVERSE_INERTIA_DIAG[("cube", 2.0)]] * 3)
        if abs(float(sf) - 1.5) < 0.0001:  # this one compares in double
            t = diag([_INVERSE_INERTIA_DIAG[("cube", 1.5)]] * 3)
    return np.array([t[c][r] for c in range(3) for r in range(3)], np.float32)


def inverse_inertia(rel: np.ndarray, model: str = "", scale: float = 1.0,
                    reference_inertia: bool = False) -> np.ndarray:
    """Inverse inertia (glm::mat3 layout, 9 floats) of unit-mass particles at offsets `rel`
    (the physical tensor, computed in double), or with ``reference_inertia`` the one the
    reference computes for this model and scale."""
    if reference_inertia:
        return _reference_inverse_inertia(rel, model, scale)
    r = np.asarray(rel, np.float64)
    inertia = (r * r).sum() * np.eye(3) - r.T @ r
    return np.linalg.inv(inertia).astype(np.float32).T.reshape(9)


def load_body(root: str | Path, model: str, scale: float, radius: float,
              reference_inertia: bool = False):
    """(offsets [N, 3], inverse inertia [9], mass) of a model at a scale."""
    pts = read_points(body_file(root, model, scale))
    rel = centre(pts, model, radius)
    mass = 1.0 if reference_inertia else float(len(rel))
    return rel, inverse_inertia(rel, model, scale, reference_inertia), mass


def scene_from_files(root: str | Path, placements: list[tuple[str, float]], centres,
                     quats, radius: float, box_min, box_max, velocities=None,
                     reference_inertia: bool = False, **kw) -> Scene:
    """A scene of bodies read from particle-body files: placements[i] = (model, scale) of
    body i, placed at centres[i] with orientation quats[i] (x, y, z, w)."""
    cache: dict = {}
    rels, invs, masses = [], [], []
    for model, scale in placements:
        key = (model, file_suffix(scale))
        if key not in cache:
            cache[key] = load_body(root, model, scale, radius, reference_inertia)
        rel, inv, m = cache[key]
        rels.append(rel)
        invs.append(inv)
        masses.append(m)
    nb = len(placements)
    offsets = np.zeros(nb + 1, np.int32)
    offsets[1:] = np.cumsum([len(r) for r in rels])
    prel = np.zeros((offsets[-1], 4), np.float32)
    prel[:, :3] = np.concatenate(rels)
    pos = np.zeros((nb, 4), np.float32)
    pos[:, :3] = np.asarray(centres, np.float32)
    vel = np.zeros((nb, 4), np.float32)
    if velocities is not None:
        vel[:, :3] = np.asarray(velocities, np.float32)
    return Scene(radius=radius, box_min=np.asarray(box_min, np.float32),
                 box_max=np.asarray(box_max, np.float32), body_pos=pos,
                 body_quat=np.asarray(quats, np.float32).reshape(nb, 4).copy(), body_vel=vel,
                 body_angvel=np.zeros((nb, 4), np.float32),
                 body_mass=np.asarray(masses, np.float32),
                 body_inv_inertia=np.stack(invs).astype(np.float32), body_offsets=offsets,
                 particle_rel=prel, name="from particle-body files", **kw)
