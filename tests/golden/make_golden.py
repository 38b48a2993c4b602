"""Generate the golden fixtures in this directory from the reference's own kernel bodies.

    python tests/golden/make_golden.py

Needs oracle/_ref/libref_cpu.so (built from the reference checkout by oracle/ref_build.py).
Every array saved here is an output of the reference code (run on the CPU) on seeded
inputs that are saved alongside; the oracle and the CUDA library are checked against them.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from diploma_thesis_b200 import scenes  # noqa: E402
from oracle import ref  # noqa: E402
from oracle.ref import SimParams  # noqa: E402  (the reference's struct layout)

OUT = Path(__file__).resolve().parent


def params_for(radius, origin, cell, dims, spring, damping, shear, attraction=0.0,
               gravity=(0.0, -0.012, 0.0), w_damping=0.99):
    p = SimParams()
    p.particle_radius = radius
    for a in range(3):
        p.world_origin[a] = origin[a]
        p.cell_size[a] = cell
        p.grid_size[a] = dims[a]
        p.gravity[a] = gravity[a]
    p.num_cells = int(np.prod(dims))
    p.spring, p.damping, p.shear, p.attraction = spring, damping, shear, attraction
    p.w_damping = w_damping
    return p


def lbvh_case(seed: int, n: int, dup_frac: float):
    rng = np.random.default_rng(seed)
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = rng.random((n, 3), dtype=np.float32)
    ndup = int(n * dup_frac)
    src = rng.integers(0, n, ndup)
    dst = rng.integers(0, n, ndup)
    pos[dst] = pos[src]
    mn, mx = ref.aabb(pos)
    codes, idx = ref.morton30(pos, mn, mx)
    skeys, svals = ref.sort_pairs_u32(codes, idx.view(np.uint32))
    tree = ref.radix_tree(skeys)
    r = np.float32(0.002)
    cms, leaf_bounds, bounds, radii = ref.leaves_and_refit(tree, svals.astype(np.int32), pos, r)
    return dict(pos=pos, mn=mn, mx=mx, codes=codes, skeys=skeys, svals=svals,
                is_leaf=tree["is_leaf"], left=tree["left"], right=tree["right"],
                parent=tree["parent"], min_r=tree["min_r"], max_r=tree["max_r"],
                radius=np.float32(r), cms=cms, leaf_bounds=leaf_bounds, bounds=bounds)


def dem_case(seed: int):
    sc = scenes.small_scene(seed, nb_side=5, packed=True)
    rng = np.random.default_rng(seed + 100)
    pos = sc.world_positions()
    n = len(pos)
    vel = np.zeros((n, 4), np.float32)
    vel[:, :3] = rng.normal(0, 0.3, (n, 3))
    rel = sc.particle_rel.copy()
    rb = sc.body_index()
    dims = (16, 16, 16)  # wrapped grid (exercises the & (G-1) aliasing)
    cell = np.float32(2 * sc.radius)
    prm = params_for(sc.radius, (0.0, 0.0, 0.0), cell, dims, 0.5, 0.02, 0.1, 0.001)
    h, idx = ref.calc_hash(prm, pos)
    sh, si = ref.sort_pairs_u32(h, idx)
    cs, ce, sp, sv = ref.reorder(sh, si, pos, vel, int(np.prod(dims)))
    pf, pt = ref.collide_grid_dem(prm, rb, sp, sv, rel, si, cs, ce)
    # BVH path on the same particles
    mn, mx = ref.aabb(pos)
    codes, cidx = ref.morton30(pos, mn, mx)
    bk, bv = ref.sort_pairs_u32(codes, cidx.view(np.uint32))
    tree = ref.radix_tree(bk)
    cms, _, bounds, radii = ref.leaves_and_refit(tree, bv.astype(np.int32), pos, sc.radius)
    bpf, bpt, bpp = ref.collide_bvh_rigid(prm, rb, rel, vel, tree, cms, bounds,
                                          bv.astype(np.int32), radii)
    cd, cpi, cbi = ref.find_rb_collisions_bvh(prm, rb, tree, cms, bounds, bv.astype(np.int32),
                                              radii, np.zeros(n, np.float32))
    # per-body reduction as the reference does it (scan differences)
    nb = sc.num_bodies
    bvel = rng.normal(0, 1, (nb, 4)).astype(np.float32)
    bang = rng.normal(0, 1, (nb, 4)).astype(np.float32)
    counts = np.diff(sc.body_offsets).astype(np.int32)
    rvel, rang = ref.reduce_impulses(pf, pt, bvel, bang, sc.body_mass, sc.body_inv_inertia,
                                     counts)
    return dict(pos=pos, vel=vel, rel=rel, rb=rb, offsets=sc.body_offsets, radius=np.float32(sc.radius),
                cell=cell, dims=np.array(dims, np.uint32), prm=np.array([0.5, 0.02, 0.1, 0.001], np.float32),
                hash=h, shash=sh, sidx=si, cell_start=cs, cell_end=ce, spos=sp, svel=sv,
                pforce=pf, ptorque=pt, mn=mn, mx=mx, bvh_keys=bk, bvh_idx=bv, cms=cms,
                bounds=bounds, radii=radii, bvh_pforce=bpf, bvh_ptorque=bpt, bvh_ppos=bpp,
                contact_distance=cd, contact_particle=cpi, contact_body=cbi,
                body_mass=sc.body_mass, body_inv_inertia=sc.body_inv_inertia, bvel=bvel,
                bang=bang, ref_reduced_vel=rvel, ref_reduced_ang=rang)


def static_scene_case(seed: int):
    """Particles of a packed scene against a wavy static point cloud with normals (the AR
    scene) that cuts through them."""
    sc = scenes.small_scene(seed, nb_side=4, packed=True)
    rng = np.random.default_rng(seed + 200)
    pos = sc.world_positions()
    n = len(pos)
    vel = np.zeros((n, 4), np.float32)
    vel[:, :3] = rng.normal(0, 0.3, (n, 3))
    rel = sc.particle_rel.copy()
    r = sc.radius
    lo, hi = pos[:, :3].min(0), pos[:, :3].max(0)
    xs = np.arange(lo[0] - 2 * r, hi[0] + 2 * r, 2 * r, dtype=np.float32)
    zs = np.arange(lo[2] - 2 * r, hi[2] + 2 * r, 2 * r, dtype=np.float32)
    X, Z = np.meshgrid(xs, zs, indexing="ij")
    ymid = 0.5 * (lo[1] + hi[1])
    Y = ymid + 3 * r * np.sin(X * 40.0) * np.cos(Z * 30.0)
    m = X.size
    spos = np.zeros((m, 4), np.float32)
    spos[:, 0], spos[:, 1], spos[:, 2] = X.ravel(), Y.ravel(), Z.ravel()
    nrm = np.zeros((m, 4), np.float32)
    gx = -3 * r * 40.0 * np.cos(X * 40.0) * np.cos(Z * 30.0)
    gz = 3 * r * 30.0 * np.sin(X * 40.0) * np.sin(Z * 30.0)
    nv = np.stack([-gx.ravel(), np.ones(m), -gz.ravel()], 1)
    nrm[:, :3] = nv / np.linalg.norm(nv, axis=1, keepdims=True)
    dims = (16, 16, 16)
    cell = np.float32(2 * r)
    prm = params_for(r, (0.0, 0.0, 0.0), cell, dims, 0.5, 0.02, 0.1, 0.001)
    h, idx = ref.calc_hash(prm, pos)
    sh, si = ref.sort_pairs_u32(h, idx)
    _, _, sp, sv = ref.reorder(sh, si, pos, vel, int(np.prod(dims)))
    ah, aidx = ref.calc_hash(prm, spos)
    ash, asi = ref.sort_pairs_u32(ah, aidx)
    acs, ace, asp, _ = ref.reorder(ash, asi, spos, np.zeros_like(spos), int(np.prod(dims)))
    lin0 = rng.normal(0, 1, (n, 4)).astype(np.float32)
    ang0 = rng.normal(0, 1, (n, 4)).astype(np.float32)
    lin, ang, color = ref.collide_static_scene(prm, sp, sv, rel, asp, nrm, si, asi, acs, ace,
                                               lin0, ang0)
    return dict(radius=np.float32(r), cell=cell, dims=np.array(dims, np.uint32),
                prm=np.array([0.5, 0.02, 0.1, 0.001], np.float32), spos=sp, svel=sv, rel=rel,
                sidx=si, scene_pos=spos, scene_normals=nrm, scene_spos=asp, scene_sidx=asi,
                scene_cell_start=acs, scene_cell_end=ace, lin0=lin0, ang0=ang0, lin=lin,
                ang=ang, color=color)


def body_case(seed: int):
    sc = scenes.small_scene(seed, nb_side=3, v_sigma=1.0)
    rng = np.random.default_rng(seed + 7)
    nb = sc.num_bodies
    st = {"cms": sc.body_pos.copy(), "vel": rng.normal(0, 1, (nb, 4)).astype(np.float32),
          "ang": rng.normal(0, 3, (nb, 4)).astype(np.float32), "quat": sc.body_quat.copy(),
          "ib": sc.body_inv_inertia.copy(), "cur": np.zeros((nb, 9), np.float32),
          "model": np.zeros((nb, 16), np.float32), "cum": scenes.random_quaternions(rng, nb).astype(np.float32)}
    st["ang"][0] = 0.0  # below the rotation threshold: identity branch
    prm = params_for(sc.radius, (0, 0, 0), 1.0, (1, 1, 1), 0.5, 0.0, 0.0)
    out = ref.gpu_integrator(prm, 0.05, st)
    rb = sc.body_index()
    rel, pos, vel, q = ref.global_attributes(out["cms"], out["vel"], out["ang"], out["quat"], rb,
                                             sc.particle_rel)
    # walls: push the scene against the -x / +y walls with velocities toward them
    ppos = pos.copy()
    bpos = out["cms"].copy()
    ppos[:, 0] -= 0.47
    bpos[:, 0] -= 0.47
    ppos[:, 1] += 0.47
    bpos[:, 1] += 0.47
    wv = out["vel"].copy()
    wv[:, 0] = -np.abs(wv[:, 0])
    wv[:, 1] = np.abs(wv[:, 1])
    counts = np.diff(sc.body_offsets).astype(np.int32)
    wvel, wang = ref.wall_collisions(ppos, bpos, [0, 0, 0], [1, 1, 1], wv, out["ang"],
                                     sc.body_inv_inertia, sc.body_mass, rb, counts, sc.radius)
    return dict(in_cms=st["cms"], in_vel=st["vel"], in_ang=st["ang"], in_quat=st["quat"],
                in_cum=st["cum"], ib=st["ib"], dt=np.float32(0.05),
                gravity=np.array([0, -0.012, 0], np.float32), w_damping=np.float32(0.99),
                out_cms=out["cms"], out_vel=out["vel"], out_ang=out["ang"], out_quat=out["quat"],
                out_cur=out["cur"], out_model=out["model"], out_cum=out["cum"],
                rb=rb, in_rel=sc.particle_rel, out_rel=rel, out_pos=pos, out_pvel=vel,
                out_q_reset=q, wall_ppos=ppos, wall_bpos=bpos, wall_vel_in=wv,
                wall_ang_in=out["ang"], mass=sc.body_mass, offsets=sc.body_offsets,
                radius=np.float32(sc.radius), wall_vel_out=wvel, wall_ang_out=wang)


def extra_case(seed: int):
    """integrateRigidBody, integrate_functor and collideD on seeded inputs."""
    rng = np.random.default_rng(seed)
    sc = scenes.small_scene(seed, nb_side=3, v_sigma=1.0)
    nb = sc.num_bodies
    st = {"cms": sc.body_pos.copy(), "vel": np.zeros((nb, 4), np.float32),
          "force": rng.normal(0, 2, (nb, 4)).astype(np.float32),
          "ang": np.zeros((nb, 4), np.float32), "quat": sc.body_quat.copy(),
          "torque": rng.normal(0, 0.5, (nb, 4)).astype(np.float32),
          "angmom": rng.normal(0, 0.05, (nb, 4)).astype(np.float32),
          "linmom": rng.normal(0, 3, (nb, 4)).astype(np.float32),
          "ib": sc.body_inv_inertia.copy(), "cur": np.zeros((nb, 9), np.float32),
          "acc": np.zeros((nb, 3), np.float32)}
    st["cms"][:3, 0] = [-0.2, 1.3, 0.5]  # exercise the box clamps
    st["cms"][3:5, 2] = [-1.5, 1.2]
    radii = np.full(nb, 0.05, np.float32)
    inv_mass = (1.0 / sc.body_mass).astype(np.float32)
    prm = params_for(sc.radius, (0, 0, 0), 1.0, (1, 1, 1), 0.5, 0.0, 0.0, gravity=(0, -0.5, 0))
    prm.boundary_damping = -0.5
    prm.global_damping = 0.999
    mom = ref.integrate_momentum(prm, st, 0.02, radii, inv_mass, [0, 0, 0], [1, 1, 1])
    # free particles (rb_idx -1) mixed with rigid ones
    n = 500
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = rng.uniform(-0.05, 1.05, (n, 3))
    pos[:, 3] = 1.0
    vel = np.zeros((n, 4), np.float32)
    vel[:, :3] = rng.normal(0, 1, (n, 3))
    rbi = np.where(rng.random(n) < 0.5, -1, 0).astype(np.int32)
    pp, pv = ref.integrate_particles(prm, pos, vel, rbi, 0.01, [0, 0, 0], [1, 1, 1])
    # collideD on the dem_small inputs (dem_case(5)) with a few free particles
    d = dem_case(5)
    rb = d["rb"].copy()
    rb[::17] = -1
    prm2 = params_for(float(d["radius"]), (0, 0, 0), float(d["cell"]), tuple(d["dims"]), 0.5,
                      0.02, 0.1, 0.001)
    nv0 = np.zeros_like(d["pos"])
    cpf, cpt, cnv = ref.collide_particles(prm2, rb, d["rel"], d["spos"], d["svel"], d["sidx"],
                                          d["cell_start"], d["cell_end"], nv0)
    out = {f"mom_in_{k}": v for k, v in st.items()}
    out.update({f"mom_out_{k}": v for k, v in mom.items()})
    out.update(dict(mom_radii=radii, mom_inv_mass=inv_mass, mom_dt=np.float32(0.02),
                    fp_pos=pos, fp_vel=vel, fp_rb=rbi, fp_pos_out=pp, fp_vel_out=pv,
                    cd_rb=rb, cd_pforce=cpf, cd_ptorque=cpt, cd_newvel=cnv))
    return out


def sis_case(seed: int):
    """FindRigidBodyCollisionsUniformGridKernel (the sequential-impulse path's contact search) on
    the dem_small inputs: deepest contact per particle."""
    d = dem_case(seed)
    prm = params_for(float(d["radius"]), (0, 0, 0), float(d["cell"]), tuple(d["dims"]), 0.5,
                     0.02, 0.1, 0.001)
    cd, cb, cp = ref.find_rb_collisions_grid(prm, d["rb"], d["spos"], d["sidx"], d["cell_start"],
                                             d["cell_end"], np.zeros(len(d["pos"]), np.float32))
    return dict(rb=d["rb"], spos=d["spos"], sidx=d["sidx"], cell_start=d["cell_start"],
                cell_end=d["cell_end"], radius=d["radius"], cell=d["cell"], dims=d["dims"],
                contact_distance=cd, contact_body=cb, contact_particle=cp)


def sis_solve_case(seed: int):
    """The reference's sequential-impulse host loops (GatherRigidBodyCollisions /
    GatherAugmentedRealityCollisions, then SequentialImpulseSolver; Particles/
    updateFunctions.cpp:1431-1874) on seeded body state.  rb_*: the grid contacts of sis_find
    (body against body); ar_*: one contact per chosen particle against a static point cloud
    with seeded normals (body against scene, the solver's one-body branch)."""
    f = sis_case(5)
    d = dem_case(5)
    rng = np.random.default_rng(seed)
    nb = len(d["offsets"]) - 1
    cms = np.zeros((nb, 4), np.float32)
    cms[:, :3] = rng.uniform(0.2, 0.8, (nb, 3))
    vel = rng.normal(0, 1, (nb, 4)).astype(np.float32)
    ang = rng.normal(0, 1, (nb, 4)).astype(np.float32)
    vel[:, 3] = ang[:, 3] = 0
    rel = d["rel"].copy()
    rel[:, 3] = 0
    prm = ref.sim_params(float(f["radius"]), (0, 0, 0), float(f["cell"]), f["dims"],
                         gravity=(0.0, -9.81, 0.0))
    prm.rb_restitution, prm.rb_friction = 0.5, 0.1
    prm.ar_restitution, prm.ar_friction = 0.3, 0.3
    ib, mass = d["body_inv_inertia"].astype(np.float32), d["body_mass"].astype(np.float32)
    rb = ref.sis_step(prm, f["rb"], d["offsets"], cms, vel, ang, ib, mass, rel,
                      f["contact_distance"], f["contact_body"], f["contact_particle"])
    n, m = len(f["rb"]), 500
    nrm = rng.normal(0, 1, (m, 3))
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    scene_normals = np.concatenate([nrm, np.zeros((m, 1))], 1).astype(np.float32)
    ar_cd = np.where(rng.random(n) < 0.05, rng.uniform(1e-4, 1e-3, n), 0).astype(np.float32)
    ar_cp = rng.integers(0, m, n).astype(np.int32)
    ar = ref.sis_step(prm, f["rb"], d["offsets"], cms, vel, ang, ib, mass, rel, ar_cd, None,
                      ar_cp, scene_normals4=scene_normals)
    out = dict(radius=f["radius"], cell=f["cell"], dims=f["dims"], rb_idx=f["rb"],
               offsets=d["offsets"], cms=cms, vel=vel, ang=ang, inv_inertia=ib, mass=mass,
               rel=rel, contact_distance=f["contact_distance"], contact_body=f["contact_body"],
               contact_particle=f["contact_particle"], scene_normals=scene_normals,
               ar_contact_distance=ar_cd, ar_contact_particle=ar_cp,
               restitution=np.float32(0.5), rb_friction=np.float32(0.1),
               ar_restitution=np.float32(0.3), ar_friction=np.float32(0.3),
               gravity_y=np.float32(-9.81), iterations=np.int32(18))
    for tag, r in (("rb", rb), ("ar", ar)):
        for key in ("normal", "point", "body1", "body2", "bias", "acc", "vel", "ang"):
            out[f"{tag}_{key}"] = r[key]
    return out


def static_scene_ar_case(seed: int):
    """The static-scene inputs of static_scene_case through the reference's impulse variant
    (ARcollisionsUniformGridKernel), its deepest-contact search
    (FindAugmentedRealityCollisionsUniformGridKernel), the contact gather and the solver
    (GatherAugmentedRealityCollisions + SequentialImpulseSolver) -- the reference's augmented-
    reality sequential-impulse update, stage by stage."""
    d = static_scene_case(seed)
    sc = scenes.small_scene(seed, nb_side=4, packed=True)
    rng = np.random.default_rng(seed + 300)
    n, nb = sc.num_particles, sc.num_bodies
    rb = sc.body_index().astype(np.int32)
    r = float(d["radius"])
    m = len(d["scene_pos"])
    scene_radii = (r * rng.uniform(0.8, 1.2, m)).astype(np.float32)
    inertia = np.zeros((nb, 9), np.float32)
    inertia[:, [0, 4, 8]] = rng.uniform(5, 50, (nb, 3))
    inertia[:, [1, 3]] = rng.uniform(-1, 1, (nb, 1))  # symmetric off-diagonal terms
    mass = rng.uniform(0.5, 2.0, nb).astype(np.float32)
    prm = ref.sim_params(r, (0, 0, 0), float(d["cell"]), d["dims"], gravity=(0.0, -9.81, 0.0))
    prm.ar_restitution, prm.ar_friction = 0.4, 0.3
    pf, pt, count, color, _ = ref.ar_collide_impulse(
        prm, rb, d["rel"], inertia, mass, scene_radii, d["spos"], d["svel"], d["scene_spos"],
        d["scene_normals"], d["sidx"], d["scene_sidx"], d["scene_cell_start"],
        d["scene_cell_end"], np.zeros((n, 4), np.float32))
    cd0 = np.zeros(n, np.float32)
    cp0 = np.full(n, -1, np.int32)
    cd, cp, fcolor = ref.ar_find_contacts(prm, d["spos"], d["scene_spos"], d["sidx"],
                                          d["scene_sidx"], d["scene_cell_start"],
                                          d["scene_cell_end"], cd0, cp0)
    cms = np.zeros((nb, 4), np.float32)
    cms[:, :3] = sc.body_pos[:, :3]
    vel = np.zeros((nb, 4), np.float32)
    vel[:, :3] = rng.normal(0, 0.5, (nb, 3))
    ang = np.zeros((nb, 4), np.float32)
    ang[:, :3] = rng.normal(0, 2, (nb, 3))
    solve = ref.sis_step(prm, rb, sc.body_offsets, cms, vel, ang, inertia, mass, d["rel"], cd,
                         None, cp, scene_normals4=d["scene_normals"])
    out = dict(radius=d["radius"], cell=d["cell"], dims=d["dims"], rb_idx=rb, rel=d["rel"],
               spos=d["spos"], svel=d["svel"], sidx=d["sidx"], scene_normals=d["scene_normals"],
               scene_spos=d["scene_spos"], scene_sidx=d["scene_sidx"],
               scene_cell_start=d["scene_cell_start"], scene_cell_end=d["scene_cell_end"],
               scene_radii=scene_radii, inertia=inertia, mass=mass,
               ar_restitution=np.float32(0.4), ar_friction=np.float32(0.3),
               impulse_force=pf, impulse_torque=pt, impulse_count=count, impulse_color=color,
               contact_distance=cd, contact_point=cp, find_color=fcolor, cms=cms, vel=vel,
               ang=ang, offsets=sc.body_offsets.astype(np.int32))
    for key in ("normal", "point", "body1", "body2", "bias", "acc", "vel", "ang"):
        out["sis_" + key] = solve[key]
    return out


def static_scene_bvh_case(seed: int):
    """Particles against a BVH built over the static point cloud of static_scene_case (the
    reference's own Morton codes, sort, Karras build, leaves and refit), through
    staticCollideBVHSoARigidBody and FindAugmentedRealityCollisionsBVHKernel.  Each particle is
    its own body here, so the reference kernel's per-body read-modify-writes do not collide and
    its body totals are the particles' own; a few particles are free (body -1)."""
    d = static_scene_case(seed)
    rng = np.random.default_rng(seed + 400)
    r = float(d["radius"])
    pos = d["spos"].copy()
    n = len(pos)
    vel = np.zeros((n, 4), np.float32)
    vel[:, :3] = rng.normal(0, 0.3, (n, 3))
    rel = d["rel"].copy()
    rb = np.arange(n, dtype=np.int32)
    rb[rng.random(n) < 0.05] = -1
    cloud = d["scene_pos"]
    m = len(cloud)
    mn, mx = ref.aabb(cloud)
    codes, idx = ref.morton30(cloud, mn, mx)
    sk, si = ref.sort_pairs_u32(codes, idx.view(np.uint32))
    tree = ref.radix_tree(sk)
    cms, _, bounds, radii = ref.leaves_and_refit(tree, si.astype(np.int32), cloud, np.float32(r))
    prm = params_for(r, (0.0, 0.0, 0.0), d["cell"], tuple(d["dims"]), 0.5, 0.02, 0.1, 0.001)
    f0 = np.zeros((n, 4), np.float32)
    mass = np.ones(n, np.float32)
    bf, bt, bvel, color = ref.collide_bvh_static(prm, rb, rel, pos, vel, tree, cms, bounds,
                                                 si.astype(np.int32), radii, f0, f0, mass)
    # the reference reads the query's radius from the scene's radius array at the query's
    # index (RB_BVHKernels.cu:955): give it an array long enough, every radius r, as the
    # reference assumes ("currently the same for all particles")
    padded = np.full(max(n, m), np.float32(r), np.float32)
    cd, cp, fcolor = ref.find_contacts_bvh_static(prm, pos, tree, cms, bounds,
                                                  si.astype(np.int32), padded,
                                                  np.zeros(n, np.float32), np.full(n, -1, np.int32))
    return dict(radius=np.float32(r), prm=np.array([0.5, 0.02, 0.1, 0.001], np.float32),
                pos=pos, vel=vel, rel=rel, rb_idx=rb, is_leaf=tree["is_leaf"], left=tree["left"],
                right=tree["right"], parent=tree["parent"], cms=cms, bounds=bounds,
                sorted_idx=si.astype(np.int32), radii=radii, body_force=bf, body_torque=bt,
                vel_out=bvel, color=color, contact_distance=cd, contact_point=cp,
                find_color=fcolor)


CASES = {
    "lbvh_uniform": lambda: lbvh_case(11, 3000, 0.0),
    "lbvh_duplicates": lambda: lbvh_case(12, 3000, 0.2),
    "dem_small": lambda: dem_case(5),
    "bodies_small": lambda: body_case(9),
    "reference_extra": lambda: extra_case(21),
    "static_scene": lambda: static_scene_case(31),
    "sis_find": lambda: sis_case(5),
    "sis_solve": lambda: sis_solve_case(2),
    "static_scene_ar": lambda: static_scene_ar_case(31),
    "static_scene_bvh": lambda: static_scene_bvh_case(31),
    "range_image": lambda: range_image_case(41),
}


def range_image_case(seed: int):
    """A 96 x 64 depth image (whole 16 x 32 blocks, as loadRangeImage launches): a tilted plane
    with a sphere cap, holes of zero depth and noise, in the TUM depth scale (5000 per metre);
    a rotated and shifted camera."""
    rng = np.random.default_rng(seed)
    h, w = 64, 96
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    z = 1.2 + 0.004 * xx + 0.002 * yy
    cap = 0.25 - ((xx - 40) ** 2 + (yy - 30) ** 2) / 400.0
    z = z - np.clip(cap, 0, None)
    z = z + rng.normal(0, 0.002, z.shape)
    depth = np.clip(np.round(z * 5000.0), 0, 65535).astype(np.uint16)
    depth[rng.random(depth.shape) < 0.03] = 0
    ang = 0.3
    cam = np.eye(4, dtype=np.float32)  # glm::mat4, column-major: cam[column][row]
    cam[0, 0], cam[0, 2], cam[2, 0], cam[2, 2] = np.cos(ang), -np.sin(ang), np.sin(ang), np.cos(ang)
    cam[3, :3] = (0.1, -0.2, 0.3)
    out = ref.range_image(depth, cam.reshape(16), 1.0 / 128)
    return {"depth": depth, "camera16": cam.reshape(16), "radius": np.float32(1.0 / 128), **out}


def main() -> None:
    """python tests/golden/make_golden.py [name ...]: (re)generate the named fixtures, or all."""
    if not ref.available():
        raise SystemExit("oracle/_ref/libref_cpu.so is not built (run oracle/ref_build.py)")
    ref.set_threads(1)
    for name in sys.argv[1:] or CASES:
        np.savez_compressed(OUT / f"{name}.npz", **CASES[name]())
    for f in sorted(OUT.glob("*.npz")):
        print(f.name, f.stat().st_size)


if __name__ == "__main__":
    main()
