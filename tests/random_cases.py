"""Seeded random single-block cases for parity checks: block shapes from
two nodes to a few dozen per axis, every boundary surface defined in a
random order, walls moving in random directions (normal components too,
so some walls are inlets), an optional pressure outlet, optional
periodic axes, an optional first-order body force with or without the
force-shifted velocity moments, random relaxation time and initial state.
Each case is small enough for the reference's CPU build to run in well
under a second."""
import math

import numpy as np

from mplb_b200 import config

SQRT3 = math.sqrt(3.0)
FACES = {2: ("Left", "Right", "Top", "Bottom"),
         3: ("Left", "Right", "Top", "Bottom", "Front", "Back")}
# surfaces paired across each axis (x, y, z)
AXES = (("Left", "Right"), ("Bottom", "Top"), ("Back", "Front"))

SEEDS = list(range(24))


def random_case(seed: int):
    """(case, steps) for one seed; check period = half the steps."""
    rng = np.random.default_rng(1000 + seed)
    dim = 2 if seed % 2 == 0 else 3
    hi = 17 if dim == 2 else 9
    size = tuple(int(rng.integers(2, hi)) for _ in range(dim))
    mesh = 1.0 / (max(size) - 1)
    dt = mesh / SQRT3
    tau_l = float(rng.uniform(0.52, 1.3))
    mt = ("Variable_U", "Variable_V", "Variable_W")[:dim]

    # periodic axes: x in a third of the cases, z in a third of the 3D ones
    periodic = []
    if rng.random() < 1 / 3:
        periodic.append(0)
    if dim == 3 and rng.random() < 1 / 3:
        periodic.append(2)
    faces = [f for f in FACES[dim]
             if not any(f in AXES[a] for a in periodic)]
    outlet = faces[int(rng.integers(len(faces)))] \
        if rng.random() < 0.3 else None
    # every surface, periodic ones included, in a random definition order
    order = list(FACES[dim])
    rng.shuffle(order)
    bounds = []
    for f in order:
        if f not in faces:
            bounds.append(config.BoundaryDef(0, f, "MDPeriodic", "MDPeriodic"))
        elif f == outlet:
            bounds.append(config.BoundaryDef(
                0, f, "ExtrapolPressure1ST", "OutLet",
                (float(rng.uniform(0.99, 1.01)),), ("Variable_Rho",)))
        else:
            u = tuple(float(v) for v in SQRT3 * rng.uniform(-0.04, 0.04, dim))
            bounds.append(config.BoundaryDef(0, f, "EQMDiffuseRefl", "Wall",
                                             u, mt))
    conns = []
    for a in periodic:
        lo, hi_face = AXES[a]
        conns.append(config.ConnectionDef(0, lo, 0, hi_face, "MDPeriodic"))
        conns.append(config.ConnectionDef(0, hi_face, 0, lo, "MDPeriodic"))

    force = rng.random() < 0.5
    accel = (0.0, 0.0, 0.0)
    if force:
        g = rng.uniform(-1e-4, 1e-4, 3) * mesh / (dt * dt)
        accel = tuple(float(v) for v in g[:dim]) + (0.0,) * (3 - dim)
    rho0 = float(rng.uniform(0.98, 1.02))
    u0 = tuple(float(v) for v in SQRT3 * rng.uniform(-0.02, 0.02, 3))
    steps = int(rng.integers(8, 31))
    case = config.CaseConfig(
        case_name=f"random{seed}", space_dim=dim, block_ids=[0],
        block_names=["Box"], block_sizes=[size], mesh_size=mesh,
        tau_ref=config.lattice_tau_to_tauref(tau_l, dt), boundaries=bounds,
        connections=conns,
        force_velocity=bool(force and rng.random() < 0.5),
        body_force="BodyForce_1st" if force else "BodyForce_None",
        accel=accel, initial=(rho0,) + u0[:dim] + (0.0,) * (3 - dim),
        check_period=max(1, steps // 2))
    return case, steps


MULTI_SEEDS = list(range(12))


def random_two_blocks(seed: int):
    """(case, steps): two blocks joined through VirtualBoundary connections
    along a random axis (block 0 below, block 1 above), equal extents
    across the joint; every other surface of both blocks a moving wall, an
    outlet or periodic, all defined in one random order."""
    rng = np.random.default_rng(5000 + seed)
    dim = 2 if seed % 2 == 0 else 3
    hi = 13 if dim == 2 else 8
    axis = int(rng.integers(dim))
    base = [int(rng.integers(2, hi)) for _ in range(dim)]
    sizes = []
    for _ in range(2):
        s = list(base)
        s[axis] = int(rng.integers(2, hi))
        sizes.append(tuple(s))
    mesh = 1.0 / (max(max(s) for s in sizes) - 1)
    dt = mesh / SQRT3
    tau_l = float(rng.uniform(0.52, 1.3))
    mt = ("Variable_U", "Variable_V", "Variable_W")[:dim]
    lo_face, hi_face = AXES[axis]
    # one periodic axis other than the joint's in a third of the cases
    others = [a for a in range(dim) if a != axis]
    periodic = int(rng.choice(others)) if rng.random() < 1 / 3 else None
    items = [(b, f) for b in (0, 1) for f in FACES[dim]]
    rng.shuffle(items)
    outlet = None
    if rng.random() < 0.4:
        cand = [(b, f) for b, f in items
                if not (b == 0 and f == hi_face) and not (b == 1 and f == lo_face)
                and (periodic is None or f not in AXES[periodic])]
        outlet = cand[int(rng.integers(len(cand)))]
    bounds = []
    for b, f in items:
        if (b == 0 and f == hi_face) or (b == 1 and f == lo_face):
            bounds.append(config.BoundaryDef(b, f, "None", "VirtualBoundary"))
        elif periodic is not None and f in AXES[periodic]:
            bounds.append(config.BoundaryDef(b, f, "MDPeriodic", "MDPeriodic"))
        elif (b, f) == outlet:
            bounds.append(config.BoundaryDef(
                b, f, "ExtrapolPressure1ST", "OutLet",
                (float(rng.uniform(0.99, 1.01)),), ("Variable_Rho",)))
        else:
            u = tuple(float(v) for v in SQRT3 * rng.uniform(-0.04, 0.04, dim))
            bounds.append(config.BoundaryDef(b, f, "EQMDiffuseRefl", "Wall",
                                             u, mt))
    conns = [config.ConnectionDef(0, hi_face, 1, lo_face, "VirtualBoundary"),
             config.ConnectionDef(1, lo_face, 0, hi_face, "VirtualBoundary")]
    if periodic is not None:
        p_lo, p_hi = AXES[periodic]
        for b in (0, 1):
            conns += [config.ConnectionDef(b, p_lo, b, p_hi, "MDPeriodic"),
                      config.ConnectionDef(b, p_hi, b, p_lo, "MDPeriodic")]
    start = {0: [0.0] * dim, 1: [0.0] * dim}
    start[1][axis] = sizes[0][axis] * mesh
    force = rng.random() < 0.5
    accel = (0.0, 0.0, 0.0)
    if force:
        g = rng.uniform(-1e-4, 1e-4, 3) * mesh / (dt * dt)
        accel = tuple(float(v) for v in g[:dim]) + (0.0,) * (3 - dim)
    rho0 = float(rng.uniform(0.98, 1.02))
    u0 = tuple(float(v) for v in SQRT3 * rng.uniform(-0.02, 0.02, 3))
    steps = int(rng.integers(8, 25))
    case = config.CaseConfig(
        case_name=f"random2b{seed}", space_dim=dim, block_ids=[0, 1],
        block_names=["Low", "High"], block_sizes=sizes, mesh_size=mesh,
        tau_ref=config.lattice_tau_to_tauref(tau_l, dt), boundaries=bounds,
        connections=conns, start_pos=start,
        force_velocity=bool(force and rng.random() < 0.5),
        body_force="BodyForce_1st" if force else "BodyForce_None",
        accel=accel, initial=(rho0,) + u0[:dim] + (0.0,) * (3 - dim),
        check_period=max(1, steps // 2))
    return case, steps


SWAP_SEEDS = list(range(8))


def random_swap_box(seed: int):
    """(case, steps) for the one-array swap scheme: a 3D box (the scheme's
    scope: one block, every surface an EQMDiffuseRefl wall) with random
    shape, wall velocities, definition order, body force and initial
    state."""
    rng = np.random.default_rng(9000 + seed)
    size = tuple(int(rng.integers(3, 12)) for _ in range(3))
    mesh = 1.0 / (max(size) - 1)
    dt = mesh / SQRT3
    tau_l = float(rng.uniform(0.52, 1.3))
    mt = ("Variable_U", "Variable_V", "Variable_W")
    order = list(FACES[3])
    rng.shuffle(order)
    bounds = [config.BoundaryDef(
        0, f, "EQMDiffuseRefl", "Wall",
        tuple(float(v) for v in SQRT3 * rng.uniform(-0.04, 0.04, 3)), mt)
        for f in order]
    force = rng.random() < 0.5
    accel = (0.0, 0.0, 0.0)
    if force:
        accel = tuple(float(v) for v in
                      rng.uniform(-1e-4, 1e-4, 3) * mesh / (dt * dt))
    rho0 = float(rng.uniform(0.98, 1.02))
    u0 = tuple(float(v) for v in SQRT3 * rng.uniform(-0.02, 0.02, 3))
    steps = int(rng.integers(8, 31))
    case = config.CaseConfig(
        case_name=f"randomswap{seed}", space_dim=3, block_ids=[0],
        block_names=["Box"], block_sizes=[size], mesh_size=mesh,
        tau_ref=config.lattice_tau_to_tauref(tau_l, dt), boundaries=bounds,
        body_force="BodyForce_1st" if force else "BodyForce_None",
        accel=accel, initial=(rho0,) + u0, check_period=max(1, steps // 2),
        scheme="Scheme_StreamCollision_Swap")
    return case, steps
