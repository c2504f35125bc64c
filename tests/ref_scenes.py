"""Scenes built in the reference engine (through the oracle harness) for the parity tests.

Each builder returns a RefWorld whose full world step (pairs, narrow phase, solver, islands)
is the reference's; the tests cut it at the solver stage (collide, export the view, solve
both ways, compare, finish).
"""
from __future__ import annotations

import numpy as np

from nepheline_b200 import abi, scenes


def pyramid(rows: int = 20, jitter: float = 1e-3, seed: int = 1, params=None, workers: int = 0):
    """The box pyramid: row r holds rows - r unit boxes at x = (j - (n-1)/2) * 1.05,
    y = 0.5 + r (benchmarks/physics/bench_physics.c:1233-1252), +-jitter in x and z, on a
    static ground slab whose top is y = 0 (test_world_support.h:64-68)."""
    from oracle.refworld import RefWorld
    rng = np.random.default_rng(seed)
    w = RefWorld(params or abi.WorldParams.default(), enable_sleep=False, workers=workers)
    w.add_ground(0.0)
    for row in range(rows):
        n = rows - row
        for j in range(n):
            dx, dz = (rng.uniform(-jitter, jitter, 2) if jitter > 0 else (0.0, 0.0))
            w.add_box(((j - (n - 1) / 2) * 1.05 + dx, 0.5 + row, dz))
    return w


def sphere_pour(count: int = 512, seed: int = 2, extent: float = 12.0, params=None,
                workers: int = 0, hit_events: bool = False):
    """Spheres of radius 0.5 with density U[500, 2000], friction U[0.2, 0.9], restitution
    U[0, 0.3], at seeded non-overlapping lattice sites of a box above the ground (every other
    sphere reporting hits when `hit_events`)."""
    from oracle.refworld import RefWorld
    rng = np.random.default_rng(seed)
    w = RefWorld(params or abi.WorldParams.default(), enable_sleep=False, workers=workers)
    w.add_ground(0.0, friction=0.6)
    side = int(np.ceil(count ** (1.0 / 3.0)))
    spacing = max(1.05, extent / side)
    sites = np.stack(np.meshgrid(np.arange(side), np.arange(side), np.arange(side),
                                 indexing="ij"), -1).reshape(-1, 3)[:count]
    rng.shuffle(sites)
    for s in sites:
        p = (s - side / 2) * spacing
        p[1] = 0.6 + s[1] * spacing
        p[[0, 2]] += rng.uniform(-0.02, 0.02, 2)
        w.add_sphere(tuple(p), 0.5, density=float(rng.uniform(500, 2000)),
                     friction=float(rng.uniform(0.2, 0.9)),
                     restitution=float(rng.uniform(0.0, 0.3)),
                     velocity=tuple(rng.uniform(-1.0, 1.0, 3) + np.array([0, -2.0, 0])),
                     hit_events=hit_events and (int(s.sum()) % 2 == 0))
    return w


def box_pile(count: int = 60, seed: int = 3, params=None, workers: int = 0):
    """Boxes of half extents U[0.2, 1.0] at random orientations dropped on the ground."""
    from oracle.refworld import RefWorld
    rng = np.random.default_rng(seed)
    w = RefWorld(params or abi.WorldParams.default(), enable_sleep=False, workers=workers)
    w.add_ground(0.0)
    side = int(np.ceil(np.sqrt(count)))
    for i in range(count):
        half = rng.uniform(0.2, 1.0, 3)
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        x, z = (i % side) * 2.2 - side, (i // side) * 2.2 - side
        w.add_box((x, 1.5 + 2.0 * (i % 3), z), half=tuple(half), rotation=tuple(q))
    return w


_S = 0.70710678


def _qmul(a, b):
    ax, ay, az, aw = a
    bx, by, bz, bw = b
    return (aw * bx + ax * bw + ay * bz - az * by, aw * by - ax * bz + ay * bw + az * bx,
            aw * bz + ax * by - ay * bx + az * bw, aw * bw - ax * bx - ay * by - az * bz)


_RZ90 = (0.0, 0.0, _S, _S)
_RX90 = (_S, 0.0, 0.0, _S)


def hinge_chain(links: int = 12, seed: int = 4, params=None, limits=True, motor=True, spring=True):
    """A chain of capsules on hinge joints hanging from a static anchor, with limits, a motor
    and a spring on alternating links, and a ball-jointed tail with a cone, twist limits and
    friction: every ball and hinge row of the joint solver."""
    from oracle.refworld import RefWorld
    rng = np.random.default_rng(seed)
    w = RefWorld(params or abi.WorldParams.default(), enable_sleep=False)
    anchor = w.add_body(abi.BODY_STATIC, (0.0, 10.0, 0.0))
    bodies = [anchor]
    for i in range(links):
        b = w.add_capsule((0.5 + i * 1.0, 10.0, 0.0), 0.25, 0.25, rotation=_RZ90,
                          velocity=tuple(rng.uniform(-0.5, 0.5, 3)))
        bodies.append(b)
    joints = np.zeros(links, abi.JOINT_DTYPE)
    for i in range(links):
        j = joints[i]
        ball = i >= links - 3
        j["type"] = abi.JOINT_BALL if ball else abi.JOINT_HINGE
        # Anchor at x = i (the previous link's end), frames with X along world z.
        j["frame_a_position"] = (0.0, 0.0, 0.0) if i == 0 else (0.0, -0.5, 0.0)
        j["frame_b_position"] = (0.0, 0.5, 0.0)
        # Frame X along world z on both sides: link rotation Rz(90) times Rx(90) on a link,
        # the product itself on the static anchor.
        j["frame_a_rotation"] = _qmul(_RZ90, _RX90) if i == 0 else _RX90
        j["frame_b_rotation"] = _RX90
        if ball:
            j["ball_enable_swing_limit"] = 1
            j["ball_swing_y"] = 0.6
            j["ball_swing_z"] = 0.4
            j["ball_enable_twist_limit"] = 1
            j["ball_twist_lower"] = -0.3
            j["ball_twist_upper"] = 0.3
            j["ball_friction_torque"] = 0.5
        else:
            if limits and i % 3 == 0:
                j["hinge_enable_limit"] = 1
                j["hinge_lower"] = -0.4
                j["hinge_upper"] = 0.4
            if motor and i % 3 == 1:
                j["hinge_enable_motor"] = 1
                j["hinge_motor_speed"] = 1.5
                j["hinge_max_motor_torque"] = 20.0
            if spring and i % 3 == 2:
                j["hinge_enable_spring"] = 1
                j["hinge_spring_hertz"] = 2.0
                j["hinge_spring_damping_ratio"] = 0.3
                j["hinge_spring_target"] = 0.2
        j["body_a"] = bodies[i]
        j["body_b"] = bodies[i + 1]
    w.add_joints(joints)
    return w


def lattice(edge: int = 6, seed: int = 3, joint_fraction: float = 0.1, params=None,
            workers: int = 0):
    """The synthetic constraint graph in the reference: shapeless bodies, joints created,
    manifolds injected in insertion order (coloured by the reference's phys_graph_add)."""
    from oracle.refworld import lattice_world
    return lattice_world(edge, seed=seed, joint_fraction=joint_fraction, params=params,
                         workers=workers)


def featured_lattice(edge: int = 8, seed: int = 7, params=None):
    """The jointed lattice with every body feature the solver stage reads: a tenth of the bodies
    kinematic and moving, a tenth with lock bits, every body damped (linear and angular, 0-2)
    and gravity-scaled (-1 to 2), a fifth pushed by forces and torques, a fifth with unequal
    principal inertias and spin (the gyroscopic step), and some past the angular and linear
    speed caps."""
    from oracle.refworld import RefWorld
    rng = np.random.default_rng(seed)
    sc = scenes.lattice_graph(edge, seed=seed, joint_fraction=0.15)
    b = sc.bodies
    n = len(b)
    kin = rng.random(n) < 0.1
    # The reference creates no joint between two bodies that are not dynamic.
    both = kin[sc.joints["body_a"]] & kin[sc.joints["body_b"]]
    kin[sc.joints["body_b"][both]] = False
    b["type"][kin] = abi.BODY_KINEMATIC
    b["linear_velocity"][kin] = rng.normal(0.0, 1.0, (int(kin.sum()), 3))
    b["angular_velocity"][kin] = rng.normal(0.0, 1.0, (int(kin.sum()), 3))
    locked = (rng.random(n) < 0.1) & ~kin
    b["locks"][locked] = rng.integers(1, 64, int(locked.sum()))
    b["linear_damping"] = rng.uniform(0.0, 2.0, n)
    b["angular_damping"] = rng.uniform(0.0, 2.0, n)
    b["gravity_scale"] = rng.uniform(-1.0, 2.0, n)
    pushed = rng.random(n) < 0.2
    b["force"][pushed] = rng.normal(0.0, 50.0, (int(pushed.sum()), 3))
    b["torque"][pushed] = rng.normal(0.0, 20.0, (int(pushed.sum()), 3))
    odd = (rng.random(n) < 0.2) & ~kin
    inertia = np.zeros((n, 9), np.float32)
    diag = np.repeat((sc.mass / 6.0)[:, None], 3, axis=1)
    diag[odd] *= rng.uniform(0.3, 3.0, (int(odd.sum()), 3))
    inertia[:, 0], inertia[:, 4], inertia[:, 8] = diag[:, 0], diag[:, 1], diag[:, 2]
    scenes.set_mass(b, sc.mass, inertia)
    b["angular_velocity"][odd] = rng.normal(0.0, 5.0, (int(odd.sum()), 3))
    spin = (rng.random(n) < 0.05) & ~kin
    b["angular_velocity"][spin] = rng.normal(0.0, 300.0, (int(spin.sum()), 3))
    fast = (rng.random(n) < 0.05) & ~kin
    b["linear_velocity"][fast] = rng.normal(0.0, 500.0, (int(fast.sum()), 3))
    w = RefWorld(params or abi.WorldParams.default(), enable_sleep=False)
    w.add_shapeless_bodies(b, sc.mass)
    w.add_joints(sc.joints)
    w.inject_contacts(sc.contacts)
    return w


def _random_quat(rng):
    q = rng.normal(size=4)
    return tuple(q / np.linalg.norm(q))


def _d6_axes(rng, joint, kind):
    """A 6-DOF joint's axes: each locked, limited or free at random, with motors and springs on
    some free or limited axes; `kind` forces the rotation, swing or point block."""
    ax = joint["d6_axes"]
    for i in range(abi.D6_AXES):
        motion = int(rng.choice([abi.AXIS_LOCKED, abi.AXIS_LIMITED, abi.AXIS_FREE], p=[0.4, 0.35, 0.25]))
        if kind == "rotation" and i >= 3:
            motion = abi.AXIS_LOCKED
        if kind == "swing" and i >= 4:
            motion = abi.AXIS_LOCKED
        if kind == "point" and i < 3:
            motion = abi.AXIS_LOCKED
        ax["motion"][i] = motion
        if i < 3:
            lo, hi = sorted(rng.uniform(-0.4, 0.4, 2))
        elif i == 3:
            lo, hi = sorted(rng.uniform(-2.5, 2.5, 2))
        else:
            lo, hi = sorted(rng.uniform(-1.2, 1.2, 2))
        ax["lower"][i], ax["upper"][i] = lo, hi
        if motion != abi.AXIS_LOCKED and rng.random() < 0.4:
            ax["enable_motor"][i] = 1
            ax["motor_speed"][i] = rng.uniform(-1.5, 1.5)
            ax["max_motor_force"][i] = rng.uniform(5.0, 200.0)
        if motion != abi.AXIS_LOCKED and rng.random() < 0.4:
            ax["enable_spring"][i] = 1
            ax["spring_hertz"][i] = rng.uniform(0.5, 5.0)
            ax["spring_damping_ratio"][i] = rng.uniform(0.0, 1.5)
            ax["spring_target"][i] = rng.uniform(-0.2, 0.2)


def joint_zoo(seed: int = 5, params=None, types=None):
    """Every joint type the solver runs, on boxes hanging from static anchors (and from each
    other), apart so that only the joints act: welded cantilevers (fixed); sliders with
    limits, motors and springs; distance joints rigid, as ropes, as limited springs and
    motor-driven; 6-DOF joints with random axes (every block: rotation, swing pair, anchors,
    none); ball and hinge joints between them."""
    from oracle.refworld import RefWorld
    rng = np.random.default_rng(seed)
    w = RefWorld(params or abi.WorldParams.default(), enable_sleep=False)
    types = types or ("fixed", "slider", "distance", "d6", "ball", "hinge")
    joints = []
    x = 0.0

    def new(jt, a, b, fa=(0.0, 0.0, 0.0), fb=(0.0, 0.0, 0.0), qa=None, qb=None):
        j = np.zeros(1, abi.JOINT_DTYPE)[0]
        j["type"] = jt
        j["body_a"], j["body_b"] = a, b
        j["frame_a_position"], j["frame_b_position"] = fa, fb
        j["frame_a_rotation"] = qa if qa is not None else (0.0, 0.0, 0.0, 1.0)
        j["frame_b_rotation"] = qb if qb is not None else (0.0, 0.0, 0.0, 1.0)
        joints.append(j)
        return j

    def box(pos, half=(0.3, 0.2, 0.25)):
        return w.add_box(pos, half=half, rotation=_random_quat(rng) if rng.random() < 0.5 else (0, 0, 0, 1),
                         velocity=tuple(rng.uniform(-0.5, 0.5, 3)),
                         angular_velocity=tuple(rng.uniform(-1.0, 1.0, 3)))

    for kind in types:
        for variant in range(4):
            x += 3.0
            anchor = w.add_body(abi.BODY_STATIC, (x, 10.0, 0.0))
            if kind == "fixed":
                prev = anchor
                for k in range(3):
                    b = box((x + 0.7 * (k + 1), 10.0, 0.0))
                    new(abi.JOINT_FIXED, prev, b, fa=(0.35, 0.0, 0.0) if k else (0.0, 0.0, 0.0),
                        fb=(-0.35, 0.0, 0.0), qa=_random_quat(rng), qb=_random_quat(rng))
                    prev = b
            elif kind == "slider":
                b = box((x + 0.5, 9.5, 0.0))
                j = new(abi.JOINT_SLIDER, anchor, b, qa=_random_quat(rng), qb=_random_quat(rng))
                j["slider_enable_limit"] = int(variant > 0)
                j["slider_lower"], j["slider_upper"] = -0.5, 0.3
                if variant >= 2:
                    j["slider_enable_motor"] = 1
                    j["slider_motor_speed"] = 0.8 if variant == 2 else -0.6
                    j["slider_max_motor_force"] = 60.0
                if variant in (1, 3):
                    j["slider_enable_spring"] = 1
                    j["slider_spring_hertz"] = 2.0
                    j["slider_spring_damping_ratio"] = 0.5
                    j["slider_spring_target"] = 0.1
            elif kind == "distance":
                b = box((x + 1.0, 9.2, 0.3))
                j = new(abi.JOINT_DISTANCE, anchor, b, fb=(0.1, 0.2, 0.0))
                j["distance_length"] = 1.2
                if variant == 1:  # a rope
                    j["distance_enable_limit"] = 1
                    j["distance_min_length"], j["distance_max_length"] = 0.0, 1.2
                if variant == 2:  # a limited spring
                    j["distance_enable_spring"] = 1
                    j["distance_spring_hertz"] = 3.0
                    j["distance_spring_damping_ratio"] = 0.3
                    j["distance_enable_limit"] = 1
                    j["distance_min_length"], j["distance_max_length"] = 0.8, 1.5
                if variant == 3:  # motor-driven, rigid otherwise
                    j["distance_enable_motor"] = 1
                    j["distance_motor_speed"] = 0.5
                    j["distance_max_motor_force"] = 30.0
                # a second box hanging from the first (two dynamic bodies)
                c = box((x + 1.0, 8.0, 0.3))
                j2 = new(abi.JOINT_DISTANCE, b, c, fa=(0.0, -0.2, 0.0), fb=(0.0, 0.2, 0.0))
                j2["distance_length"] = 0.9
            elif kind == "d6":
                b = box((x + 0.6, 9.6, 0.0))
                j = new(abi.JOINT_D6, anchor, b, fb=(-0.3, 0.1, 0.0), qa=_random_quat(rng),
                        qb=_random_quat(rng))
                _d6_axes(rng, j, ("rotation", "swing", "point", None)[variant])
                c = box((x + 1.3, 9.6, 0.0))
                j2 = new(abi.JOINT_D6, b, c, fa=(0.3, 0.0, 0.0), fb=(-0.3, 0.0, 0.0),
                         qa=_random_quat(rng), qb=_random_quat(rng))
                _d6_axes(rng, j2, (None, "point", "swing", "rotation")[variant])
            elif kind == "ball":
                b = box((x + 0.6, 10.0, 0.0))
                j = new(abi.JOINT_BALL, anchor, b, fb=(-0.6, 0.0, 0.0))
                j["ball_enable_swing_limit"] = variant % 2
                j["ball_swing_y"], j["ball_swing_z"] = 0.5, 0.3
                j["ball_enable_twist_limit"] = variant // 2
                j["ball_twist_lower"], j["ball_twist_upper"] = -0.4, 0.4
            else:
                b = box((x + 0.6, 10.0, 0.0))
                j = new(abi.JOINT_HINGE, anchor, b, fb=(-0.6, 0.0, 0.0), qa=_random_quat(rng),
                        qb=_random_quat(rng))
                j["hinge_enable_limit"] = variant % 2
                j["hinge_lower"], j["hinge_upper"] = -0.5, 0.5
                j["hinge_enable_motor"] = int(variant >= 2)
                j["hinge_motor_speed"], j["hinge_max_motor_torque"] = 1.0, 15.0
    w.add_joints(np.array(joints, abi.JOINT_DTYPE))
    return w
