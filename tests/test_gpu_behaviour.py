"""Behavioural pins: the reference engine's own scene tests (engine/physics/tests/test_world.c)
with the device solver as the world step's solver stage. The reference world collides and runs
its islands and sleep; each step's solver stage is nph_gpu_phys_solve on the world's view,
written back into the world as phys_solve writes it (the drop-in at world.c:346). The
expectations and tolerances are the reference tests' own."""
from __future__ import annotations

import math

import numpy as np
import pytest

from nepheline_b200 import abi

pytestmark = pytest.mark.gpu

DT = 1.0 / 240.0  # the reference tests' step


def gpu_steps(w, solver, params, count):
    for _ in range(count):
        w.collide()
        v = w.export_view()
        solver.phys_solve(v, params, DT)
        w.import_view(v, DT)
        w.finish()


def world(enable_sleep=True):
    from oracle.refworld import RefWorld
    params = abi.WorldParams.default()
    return RefWorld(params, enable_sleep=enable_sleep), params


def awake(w, body):
    return (w.body_state(body)["flags"] & 1) != 0


def test_free_fall_matches_the_integrator(solver, ref_lib):
    """test_world.c:46-62: semi-implicit Euler over n substeps of h."""
    w, params = world()
    b = w.add_sphere((0.0, 100.0, 0.0), 0.5)
    gpu_steps(w, solver, params, 240)
    n, h = 240.0 * 4.0, 1.0 / 960.0
    st = w.body_state(b)
    assert abs(st["v"][1] - (-9.81 * n * h)) <= 1e-3
    assert abs(st["center"][1] - (100.0 - 9.81 * h * h * n * (n + 1.0) / 2.0)) <= 1e-3
    assert st["center"][0] == 0.0
    w.close()


def test_a_dropped_sphere_comes_to_rest_and_sleeps(solver, ref_lib):
    """test_world.c:64-79."""
    w, params = world()
    w.add_ground(0.0)
    b = w.add_sphere((0.0, 2.0, 0.0), 0.5)
    gpu_steps(w, solver, params, 480)
    st = w.body_state(b)
    assert abs(st["center"][1] - 0.5) <= 0.01
    assert np.linalg.norm(st["v"]) < 0.01
    gpu_steps(w, solver, params, 240)
    assert not awake(w, b)
    w.close()


def test_a_resting_box_does_not_drift(solver, ref_lib):
    """test_world.c:81-103."""
    w, params = world()
    w.add_ground(0.0)
    b = w.add_box((1.0, 0.5, -2.0), half=(0.5, 0.5, 0.5), enable_sleep=False)
    gpu_steps(w, solver, params, 240 * 5)
    st = w.body_state(b)
    assert abs(st["center"][0] - 1.0) <= 1e-3
    assert abs(st["center"][2] + 2.0) <= 1e-3
    assert abs(st["center"][1] - 0.5) <= 6e-3
    q = st["rotation"].astype(np.float64)
    assert 2.0 * math.acos(min(1.0, abs(q[3]))) < 1e-3
    w.close()


def test_a_pyramid_stands(solver, ref_lib):
    """test_world.c:365-392: 20 rows (210 boxes), five seconds."""
    w, params = world()
    w.add_ground(0.0)
    rows = 20
    top = None
    for row in range(rows):
        count = rows - row
        for i in range(count):
            x = (i - (count - 1) * 0.5) * 1.05
            top = w.add_box((x, 0.5 + row, 0.0), half=(0.5, 0.5, 0.5))
    gpu_steps(w, solver, params, 240 * 5)
    st = w.body_state(top)
    assert abs(st["center"][0]) <= 0.003
    assert abs(st["center"][1] - (0.5 + rows - 1)) <= 0.005
    assert not awake(w, top)
    w.close()


def test_a_heavy_box_rests_on_a_light_one(solver, ref_lib):
    """test_world.c:394-418: a 100:1 mass ratio."""
    w, params = world()
    w.add_ground(0.0)
    light = w.add_box((0.0, 0.5, 0.0), half=(0.5, 0.5, 0.5))
    heavy = w.add_box((0.0, 1.5, 0.0), half=(0.5, 0.5, 0.5), density=100_000.0)
    gpu_steps(w, solver, params, 240 * 3)
    assert 0.5 - w.body_state(light)["center"][1] < 0.001
    assert 1.5 - w.body_state(heavy)["center"][1] < 0.004
    assert abs(w.body_state(heavy)["center"][0]) <= 1e-3
    w.close()


def ramp_slide(solver, theta, mu, seconds):
    """test_world.c:420-455: a box on a static ramp of angle theta, friction mu on both."""
    w, params = world(enable_sleep=False)
    q = (0.0, 0.0, math.sin(0.5 * theta), math.cos(0.5 * theta))
    w.add_box((0.0, 0.0, 0.0), half=(20.0, 0.5, 5.0), type_=abi.BODY_STATIC, rotation=q,
              friction=mu)
    up = np.array([-math.sin(theta), math.cos(theta), 0.0])
    along = np.array([math.cos(theta), math.sin(theta), 0.0])
    start = up * (0.5 + 0.25 - 0.001)
    b = w.add_box(tuple(start), half=(0.25, 0.25, 0.25), rotation=q, friction=mu,
                  enable_sleep=False)
    gpu_steps(w, solver, params, 24)
    s0 = w.body_state(b)
    steps = int(seconds * 240.0)
    gpu_steps(w, solver, params, steps)
    s1 = w.body_state(b)
    accel = (float(s1["v"] @ along) - float(s0["v"] @ along)) / (steps * DT)
    moved = float((s1["center"] - s0["center"]) @ along)
    w.close()
    return moved, accel


def test_friction_holds_below_its_angle_and_slides_above(solver, ref_lib):
    """test_world.c:457-470: tan 20 deg < 0.6 holds; tan 35 deg > 0.3 slides at
    g (sin - mu cos)."""
    held, _ = ramp_slide(solver, 0.349066, 0.6, 2.0)
    assert abs(held) < 0.005
    slid, accel = ramp_slide(solver, 0.610865, 0.3, 1.0)
    assert slid < -1.0
    expected = 9.81 * (math.sin(0.610865) - 0.3 * math.cos(0.610865))
    assert abs(-accel - expected) <= 0.005 * expected


def bounce_height(solver, restitution):
    """test_world.c:472-500: fall 2 m, bounce, the peak of the first rebound."""
    w, params = world()
    w.add_box((0.0, -1.0, 0.0), half=(10.0, 1.0, 10.0), type_=abi.BODY_STATIC,
              restitution=restitution)
    b = w.add_sphere((0.0, 2.5, 0.0), 0.5, restitution=restitution)
    peak, bounced = -1.0, False
    for _ in range(240 * 3):
        gpu_steps(w, solver, params, 1)
        st = w.body_state(b)
        if not bounced and st["v"][1] > 0.0:
            bounced = True
        if bounced:
            peak = max(peak, float(st["center"][1]))
            if st["v"][1] < 0.0:
                break
    w.close()
    return peak - 0.5


def test_restitution_bounces_to_its_height(solver, ref_lib):
    """test_world.c:502-507: e = 1 back to 2 m, e = 0.5 to 0.5 m."""
    assert abs(bounce_height(solver, 1.0) - 2.0) <= 0.08
    assert abs(bounce_height(solver, 0.5) - 0.5) <= 0.05
