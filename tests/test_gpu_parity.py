"""Parity of the device solver with the reference and the oracle, through the C ABI.

Every scene is cut at the solver stage: the reference's world exports the solver's input
view; the device solves a copy through nph_gpu_phys_solve; the reference's own phys_solve
(or the CPU restatement pinned to it) solves the same input. Outputs must agree value for
value (IEEE equality, so +0 and -0 are equal). The joint rows whose angle goes through an
arctangent (hinge limits and springs, ball cones and twists) take it from nph_atan2f, the
reference's C library atan2f restated in FP32 operations, so they are compared exactly too.
"""
from __future__ import annotations

import numpy as np
import pytest

from nepheline_b200 import abi, scenes
from tests import helpers, ref_scenes

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0
ANGLE_TOL = 1e-5


def gpu_solve(solver, view, params, dt=DT):
    out = view.copy()
    solver.phys_solve(out, params, dt)
    return out


def cut_and_compare(solver, w, steps, params, dt=DT, every=1, exact=True, stats=None):
    """The world steps with the reference's solver; every `every` steps the device solves the
    same input and its results are compared with the reference's."""
    worst_bits = 1.0
    for s in range(steps):
        w.collide()
        if s % every:
            w.solve(dt)
            w.finish()
            continue
        vin = w.export_view()
        dev = gpu_solve(solver, vin, params, dt)
        if stats is not None:
            stats.append((s, len(vin.bodies), len(vin.contacts), vin.colors_used))
        w.solve(dt)
        w.finish()
        ref = w.export_view()
        if exact:
            bad = helpers.mismatches(dev, ref)
            assert not bad, f"step {s}: {bad}"
            worst_bits = min(worst_bits, helpers.bitwise_fraction(dev, ref))
        else:
            err = helpers.max_normwise_err(dev, ref)
            assert max(err.values()) < ANGLE_TOL, f"step {s}: {err}"
    return worst_bits


def test_pyramid_matches_reference(solver, ref_lib):
    params = abi.WorldParams.default()
    w = ref_scenes.pyramid(rows=20, jitter=1e-3)
    bits = cut_and_compare(solver, w, 150, params, every=5)
    assert bits > 0.999


def test_sphere_pour_matches_reference(solver, ref_lib):
    """Single-point manifolds, restitution, mixed group point counts."""
    params = abi.WorldParams.default()
    w = ref_scenes.sphere_pour(count=343)
    cut_and_compare(solver, w, 120, params, every=4)


def test_box_pile_matches_reference(solver, ref_lib):
    """Impacts (the seven extra sweeps), tumbling boxes, the gyroscopic step."""
    params = abi.WorldParams.default()
    w = ref_scenes.box_pile(count=64)
    cut_and_compare(solver, w, 120, params, every=4)


def test_lattice_with_joints_matches_reference(solver, ref_lib):
    params = abi.WorldParams.default()
    w, _ = ref_scenes.lattice(edge=8, joint_fraction=0.15)
    for s in range(10):
        vin = w.export_view()
        dev = gpu_solve(solver, vin, params)
        w.solve(DT)
        bad = helpers.mismatches(dev, w.export_view())
        assert not bad, f"step {s}: {bad}"


def test_jointed_chain_matches_reference_every_step(solver, ref_lib):
    """Hinge limits, motors and springs, ball cones, twists and friction: every step the device
    solves the reference's own input and every value equals the reference's output, angle rows
    included (the arctangent is the reference's, restated)."""
    params = abi.WorldParams.default()
    w = ref_scenes.hinge_chain(links=12)
    cut_and_compare(solver, w, 120, params)
    w.close()


def test_other_settings_match_reference(solver, ref_lib):
    params = abi.WorldParams.default(substeps=8, contact_hertz=45.0, contact_damping_ratio=3.0,
                                     joint_hertz=60.0, restitution_threshold=0.5,
                                     max_linear_speed=30.0, gravity=(0.5, -12.0, 0.0))
    w = ref_scenes.sphere_pour(count=125, params=params)
    cut_and_compare(solver, w, 40, params, dt=1.0 / 120.0, every=2)


def test_large_lattice_matches_port(solver):
    """A 24^3 lattice (13k bodies, 40k manifolds, 4k joints): the device against the CPU
    restatement, both coloured by the device colouring."""
    from oracle.refworld import port32
    params = abi.WorldParams.default()
    sc = scenes.lattice_graph(24, seed=7, joint_fraction=0.1)
    color, slot = solver.graph_color(*sc.constraint_arrays(), len(sc.bodies))
    view = sc.to_view(color, slot)
    dev = gpu_solve(solver, view, params)
    cpu = port32(view, params, DT)
    assert not helpers.mismatches(dev, cpu)


def test_resident_steps_match_repeated_solves(solver):
    """Device-resident stepping equals calling the drop-in again on its own results."""
    from oracle.refworld import port32
    params = abi.WorldParams.default()
    sc = scenes.lattice_graph(10, seed=9, joint_fraction=0.1)
    color, slot = solver.graph_color(*sc.constraint_arrays(), len(sc.bodies))
    view = sc.to_view(color, slot)
    solver.upload(view)
    solver.step_async(params, DT, 5)
    dev = view.copy()
    solver.download(dev)
    cpu = view
    for _ in range(5):
        cpu = port32(cpu, params, DT)
    assert not helpers.mismatches(dev, cpu)


def test_graph_replay_equals_direct_launches():
    from nepheline_b200.solver import Solver
    params = abi.WorldParams.default()
    sc = scenes.lattice_graph(6, seed=2, joint_fraction=0.2)
    color, slot = scenes.host_color(sc)
    view = sc.to_view(color, slot)
    a = Solver(use_graph=True)
    b = Solver(use_graph=False)
    va, vb = view.copy(), view.copy()
    for _ in range(3):
        a.phys_solve(va, params, DT)
        b.phys_solve(vb, params, DT)
    assert va.bodies.tobytes() == vb.bodies.tobytes()
    assert va.contacts.tobytes() == vb.contacts.tobytes()
    a.close()
    b.close()


def test_overflow_is_solved_serially_in_list_order(solver):
    """A hub body touching 30 dynamic bodies: colours 0..19 fill, the rest overflow, and the
    overflow runs one constraint at a time before the colours."""
    from oracle.refworld import port32
    params = abi.WorldParams.default()
    nb = 31
    bodies = scenes.body_records(nb)
    mass = np.full(nb, 2.0, np.float32)
    inertia = np.zeros((nb, 9), np.float32)
    inertia[:, [0, 4, 8]] = 2.0 / 6.0
    scenes.set_mass(bodies, mass, inertia)
    ang = np.linspace(0, 2 * np.pi, nb - 1, endpoint=False)
    bodies["center"][1:, 0] = 1.0 * np.cos(ang)
    bodies["center"][1:, 2] = 1.0 * np.sin(ang)
    bodies["linear_velocity"][1:, 0] = -0.5 * np.cos(ang)
    contacts = np.zeros(nb - 1, abi.CONTACT_DTYPE)
    contacts["body_a"] = 0
    contacts["body_b"] = np.arange(1, nb)
    contacts["point_count"] = 1
    contacts["friction"] = 0.5
    n = np.stack([np.cos(ang), np.zeros_like(ang), np.sin(ang)], 1).astype(np.float32)
    contacts["normal"] = n
    pts = contacts["points"]
    pts["anchor_a"][:, 0] = n * 0.5
    pts["anchor_b"][:, 0] = -n * 0.5
    pts["separation"][:, 0] = -0.01
    sc = scenes.SolverScene(bodies, mass, np.zeros(0, abi.JOINT_DTYPE), contacts)
    color, slot = scenes.host_color(sc)
    assert (color == abi.OVERFLOW).sum() == 10
    view = sc.to_view(color, slot)
    dev = gpu_solve(solver, view, params)
    assert not helpers.mismatches(dev, port32(view, params, DT))


def test_invalid_view_is_refused_and_left_untouched(solver):
    params = abi.WorldParams.default()
    sc = scenes.lattice_graph(4, seed=3)
    color, slot = scenes.host_color(sc)
    view = sc.to_view(color, slot)
    bad = view.copy()
    bad.contacts["body_b"][3] = 99999
    before = bad.copy()
    assert solver.phys_solve_code(bad, params, DT) == abi.INVALID_ARGUMENT
    assert bad.bodies.tobytes() == before.bodies.tobytes()
    bad = view.copy()
    bad.contacts["point_count"][0] = 0
    assert solver.phys_solve_code(bad, params, DT) == abi.INVALID_ARGUMENT
    bad = view.copy()
    bad.contact_color_counts[1] += 1
    assert solver.phys_solve_code(bad, params, DT) == abi.INVALID_ARGUMENT
    # The solver stays usable after a refusal.
    good = view.copy()
    solver.phys_solve(good, params, DT)


def test_unsupported_settings_are_refused(solver):
    sc = scenes.lattice_graph(3, seed=4, joint_fraction=0.5)
    color, slot = scenes.host_color(sc)
    view = sc.to_view(color, slot)
    p = abi.WorldParams.default(enable_continuous=1)
    assert solver.phys_solve_code(view.copy(), p, DT) == abi.UNSUPPORTED
    p = abi.WorldParams.default(solver=2)
    assert solver.phys_solve_code(view.copy(), p, DT) == abi.UNSUPPORTED
    bad = view.copy()
    bad.joints["type"][0] = 6  # no such joint type
    assert solver.phys_solve_code(bad, abi.WorldParams.default(), DT) == abi.UNSUPPORTED
    bad = view.copy()
    bad.joints["type"][0] = abi.JOINT_D6
    bad.joints["d6_axes"]["motion"][0] = 0
    bad.joints["d6_axes"]["motion"][0, 2] = 3  # no such motion
    assert solver.phys_solve_code(bad, abi.WorldParams.default(), DT) == abi.INVALID_ARGUMENT
    assert solver.phys_solve_code(view.copy(), abi.WorldParams.default(), 0.0) == abi.INVALID_ARGUMENT


def test_empty_world_is_a_no_op(solver):
    empty = abi.View(np.zeros(0, abi.BODY_DTYPE), None, np.zeros(0, abi.CONTACT_DTYPE), None,
                     np.zeros(25, np.uint32), np.zeros(25, np.uint32))
    solver.phys_solve(empty, abi.WorldParams.default(), DT)


def test_every_pass_configuration_gives_the_same_bits(ref_lib):
    """Every launch configuration the autotuner chooses from (plain, staged and pipelined
    kernels) for every pass kind: the same bits as the restatement, on a jointed lattice large
    enough for the pipelined passes' blocks to walk several chunks, and on a batch world."""
    from nepheline_b200.solver import Solver
    from oracle.refworld import port32
    params = abi.WorldParams.default()
    views = []
    sc = scenes.lattice_graph((80, 80, 24), seed=3, joint_fraction=0.1)
    c, s_ = scenes.host_color(sc)
    views.append(sc.to_view(c, s_))
    sc = scenes.mixed_world(800, 5)
    c, s_ = scenes.host_color(sc)
    views.append(sc.to_view(c, s_))
    want = [port32(v, params, DT) for v in views]
    solver = Solver(device=0)
    for config in range(solver.pass_config_count()):
        for kind in range(4):
            solver.set_pass_config(kind, config)
        for v, w in zip(views, want):
            got = v.copy()
            solver.phys_solve(got, params, DT)
            assert not helpers.mismatches(got, w), f"configuration {config}"
    solver.close()


def test_pyramid_configuration_600_steps_every_step(solver, ref_lib):
    """The pyramid configuration at its size: 20 rows (210 boxes, +-1 mm jitter) on a ground,
    600 steps, the device's solve compared with the reference's at every step."""
    params = abi.WorldParams.default()
    w = ref_scenes.pyramid(rows=20, jitter=1e-3)
    bits = cut_and_compare(solver, w, 600, params, every=1)
    assert bits > 0.999
    w.close()


def test_sphere_pour_configuration_65536_spheres(solver, ref_lib):
    """The pour configuration at its size: 65,536 spheres (radius 0.5 m, density, friction and
    restitution seeded per sphere) dropped from a 43 m lattice onto the ground, 300 steps of
    the reference's collision, the device's solve compared with the reference's every 30 steps
    (each with tens of thousands of contacts once the pour lands)."""
    params = abi.WorldParams.default()
    w = ref_scenes.sphere_pour(count=65536, extent=40.0, workers=-1)
    stats = []
    cut_and_compare(solver, w, 300, params, every=30, stats=stats)
    assert max(c for _, _, c, _ in stats) > 10000
    assert all(colours <= abi.COLORS for _, _, _, colours in stats)
    w.close()


def test_every_body_feature_matches(solver, ref_lib):
    """Kinematic bodies, locks, damping, gravity scale, forces and torques, unequal inertias
    (the gyroscopic step) and both speed caps, with joints: the device equals the reference
    value for value every step."""
    params = abi.WorldParams.default()
    w = ref_scenes.featured_lattice(edge=9, seed=11)
    for s in range(12):
        vin = w.export_view()
        dev = gpu_solve(solver, vin, params)
        w.solve(DT)
        bad = helpers.mismatches(dev, w.export_view())
        assert not bad, f"step {s}: {bad}"
    w.close()
