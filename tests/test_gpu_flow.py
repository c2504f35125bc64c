"""The dependency-driven passes (one launch a pass, csrc/solver.cu k_pass_flow) on what the
every-configuration test does not hold: every joint type (slider, 6-DOF and distance rows out
of line), an overflow that runs before the pass, many resident steps in one graph, and the
batch's merged packing. Each against the reference's phys_solve (joints), the FP32 restatement
or the launch-per-colour configuration, value for value."""
from __future__ import annotations

import numpy as np
import pytest

from nepheline_b200 import abi, scenes
from tests import helpers, ref_scenes

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0
SOLVERS = {"soft_step": abi.SOLVER_SOFT_STEP, "tgs": abi.SOLVER_TGS}


def flow_solver(config):
    from nepheline_b200.solver import Solver
    s = Solver(device=0)
    for kind in (0, 1, 2):  # warm start, solve, relax
        s.set_pass_config(kind, config)
    return s


@pytest.mark.parametrize("solver_name", list(SOLVERS))
def test_every_joint_type_matches_the_reference(ref_lib, solver_name):
    params = abi.WorldParams.default(solver=SOLVERS[solver_name])
    w = ref_scenes.joint_zoo(seed=5, params=params)
    s = flow_solver(abi.PASS_CONFIGS_FLOW[0])
    try:
        for step in range(60):
            w.collide()
            dev = w.export_view()
            s.phys_solve(dev, params, DT)
            w.solve(DT)
            w.finish()
            bad = helpers.mismatches(dev, w.export_view())
            assert not bad, f"step {step}: {bad}"
    finally:
        s.close()
        w.close()


def hub_view(spokes=30):
    """A hub body touching `spokes` dynamic bodies: colours fill and the rest overflow."""
    nb = spokes + 1
    bodies = scenes.body_records(nb)
    mass = np.full(nb, 2.0, np.float32)
    inertia = np.zeros((nb, 9), np.float32)
    inertia[:, [0, 4, 8]] = 2.0 / 6.0
    scenes.set_mass(bodies, mass, inertia)
    ang = np.linspace(0, 2 * np.pi, spokes, endpoint=False)
    bodies["center"][1:, 0] = np.cos(ang)
    bodies["center"][1:, 2] = np.sin(ang)
    bodies["linear_velocity"][1:, 0] = -0.5 * np.cos(ang)
    contacts = np.zeros(spokes, abi.CONTACT_DTYPE)
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
    assert (color == abi.OVERFLOW).sum() > 0
    return sc.to_view(color, slot)


@pytest.mark.parametrize("config", list(abi.PASS_CONFIGS_FLOW))
def test_overflow_then_the_colours(ref_lib, config):
    from oracle.refworld import port32
    params = abi.WorldParams.default()
    view = hub_view()
    s = flow_solver(config)
    try:
        dev = view.copy()
        s.phys_solve(dev, params, DT)
        assert not helpers.mismatches(dev, port32(view, params, DT))
    finally:
        s.close()


def test_resident_steps_equal_a_colour_a_launch(ref_lib):
    """Twenty resident steps of a jointed lattice in the step graph: the dependency-driven
    passes and the lean launch-per-colour passes end on the same bits."""
    sc = scenes.lattice_graph((24, 24, 12), seed=7, joint_fraction=0.1)
    view = sc.to_view(*scenes.host_color(sc))
    params = abi.WorldParams.default()
    out = []
    for config in (abi.PASS_CONFIGS_LEAN[0], abi.PASS_CONFIGS_FLOW[-1]):
        s = flow_solver(config)
        try:
            v = view.copy()
            s.upload(v)
            s.step_async(params, DT, 20)
            s.download(v)
            out.append(v)
        finally:
            s.close()
    assert not helpers.mismatches(out[1], out[0])


def test_merged_batch_with_dependency_driven_passes(ref_lib):
    """The batch's merged packing runs the single-world solver; with its passes set to the
    dependency-driven form every world equals the world solved alone."""
    from nepheline_b200.solver import Batch
    from oracle.refworld import port32
    params = abi.WorldParams.default()
    views = []
    for i, bodies in enumerate((40, 300, 90, 700)):
        sc = scenes.mixed_world(bodies, 40 + i)
        views.append(sc.to_view(*scenes.host_color(sc)))
    b = Batch()
    try:
        b.set_config(packing=abi.BATCH_MERGED)
        b.set_merged_pass_configs([abi.PASS_CONFIGS_FLOW[0]] * 3 + [0])
        together = [v.copy() for v in views]
        b.phys_solve_worlds(together, params, DT)
        for v, got in zip(views, together):
            assert not helpers.mismatches(got, port32(v, params, DT))
    finally:
        b.close()
