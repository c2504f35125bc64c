"""Every joint type the reference's joint solver runs (joint_solver.c): ball, hinge, fixed
(rotation lock, 232-262), slider and 6-DOF (rows per axis with the rotation, swing-pair and
anchor blocks, 395-682), distance (683-720), with their prepare-time resets (726-824) and
block flags, under the soft step and TGS.

CPU: the restatement against the reference's phys_solve, value for value, step by step.
GPU: the device solver against the reference, value for value every step (its angle rows take
the reference's arctangent, restated), alone and in both batch packings."""
from __future__ import annotations

import numpy as np
import pytest

from nepheline_b200 import abi
from tests import helpers, ref_scenes

DT = 1.0 / 60.0

SOLVERS = {"soft_step": abi.SOLVER_SOFT_STEP, "tgs": abi.SOLVER_TGS}
KINDS = ("fixed", "slider", "distance", "d6", "ball", "hinge")


def params_for(name):
    return abi.WorldParams.default(solver=SOLVERS[name])


@pytest.mark.parametrize("solver_name", list(SOLVERS))
def test_port_matches_reference_every_joint_type(ref_lib, solver_name):
    from oracle.refworld import port32
    p = params_for(solver_name)
    w = ref_scenes.joint_zoo(seed=5, params=p)
    v0 = w.export_view()
    assert set(int(t) for t in v0.joints["type"]) == set(range(6))
    for s in range(120):
        w.collide()
        vin = w.export_view()
        mine = port32(vin, p, DT)
        w.solve(DT)
        w.finish()
        bad = helpers.mismatches(mine, w.export_view())
        assert not bad, f"step {s}: {bad}"
    out = w.export_view()
    # Every row kind took load (lock or lower limit, upper limit, motor, spring), and every
    # type's rows some.
    rows = np.isin(out.joints["type"], (abi.JOINT_SLIDER, abi.JOINT_DISTANCE, abi.JOINT_D6))
    assert np.abs(out.joints["axis_impulse"][rows]).sum(axis=(0, 1)).min() > 0.0
    for t in (abi.JOINT_SLIDER, abi.JOINT_DISTANCE, abi.JOINT_D6):
        assert np.abs(out.joints["axis_impulse"][out.joints["type"] == t]).sum() > 0.0
    fixed = out.joints["type"] == abi.JOINT_FIXED
    assert np.abs(out.joints["angular_impulse"][fixed]).max() > 0.0
    # Every block shows in the flags.
    d6 = out.joints["flags"][out.joints["type"] == abi.JOINT_D6]
    for bit in (abi.JOINT_BLOCK_ROTATION, abi.JOINT_BLOCK_SWING, abi.JOINT_BLOCK_POINT):
        assert (d6 & bit).any()
    w.close()


@pytest.mark.parametrize("kind", KINDS)
def test_port_matches_reference_joint_type_alone(ref_lib, kind):
    from oracle.refworld import port32
    p = abi.WorldParams.default()
    w = ref_scenes.joint_zoo(seed=11, params=p, types=(kind,))
    for s in range(60):
        w.collide()
        vin = w.export_view()
        mine = port32(vin, p, DT)
        w.solve(DT)
        w.finish()
        bad = helpers.mismatches(mine, w.export_view())
        assert not bad, f"step {s}: {bad}"
    w.close()


def test_a_block_change_restarts_its_impulse(ref_lib):
    """A 6-DOF joint whose axes change between steps (the rotation block released) starts the
    block's impulse from nothing, as the reference's prepare does."""
    from oracle.refworld import port32
    p = abi.WorldParams.default()
    w = ref_scenes.joint_zoo(seed=5, params=p, types=("d6",))
    for _ in range(10):
        w.step(DT)
    w.collide()
    v = w.export_view()
    d6 = np.nonzero((v.joints["flags"] & abi.JOINT_BLOCK_ROTATION) != 0)[0]
    assert len(d6) > 0
    i = d6[0]
    assert np.abs(v.joints["angular_impulse"][i]).max() > 0.0
    v.joints["d6_axes"]["motion"][i, 3] = abi.AXIS_FREE  # the twist freed: no rotation block
    out = port32(v, p, DT)
    assert (out.joints["flags"][i] & abi.JOINT_BLOCK_ROTATION) == 0
    w.close()


def test_port_refuses_bad_joint_records():
    from nepheline_b200 import scenes
    from oracle.refworld import port32_result
    sc = scenes.lattice_graph(3, seed=4, joint_fraction=0.5)
    v = sc.to_view(*scenes.host_color(sc))
    bad = v.copy()
    bad.joints["type"][0] = 6
    assert port32_result(bad, abi.WorldParams.default(), DT) == abi.UNSUPPORTED
    bad = v.copy()
    bad.joints["type"][0] = abi.JOINT_D6
    bad.joints["d6_axes"]["motion"][0] = 0
    bad.joints["d6_axes"]["motion"][0, 4] = 7
    assert port32_result(bad, abi.WorldParams.default(), DT) == abi.INVALID_ARGUMENT


# ---------------------------------------------------------------------------------------
# The device
# ---------------------------------------------------------------------------------------

@pytest.mark.gpu
@pytest.mark.parametrize("solver_name", list(SOLVERS))
def test_device_matches_every_joint_type(solver, ref_lib, solver_name):
    """Every step the device solves the reference's input; every value equals the reference's
    output, the 6-DOF twist and swing rows and the hinge and ball angles included."""
    p = params_for(solver_name)
    w = ref_scenes.joint_zoo(seed=5, params=p)
    for s in range(120):
        w.collide()
        vin = w.export_view()
        dev = vin.copy()
        solver.phys_solve(dev, p, DT)
        w.solve(DT)
        w.finish()
        bad = helpers.mismatches(dev, w.export_view())
        assert not bad, f"step {s}: {bad}"
    w.close()


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["fixed", "slider", "distance"])
def test_device_equals_reference_where_no_angle_row_runs(solver, ref_lib, kind):
    """The fixed joint's rotation lock, the slider (its rotation is one block) and the distance
    joint take no arctangent: bit for bit with the reference."""
    p = abi.WorldParams.default()
    w = ref_scenes.joint_zoo(seed=11, params=p, types=(kind,))
    for s in range(60):
        w.collide()
        vin = w.export_view()
        dev = vin.copy()
        solver.phys_solve(dev, p, DT)
        w.solve(DT)
        w.finish()
        bad = helpers.mismatches(dev, w.export_view())
        assert not bad, f"step {s}: {bad}"
    w.close()


@pytest.mark.gpu
@pytest.mark.parametrize("packing", [abi.BATCH_PERSISTENT, abi.BATCH_MERGED])
def test_batch_runs_every_joint_type(ref_lib, packing):
    from nepheline_b200.solver import Batch
    from oracle.refworld import port32
    p = abi.WorldParams.default()
    worlds = []
    for seed in (5, 6, 7):
        w = ref_scenes.joint_zoo(seed=seed, params=p)
        for _ in range(5):
            w.step(DT)
        w.collide()
        worlds.append(w.export_view())
        w.close()
    batch = Batch(device=0)
    batch.set_config(packing=packing)
    mine = [v.copy() for v in worlds]
    want = [v.copy() for v in worlds]
    for _ in range(3):
        batch.phys_solve_worlds(mine, p, DT)
        want = [port32(v, p, DT) for v in want]
    for m, r in zip(mine, want):
        assert not helpers.mismatches(m, r)
    batch.close()
