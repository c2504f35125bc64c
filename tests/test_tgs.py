"""The TGS solver (NPH_PHYSICS_SOLVER_TGS, solver.c:1007-1017 and 1036-1060): rigid rows with a
Baumgarte fifth of the error per substep and a linear slop, no relax pass inside the substeps and
one after them, and a hit or bounce scaling the next warm start (solver_impl.h:172-238, 528-532,
662-665; store_group's HIT flag, solver.c:475-499).

CPU: the restatement against the reference's phys_solve under TGS, step by step, on every scene
kind. GPU: the device solver (single world and both batch packings) against the reference."""
from __future__ import annotations

import numpy as np
import pytest

from nepheline_b200 import abi
from tests import helpers, ref_scenes

DT = 1.0 / 60.0


def tgs(**kw):
    return abi.WorldParams.default(solver=abi.SOLVER_TGS, **kw)


def hits(view) -> int:
    return int(((view.contacts["flags"] & abi.CONTACT_HIT) != 0).sum())


def compare(w, steps, params, solve, dt=DT, exact=True, skip_joint=False):
    """Cuts the reference's step at the solver; returns how many steps carried HIT flags in."""
    with_hits = 0
    for s in range(steps):
        w.collide()
        vin = w.export_view()
        with_hits += hits(vin) > 0
        mine = solve(vin, params, dt)
        w.solve(dt)
        w.finish()
        ref = w.export_view()
        if exact:
            bad = helpers.mismatches(mine, ref)
            if skip_joint:
                bad = {k: v for k, v in bad.items() if not k.startswith("joint.")}
            assert not bad, f"step {s}: {bad}"
        err = helpers.max_normwise_err(mine, ref)
        assert max(err.values()) < 1e-5, f"step {s}: {err}"
    return with_hits


def scene(kind):
    p = tgs()
    if kind == "pyramid":
        return ref_scenes.pyramid(rows=12, jitter=1e-3, params=p), 90
    if kind == "sphere_pour":
        return ref_scenes.sphere_pour(count=216, params=p), 90
    if kind == "box_pile":
        return ref_scenes.box_pile(count=40, params=p), 90
    if kind == "hinge_chain":
        return ref_scenes.hinge_chain(links=12, params=p), 90
    raise ValueError(kind)


@pytest.mark.parametrize("kind", ["pyramid", "sphere_pour", "box_pile", "hinge_chain"])
def test_port_matches_reference_under_tgs(ref_lib, kind):
    from oracle.refworld import port32
    w, steps = scene(kind)
    carried = compare(w, steps, tgs(), port32)
    if kind in ("sphere_pour", "box_pile"):
        assert carried > 0, "no hit reached a later step's warm start"
    w.close()


def test_port_matches_reference_under_tgs_lattice_with_joints(ref_lib):
    from oracle.refworld import port32
    params = tgs()
    w, _ = ref_scenes.lattice(edge=6, joint_fraction=0.2, params=params)
    for s in range(20):
        vin = w.export_view()
        mine = port32(vin, params, DT)
        w.solve(DT)
        bad = helpers.mismatches(mine, w.export_view())
        assert not bad, f"step {s}: {bad}"
    w.close()


def test_tgs_differs_from_the_soft_step(ref_lib):
    """The two stage lists give different steps on the same input (the parameter is read)."""
    from oracle.refworld import port32
    w = ref_scenes.box_pile(count=20)
    for _ in range(20):
        w.step(DT)
    w.collide()
    v = w.export_view()
    a = port32(v, abi.WorldParams.default(), DT)
    b = port32(v, tgs(), DT)
    assert a.bodies.tobytes() != b.bodies.tobytes()
    w.close()


def test_port_takes_tgs_and_refuses_xpbd():
    from oracle.refworld import port32_result
    from nepheline_b200 import scenes
    sc = scenes.lattice_graph(3, seed=1)
    v = sc.to_view(*scenes.host_color(sc))
    assert port32_result(v, abi.WorldParams.default(solver=2), DT) == abi.INVALID_ARGUMENT
    assert port32_result(v, tgs(), DT) == abi.OK


# ---------------------------------------------------------------------------------------
# The device under TGS
# ---------------------------------------------------------------------------------------

@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["pyramid", "sphere_pour", "box_pile", "hinge_chain"])
def test_device_matches_reference_under_tgs(solver, ref_lib, kind):
    """Every step the device solves the reference's input under TGS; every value equals the
    reference's output, the hinge chain's angle rows included."""
    w, steps = scene(kind)
    params = tgs()
    for s in range(steps):
        w.collide()
        vin = w.export_view()
        dev = vin.copy()
        solver.phys_solve(dev, params, DT)
        w.solve(DT)
        w.finish()
        bad = helpers.mismatches(dev, w.export_view())
        assert not bad, f"step {s}: {bad}"
    w.close()


@pytest.mark.gpu
def test_device_matches_the_restatement_under_tgs_every_pass_configuration(ref_lib):
    from nepheline_b200.solver import Solver
    from oracle.refworld import port32
    w = ref_scenes.box_pile(count=40, params=tgs())
    for _ in range(30):
        w.step(DT)
    w.collide()
    vin = w.export_view()
    want = port32(vin, tgs(), DT)
    solver = Solver(device=0)
    for config in range(solver.pass_config_count()):
        for kind in range(4):
            solver.set_pass_config(kind, config)
        v = vin.copy()
        solver.phys_solve(v, tgs(), DT)
        assert not helpers.mismatches(v, want), f"pass config {config}"
    solver.close()
    w.close()


@pytest.mark.gpu
@pytest.mark.parametrize("packing", [abi.BATCH_PERSISTENT, abi.BATCH_MERGED])
def test_batch_matches_the_restatement_under_tgs(ref_lib, packing):
    from nepheline_b200 import scenes
    from nepheline_b200.solver import Batch
    from oracle.refworld import port32
    worlds = []
    for i, bodies in enumerate((40, 300, 90)):
        sc = scenes.mixed_world(bodies, 20 + i)
        worlds.append(sc.to_view(*scenes.host_color(sc)))
    batch = Batch(device=0)
    batch.set_config(packing=packing)
    mine = [w.copy() for w in worlds]
    want = [w.copy() for w in worlds]
    for _ in range(3):
        batch.phys_solve_worlds(mine, tgs(), DT)
        want = [port32(w, tgs(), DT) for w in want]
    for m, r in zip(mine, want):
        assert not helpers.mismatches(m, r)
    batch.close()


@pytest.mark.gpu
def test_learned_calls_refuse_tgs(solver):
    from nepheline_b200 import scenes
    from nepheline_b200.solver import SolverError
    sc = scenes.lattice_graph(3, seed=1)
    v = sc.to_view(*scenes.host_color(sc))
    solver.upload(v)
    with pytest.raises(SolverError):
        solver.features(tgs(), DT)
    solver.features(abi.WorldParams.default(), DT)
