"""Batched worlds: every world of a batch gives the same bits as the world solved alone."""
from __future__ import annotations

import numpy as np
import pytest

from nepheline_b200 import abi, scenes
from tests import helpers, ref_scenes

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0


def reference_views(steps_warm=30):
    """Solver inputs cut from reference scenes of different kinds and sizes."""
    views = []
    for w in (ref_scenes.pyramid(rows=8), ref_scenes.sphere_pour(count=125),
              ref_scenes.box_pile(count=30), ref_scenes.hinge_chain(links=6, limits=False,
                                                                    spring=False),
              ref_scenes.pyramid(rows=3)):
        for _ in range(steps_warm):
            w.step(DT)
        w.collide()
        views.append(w.export_view())
    for edge, seed in ((3, 1), (5, 2), (9, 3)):
        sc = scenes.lattice_graph(edge, seed=seed, joint_fraction=0.2)
        color, slot = scenes.host_color(sc)
        views.append(sc.to_view(color, slot))
    return views


@pytest.mark.parametrize("config", [0, 1, 2, 3, 4])
@pytest.mark.parametrize("shared", [False, True])
def test_batch_equals_worlds_solved_alone(solver, ref_lib, config, shared):
    from nepheline_b200.solver import Batch
    params = abi.WorldParams.default()
    views = reference_views()
    alone = []
    for v in views:
        out = v.copy()
        solver.phys_solve(out, params, DT)
        alone.append(out)
    batch = Batch()
    batch.set_config(config, shared)
    together = [v.copy() for v in views]
    batch.phys_solve_worlds(together, params, DT)
    for i, (a, b) in enumerate(zip(together, alone)):
        assert a.bodies.tobytes() == b.bodies.tobytes(), f"world {i}"
        assert a.contacts.tobytes() == b.contacts.tobytes(), f"world {i}"
        assert a.joints.tobytes() == b.joints.tobytes(), f"world {i}"
    batch.close()


def test_resident_batch_steps_match_repeated_solves(solver):
    from nepheline_b200.solver import Batch
    params = abi.WorldParams.default()
    views = []
    for edge, seed in ((4, 5), (7, 6), (6, 7), (2, 8)):
        sc = scenes.lattice_graph(edge, seed=seed, joint_fraction=0.1)
        c, s = scenes.host_color(sc)
        views.append(sc.to_view(c, s))
    batch = Batch()
    batch.upload(views)
    batch.step_async(params, DT, 4)
    got = [v.copy() for v in views]
    batch.download(got)
    for v, g in zip(views, got):
        want = v.copy()
        for _ in range(4):
            solver.phys_solve(want, params, DT)
        assert not helpers.mismatches(g, want)
    batch.close()


def test_batch_autotuner_keeps_results(solver):
    from nepheline_b200.solver import Batch
    params = abi.WorldParams.default()
    views = []
    for edge, seed in ((5, 1), (8, 2), (3, 3)):
        sc = scenes.lattice_graph(edge, seed=seed)
        c, s = scenes.host_color(sc)
        views.append(sc.to_view(c, s))
    batch = Batch()
    batch.upload(views)
    tuned = batch.autotune(params, DT, rounds=1)
    assert tuned["threads"] in (128, 256, 512, 1024)
    batch.upload(views)
    batch.step_async(params, DT, 1)
    got = [v.copy() for v in views]
    batch.download(got)
    for v, g in zip(views, got):
        want = v.copy()
        solver.phys_solve(want, params, DT)
        assert not helpers.mismatches(g, want)
    batch.close()


def test_batch_refuses_malformed_worlds(solver):
    from nepheline_b200.solver import Batch
    params = abi.WorldParams.default()
    sc = scenes.lattice_graph(3, seed=1)
    c, s = scenes.host_color(sc)
    good = sc.to_view(c, s)
    bad = good.copy()
    bad.contacts["body_a"][0] = 10_000
    batch = Batch()
    before = bad.copy()
    assert batch.phys_solve_worlds_code([good.copy(), bad], params, DT) == abi.INVALID_ARGUMENT
    assert bad.bodies.tobytes() == before.bodies.tobytes()
    batch.close()
