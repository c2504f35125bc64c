"""Hit events (hit_events, solver.c:919-960): per manifold whose shapes report hits, its point
of fastest approach above the world's threshold among those that took load, in the colour
lists' order.

CPU: the restatement (oracle/hits.py) on the records the reference's phys_solve wrote equals
the reference's own events, approach speed, world point and normal bit for bit, over a sphere
pour in which half the spheres report hits. GPU: the device's nph_gpu_world_hit_events after
the device's step equals the reference's events the same way."""
from __future__ import annotations

import numpy as np
import pytest

from nepheline_b200 import abi
from tests import helpers, ref_scenes

DT = 1.0 / 60.0


def same_events(events, view, ref):
    speed, point, normal = ref
    assert len(events) == len(speed)
    assert events["approach_speed"].tobytes() == speed.tobytes()
    p, n = abi.hit_points(view, events)
    assert p.tobytes() == point.tobytes()
    assert n.tobytes() == normal.tobytes()


@pytest.mark.parametrize("threshold", [1.0, 0.25])
def test_restatement_matches_reference_hit_events(ref_lib, threshold):
    from oracle.hits import hit_events_of
    w = ref_scenes.sphere_pour(count=216, hit_events=True)
    w.set_hit_threshold(threshold)
    seen = 0
    for s in range(90):
        w.collide()
        w.solve(DT)
        out = w.export_view()
        ref = w.hit_events()
        same_events(hit_events_of(out, threshold), out, ref)
        seen += len(ref[0])
        w.finish()
    assert seen > 20, seen
    # Contacts of spheres that do not report hits carry no flag: some manifolds have none.
    flags = w.export_view().contacts["flags"]
    assert ((flags & abi.CONTACT_HIT_EVENTS) == 0).any() and ((flags & abi.CONTACT_HIT_EVENTS) != 0).any()
    w.close()


@pytest.mark.gpu
@pytest.mark.parametrize("threshold", [1.0, 0.25])
def test_device_hit_events_match_reference(solver, ref_lib, threshold):
    from oracle.hits import hit_events_of
    w = ref_scenes.sphere_pour(count=216, hit_events=True)
    w.set_hit_threshold(threshold)
    p = abi.WorldParams.default()
    seen = 0
    for s in range(90):
        w.collide()
        vin = w.export_view()
        dev = vin.copy()
        solver.phys_solve(dev, p, DT)
        events = solver.hit_events(threshold)
        w.solve(DT)
        ref_view = w.export_view()
        assert not helpers.mismatches(dev, ref_view), f"step {s}"
        same_events(events, dev, w.hit_events())
        assert events.tobytes() == hit_events_of(dev, threshold).tobytes()
        seen += len(events)
        if len(events) > 1:
            # A smaller buffer takes the first events; the count is all of them.
            head = solver.hit_events(threshold, capacity=1)
            assert head.tobytes() == events[:1].tobytes()
        w.finish()
    assert seen > 20, seen
    w.close()


@pytest.mark.gpu
def test_device_hit_events_on_many_manifolds(solver):
    """Hits spread over many blocks of manifolds (the ordered write across blocks), read from
    uploaded records whose flags, approach speeds and impulses are set on the host: 70 % of the
    manifolds report hits, a quarter of the points took no load, ties included."""
    from oracle.hits import hit_events_of
    from nepheline_b200 import scenes
    sc = scenes.lattice_graph(24, seed=3, joint_fraction=0.0)
    v = sc.to_view(*scenes.host_color(sc))
    rng = np.random.default_rng(4)
    c = v.contacts
    c["flags"] |= np.where(rng.random(len(c)) < 0.7, abi.CONTACT_HIT_EVENTS, 0).astype(np.uint32)
    pts = c["points"]
    pts["relative_velocity"] = np.round(rng.uniform(-4.0, 1.0, pts["relative_velocity"].shape), 1)
    pts["max_normal_impulse"] = np.where(rng.random(pts["max_normal_impulse"].shape) < 0.25, 0.0,
                                         rng.uniform(0.0, 2.0, pts["max_normal_impulse"].shape))
    solver.upload(v)
    for threshold in (0.5, 2.0):
        events = solver.hit_events(threshold)
        want = hit_events_of(v, threshold)
        assert len(want) > 1000
        assert events.tobytes() == want.tobytes()
    assert len(solver.hit_events(10.0)) == 0


@pytest.mark.gpu
def test_device_hit_events_edge_cases():
    """Before any upload the call is refused; a world without manifolds has no hits."""
    from nepheline_b200 import scenes
    from nepheline_b200.solver import Solver, SolverError
    s = Solver(device=0)
    with pytest.raises(SolverError):
        s.hit_events(1.0)
    sc = scenes.lattice_graph(3, seed=1, joint_fraction=0.5)
    sc.contacts = sc.contacts[:0]
    v = sc.to_view(*scenes.host_color(sc))
    s.phys_solve(v, abi.WorldParams.default(), DT)
    assert len(s.hit_events(0.0)) == 0
    s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("parts", [1, 2])
@pytest.mark.parametrize("packing", [abi.BATCH_PERSISTENT, abi.BATCH_MERGED])
def test_batch_hit_events_equal_each_world_alone(solver, ref_lib, parts, packing):
    """A batch of sphere pours (and a world without hits between them), split or not: the
    batch's hits are each world's own hits, world by world, tagged with the world."""
    from nepheline_b200.solver import Batch
    p = abi.WorldParams.default()
    views = []
    for seed in (2, 5, 7):
        w = ref_scenes.sphere_pour(count=125, seed=seed, hit_events=True)
        for _ in range(20):
            w.step(DT)
        w.collide()
        views.append(w.export_view())
        w.close()
    quiet = ref_scenes.sphere_pour(count=27, seed=9)  # no step yet: bodies, no manifolds
    views.insert(1, quiet.export_view())
    quiet.close()
    batch = Batch(device=0)
    batch.set_config(packing=packing)
    batch.set_pipeline(parts)
    mine = abi.pack_views([v.copy() for v in views])
    batch.phys_solve_worlds(mine, p, DT)
    got = batch.hit_events(0.25)
    want = []
    for i, v in enumerate(views):
        alone = v.copy()
        solver.phys_solve(alone, p, DT)
        e = solver.hit_events(0.25)
        e["world"] = i
        want.append(e)
    want = np.concatenate(want)
    assert len(want) > 5
    assert got.tobytes() == want.tobytes()
    batch.close()
