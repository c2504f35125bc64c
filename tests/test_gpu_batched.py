"""Batched worlds: every world of a batch gives the same bits as the world solved alone."""
from __future__ import annotations

import numpy as np
import pytest

from nepheline_b200 import abi, scenes
from tests import helpers, ref_scenes

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0


def hub_view(spokes=30):
    """A hub body touching `spokes` dynamic bodies: colours 0..19 fill, the rest overflow."""
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
    return sc.to_view(color, slot)


def reference_views(steps_warm=30):
    """Solver inputs cut from reference scenes of different kinds and sizes, lattices, mixed
    batch worlds, a world with overflow constraints and a world without constraints."""
    views = []
    for w in (ref_scenes.pyramid(rows=8), ref_scenes.sphere_pour(count=125),
              ref_scenes.box_pile(count=30), ref_scenes.hinge_chain(links=6, limits=False,
                                                                    spring=False),
              ref_scenes.pyramid(rows=3)):
        for _ in range(steps_warm):
            w.step(DT)
        w.collide()
        views.append(w.export_view())
    for edge, seed in ((3, 1), (5, 2), (9, 3), (14, 4)):
        sc = scenes.lattice_graph(edge, seed=seed, joint_fraction=0.2)
        color, slot = scenes.host_color(sc)
        views.append(sc.to_view(color, slot))
    for bodies, seed in ((12, 1), (90, 2), (700, 3)):
        sc = scenes.mixed_world(bodies, seed)
        color, slot = scenes.host_color(sc)
        views.append(sc.to_view(color, slot))
    views.append(hub_view())
    sc = scenes.lattice_graph(2, seed=9, joint_fraction=0.0)
    sc.contacts = sc.contacts[:0]
    color, slot = scenes.host_color(sc)
    views.append(sc.to_view(color, slot))
    return views


@pytest.fixture(scope="module")
def solved_alone(solver):
    params = abi.WorldParams.default()
    views = reference_views()
    alone = []
    for v in views:
        out = v.copy()
        solver.phys_solve(out, params, DT)
        alone.append(out)
    return views, alone


@pytest.mark.parametrize("shared", [abi.BATCH_SHARED_NONE, abi.BATCH_SHARED_SMALL,
                                    abi.BATCH_SHARED_LARGE])
def test_batch_equals_worlds_solved_alone(solved_alone, ref_lib, shared):
    """Every launch shape, with every world on a block, on a warp, or on teams sized to it."""
    from nepheline_b200.solver import Batch
    params = abi.WorldParams.default()
    views, alone = solved_alone
    batch = Batch()
    for config in range(batch.config_count()):
        for per_thread in (0, 1, 1 << 20):
            batch.set_config(config, shared, per_thread)
            together = [v.copy() for v in views]
            batch.phys_solve_worlds(together, params, DT)
            info = batch.info()
            if per_thread == 0:
                assert info["block_worlds"] == len(views)
            if per_thread == 1 << 20:
                assert info["warp_worlds"] == len(views)
            for i, (a, b) in enumerate(zip(together, alone)):
                where = f"world {i}, config {config}, shared {shared}, per thread {per_thread}"
                assert a.bodies.tobytes() == b.bodies.tobytes(), where
                assert a.contacts.tobytes() == b.contacts.tobytes(), where
                assert a.joints.tobytes() == b.joints.tobytes(), where
    batch.close()


def test_packed_worlds_copy_back_to_their_slices(solved_alone):
    """Worlds whose records are consecutive slices of shared host arrays (the coalesced copy
    path) get the same results as separately allocated worlds."""
    from nepheline_b200.solver import Batch
    params = abi.WorldParams.default()
    views, alone = solved_alone
    packed = abi.pack_views([v.copy() for v in views])
    batch = Batch()
    batch.phys_solve_worlds(packed, params, DT)
    for i, (a, b) in enumerate(zip(packed, alone)):
        assert a.bodies.tobytes() == b.bodies.tobytes(), f"world {i}"
        assert a.contacts.tobytes() == b.contacts.tobytes(), f"world {i}"
        assert a.joints.tobytes() == b.joints.tobytes(), f"world {i}"
    # A smaller batch after a larger one reuses the device arrays.
    few = abi.pack_views([v.copy() for v in views[:3]])
    batch.phys_solve_worlds(few, params, DT)
    for i in range(3):
        assert few[i].bodies.tobytes() == alone[i].bodies.tobytes()
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
    assert tuned["threads"] in (128, 256, 512)
    assert tuned["shared_velocities"] in (0, 1, 2)
    assert tuned["packing"] in (abi.BATCH_PERSISTENT, abi.BATCH_MERGED)
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


def test_merged_packing_equals_worlds_solved_alone(solved_alone):
    """The batch as one world (colour lists padded to whole groups of eight per world) gives
    each world the bits it has alone; so do switches between the packings."""
    from nepheline_b200.solver import Batch
    params = abi.WorldParams.default()
    views, alone = solved_alone
    batch = Batch()
    for packing in (abi.BATCH_MERGED, abi.BATCH_PERSISTENT, abi.BATCH_MERGED):
        batch.set_config(packing=packing)
        together = [v.copy() for v in views]
        batch.phys_solve_worlds(together, params, DT)
        assert batch.info()["packing"] == packing
        for i, (a, b) in enumerate(zip(together, alone)):
            assert a.bodies.tobytes() == b.bodies.tobytes(), f"world {i}, packing {packing}"
            assert a.contacts.tobytes() == b.contacts.tobytes(), f"world {i}, packing {packing}"
            assert a.joints.tobytes() == b.joints.tobytes(), f"world {i}, packing {packing}"
    batch.close()


def test_merged_resident_steps_and_packing_switches(solver):
    """Resident steps alternating between the packings equal repeated solves of each world."""
    from nepheline_b200.solver import Batch
    params = abi.WorldParams.default()
    views = []
    for edge, seed in ((4, 5), (7, 6), (6, 7), (2, 8)):
        sc = scenes.lattice_graph(edge, seed=seed, joint_fraction=0.1)
        c, s = scenes.host_color(sc)
        views.append(sc.to_view(c, s))
    views.append(hub_view(27))
    batch = Batch()
    batch.upload(views)
    for packing in (abi.BATCH_MERGED, abi.BATCH_MERGED, abi.BATCH_PERSISTENT, abi.BATCH_MERGED):
        batch.set_config(packing=packing)
        batch.step_async(params, DT, 1)
    got = [v.copy() for v in views]
    batch.download(got)
    for v, g in zip(views, got):
        want = v.copy()
        for _ in range(4):
            solver.phys_solve(want, params, DT)
        assert not helpers.mismatches(g, want)
    batch.close()


def test_merged_packing_refuses_malformed_worlds(solver):
    from nepheline_b200.solver import Batch
    params = abi.WorldParams.default()
    sc = scenes.lattice_graph(3, seed=1)
    c, s = scenes.host_color(sc)
    good = sc.to_view(c, s)
    bad = good.copy()
    bad.contacts["body_a"][0] = 10_000
    batch = Batch()
    batch.set_config(packing=abi.BATCH_MERGED)
    before = bad.copy()
    assert batch.phys_solve_worlds_code([good.copy(), bad], params, DT) == abi.INVALID_ARGUMENT
    assert bad.bodies.tobytes() == before.bodies.tobytes()
    batch.close()


def empty_view():
    """A world whose islands all sleep: no awake body, so no constraint in its view."""
    z = np.zeros(abi.COLOR_SLOTS, np.uint32)
    return abi.View(np.zeros(0, abi.BODY_DTYPE), np.zeros(0, abi.BODY_DTYPE),
                    np.zeros(0, abi.CONTACT_DTYPE), np.zeros(0, abi.JOINT_DTYPE), z, z.copy())


@pytest.mark.parametrize("packing", [abi.BATCH_PERSISTENT, abi.BATCH_MERGED])
def test_sleeping_worlds_are_left_out(solved_alone, packing):
    """Worlds without awake bodies between the others: the others step as alone, resident or
    not, and the batch's queue leaves the sleeping ones out (phys_solve does nothing for a
    world without awake bodies, solver.c:963-966)."""
    from nepheline_b200.solver import Batch
    views, alone = solved_alone
    params = abi.WorldParams.default()
    mixed, where = [], []
    for i, v in enumerate(views):
        mixed.append(empty_view())
        where.append(len(mixed))
        mixed.append(v.copy())
    mixed.append(empty_view())
    batch = Batch(device=0)
    batch.set_config(packing=packing)
    batch.phys_solve_worlds(mixed, params, DT)
    for i, k in enumerate(where):
        assert not helpers.mismatches(mixed[k], alone[i]), i
    for v in mixed:
        if len(v.bodies) == 0:
            assert len(v.contacts) == 0 and len(v.joints) == 0
    assert batch.info()["worlds"] == len(mixed)
    batch.close()


@pytest.mark.parametrize("packing", [abi.BATCH_PERSISTENT, abi.BATCH_MERGED])
def test_drop_in_steps_with_the_same_shapes(solver, packing):
    """Consecutive drop-in calls on worlds of unchanged shapes (the step graph and the merged
    lists are kept between them, only records move) equal each world solved alone as often;
    a call with two worlds swapped (the same totals) is taken as a new batch."""
    from nepheline_b200.solver import Batch
    params = abi.WorldParams.default()
    views = []
    for edge, seed in ((4, 5), (7, 6), (6, 7), (2, 8)):
        sc = scenes.lattice_graph(edge, seed=seed, joint_fraction=0.1)
        c, s = scenes.host_color(sc)
        views.append(sc.to_view(c, s))
    views.append(hub_view(27))
    batch = Batch(device=0)
    batch.set_config(packing=packing)
    mine = abi.pack_views([v.copy() for v in views])
    want = [v.copy() for v in views]
    for _ in range(3):
        batch.phys_solve_worlds(mine, params, DT)
        for w in want:
            solver.phys_solve(w, params, DT)
        for m, w in zip(mine, want):
            assert not helpers.mismatches(m, w)
    # The first two worlds swapped: the same totals, other offsets, so a new batch.
    swapped = [mine[1], mine[0]] + mine[2:]
    want = [want[1], want[0]] + want[2:]
    assert len(mine[0].contacts) != len(mine[1].contacts)
    batch.phys_solve_worlds(swapped, params, DT)
    for w in want:
        solver.phys_solve(w, params, DT)
    for m, w in zip(swapped, want):
        assert not helpers.mismatches(m, w)
    batch.close()


@pytest.mark.parametrize("packing", [abi.BATCH_PERSISTENT, abi.BATCH_MERGED])
@pytest.mark.parametrize("parts", [2, 3, 8])
def test_drop_in_in_parts_equals_worlds_solved_alone(solved_alone, packing, parts):
    """The drop-in call split into parts (each on its own stream, uploads chained) gives each
    world the bits it has alone, packed or not, twice in a row, with sleeping worlds between."""
    from nepheline_b200.solver import Batch
    params = abi.WorldParams.default()
    views, alone = solved_alone
    batch = Batch(device=0)
    batch.set_config(packing=packing)
    batch.set_pipeline(parts)
    for packed in (True, False):
        mixed, where = [], []
        for v in views:
            mixed.append(empty_view())
            where.append(len(mixed))
            mixed.append(v.copy())
        worlds = abi.pack_views(mixed) if packed else mixed
        batch.phys_solve_worlds(worlds, params, DT)
        for i, k in enumerate(where):
            assert not helpers.mismatches(worlds[k], alone[i]), (packed, i)
    batch.close()


def test_drop_in_in_parts_refuses_before_writing_back(solver):
    """A malformed record in the last part: the call is refused and no world, in any part, is
    written back."""
    from nepheline_b200.solver import Batch
    params = abi.WorldParams.default()
    views = []
    for edge, seed in ((4, 5), (7, 6), (6, 7), (5, 8)):
        sc = scenes.lattice_graph(edge, seed=seed, joint_fraction=0.1)
        c, s = scenes.host_color(sc)
        views.append(sc.to_view(c, s))
    batch = Batch(device=0)
    batch.set_pipeline(4)
    for field, value in (("body_a", 10_000), ("point_count", 0), ("point_count", 5)):
        worlds = abi.pack_views([v.copy() for v in views])
        worlds[-1].contacts[field][3] = value
        before = [w.copy() for w in worlds]
        assert batch.phys_solve_worlds_code(worlds, params, DT) == abi.INVALID_ARGUMENT
        for w, b in zip(worlds, before):
            assert w.bodies.tobytes() == b.bodies.tobytes()
            assert w.contacts.tobytes() == b.contacts.tobytes()
    worlds = abi.pack_views([v.copy() for v in views])
    worlds[-1].joints["body_b"][0] = 10_000
    before = worlds[0].copy()
    assert batch.phys_solve_worlds_code(worlds, params, DT) == abi.INVALID_ARGUMENT
    assert worlds[0].bodies.tobytes() == before.bodies.tobytes()
    # And the same batch then solves good worlds.
    worlds = abi.pack_views([v.copy() for v in views])
    batch.phys_solve_worlds(worlds, params, DT)
    for w, v in zip(worlds, views):
        want = v.copy()
        solver.phys_solve(want, params, DT)
        assert not helpers.mismatches(w, want)
    with pytest.raises(Exception):
        batch.set_pipeline(0)
    # One part: the parts released, the call unsplit, the same bits.
    batch.set_pipeline(1)
    worlds = abi.pack_views([v.copy() for v in views])
    batch.phys_solve_worlds(worlds, params, DT)
    for w, v in zip(worlds, views):
        want = v.copy()
        solver.phys_solve(want, params, DT)
        assert not helpers.mismatches(w, want)
    batch.close()


def test_drop_in_in_parts_follows_the_batch(solver):
    """The parts take the batch's packing when it changes between calls, and TGS steps as alone."""
    from nepheline_b200.solver import Batch
    views = []
    for edge, seed in ((4, 5), (7, 6), (6, 7), (5, 8), (3, 9)):
        sc = scenes.lattice_graph(edge, seed=seed, joint_fraction=0.1)
        views.append(sc.to_view(*scenes.host_color(sc)))
    batch = Batch(device=0)
    batch.set_pipeline(3)
    mine = abi.pack_views([v.copy() for v in views])
    want = [v.copy() for v in views]
    for packing, solver_kind in ((abi.BATCH_PERSISTENT, abi.SOLVER_SOFT_STEP), (abi.BATCH_MERGED, abi.SOLVER_TGS),
                                 (abi.BATCH_PERSISTENT, abi.SOLVER_TGS)):
        params = abi.WorldParams.default(solver=solver_kind)
        batch.set_config(packing=packing)
        batch.phys_solve_worlds(mine, params, DT)
        for w in want:
            solver.phys_solve(w, params, DT)
        for m, w in zip(mine, want):
            assert not helpers.mismatches(m, w), (packing, solver_kind)
    batch.close()


@pytest.mark.parametrize("packing", [abi.BATCH_PERSISTENT, abi.BATCH_MERGED])
def test_batched_worlds_match_the_restatement(packing):
    """Worlds of the batched configuration's generator (box pyramids, piles and capsule chains on
    hinges, 8 to 600 bodies) solved in one batch, three steps, against the CPU restatement
    pinned to the reference, world by world: a direct check, not through the single-world
    device solver."""
    from nepheline_b200.solver import Batch
    from oracle.refworld import port32
    params = abi.WorldParams.default()
    worlds = [w.to_view(*scenes.host_color(w))
              for w in scenes.batched_worlds(12, seed=9, max_bodies=600)]
    batch = Batch(device=0)
    batch.set_config(packing=packing)
    mine = [v.copy() for v in worlds]
    want = [v.copy() for v in worlds]
    for _ in range(3):
        batch.phys_solve_worlds(mine, params, DT)
        want = [port32(v, params, DT) for v in want]
    for i, (m, r) in enumerate(zip(mine, want)):
        assert not helpers.mismatches(m, r), f"world {i}"
    batch.close()
