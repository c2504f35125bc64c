"""The island sleep decision (phys_island_sleep_and_split, island.c:675-735) on the device
(nph_gpu_world_sleep_decision) against the reference's own island stage: a sleep-enabled world
whose stacks come to rest and sleep, whose body that may not sleep keeps its island awake, whose
kinematic bodies sleep on their own clocks, and whose island loses a contact and is split. Each
step: the reference collides, the device solves (the drop-in), the reference merges its islands;
the decision is taken from the islands and the bodies' clocks and compared with what the
reference's own sleep-and-split then does. The CPU test runs the same comparison with the
decision restated in numpy."""
from __future__ import annotations

import numpy as np
import pytest

from nepheline_b200 import abi

DT = 1.0 / 60.0
TIME_TO_SLEEP = 0.5  # the reference's default (world.c:98)


def scene():
    from oracle.refworld import RefWorld
    params = abi.WorldParams.default()
    w = RefWorld(params, enable_sleep=True)
    w.add_ground(0.0)
    for s in range(3):  # stacks that settle and sleep
        for k in range(3):
            w.add_box((-6.0 + 2.5 * s, 0.5 + k * 1.0, 0.0), half=(0.5, 0.5, 0.5))
    w.add_box((4.0, 0.5, 0.0), half=(0.5, 0.5, 0.5))  # a pair whose top box may not sleep
    w.add_box((4.0, 1.5, 0.0), half=(0.5, 0.5, 0.5), enable_sleep=False)
    # Two boxes side by side, one pushed away: the island loses its contact and is split.
    w.add_box((0.0, 0.5, 4.0), half=(0.5, 0.5, 0.5))
    w.add_box((1.0, 0.5, 4.0), half=(0.5, 0.5, 0.5), velocity=(2.0, 0.0, 0.0))
    w.add_box((-4.0, 3.0, -4.0), half=(0.5, 0.5, 0.5), type_=abi.BODY_KINEMATIC)  # sleeps alone
    w.add_box((4.0, 3.0, -4.0), half=(0.5, 0.5, 0.5), type_=abi.BODY_KINEMATIC,
              velocity=(0.3, 0.0, 0.0))  # keeps moving
    return w, params


def decision_numpy(bodies, island_of, removed, time_to_sleep):
    """phys_island_sleep_and_split's decision restated (island.c:684-734)."""
    n_is = len(removed)
    t = np.full(n_is, 1e30, np.float32)
    sleepiest = np.zeros(n_is, np.float32)
    bt = np.where((bodies["flags"] & abi.BODY_ENABLE_SLEEP) != 0, bodies["sleep_time"], 0.0).astype(np.float32)
    for i, k in enumerate(island_of):
        if k != abi.NULL:
            t[k] = min(t[k], bt[i])
            sleepiest[k] = max(sleepiest[k], bt[i])
    sleep = np.zeros(n_is, bool)
    split, split_time = None, 0.0
    for k in range(n_is):
        if removed[k] > 0:
            if sleepiest[k] >= time_to_sleep and sleepiest[k] > split_time:
                split, split_time = k, sleepiest[k]
        elif t[k] >= time_to_sleep:
            sleep[k] = True
    kin = ((bodies["type"] == abi.BODY_KINEMATIC) & ((bodies["flags"] & abi.BODY_ENABLE_SLEEP) != 0)
           & (bodies["sleep_time"] >= time_to_sleep))
    return sleep, split, kin


def run(decide, solve, steps=150):
    """Steps the scene, comparing each step's decision with the reference's outcome; returns how
    many islands slept, kinematic bodies slept and islands were split."""
    w, params = scene()
    slept = kin_slept = splits = 0
    for s in range(steps):
        w.collide()
        view = w.export_view()
        n = len(view.bodies)
        if n == 0:
            break
        out = solve(view, params)
        w.import_view(out, DT)
        w.merge_islands()
        island_of, ids, removed = w.island_view(n)
        sleep, split, kin = decide(out, island_of, removed)
        awake_ids = w.awake_creation_ids(n)
        w.sleep_islands()
        fell = {int(awake_ids[i]) for i in range(n)
                if (w.body_state(int(awake_ids[i]))["flags"] & 1) == 0}
        want = {int(awake_ids[i]) for i in range(n)
                if (island_of[i] != abi.NULL and sleep[island_of[i]]) or kin[i]}
        assert fell == want, f"step {s}: fell asleep {sorted(fell)}, decided {sorted(want)}"
        for k in range(len(removed)):
            after_removed, after_awake = w.island_state(int(ids[k]))
            if split is not None and k == split:
                assert after_removed == 0, f"step {s}: island {k} was to be split"
            elif removed[k] > 0:
                assert after_removed == removed[k], f"step {s}: island {k} split, not decided"
        slept += int(sleep.sum())
        kin_slept += int(kin.sum())
        splits += split is not None
    w.close()
    return slept, kin_slept, splits


def test_numpy_decision_matches_reference(ref_lib):
    from oracle.refworld import port32

    def solve(view, params):
        return port32(view, params, DT)

    def decide(out, island_of, removed):
        return decision_numpy(out.bodies, island_of, removed, TIME_TO_SLEEP)

    slept, kin_slept, splits = run(decide, solve)
    assert slept >= 3 and kin_slept >= 1 and splits >= 1, (slept, kin_slept, splits)


@pytest.mark.gpu
def test_device_decision_matches_reference(solver, ref_lib):
    def solve(view, params):
        out = view.copy()
        solver.phys_solve(out, params, DT)
        return out

    def decide(out, island_of, removed):
        return solver.sleep_decision(island_of, removed, TIME_TO_SLEEP)

    slept, kin_slept, splits = run(decide, solve)
    assert slept >= 3 and kin_slept >= 1 and splits >= 1, (slept, kin_slept, splits)


@pytest.mark.gpu
def test_device_decision_refuses_bad_island_indices(solver):
    from nepheline_b200 import scenes
    from nepheline_b200.solver import SolverError
    sc = scenes.lattice_graph(3, seed=1)
    v = sc.to_view(*scenes.host_color(sc))
    solver.phys_solve(v, abi.WorldParams.default(), DT)
    island_of = np.zeros(len(v.bodies), np.uint32)
    island_of[0] = 5
    with pytest.raises(SolverError):
        solver.sleep_decision(island_of, np.zeros(2, np.uint32), TIME_TO_SLEEP)
