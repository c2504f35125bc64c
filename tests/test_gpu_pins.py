"""The strongest pins and the failure paths, through the C ABI.

* The reference build's own determinism pin: a 20-row pyramid, no jitter, dt 1/60, 4 substeps,
  sleep off, 600 steps, ends at world hash 0xBE0527E5EE2697B2 (nph_physics_world_hash,
  world.c:436-462: every body's handle, awake flag, origin, rotation and velocity bits). Here the
  reference's world steps with the device as its solver stage (the drop-in at world.c:346), free
  running, beside the same world stepped by the reference's own phys_solve.
* Failure paths injected on the host, as the reference's failing-allocator test does
  (test_sensor.c:342-392): a device-array growth beyond the solver's memory budget returns
  OUT_OF_MEMORY and leaves the view untouched (world.h:163-165: the step did not happen); a body
  with a non-finite value is refused with INVALID_ARGUMENT before anything is written back.
* A device wait that runs out, without a fault: the dependency-driven passes' waits are given
  counts that never come; each gives up after about a second, the call returns DEVICE_LOST with
  the view untouched, and the same solver then steps the view as the restatement does.
"""
from __future__ import annotations

import numpy as np
import pytest

from nepheline_b200 import abi, scenes
from tests import helpers, ref_scenes

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0
PYRAMID_HASH = 0xBE0527E5EE2697B2


def body_bits_differ(a: abi.View, b: abi.View) -> dict:
    """Body fields whose bits differ, and how many of those differ in value too."""
    out = {}
    for f in ("center", "origin", "rotation", "linear_velocity", "angular_velocity"):
        x, y = np.ascontiguousarray(a.bodies[f]), np.ascontiguousarray(b.bodies[f])
        bits = x.view(np.uint8).reshape(len(x), -1) != y.view(np.uint8).reshape(len(y), -1)
        if bits.any():
            out[f] = {"bits": int(bits.any(axis=1).sum()), "values": int((x != y).any(axis=-1).sum())}
    return out


def test_pyramid_600_steps_free_running_hash(solver, ref_lib):
    params = abi.WorldParams.default()
    dev = ref_scenes.pyramid(rows=20, jitter=0.0)
    ref = ref_scenes.pyramid(rows=20, jitter=0.0)
    first_diff = None
    try:
        for s in range(600):
            dev.collide()
            v = dev.export_view()
            solver.phys_solve(v, params, DT)
            dev.import_view(v, DT)
            dev.finish()
            ref.step(DT)
            if first_diff is None and dev.hash() != ref.hash():
                first_diff = (s, body_bits_differ(dev.export_view(), ref.export_view()))
        assert ref.hash() == PYRAMID_HASH
        assert dev.hash() == PYRAMID_HASH, f"first step whose hash differs: {first_diff}"
    finally:
        dev.close()
        ref.close()


def lattice_view(edge=6, seed=3):
    sc = scenes.lattice_graph(edge, seed=seed, joint_fraction=0.2)
    return sc.to_view(*scenes.host_color(sc))


def test_growth_beyond_the_memory_budget_fails_and_leaves_the_view_untouched(ref_lib):
    from nepheline_b200.solver import Solver, SolverError
    from oracle.refworld import port32
    params = abi.WorldParams.default()
    small = lattice_view(3, seed=1)
    big = lattice_view(8, seed=2)
    s = Solver(device=0)
    try:
        s.phys_solve(small.copy(), params, DT)
        held = s.memory()
        s.set_memory_limit(held)  # what it holds now: enough for the small world, not the big
        again = small.copy()
        s.phys_solve(again, params, DT)
        assert not helpers.mismatches(again, port32(small, params, DT))
        v = big.copy()
        with pytest.raises(SolverError) as err:
            s.phys_solve(v, params, DT)
        assert err.value.code == abi.OUT_OF_MEMORY
        for name in ("bodies", "contacts", "joints"):
            assert getattr(v, name).tobytes() == getattr(big, name).tobytes(), name
        assert s.memory() == held
        s.set_memory_limit(0)
        s.phys_solve(v, params, DT)
        assert not helpers.mismatches(v, port32(big, params, DT))
    finally:
        s.close()


@pytest.mark.parametrize("field,index,value", [
    ("linear_velocity", 1, np.nan), ("angular_velocity", 2, np.inf), ("rotation", 3, np.nan),
    ("center", 0, -np.inf), ("force", 0, np.nan), ("inv_inertia", 4, np.inf),
])
def test_a_body_with_a_non_finite_value_is_refused(solver, ref_lib, field, index, value):
    from nepheline_b200.solver import SolverError
    from oracle.refworld import port32
    params = abi.WorldParams.default()
    good = lattice_view()
    bad = good.copy()
    bad.bodies[field][7][index] = value
    before = bad.copy()
    with pytest.raises(SolverError) as err:
        solver.phys_solve(bad, params, DT)
    assert err.value.code == abi.INVALID_ARGUMENT
    for name in ("bodies", "contacts", "joints"):
        assert getattr(bad, name).tobytes() == getattr(before, name).tobytes(), name
    # The next call with a clean view steps as if the refused one never happened.
    v = good.copy()
    solver.phys_solve(v, params, DT)
    assert not helpers.mismatches(v, port32(good, params, DT))


def test_a_wait_that_runs_out_fails_the_call_and_the_next_call_works(ref_lib):
    import time

    from nepheline_b200.solver import Solver, SolverError
    from oracle.refworld import port32
    params = abi.WorldParams.default()
    good = lattice_view(5, seed=4)
    s = Solver(device=0)
    try:
        for kind in (1, 2):  # solve and relax, dependency-driven
            s.set_pass_config(kind, abi.PASS_CONFIGS_FLOW[0])
        s.set_wait_injection(1)
        v = good.copy()
        t0 = time.perf_counter()
        with pytest.raises(SolverError) as err:
            s.phys_solve(v, params, DT)
        assert err.value.code == abi.DEVICE_LOST
        assert time.perf_counter() - t0 < 60.0
        for name in ("bodies", "contacts", "joints"):
            assert getattr(v, name).tobytes() == getattr(good, name).tobytes(), name
        s.set_wait_injection(0)
        s.phys_solve(v, params, DT)
        assert not helpers.mismatches(v, port32(good, params, DT))
    finally:
        s.close()
