"""The oracle pinned against the reference (CPU only).

The reference engine's own solver, built from its sources into oracle/_ref, is the judge:
  - the harness reproduces the reference's own pyramid run (the world hash of a 600-step
    run measured on the reference build);
  - the CPU restatement (oracle/port_impl.h) agrees with the reference's phys_solve value
    for value on identical inputs, step by step, on every scene kind the device runs;
  - its colouring agrees with the reference's phys_graph_add colouring;
  - the FP64 re-run stays within FP32 rounding of both.
"""
from __future__ import annotations

import numpy as np
import pytest

from nepheline_b200 import abi, scenes
from tests import helpers, ref_scenes

DT = 1.0 / 60.0


def step_compare(w, steps, params, dt=DT, check_every=1):
    """Cuts the reference's step at the solver: the port solves the exported input, the
    reference solves its world; their outputs must agree."""
    from oracle.refworld import port32
    worst = {}
    for s in range(steps):
        w.collide()
        vin = w.export_view()
        mine = port32(vin, params, dt)
        w.solve(dt)
        w.finish()
        if s % check_every == 0:
            vout = w.export_view()
            bad = helpers.mismatches(mine, vout)
            assert not bad, f"step {s}: {bad}"
            worst[s] = helpers.bitwise_fraction(mine, vout)
    return worst


def test_pyramid_hash_matches_reference_build(ref_lib):
    """20-row pyramid, no jitter, dt 1/60, 4 substeps, sleep off, 600 steps: the world hash
    the reference build gives (be0527e5ee2697b2)."""
    w = ref_scenes.pyramid(rows=20, jitter=0.0)
    for _ in range(600):
        w.step(DT)
    assert w.hash() == 0xBE0527E5EE2697B2
    st = w.stats()
    assert (st["touching"], st["points"], st["colors_used"]) == (400, 1600, 4)


def test_port_matches_reference_pyramid(ref_lib):
    params = abi.WorldParams.default()
    w = ref_scenes.pyramid(rows=12, jitter=1e-3)
    frac = step_compare(w, 120, params, check_every=3)
    assert min(frac.values()) > 0.999


def test_port_matches_reference_sphere_pour(ref_lib):
    params = abi.WorldParams.default()
    w = ref_scenes.sphere_pour(count=216)
    step_compare(w, 90, params, check_every=3)


def test_port_matches_reference_box_pile(ref_lib):
    params = abi.WorldParams.default()
    w = ref_scenes.box_pile(count=40)
    step_compare(w, 90, params, check_every=3)


def test_port_matches_reference_lattice_with_joints(ref_lib):
    params = abi.WorldParams.default()
    w, _ = ref_scenes.lattice(edge=6, joint_fraction=0.2)
    from oracle.refworld import port32
    for s in range(20):
        vin = w.export_view()
        mine = port32(vin, params, DT)
        w.solve(DT)
        bad = helpers.mismatches(mine, w.export_view())
        assert not bad, f"step {s}: {bad}"


def test_port_matches_reference_jointed_chain(ref_lib):
    """Every ball and hinge row: limits, motor, spring, cone, twist, friction (the angle rows
    use atan2f of the host C library on both sides)."""
    params = abi.WorldParams.default()
    w = ref_scenes.hinge_chain(links=12)
    step_compare(w, 120, params, check_every=2)


def test_port_matches_reference_substeps_and_settings(ref_lib):
    params = abi.WorldParams.default(substeps=8, contact_hertz=45.0, contact_damping_ratio=3.0,
                                     joint_hertz=60.0, restitution_threshold=0.5,
                                     max_linear_speed=30.0, gravity=(0.5, -12.0, 0.0))
    w = ref_scenes.sphere_pour(count=64, params=params)
    step_compare(w, 40, params, dt=1.0 / 120.0, check_every=2)


def test_port_colouring_matches_reference(ref_lib):
    from oracle.refworld import port_graph_color
    w, sc = ref_scenes.lattice(edge=7, joint_fraction=0.15, seed=11)
    c = w.constraints()
    color, slot = port_graph_color(*sc.constraint_arrays(), c["body_slots"])
    assert np.array_equal(color, c["color"]) and np.array_equal(slot, c["slot"])
    hc, hs = scenes.host_color(sc)
    assert np.array_equal(hc, c["color"]) and np.array_equal(hs, c["slot"])


def test_scene_view_equals_reference_export(ref_lib):
    w, sc = ref_scenes.lattice(edge=5, joint_fraction=0.2, seed=5)
    c = w.constraints()
    v = w.export_view()
    mine = sc.to_view(c["color"], c["slot"])
    assert v.bodies.tobytes() == mine.bodies.tobytes()
    assert v.contacts.tobytes() == mine.contacts.tobytes()
    assert v.joints.tobytes() == mine.joints.tobytes()
    assert np.array_equal(v.contact_color_counts, mine.contact_color_counts)


def test_fp64_baseline_is_within_fp32_rounding(ref_lib):
    """The error baseline: the FP32 step's distance from the FP64 re-run of the same step."""
    from oracle.refworld import port32, port64
    params = abi.WorldParams.default()
    w = ref_scenes.pyramid(rows=10, jitter=1e-3)
    for _ in range(30):
        w.step(DT)
    w.collide()
    vin = w.export_view()
    f32 = port32(vin, params, DT)
    f64 = port64(vin, params, DT)
    v = f32.bodies["linear_velocity"].astype(np.float64)
    # Resting bodies move at a step's gravity at most: the velocity scale of the step.
    scale = max(np.abs(f64["linear_velocity"]).max(), 9.81 * DT)
    assert np.abs(v - f64["linear_velocity"]).max() / scale < 1e-4
    ni = f32.contacts["points"]["normal_impulse"].astype(np.float64)
    assert np.abs(ni - f64["normal_impulse"]).max() / max(np.abs(f64["normal_impulse"]).max(), 1e-6) < 1e-3


def test_port_rejects_malformed_views():
    from oracle.refworld import port32_result
    params = abi.WorldParams.default()
    sc = scenes.lattice_graph(3, seed=1)
    color, slot = scenes.host_color(sc)
    v = sc.to_view(color, slot)
    bad = v.copy()
    bad.contacts["body_a"][0] = 10_000
    assert port32_result(bad, params, DT) == abi.INVALID_ARGUMENT
    bad = v.copy()
    bad.contacts["point_count"][0] = 5
    assert port32_result(bad, params, DT) == abi.INVALID_ARGUMENT
    bad = v.copy()
    bad.contact_color_counts[0] += 1
    assert port32_result(bad, params, DT) == abi.INVALID_ARGUMENT
    bad = v.copy()
    if len(bad.joints):
        bad.joints["type"][0] = 6
        assert port32_result(bad, params, DT) == abi.UNSUPPORTED


@pytest.mark.parametrize("bodies,seed", [(40, 1), (300, 2), (1200, 3)])
def test_port_matches_reference_mixed_batch_world(ref_lib, bodies, seed):
    """The batched workload's worlds (pyramids, piles and hinge chains on a fixed ground):
    the reference colours them as the host colouring does and solves them as the port does."""
    from oracle.refworld import port32, scene_world
    params = abi.WorldParams.default()
    sc = scenes.mixed_world(bodies, seed)
    w = scene_world(sc, params)
    c = w.constraints()
    hc, hs = scenes.host_color(sc)
    assert np.array_equal(hc, c["color"]) and np.array_equal(hs, c["slot"])
    for s in range(5):
        vin = w.export_view()
        mine = port32(vin, params, DT)
        w.solve(DT)
        bad = helpers.mismatches(mine, w.export_view())
        assert not bad, f"step {s}: {bad}"
    w.close()


def aligned_old(old: abi.View, new: abi.View) -> np.ndarray:
    """Last step's record of each of this step's contacts, found by its pair (a zero record,
    no points, for a pair that starts touching)."""
    by_pair = {(int(c["body_a"]), int(c["body_b"])): c for c in old.contacts}
    out = np.zeros(len(new.contacts), abi.CONTACT_DTYPE)
    for i, c in enumerate(new.contacts):
        rec = by_pair.get((int(c["body_a"]), int(c["body_b"])))
        if rec is not None:
            out[i] = rec
        else:
            out[i]["body_a"] = c["body_a"]
            out[i]["body_b"] = c["body_b"]
    return out


def raw_manifolds(view: abi.View) -> np.ndarray:
    """The narrow phase's manifolds of an updated view: its points without their impulses."""
    raw = view.contacts.copy()
    raw["points"]["normal_impulse"] = 0.0
    raw["points"]["tangent_impulse"] = 0.0
    return raw


def test_port_warm_update_matches_the_reference_contact_update(ref_lib):
    """contact.c:516-565 on a box pile settling: every contact's warm start, by id and by
    place, equals the reference's, step after step."""
    from oracle.refworld import port_warm_update
    w = ref_scenes.box_pile(count=40, seed=4)
    old = None
    carried = 0
    for s in range(150):
        w.collide()
        new = w.export_view()
        if old is not None and len(new.contacts):
            got = port_warm_update(aligned_old(old, new), raw_manifolds(new))
            assert got.tobytes() == new.contacts.tobytes(), f"step {s}"
            carried += int(np.count_nonzero(new.contacts["points"]["normal_impulse"]))
        w.solve(DT)
        w.finish()
        old = w.export_view()
    assert carried > 0
    w.close()


def test_port_matches_reference_with_every_body_feature(ref_lib):
    """Kinematic bodies, locks, damping, gravity scale, forces and torques, the gyroscopic step
    and both speed caps, with joints: value for value every step."""
    from oracle.refworld import port32
    params = abi.WorldParams.default()
    w = ref_scenes.featured_lattice(edge=7, seed=7)
    v0 = w.export_view()
    assert (v0.bodies["type"] == abi.BODY_KINEMATIC).any() and v0.bodies["locks"].any()
    for s in range(12):
        vin = w.export_view()
        mine = port32(vin, params, DT)
        w.solve(DT)
        bad = helpers.mismatches(mine, w.export_view())
        assert not bad, f"step {s}: {bad}"
    w.close()
