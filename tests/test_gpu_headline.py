"""Parity at the headline workload's size, against the reference itself.

The synthetic constraint graph is built in the reference (bodies created, joints made,
manifolds injected in insertion order and coloured by its phys_graph_add, island.c:34-118):
the 128 x 128 x 64 lattice the bench measures (1,048,576 bodies, the most a reference world
holds: NPH_PHYSICS_MAX_OBJECTS, world.h:80, 2^20 body slots). The device's colouring must equal
the reference's colour and slot for every constraint, and for three steps the device's drop-in
step on the reference's own input must equal the reference's phys_solve (solver.c:961-1105)
value for value: bodies, contact points, joints. The FP64 restatement of the first step is
printed as the error baseline of both FP32 results.

The 128^3 cube (2,097,152 bodies) is beyond the reference's world; there the device's colouring
and step are checked against the CPU restatement pinned to the reference.
"""
from __future__ import annotations

import numpy as np
import pytest

from nepheline_b200 import abi
from tests import helpers

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0


def fp64_baseline(vin, fp32_views, params):
    """Per field, max |f32 - f64| / max |f64| of each FP32 result against the FP64 restatement
    of the same step."""
    from oracle.refworld import port64
    f64 = port64(vin, params, DT)
    mask = np.arange(4)[None, :] < vin.contacts["point_count"][:, None]
    out = {}
    for name, (key, sub) in {"linear_velocity": ("linear_velocity", "bodies"),
                             "angular_velocity": ("angular_velocity", "bodies"),
                             "center": ("center", "bodies"),
                             "normal_impulse": ("normal_impulse", "points"),
                             "tangent_impulse": ("tangent_impulse", "points"),
                             "joint_linear_impulse": ("linear_impulse", "joints")}.items():
        ref64 = f64[name][mask] if sub == "points" else f64[name]
        scale = float(np.abs(ref64).max())
        errs = []
        for v in fp32_views:
            if sub == "bodies":
                x = v.bodies[key]
            elif sub == "points":
                x = v.contacts["points"][key][mask]
            else:
                x = v.joints[key]
            errs.append(float(np.abs(np.asarray(x, np.float64) - ref64).max()) / scale)
        out[name] = errs
    return out


def test_headline_lattice_colouring_and_steps_match_reference(solver, ref_lib):
    dims = (128, 128, 64)
    params = abi.WorldParams.default()
    w, sc = ref_lib.lattice_world(dims, seed=0, joint_fraction=0.1, params=params, workers=-1)
    try:
        c = w.constraints()
        a, b, d = sc.constraint_arrays()
        assert np.array_equal(a, c["body_a"]) and np.array_equal(b, c["body_b"])
        color, slot = solver.graph_color(a, b, d, c["body_slots"])
        assert np.array_equal(color, c["color"]), "device colouring differs from phys_graph_add"
        assert np.array_equal(slot, c["slot"]), "device colour slots differ from phys_graph_add"
        for s in range(3):
            vin = w.export_view()
            dev = vin.copy()
            solver.phys_solve(dev, params, DT)
            w.solve(DT)
            ref = w.export_view()
            bad = helpers.mismatches(dev, ref)
            assert not bad, f"step {s}: {bad}"
            if s == 0:
                err = fp64_baseline(vin, (dev, ref), params)
                print(f"{dims}: FP64 error baseline (device, reference): {err}")
    finally:
        w.close()


def test_cube_lattice_colouring_and_step_match_the_restatement(solver, ref_lib):
    from oracle.refworld import port32, port_graph_color
    from nepheline_b200 import scenes
    params = abi.WorldParams.default()
    sc = scenes.lattice_graph((128, 128, 128), seed=0, joint_fraction=0.1)
    a, b, d = sc.constraint_arrays()
    color, slot = solver.graph_color(a, b, d, len(sc.bodies))
    pc, ps = port_graph_color(a, b, d, len(sc.bodies))
    assert np.array_equal(color, pc) and np.array_equal(slot, ps)
    vin = sc.to_view(color, slot)
    dev = vin.copy()
    solver.phys_solve(dev, params, DT)
    bad = helpers.mismatches(dev, port32(vin, params, DT))
    assert not bad, bad
