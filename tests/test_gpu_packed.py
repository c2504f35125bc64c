"""The packed drop-in (nph_gpu_phys_solve_packed) against the whole-record one.

The packed call moves only the fields the solver stage reads and writes; the device expands and
packs the records around the same step. Its outputs must equal the whole-record call's field
for field (the arithmetic is the same), step after step, on worlds with every kind of record,
and its refusals must leave the outputs untouched."""
from __future__ import annotations

import numpy as np
import pytest

from nepheline_b200 import abi, scenes
from tests import helpers, ref_scenes

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0


def both(solver, view, params, steps=2):
    """`steps` whole-record solves and `steps` packed solves of the same view."""
    whole = view.copy()
    packed_view = view.copy()
    for _ in range(steps):
        solver.phys_solve(whole, params, DT)
        pk = abi.Packed(packed_view)
        solver.phys_solve_packed(pk, params, DT)
        pk.scatter(packed_view)
    return whole, packed_view


@pytest.mark.parametrize("solver_name", ["soft_step", "tgs"])
def test_packed_equals_whole_records_on_a_jointed_lattice(solver, solver_name):
    params = abi.WorldParams.default(solver=abi.SOLVER_TGS if solver_name == "tgs" else abi.SOLVER_SOFT_STEP)
    sc = scenes.lattice_graph((12, 10, 8), seed=7, joint_fraction=0.3)
    view = sc.to_view(*scenes.host_color(sc))
    whole, packed = both(solver, view, params)
    assert not helpers.mismatches(packed, whole)
    assert packed.bodies.tobytes() == whole.bodies.tobytes()


def test_packed_equals_whole_records_on_reference_scenes(solver, ref_lib):
    """Every joint type, fixed bodies, hits and restitution: scenes cut at the solver stage."""
    params = abi.WorldParams.default()
    for w in (ref_scenes.joint_zoo(seed=5, params=params), ref_scenes.sphere_pour(count=300)):
        for _ in range(20):
            w.step(DT)
        w.collide()
        view = w.export_view()
        w.close()
        whole, packed = both(solver, view, params, steps=3)
        assert not helpers.mismatches(packed, whole)


def test_packed_refusal_leaves_the_outputs_untouched(solver):
    params = abi.WorldParams.default()
    sc = scenes.lattice_graph(5, seed=2)
    view = sc.to_view(*scenes.host_color(sc))
    pk = abi.Packed(view)
    pk.out_bodies[...] = np.frombuffer(np.full(pk.out_bodies.nbytes, 0xAB, np.uint8).tobytes(),
                                       abi.BODY_OUTPUT_DTYPE)
    before = pk.out_bodies.tobytes()
    pk.contacts["body_a"][3] = len(view.bodies) + 1000  # an index out of range
    from nepheline_b200.solver import SolverError
    with pytest.raises(SolverError) as err:
        solver.phys_solve_packed(pk, params, DT)
    assert err.value.code == abi.INVALID_ARGUMENT
    assert pk.out_bodies.tobytes() == before
