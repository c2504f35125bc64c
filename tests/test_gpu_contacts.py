"""The contact update on the device (nph_gpu_world_update_contacts) against the reference's
own (contact.c:516-565): on steps that keep their contact set, the device's warm-started
records equal the reference's bit for bit, and a world stepped with the bodies resident and
only the manifolds updated equals the reference's step after step."""
from __future__ import annotations

import numpy as np
import pytest

from nepheline_b200 import abi
from tests import helpers, ref_scenes
from tests.test_oracle import aligned_old, raw_manifolds

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0


def same_pairs(a: abi.View, b: abi.View) -> bool:
    return (len(a.contacts) == len(b.contacts)
            and np.array_equal(a.contacts["body_a"], b.contacts["body_a"])
            and np.array_equal(a.contacts["body_b"], b.contacts["body_b"])
            and np.array_equal(a.contact_color_counts, b.contact_color_counts))


def test_device_update_matches_the_reference(solver, ref_lib):
    w = ref_scenes.box_pile(count=40, seed=4)
    old = None
    checked = 0
    for s in range(150):
        w.collide()
        new = w.export_view()
        if old is not None and same_pairs(old, new) and len(new.contacts):
            solver.upload(old)
            solver.update_contacts(raw_manifolds(new))
            got = old.copy()
            solver.download(got)
            assert got.contacts.tobytes() == new.contacts.tobytes(), f"step {s}"
            checked += 1
        w.solve(DT)
        w.finish()
        old = w.export_view()
    assert checked > 20
    w.close()


def test_resident_world_with_updated_contacts_matches_the_reference(solver, ref_lib):
    """A pyramid at rest, stepped by the reference and by the device side by side: the device
    keeps its bodies and contacts between steps and each step receives only the narrow phase's
    manifolds, warm-started on the device from its own stored impulses; its results equal the
    reference's step after step."""
    params = abi.WorldParams.default()
    w = ref_scenes.pyramid(rows=6)
    for _ in range(60):
        w.step(DT)
    w.collide()
    prev = w.export_view()
    solver.upload(prev)
    solver.step_async(params, DT, 1)
    w.solve(DT)
    w.finish()
    steps = 0
    for s in range(30):
        w.collide()
        ref_in = w.export_view()
        assert same_pairs(prev, ref_in), f"the contact set changed at step {s}"
        solver.update_contacts(raw_manifolds(ref_in))
        solver.step_async(params, DT, 1)
        w.solve(DT)
        w.finish()
        ref_out = w.export_view()
        got = ref_out.copy()
        solver.download(got)
        assert not helpers.mismatches(got, ref_out), f"step {s}"
        prev = ref_in
        steps += 1
    assert steps == 30
    w.close()
