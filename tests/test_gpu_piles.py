"""The stages around the narrow phase that the library's own pile simulation uses, on the device:
the broad phase against a brute-force pass over every pair, the contact update's warm start on
host arrays against the CPU restatement of the reference's (contact.c:516-565), and dropped box
piles stepped by the whole pipeline (broad phase, narrow phase, warm start, colouring, solver
stage) coming to rest on their grounds."""
from __future__ import annotations

import numpy as np
import pytest

from nepheline_b200 import abi

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0


def brute_pairs(lo, hi, group):
    n = len(lo)
    i, j = np.triu_indices(n, 1)
    ok = (group[i] == group[j]) & np.all(lo[i] <= hi[j], axis=1) & np.all(lo[j] <= hi[i], axis=1)
    return set(zip(i[ok].tolist(), j[ok].tolist()))


@pytest.mark.parametrize("seed", [1, 2])
def test_broad_phase_equals_every_pair_checked(solver, seed):
    from nepheline_b200.solver import broad_phase
    rng = np.random.default_rng(seed)
    n = 3000
    group = rng.integers(0, 5, n).astype(np.uint32)
    center = rng.uniform(-12.0, 12.0, (n, 3)).astype(np.float32)
    center[:50] = center[50:100] + rng.uniform(-0.5, 0.5, (50, 3)).astype(np.float32)  # close ones
    ext = rng.uniform(0.05, 1.5, (n, 3)).astype(np.float32)
    lo, hi = center - ext, center + ext
    a, b = broad_phase(lo, hi, group, cell=3.01)
    got = set(zip(a.tolist(), b.tolist()))
    assert len(got) == len(a)  # each pair once
    assert got == brute_pairs(lo, hi, group)
    keys = (a.astype(np.uint64) << np.uint64(32)) | b.astype(np.uint64)
    assert np.all(np.diff(keys.astype(np.int64)) > 0)  # in (a, b) order
    assert np.all(a < b)


def test_warm_start_contacts_equals_the_restatement(ref_lib):
    from nepheline_b200 import scenes
    from nepheline_b200.solver import warm_start_contacts
    from oracle.refworld import port_warm_update
    rng = np.random.default_rng(4)
    sc = scenes.lattice_graph(6, seed=3)
    old = sc.contacts.copy()
    pts = old["points"]
    pts["normal_impulse"] = rng.uniform(0, 2, pts["normal_impulse"].shape)
    pts["tangent_impulse"] = rng.normal(0, 0.3, pts["tangent_impulse"].shape)
    pts["id"] = rng.integers(0, 6, pts["id"].shape)
    old["flags"] = rng.integers(0, 2, len(old)).astype(np.uint32) * np.uint32(abi.CONTACT_HIT)
    fresh = sc.contacts.copy()
    fp = fresh["points"]
    fp["normal_impulse"] = 0.0
    fp["tangent_impulse"] = 0.0
    fp["id"] = rng.integers(0, 8, fp["id"].shape)  # some ids persist, others move by place
    fp["anchor_a"] += rng.normal(0, 0.004, fp["anchor_a"].shape).astype(np.float32)
    fp["anchor_b"] += rng.normal(0, 0.004, fp["anchor_b"].shape).astype(np.float32)
    old["point_count"][::7] = 0  # pairs new this step
    got = warm_start_contacts(old, fresh)
    want = port_warm_update(old, fresh)
    assert got.tobytes() == want.tobytes()


def test_dropped_piles_come_to_rest(solver):
    """270 boxes in three worlds dropped from layers up to 13 m: the piles collapse and come to
    rest within 10 s, as the reference engine's world step does with the same boxes (measured:
    8 boxes still above 1 m/s after 4 s, none above 0.2 m/s from 9 s on)."""
    from nepheline_b200 import piles
    params = abi.WorldParams.default()
    p = piles.Piles([60, 120, 90], seed=5)
    speeds = []
    for s in range(600):
        view = p.step(solver, params, DT)
        assert np.isfinite(view.bodies["linear_velocity"]).all()
        v = np.linalg.norm(view.bodies["linear_velocity"], axis=1)
        speeds.append(float(v.max()))
        if s % 60 == 59:
            print(f"step {s}: max |v| {v.max():.3f}, above 1 m/s {int((v > 1).sum())}")
    assert len(p.records) > p.n // 2  # boxes rest on the ground and on each other
    assert max(speeds) > 5.0 and speeds[-1] < 0.5
    # No box sank through its ground (the slab's top is y = 0): each box's lowest corner, its
    # centre less its rotated half extents' vertical reach.
    rot = piles._rotations(p.bodies["rotation"])
    reach = np.einsum("nj,nj->n", np.abs(rot[:, 1, :]), p.half)
    lowest = p.bodies["center"][:, 1] - reach
    assert lowest.min() > -0.05
