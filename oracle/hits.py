"""Test infrastructure only: a CPU restatement of the reference's hit events, the checker of
the device's nph_gpu_world_hit_events.

hit_events (engine/physics/src/solver.c:919-960): over the colour lists and then the overflow,
each manifold whose flags carry PHYS_CONTACT_HIT_EVENTS gives at most one event, at its point of
fastest approach (-relative_velocity) strictly above the world's hit threshold among the points
with a positive max_normal_impulse. Pinned against the reference's own events in
tests/test_hits.py."""
from __future__ import annotations

import numpy as np

from nepheline_b200 import abi


def hit_events_of(view: abi.View, threshold: float) -> np.ndarray:
    """The events of a view written back by a step, as abi.HIT_EVENT_DTYPE records."""
    out = []
    best0 = np.float32(threshold)
    for i, c in enumerate(view.contacts):
        if (int(c["flags"]) & abi.CONTACT_HIT_EVENTS) == 0:
            continue
        best, found = best0, None
        for k in range(int(c["point_count"])):
            approach = -np.float32(c["points"]["relative_velocity"][k])
            if approach > best and np.float32(c["points"]["max_normal_impulse"][k]) > 0.0:
                best, found = approach, k
        if found is not None:
            out.append((i, found, best, 0))
    return np.array(out, dtype=abi.HIT_EVENT_DTYPE)
