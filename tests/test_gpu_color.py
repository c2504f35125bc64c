"""The device colouring equals the reference's sequential first-fit bit for bit."""
from __future__ import annotations

import numpy as np
import pytest

from nepheline_b200 import abi, scenes
from tests import ref_scenes

pytestmark = pytest.mark.gpu


def test_lattice_colouring_matches_reference(solver, ref_lib):
    w, sc = ref_scenes.lattice(edge=10, joint_fraction=0.1, seed=21)
    c = w.constraints()
    color, slot = solver.graph_color(*sc.constraint_arrays(), c["body_slots"])
    assert np.array_equal(color, c["color"])
    assert np.array_equal(slot, c["slot"])


def test_large_lattice_colouring_matches_port(solver):
    from oracle.refworld import port_graph_color
    sc = scenes.lattice_graph(40, seed=5, joint_fraction=0.1)
    a, b, d = sc.constraint_arrays()
    color, slot = solver.graph_color(a, b, d, len(sc.bodies))
    pc, ps = port_graph_color(a, b, d, len(sc.bodies))
    assert np.array_equal(color, pc) and np.array_equal(slot, ps)


def test_random_graph_with_static_bodies_and_overflow(solver):
    """Random pairs over a few hubs (so colours run out), static and kinematic endpoints,
    joints and contacts interleaved."""
    from oracle.refworld import port_graph_color
    rng = np.random.default_rng(8)
    slots = 400
    dynamic = rng.random(slots) < 0.85
    n = 6000
    a = rng.integers(0, slots, n).astype(np.uint32)
    b = rng.integers(0, slots, n).astype(np.uint32)
    hubs = rng.integers(0, 8, n // 4)
    a[: n // 4] = hubs
    same = a == b
    b[same] = (b[same] + 1) % slots
    keep = dynamic[a] | dynamic[b]
    a, b = a[keep], b[keep]
    d = (dynamic[a].astype(np.uint8) | (dynamic[b].astype(np.uint8) << 1))
    d |= (rng.random(len(a)) < 0.3).astype(np.uint8) * abi.CONSTRAINT_JOINT
    color, slot = solver.graph_color(a, b, d, slots)
    pc, ps = port_graph_color(a, b, d, slots)
    assert (pc == abi.OVERFLOW).any()
    assert np.array_equal(color, pc) and np.array_equal(slot, ps)


def test_colouring_refuses_bad_slots(solver):
    from nepheline_b200.solver import SolverError
    with pytest.raises(SolverError):
        solver.graph_color(np.array([0, 5], np.uint32), np.array([1, 2], np.uint32),
                           np.array([3, 3], np.uint8), 4)


def rope(links: int, seed: int):
    """A chain inserted in order: constraint i joins bodies i and i + 1, so each constraint's
    colour waits on the one before it (the longest chain of lower-index neighbours is the whole
    rope). Every seventh link is a joint, every eleventh body static."""
    rng = np.random.default_rng(seed)
    slots = links + 1
    dynamic = np.ones(slots, bool)
    dynamic[::11] = False
    a = np.arange(links, dtype=np.uint32)
    b = a + 1
    keep = dynamic[a] | dynamic[b]
    a, b = a[keep], b[keep]
    d = dynamic[a].astype(np.uint8) | (dynamic[b].astype(np.uint8) << 1)
    d[::7] |= abi.CONSTRAINT_JOINT
    order = np.arange(len(a))
    rng.shuffle(order[len(a) // 2:])  # the second half out of order: shorter chains there
    return a[order], b[order], d[order], slots


@pytest.mark.parametrize("links", [600, 100_000])
def test_long_chain_colouring_matches_port(solver, links):
    """A rope longer than the rounds' cap goes to the sequential first-fit on one warp; a
    shorter one converges in rounds. Both equal the sequential rule."""
    import time
    from oracle.refworld import port_graph_color
    a, b, d, slots = rope(links, seed=links)
    t = time.perf_counter()
    color, slot = solver.graph_color(a, b, d, slots)
    ms = 1e3 * (time.perf_counter() - t)
    pc, ps = port_graph_color(a, b, d, slots)
    assert np.array_equal(color, pc) and np.array_equal(slot, ps)
    print(f"rope of {links} links coloured in {ms:.1f} ms")
