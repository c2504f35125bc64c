"""The allocation-free colouring, nph_gpu_graph_color_static, through the C ABI.

It exists for callers that may not allocate device memory while they run (an engine that
reserves its memory up front, a fixed per-frame budget, an allocator owned by another
runtime): its scratch is one fixed device array inside the library. Its results must equal
the allocating entry point's, call after call (the array keeps the last call's contents),
and inputs beyond its fixed capacity must be refused with NPH_GPU_TOO_LARGE.

This file is collected last, so a run that stops at the first failure has run every other
test before it; it passes alone in a fresh process too.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from nepheline_b200 import abi, scenes

pytestmark = pytest.mark.gpu

TOO_LARGE = 7
MAX_CONSTRAINTS = 131072
MAX_BODY_SLOTS = 131072


def static_entry():
    from nepheline_b200.solver import lib
    fn = lib().nph_gpu_graph_color_static
    fn.restype = ctypes.c_int32
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                   ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p]
    return fn


def color_static(a, b, d, slots):
    a = np.ascontiguousarray(a, np.uint32)
    b = np.ascontiguousarray(b, np.uint32)
    d = np.ascontiguousarray(d, np.uint8)
    color = np.full(len(a), 0xFFFFFFFF, np.uint32)
    slot = np.full(len(a), 0xFFFFFFFF, np.uint32)
    code = static_entry()(None, a.ctypes.data, b.ctypes.data, d.ctypes.data, len(a), slots,
                          color.ctypes.data, slot.ctypes.data)
    return code, color, slot


def random_graph(seed, slots, count):
    rng = np.random.default_rng(seed)
    dynamic = rng.random(slots) < 0.9
    a = rng.integers(0, slots, count).astype(np.uint32)
    b = rng.integers(0, slots, count).astype(np.uint32)
    a[: count // 5] = rng.integers(0, 6, count // 5)  # hubs: colours run out, some overflow
    b[a == b] = (b[a == b] + 1) % slots
    keep = dynamic[a] | dynamic[b]
    a, b = a[keep], b[keep]
    d = dynamic[a].astype(np.uint8) | (dynamic[b].astype(np.uint8) << 1)
    d |= (rng.random(len(a)) < 0.25).astype(np.uint8) * abi.CONSTRAINT_JOINT
    return a, b, d


@pytest.fixture(scope="module")
def allocating():
    if not pytest.importorskip("torch").cuda.is_available():
        pytest.skip("no CUDA device")
    from nepheline_b200.solver import Solver
    s = Solver(device=0)
    yield s
    s.close()


def test_static_colouring_equals_allocating_colouring_two_calls_in_a_row(allocating):
    lattice = scenes.lattice_graph(20, seed=4, joint_fraction=0.1)
    first = (*lattice.constraint_arrays(), len(lattice.bodies))
    second = (*random_graph(9, 3000, 40000), 3000)
    for args in (first, second, first):
        code, color, slot = color_static(*args)
        assert code == abi.OK
        want_color, want_slot = allocating.graph_color(*args)
        assert np.array_equal(color, want_color)
        assert np.array_equal(slot, want_slot)


def test_static_colouring_takes_no_device_memory_after_its_first_call():
    """Once the library is loaded on the device (its first call), further calls leave the
    device's free memory where it was: nothing is allocated, by the entry point or a library
    it calls."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    args = (*random_graph(12, 5000, 60000), 5000)
    assert color_static(*args)[0] == abi.OK
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info(0)
    for _ in range(3):
        assert color_static(*args)[0] == abi.OK
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info(0)
    assert free_after == free_before


def test_static_colouring_at_its_capacity(allocating):
    a, b, d = random_graph(3, MAX_BODY_SLOTS, MAX_CONSTRAINTS + 4000)
    a, b, d = a[:MAX_CONSTRAINTS], b[:MAX_CONSTRAINTS], d[:MAX_CONSTRAINTS]
    code, color, slot = color_static(a, b, d, MAX_BODY_SLOTS)
    assert code == abi.OK
    want_color, want_slot = allocating.graph_color(a, b, d, MAX_BODY_SLOTS)
    assert np.array_equal(color, want_color) and np.array_equal(slot, want_slot)


def test_static_colouring_refuses_inputs_beyond_capacity():
    a, b, d = random_graph(5, 1000, MAX_CONSTRAINTS + 2000)
    a = np.resize(a, MAX_CONSTRAINTS + 1)
    b = np.resize(b, MAX_CONSTRAINTS + 1)
    d = np.resize(d, MAX_CONSTRAINTS + 1)
    code, _, _ = color_static(a, b, d, 1000)
    assert code == TOO_LARGE
    code, _, _ = color_static(a[:10], b[:10], d[:10], MAX_BODY_SLOTS + 1)
    assert code == TOO_LARGE
