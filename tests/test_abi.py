"""The C ABI on the CPU: record layouts agree with the header, and the shared library loads
and exports every entry point include/nepheline_b200.h declares (no device calls)."""
from __future__ import annotations

import re
import subprocess
from pathlib import Path

import pytest

from nepheline_b200 import abi

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "nepheline_b200.h"


def declared_entry_points() -> list[str]:
    text = HEADER.read_text()
    return sorted(set(re.findall(r"NPH_GPU_API\s+[\w\s\*]+?\b(nph_gpu_\w+)\s*\(", text)))


def test_header_declares_the_entry_points():
    names = declared_entry_points()
    for n in ("nph_gpu_solver_create", "nph_gpu_phys_solve", "nph_gpu_graph_color",
              "nph_gpu_world_upload", "nph_gpu_world_step_async", "nph_gpu_world_download"):
        assert n in names


def test_record_layouts_match_the_header(tmp_path):
    src = tmp_path / "sizes.c"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "nepheline_b200.h"\n'
        'int main(void){printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\\n",'
        'sizeof(NphGpuBody),sizeof(NphGpuContactPoint),sizeof(NphGpuContact),'
        'sizeof(NphGpuJoint),sizeof(NphGpuWorldParams),sizeof(NphGpuWorldView),'
        'offsetof(NphGpuJoint,linear_impulse),offsetof(NphGpuContact,points),'
        'sizeof(NphGpuKernelTime),sizeof(NphGpuBatchTuning),sizeof(NphGpuBatchInfo),'
        'sizeof(NphGpuStepStats),sizeof(NphGpuSolverDesc));'
        'printf("%zu %zu %zu %zu %zu %zu %zu %zu\\n",sizeof(NphGpuBodyInput),sizeof(NphGpuContactInput),'
        'sizeof(NphGpuBodyOutput),sizeof(NphGpuContactOutput),sizeof(NphGpuJointOutput),'
        'sizeof(NphGpuPackedInput),sizeof(NphGpuPackedOutput),sizeof(NphGpuConvergeStats));return 0;}\n')
    exe = tmp_path / "sizes"
    subprocess.run(["gcc", f"-I{HEADER.parent}", str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True,
                                          check=True).stdout.split()]
    sz = abi.layout_sizes()
    import ctypes
    assert got == [sz["body"], sz["point"], sz["contact"], sz["joint"], sz["params"], sz["view"],
                   abi.JOINT_DTYPE.fields["linear_impulse"][1],
                   abi.CONTACT_DTYPE.fields["points"][1], ctypes.sizeof(abi.KernelTime),
                   ctypes.sizeof(abi.BatchTuning), ctypes.sizeof(abi.BatchInfo),
                   ctypes.sizeof(abi.StepStats), ctypes.sizeof(abi.SolverDesc),
                   sz["body_input"], sz["contact_input"], sz["body_output"], sz["contact_output"],
                   sz["joint_output"], sz["packed_input"], sz["packed_output"],
                   ctypes.sizeof(abi.ConvergeStats)]


def test_library_exports_every_declared_entry_point():
    from nepheline_b200 import solver
    if not solver.LIB_PATH.exists():
        pytest.skip("library not built")
    out = subprocess.run(["nm", "-D", "--defined-only", str(solver.LIB_PATH)],
                         capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (nph_gpu_\w+)", out))
    missing = [n for n in declared_entry_points() if n not in exported]
    assert not missing, missing
    lib = solver.lib()  # loads with its signatures, no device needed
    assert "sm_100a" in solver.version()
    del lib


def test_views_array_equals_the_records_one_at_a_time():
    """The batch's view array, filled column by column, holds the bytes a ctypes record per
    world would: pointers (0 for empty arrays), counts and colour counts, plain and packed
    worlds, and a view whose arrays were replaced after a first use."""
    import ctypes

    import numpy as np
    rng = np.random.default_rng(1)
    views = []
    for _ in range(300):
        cc = rng.integers(0, 9, abi.COLOR_SLOTS).astype(np.uint32)
        jc = rng.integers(0, 3, abi.COLOR_SLOTS).astype(np.uint32)
        views.append(abi.View(np.zeros(rng.integers(0, 12), abi.BODY_DTYPE),
                              np.zeros(rng.integers(0, 2), abi.BODY_DTYPE),
                              np.zeros(rng.integers(0, 20), abi.CONTACT_DTYPE),
                              np.zeros(rng.integers(0, 3), abi.JOINT_DTYPE), cc, jc))

    def one_at_a_time(vs):
        arr = (abi.WorldView * len(vs))()
        for i, v in enumerate(vs):
            arr[i] = v.c_view()
        return bytes(arr)

    assert abi.WORLD_VIEW_DTYPE.itemsize == ctypes.sizeof(abi.WorldView)
    for vs in (views, abi.pack_views(views)):
        assert abi.views_array(vs).tobytes() == one_at_a_time(vs)
    packed = abi.pack_views(views)
    abi.views_array(packed)
    packed[5].contacts = np.zeros(3, abi.CONTACT_DTYPE)
    packed[7].contact_color_counts[0] += 1
    assert abi.views_array(packed).tobytes() == one_at_a_time(packed)
    assert len(abi.views_array([])) == 1


def test_colouring_refuses_counts_beyond_the_sort_without_touching_arrays():
    """Counts the device sort cannot index (it counts items in int) are refused before the
    solver, the arrays or the device are touched: no device is needed."""
    import ctypes

    from nepheline_b200 import solver
    if not solver.LIB_PATH.exists():
        pytest.skip("library not built")
    fn = solver.lib().nph_gpu_graph_color
    dummy = ctypes.create_string_buffer(64)
    p = ctypes.addressof(dummy)
    assert fn(p, p, p, p, 0x7FFFFFFF, 16, p, p) == abi.TOO_LARGE
    assert fn(p, p, p, p, 16, 0x7FFFFFFF, p, p) == abi.TOO_LARGE
