"""The device narrow phase's pair code built for the host (tests/narrow_host_shim.cu: the same
source with no contraction and correctly rounded division and square root) against the
reference's own nph_physics_collide, on the CPU: every pair kind the device runs, box-box with
its face, edge and GJK paths included, manifold for manifold, bit for bit."""
from __future__ import annotations

import ctypes
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from nepheline_b200 import abi
from tests import narrow_cases

ROOT = Path(__file__).resolve().parent.parent


@pytest.fixture(scope="module")
def host_collide(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(nvcc).exists():
        pytest.skip("nvcc not found")
    out = tmp_path_factory.mktemp("narrow") / "narrow_host.so"
    subprocess.run([nvcc, "-O2", "-std=c++17", "-Xcompiler", "-ffp-contract=off,-fPIC,-fno-fast-math",
                    "-shared", f"-I{ROOT / 'include'}", f"-I{ROOT / 'nepheline_b200' / 'csrc'}",
                    "-Wno-deprecated-gpu-targets", str(ROOT / "tests" / "narrow_host_shim.cu"),
                    "-o", str(out)], check=True, capture_output=True)
    lib = ctypes.CDLL(str(out))

    def run(a, pa, b, pb, spec):
        arrs = [np.ascontiguousarray(a, abi.SHAPE_DTYPE), np.ascontiguousarray(pa, abi.POSE_DTYPE),
                np.ascontiguousarray(b, abi.SHAPE_DTYPE), np.ascontiguousarray(pb, abi.POSE_DTYPE),
                np.ascontiguousarray(spec, np.float32)]
        res = np.zeros(len(a), abi.MANIFOLD_DTYPE)
        ptr = [ctypes.c_void_p(x.ctypes.data) for x in arrs]
        lib.nph_host_collide(*ptr, ctypes.c_uint(len(a)), ctypes.c_void_p(res.ctypes.data))
        return res
    return run


def live(m):
    return [r["normal"].tobytes() + r["point_count"].tobytes() + r["points"][:int(r["point_count"])].tobytes()
            for r in m]


@pytest.mark.parametrize("kind", range(len(narrow_cases.KINDS)))
def test_host_build_matches_reference(ref_lib, host_collide, kind):
    from oracle.refworld import ref_collide
    a, pa, b, pb, spec = narrow_cases.pairs(seed=kind, per_kind=3000)[kind]
    mine, ref = host_collide(a, pa, b, pb, spec), ref_collide(a, pa, b, pb, spec)
    bad = [i for i, (x, y) in enumerate(zip(live(mine), live(ref))) if x != y]
    assert not bad, (len(bad), bad[:5])


def test_host_build_matches_reference_stacked_boxes(ref_lib, host_collide):
    from oracle.refworld import ref_collide
    a, pa, b, pb, spec = narrow_cases.stacked_boxes(seed=1, n=6000)
    mine, ref = host_collide(a, pa, b, pb, spec), ref_collide(a, pa, b, pb, spec)
    bad = [i for i, (x, y) in enumerate(zip(live(mine), live(ref))) if x != y]
    assert not bad, (len(bad), bad[:5])
    # Face contacts of four points (clipped and reduced), and boxes apart measured by GJK.
    assert (ref["point_count"] == 4).mean() > 0.4
    gjk = (ref["point_count"] == 1) & (ref["points"]["id"][:, 0] == 0x40000000)
    assert gjk.sum() > 20
