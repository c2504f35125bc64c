"""The device's joint-angle arctangent equals the reference's, bit for bit, on the CPU.

The reference's hinge, ball-cone, twist and 6-DOF angle rows call the host C library's
atan2f (glibc 2.39: joint_solver.c:77-84, 303-394, 452-463 through scalar.h:239-242). The
library restates that function in nepheline_b200/csrc/atan2f.h, which the device kernels and
the CPU restatement both include; here the header is compiled for the host with the device's
floating-point contract and compared with the host library's atan2f."""
from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def test_atan2f_equals_the_host_library(tmp_path):
    if shutil.which("gcc") is None:
        pytest.skip("no host compiler")
    exe = tmp_path / "atan2f_check"
    subprocess.run(["gcc", "-O2", "-std=gnu17", "-ffp-contract=off", "-fno-builtin",
                    f"-I{ROOT / 'nepheline_b200' / 'csrc'}", str(ROOT / "tests" / "atan2f_check.c"),
                    "-o", str(exe), "-lm"], check=True)
    out = subprocess.run([str(exe), "61", "20000000"], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout
    assert out.stdout.strip().endswith("mismatches 0")
