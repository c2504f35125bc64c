"""The binding a maintainer adds to the reference engine (nepheline_b200/binding), compiled into
the engine with world.c built as -Dphys_solve=phys_solve_dispatch (oracle/Makefile, target
`binding`), driven through the engine's public world step: the reference build's determinism
scene (a 20-row box pyramid, sleep off, dt 1/60, 4 substeps, 600 steps), whose world hash the
reference build gives as 0xBE0527E5EE2697B2 (nph_physics_world_hash, world.c:436-462)."""
from __future__ import annotations

import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
EXE = ROOT / "oracle" / "_ref" / "binding_world_step"
PYRAMID_HASH = "be0527e5ee2697b2"
UNSUPPORTED = 8


def run(mode: str, steps: int) -> dict:
    if not EXE.exists():
        pytest.skip("the binding check is not built (the reference sources are absent)")
    out = subprocess.run([str(EXE), mode, str(steps)], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    m = re.search(r"mode (\w+) steps (\d+) result (-?\d+) hash ([0-9a-f]+)", out.stdout)
    assert m, out.stdout
    return {"steps": int(m.group(2)), "result": int(m.group(3)), "hash": m.group(4)}


def test_engine_step_with_the_binding_compiled_in_keeps_the_reference_hash():
    """No device solver attached: the dispatch runs the engine's own stage."""
    r = run("cpu", 600)
    assert r == {"steps": 600, "result": 0, "hash": PYRAMID_HASH}


@pytest.mark.gpu
def test_engine_step_on_the_device_reaches_the_reference_hash():
    """The device solver attached: 600 world steps through nph_physics_world_step, each solver
    stage on the device, end at the reference build's hash."""
    r = run("gpu", 600)
    assert r["result"] == 0 and r["steps"] == 600
    assert r["hash"] == PYRAMID_HASH


@pytest.mark.gpu
def test_engine_step_refuses_what_the_device_does_not_run():
    """An XPBD world's step returns NPH_RESULT_UNSUPPORTED from the device binding: no CPU
    fallback."""
    r = run("xpbd", 5)
    assert r["steps"] == 1 and r["result"] == UNSUPPORTED
