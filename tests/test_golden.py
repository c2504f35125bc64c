"""Golden vectors made by the reference itself (tests/golden/make_golden.py): one step of the
reference's phys_solve per fixture, input and output views. The CPU restatement and the
device solver must reproduce the outputs value for value, joint angle rows included."""
from __future__ import annotations

from pathlib import Path

import pytest

from tests import helpers
from tests.golden.make_golden import load

GOLDEN = sorted((Path(__file__).resolve().parent / "golden").glob("*.npz"))


def ids(p):
    return p.stem


@pytest.mark.parametrize("path", GOLDEN, ids=ids)
def test_port_reproduces_reference_golden(path):
    from oracle.refworld import port32
    vin, vout, params, dt = load(path)
    mine = port32(vin, params, dt)
    assert not helpers.mismatches(mine, vout)


@pytest.mark.gpu
@pytest.mark.parametrize("path", GOLDEN, ids=ids)
def test_device_reproduces_reference_golden(path, solver):
    vin, vout, params, dt = load(path)
    dev = vin.copy()
    solver.phys_solve(dev, params, dt)
    assert not helpers.mismatches(dev, vout)
