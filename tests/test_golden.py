"""Golden vectors made by the reference itself (tests/golden/make_golden.py): one step of the
reference's phys_solve per fixture, input and output views. The CPU restatement and the
device solver must reproduce the outputs; the device's joint angle rows (correctly rounded
arctangent) equal the restatement with that angle, and the reference within its rounding."""
from __future__ import annotations

from pathlib import Path

import pytest

from tests import helpers
from tests.golden.make_golden import load

GOLDEN = sorted((Path(__file__).resolve().parent / "golden").glob("*.npz"))
ANGLE_ROWS = {"hinge_chain_8", "joint_zoo", "joint_zoo_tgs"}


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
    if path.stem in ANGLE_ROWS:
        from oracle.refworld import port32cr
        assert not helpers.mismatches(dev, port32cr(vin, params, dt))
        err = helpers.max_normwise_err(dev, vout)
        assert max(err.values()) < 1e-3, err
    else:
        assert not helpers.mismatches(dev, vout)
