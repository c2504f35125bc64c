"""Comparison helpers for the parity tests."""
from __future__ import annotations

import numpy as np

from nepheline_b200 import abi

BODY_OUT = ["center", "origin", "rotation", "linear_velocity", "angular_velocity", "force",
            "torque", "sleep_time"]
POINT_OUT = ["normal_impulse", "max_normal_impulse", "tangent_impulse", "relative_velocity"]
JOINT_OUT = ["linear_impulse", "angular_impulse", "friction_impulse", "lower_impulse",
             "upper_impulse", "swing_impulse", "motor_impulse", "spring_impulse", "axis_impulse",
             "flags"]


def _fields(view: abi.View):
    out = {}
    for f in BODY_OUT:
        out["body." + f] = view.bodies[f]
    pc = view.contacts["point_count"]
    mask = np.arange(4)[None, :] < pc[:, None]
    for f in POINT_OUT:
        v = view.contacts["points"][f]
        out["point." + f] = v[mask]
    out["contact.flags"] = view.contacts["flags"]
    for f in JOINT_OUT:
        out["joint." + f] = view.joints[f]
    return out


def mismatches(a: abi.View, b: abi.View) -> dict:
    """Fields whose values differ (IEEE equality: +0 == -0), with counts."""
    fa, fb = _fields(a), _fields(b)
    bad = {}
    for k in fa:
        x, y = np.asarray(fa[k]), np.asarray(fb[k])
        if x.dtype.kind == "f":
            ne = ~((x == y) | (np.isnan(x) & np.isnan(y)))
        else:
            ne = x != y
        if ne.any():
            bad[k] = int(ne.sum())
    return bad


def bitwise_fraction(a: abi.View, b: abi.View) -> float:
    """Share of output values that agree bit for bit (the sign of zero included)."""
    fa, fb = _fields(a), _fields(b)
    same = total = 0
    for k in fa:
        x, y = np.ascontiguousarray(fa[k]), np.ascontiguousarray(fb[k])
        bx, by = x.view(np.uint8).reshape(x.size, -1) if x.size else x, y.view(np.uint8).reshape(y.size, -1) if y.size else y
        if x.size:
            eq = (bx == by).all(axis=1)
            same += int(eq.sum())
            total += x.size
    return same / max(total, 1)


def max_rel_err(a: abi.View, b: abi.View, floor: float = 1e-6) -> dict:
    """Per field, max |a - b| / max(|b|, floor) over the outputs."""
    fa, fb = _fields(a), _fields(b)
    out = {}
    for k in fa:
        x, y = np.asarray(fa[k], np.float64), np.asarray(fb[k], np.float64)
        if x.size == 0:
            continue
        out[k] = float(np.max(np.abs(x - y) / np.maximum(np.abs(y), floor)))
    return out


def max_normwise_err(a: abi.View, b: abi.View) -> dict:
    """Per field, max |a - b| over the field's largest magnitude in b (relative to the
    field's scale: the error measure of rows whose angle goes through atan2f)."""
    fa, fb = _fields(a), _fields(b)
    out = {}
    for k in fa:
        x, y = np.asarray(fa[k], np.float64), np.asarray(fb[k], np.float64)
        if x.size == 0:
            continue
        scale = np.max(np.abs(y))
        out[k] = float(np.max(np.abs(x - y)) / scale) if scale > 0 else float(np.max(np.abs(x)))
    return out
