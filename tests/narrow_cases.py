"""Seeded pairs of the narrow phase's device shapes: random poses near contact, the degenerate
cases the formulas branch on, and for two boxes resting contacts (one box on another's face,
tilted a little, touching, sunk or just apart: face clipping with its reduction to four points)
beside the random poses (edge pairs, and GJK for boxes apart by more than the slop)."""
from __future__ import annotations

import numpy as np

from nepheline_b200 import abi

KINDS = [(abi.SHAPE_SPHERE, abi.SHAPE_SPHERE), (abi.SHAPE_CAPSULE, abi.SHAPE_SPHERE),
         (abi.SHAPE_SPHERE, abi.SHAPE_CAPSULE), (abi.SHAPE_CAPSULE, abi.SHAPE_CAPSULE),
         (abi.SHAPE_BOX, abi.SHAPE_SPHERE), (abi.SHAPE_SPHERE, abi.SHAPE_BOX),
         (abi.SHAPE_BOX, abi.SHAPE_BOX), (abi.SHAPE_BOX, abi.SHAPE_CAPSULE),
         (abi.SHAPE_CAPSULE, abi.SHAPE_BOX)]


def _qmul(x, y):
    x1, y1, z1, w1 = x.T
    x2, y2, z2, w2 = y.T
    return np.stack([w1 * x2 + x1 * w2 + y1 * z2 - z1 * y2, w1 * y2 - x1 * z2 + y1 * w2 + z1 * x2,
                     w1 * z2 + x1 * y2 - y1 * x2 + z1 * w2, w1 * w2 - x1 * x2 - y1 * y2 - z1 * z2], 1)


def _rotate(q, v):
    u, w = q[:, :3], q[:, 3:4]
    t = 2.0 * np.cross(u, v)
    return v + w * t + np.cross(u, t)


def stacked_boxes(seed=0, n=4000):
    """Box B on box A's +y face (in A's frame): B turned by a small random rotation, offset
    across the face, its gap from -2 cm (sunk) to +3 cm (apart)."""
    rng = np.random.default_rng(seed)
    a, b = shape(rng, abi.SHAPE_BOX, n), shape(rng, abi.SHAPE_BOX, n)
    pa = np.zeros(n, abi.POSE_DTYPE)
    pb = np.zeros(n, abi.POSE_DTYPE)
    pa["position"] = rng.uniform(-2, 2, (n, 3))
    pa["rotation"] = random_quat(rng, n)
    tilt = rng.normal(0.0, 0.02, (n, 4))
    tilt[:, 3] = 1.0
    tilt /= np.linalg.norm(tilt, axis=1, keepdims=True)
    qa = pa["rotation"].astype(np.float64)
    pb["rotation"] = _qmul(qa, tilt).astype(np.float32)
    off = np.zeros((n, 3))
    off[:, 0] = rng.uniform(-0.5, 0.5, n)
    off[:, 1] = a["dims"][:, 1] + b["dims"][:, 1] + rng.uniform(-0.02, 0.03, n)
    off[:, 2] = rng.uniform(-0.5, 0.5, n)
    pb["position"] = (pa["position"] + _rotate(qa, off)).astype(np.float32)
    spec = rng.uniform(-0.01, 0.2, n).astype(np.float32)
    return a, pa, b, pb, spec


def random_quat(rng, n):
    q = rng.normal(size=(n, 4))
    return (q / np.linalg.norm(q, axis=1, keepdims=True)).astype(np.float32)


def shape(rng, kind, n):
    s = np.zeros(n, abi.SHAPE_DTYPE)
    s["type"] = kind
    if kind == abi.SHAPE_SPHERE:
        s["dims"][:, 0] = rng.uniform(0.1, 1.0, n)
    elif kind == abi.SHAPE_CAPSULE:
        s["dims"][:, 0] = rng.uniform(0.0, 1.0, n)
        s["dims"][:, 1] = rng.uniform(0.1, 0.6, n)
    else:
        s["dims"] = rng.uniform(0.2, 1.0, (n, 3))
    return s


def pairs(seed=0, per_kind=4000):
    rng = np.random.default_rng(seed)
    out = []
    for ka, kb in KINDS:
        n = per_kind
        a, b = shape(rng, ka, n), shape(rng, kb, n)
        pa = np.zeros(n, abi.POSE_DTYPE)
        pb = np.zeros(n, abi.POSE_DTYPE)
        pa["position"] = rng.uniform(-2, 2, (n, 3))
        pa["rotation"] = random_quat(rng, n)
        pb["rotation"] = random_quat(rng, n)
        pb["position"] = pa["position"] + rng.normal(0, 1.0, (n, 3)).astype(np.float32)
        spec = rng.uniform(-0.01, 0.2, n).astype(np.float32)
        # Degenerate: coincident centres, centres on a capsule core or a box face, parallel and
        # crossing capsules, zero-length cores, exact touching distance.
        m = n // 8
        pb["position"][:m] = pa["position"][:m]
        if ka == abi.SHAPE_CAPSULE and kb == abi.SHAPE_CAPSULE:
            pb["rotation"][m:2 * m] = pa["rotation"][m:2 * m]
            pb["rotation"][2 * m:3 * m] = -pa["rotation"][2 * m:3 * m]
            a["dims"][3 * m:4 * m, 0] = 0.0
        if ka == abi.SHAPE_BOX:
            pb["position"][m:2 * m] = pa["position"][m:2 * m]
            pb["position"][m:2 * m, 1] += a["dims"][m:2 * m, 1] * 0.5
        if ka == abi.SHAPE_SPHERE and kb == abi.SHAPE_SPHERE:
            d = (a["dims"][m:2 * m, 0] + b["dims"][m:2 * m, 0])
            pb["position"][m:2 * m] = pa["position"][m:2 * m]
            pb["position"][m:2 * m, 0] += d
            spec[m:2 * m] = 0.0
        out.append((a, pa, b, pb, spec))
    return out
