"""Seeded pairs of the narrow phase's closed-form shapes: random poses near contact and the
degenerate cases the formulas branch on."""
from __future__ import annotations

import numpy as np

from nepheline_b200 import abi

KINDS = [(abi.SHAPE_SPHERE, abi.SHAPE_SPHERE), (abi.SHAPE_CAPSULE, abi.SHAPE_SPHERE),
         (abi.SHAPE_SPHERE, abi.SHAPE_CAPSULE), (abi.SHAPE_CAPSULE, abi.SHAPE_CAPSULE),
         (abi.SHAPE_BOX, abi.SHAPE_SPHERE), (abi.SHAPE_SPHERE, abi.SHAPE_BOX)]


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
