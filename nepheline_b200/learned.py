"""The learned warm start's host pipeline, over the library's own kernels.

  samples()   training samples of a world: the features of its cold points at the step's
              start and, as targets, the impulses the plain solver converged to from a zero
              start (nph_gpu_world_converge), over each point's impulse scale g h / kn
  train()     a network trained on them on the device (nph_gpu_mlp_train)
  compare()   the residual-driven comparison that judges the network: the plain start and the
              learned start on the same world, passes to each tolerance of the plain start's
              initial residual, and device time
  judge()     the same with the exact start beside them: the cold points started at the very
              impulses the plain run converges to, which no predictor can beat

The reference has no counterpart (its new contact points start at zero impulse,
engine/physics/src/contact.c:547-565).
"""
from __future__ import annotations

import numpy as np

from . import abi, scenes


def merged_view(solver, scs: list) -> abi.View:
    """Disjoint worlds as one view, coloured on the device (disjoint worlds colour as they
    would alone)."""
    sc = scenes.merge_scenes(scs)
    a, b, d = sc.constraint_arrays()
    color, slot = solver.graph_color(a, b, d, len(sc.bodies) + (0 if sc.fixed is None else len(sc.fixed)))
    return sc.to_view(color, slot)


def samples(solver, view: abi.View, params: abi.WorldParams, dt: float,
            tolerance: float = 1e-4, max_passes: int = 2000):
    """(features, targets, converge stats) of the world's cold points."""
    solver.upload(view)
    f, scale, kind = solver.features(params, dt)
    run = solver.converge(params, dt, tolerance=tolerance, max_passes=max_passes, impulses=True)
    imp = run["impulses"].reshape(-1, 3)
    cold = (kind == abi.POINT_COLD) & (scale > 0)
    return f[cold], (imp[cold] / scale[cold, None]).astype(np.float32), run


def train(mlp, x: np.ndarray, t: np.ndarray, epochs: int = 40, batch: int = 1024,
          lr: float = 1e-3, seed: int = 0) -> dict:
    """Trains `mlp` on the device; the loss before and after."""
    _, before = mlp.gradients(x, t)
    after = mlp.train(x, t, epochs=epochs, batch=batch, lr=lr, seed=seed)
    return {"samples": int(len(x)), "loss_before": before, "loss_after": after,
            "loss_zero_start": float(np.mean(np.sum(t.astype(np.float64) ** 2, axis=1)))}


def passes_to(residuals: np.ndarray, tolerance: float, reference: float):
    """The first pass whose residual is within tolerance x reference (None: never)."""
    idx = np.flatnonzero(np.asarray(residuals) <= tolerance * reference)
    return int(idx[0]) if len(idx) else None


def compare(solver, mlp, view: abi.View, params: abi.WorldParams, dt: float,
            tolerances=(1e-2, 1e-3, 1e-4), max_passes: int = 2000) -> dict:
    """The plain and the learned start on the same world, judged by the plain solver's
    residual relative to the plain start's initial residual: for each tolerance, the passes
    each start needs (None: not within max_passes) and the device time of that run."""
    solver.upload(view)
    out = {"max_passes": max_passes, "tolerances": {}}
    ref = None
    for tol in sorted(tolerances, reverse=True):
        plain = solver.converge(params, dt, tolerance=tol, max_passes=max_passes)
        ref = float(plain["reference_residual"])
        solver.set_warm_start_model(mlp)
        try:
            learned = solver.converge(params, dt, learned=True, tolerance=tol,
                                      max_passes=max_passes, reference_residual=ref)
        finally:
            solver.set_warm_start_model(None)
        out["tolerances"][f"{tol:g}"] = {
            "plain": int(plain["passes"]) if plain["converged"] else None,
            "learned": int(learned["passes"]) if learned["converged"] else None,
            "plain_ms": float(plain["ms"]), "learned_ms": float(learned["ms"])}
        out["cold_points"] = int(plain["cold_points"])
        out["predicted_points"] = int(learned["predicted_points"])
        out["reference_residual"] = ref
        out["learned_initial_over_plain"] = float(learned["initial_residual"]) / ref if ref > 0 else None
        out["plain_lowest"] = float(plain["residuals"].min()) / ref if ref > 0 else None
        out["learned_lowest"] = float(learned["residuals"].min()) / ref if ref > 0 else None
    return out


def tangents(normal: np.ndarray):
    """t1 = nph_vec3_perpendicular(n) (vec.h:460-469: n crossed with the axis it is least
    aligned with, normalised) and t2 = n x t1, in FP32, for (m, 3) unit normals."""
    n = np.asarray(normal, np.float32)
    a = np.abs(n)
    axis = np.zeros_like(n)
    use_x = (a[:, 0] <= a[:, 1]) & (a[:, 0] <= a[:, 2])
    use_y = ~use_x & (a[:, 1] <= a[:, 2])
    axis[use_x, 0] = 1.0
    axis[use_y, 1] = 1.0
    axis[~use_x & ~use_y, 2] = 1.0
    t1 = np.cross(n, axis)
    t1 /= np.linalg.norm(t1, axis=1, keepdims=True)
    return t1.astype(np.float32), np.cross(n, t1).astype(np.float32)


def exact_start(view: abi.View, kind: np.ndarray, impulses: np.ndarray) -> abi.View:
    """`view` with its cold points' warm start set to `impulses` (4 x (normal, t1, t2) per
    manifold, as nph_gpu_world_converge returns them): the exact start of the new points."""
    out = view.copy()
    cold = (np.asarray(kind).reshape(-1, 4) == abi.POINT_COLD)
    t1, t2 = tangents(out.contacts["normal"])
    imp = np.asarray(impulses, np.float32).reshape(-1, 4, 3)
    pts = out.contacts["points"]
    pts["normal_impulse"] = np.where(cold, imp[..., 0], pts["normal_impulse"])
    world = imp[..., 1:2] * t1[:, None, :] + imp[..., 2:3] * t2[:, None, :]
    pts["tangent_impulse"] = np.where(cold[..., None], world, pts["tangent_impulse"])
    return out


def judge(solver, mlp, view: abi.View, params: abi.WorldParams, dt: float,
          tolerances=(1e-1, 1e-2, 1e-3, 1e-4), max_passes: int = 2000) -> dict:
    """Passes and device time to each tolerance of the plain start's initial residual, for the
    plain start, the network's start, the gated start (the network's start with the plain start
    as its fallback, abi.START_GATED) and the exact start, on one world (each run stops at its
    tolerance, so each time is the run's own)."""
    solver.upload(view)
    _, _, kind = solver.features(params, dt)
    full = solver.converge(params, dt, tolerance=min(tolerances), max_passes=max_passes,
                           impulses=True)
    ref = float(full["reference_residual"])
    exact = exact_start(view, kind, full["impulses"])
    out = {"reference_residual": ref, "cold_points": int(full["cold_points"]),
           "points": int((np.asarray(kind) != abi.POINT_NONE).sum()),
           "plain_lowest": float(full["residuals"].min()) / ref if ref > 0 else None,
           "tolerances": {}}
    for tol in sorted(tolerances, reverse=True):
        row = {}
        for name in ("plain", "learned", "gated", "exact"):
            if name == "exact":
                solver.upload(exact)
            else:
                solver.upload(view)
            start = {"learned": abi.START_LEARNED, "gated": abi.START_GATED}.get(name, abi.START_PLAIN)
            if start != abi.START_PLAIN:
                solver.set_warm_start_model(mlp)
            try:
                r = solver.converge(params, dt, learned=start, tolerance=tol,
                                    max_passes=max_passes, reference_residual=ref)
            finally:
                if start != abi.START_PLAIN:
                    solver.set_warm_start_model(None)
            row[name] = int(r["passes"]) if r["converged"] else None
            row[name + "_ms"] = float(r["ms"])
            if name == "gated":
                row["gated_fell_back"] = bool(r["fell_back"])
            if tol == max(tolerances):
                out[name + "_initial_over_plain"] = float(r["initial_residual"]) / ref if ref > 0 else None
        out["tolerances"][f"{tol:g}"] = row
    return out
