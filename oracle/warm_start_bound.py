"""TEST INFRASTRUCTURE (an analysis on the oracle), never the product.

How much any warm start of the new contact points can save on collapsing box piles, measured
on the CPU restatement of the residual-driven mode (oracle/port_impl.h) over piles that the
reference engine itself drops and collides (oracle/_ref): each view is the solver stage's
input at one step, persisted points carrying the reference's matched impulses and new points
starting at zero (contact.c:547-565).

For each view it runs the plain start, then the exact start: the new points set to the very
impulses the plain run converged to (no predictor can start them closer), and the half-exact
start. It prints the passes each needs to reach each tolerance of the plain start's initial
residual, and the lowest residual the plain run reached. Run: python oracle/warm_start_bound.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parent.parent))

from nepheline_b200 import abi  # noqa: E402
from oracle.learned_ref import features  # noqa: E402
from oracle.refworld import RefWorld, port32_converge  # noqa: E402

DT = 1.0 / 60.0
TOLERANCES = (1e-1, 3e-2, 1e-2, 3e-3, 1e-3, 1e-4)


def pile(seed: int, count: int, params) -> RefWorld:
    """`count` boxes (half extents uniform in 0.2-1.0 m, seeded random orientations) in
    layers above the ground, dropped."""
    rng = np.random.default_rng(seed)
    w = RefWorld(params, enable_sleep=False, workers=8)
    w.add_ground(0.0)
    side = max(2, int(round((count / 6) ** 0.5)))
    for i in range(count):
        half = rng.uniform(0.2, 1.0, 3)
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        x, z = (i % side) * 2.0 - side, ((i // side) % side) * 2.0 - side
        y = 1.5 + 2.0 * (i // (side * side))
        w.add_box((x + rng.uniform(-0.2, 0.2), y, z + rng.uniform(-0.2, 0.2)), half=tuple(half),
                  rotation=tuple(q))
    return w


def views(seed: int, count: int, steps, params) -> list:
    w = pile(seed, count, params)
    out = []
    for s in range(max(steps) + 1):
        w.collide()
        if s in steps:
            out.append((s, w.export_view()))
        w.solve(DT)
        w.finish()
    w.close()
    return out


def passes_to(res, tol, ref):
    idx = np.flatnonzero(res <= tol * ref)
    return int(idx[0]) if len(idx) else None


def main(seeds=(50, 51), count=300, steps=range(25, 125, 20), max_passes=1500):
    params = abi.WorldParams.default()
    print("seed step points cold | lowest plain | passes to tolerance: plain / exact / half-exact")
    for seed in seeds:
        for step, v in views(seed, count, list(steps), params):
            _, _, kind = features(v, params, DT)
            cold = kind == abi.POINT_COLD
            plain = port32_converge(v, params, DT, tol=1e-6, max_passes=max_passes)
            ref = plain["residuals"][0]
            exact = np.zeros((len(kind), 3), np.float32)
            exact[cold] = plain["impulses"].reshape(-1, 3)[cold]
            e = port32_converge(v, params, DT, init=exact.reshape(-1), tol=1e-6,
                                max_passes=max_passes, ref=ref)
            hx = port32_converge(v, params, DT, init=(0.5 * exact).reshape(-1), tol=1e-6,
                                 max_passes=max_passes, ref=ref)
            row = " ".join(f"{t:g}:{passes_to(plain['residuals'], t, ref)}/"
                           f"{passes_to(e['residuals'], t, ref)}/{passes_to(hx['residuals'], t, ref)}"
                           for t in TOLERANCES)
            print(f"{seed} {step} {int((kind > 0).sum())} {int(cold.sum())} | "
                  f"{plain['residuals'].min() / ref:.2g} | {row}", flush=True)


if __name__ == "__main__":
    main()
