"""Generates the golden solver-stage vectors in tests/golden/ from the reference itself.

Each fixture is one step of the reference's phys_solve (oracle/_ref/libnphref.so, built from
the reference's sources by oracle/Makefile) cut out of a scene: the view the solver read
(`in_*`) and the view it wrote (`out_*`), with the world settings and dt. Run here, where the
reference's sources are:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from nepheline_b200 import abi  # noqa: E402
from tests import ref_scenes  # noqa: E402

DT = 1.0 / 60.0


def save(name: str, vin: abi.View, vout: abi.View, params: abi.WorldParams, dt: float):
    arrays = {}
    # Records as raw bytes (the joint record's settings union has overlapping fields).
    for tag, v in (("in", vin), ("out", vout)):
        arrays[f"{tag}_bodies"] = v.bodies.view(np.uint8)
        arrays[f"{tag}_fixed"] = v.fixed.view(np.uint8)
        arrays[f"{tag}_contacts"] = v.contacts.view(np.uint8)
        arrays[f"{tag}_joints"] = v.joints.view(np.uint8)
    arrays["contact_color_counts"] = vin.contact_color_counts
    arrays["joint_color_counts"] = vin.joint_color_counts
    arrays["params"] = np.frombuffer(bytes(params), np.uint8)
    arrays["dt"] = np.array([dt], np.float32)
    np.savez_compressed(HERE / f"{name}.npz", **arrays)
    print(name, len(vin.bodies), "bodies", len(vin.contacts), "manifolds", len(vin.joints), "joints")


def cut(w, warm_steps: int, params, dt=DT, collide=True):
    for _ in range(warm_steps):
        w.step(dt) if collide else w.solve(dt)
    if collide:
        w.collide()
    vin = w.export_view()
    w.solve(dt)
    return vin, w.export_view()


def main():
    p = abi.WorldParams.default()
    save("pyramid_10", *cut(ref_scenes.pyramid(rows=10, jitter=1e-3), 45, p), p, DT)
    save("sphere_pour_64", *cut(ref_scenes.sphere_pour(count=64, extent=6.0), 25, p), p, DT)
    save("box_pile_24", *cut(ref_scenes.box_pile(count=24), 40, p), p, DT)
    save("hinge_chain_8", *cut(ref_scenes.hinge_chain(links=8), 30, p), p, DT)
    w, _ = ref_scenes.lattice(edge=5, joint_fraction=0.25, seed=13)
    save("lattice_5", *cut(w, 2, p, collide=False), p, DT)
    p8 = abi.WorldParams.default(substeps=8, contact_hertz=45.0, restitution_threshold=0.5)
    save("sphere_pour_substeps8", *cut(ref_scenes.sphere_pour(count=48, extent=6.0, params=p8),
                                       20, p8, dt=1.0 / 120.0), p8, 1.0 / 120.0)
    save("joint_zoo", *cut(ref_scenes.joint_zoo(seed=5, params=p), 20, p), p, DT)
    tgs = abi.WorldParams.default(solver=abi.SOLVER_TGS)
    save("joint_zoo_tgs", *cut(ref_scenes.joint_zoo(seed=6, params=tgs), 20, tgs), tgs, DT)
    save("box_pile_24_tgs", *cut(ref_scenes.box_pile(count=24, params=tgs), 40, tgs), tgs, DT)


def load(path: Path) -> tuple[abi.View, abi.View, abi.WorldParams, float]:
    """A fixture's input view, the reference's output view, the settings and dt."""
    z = np.load(path)
    views = []
    for tag in ("in", "out"):
        views.append(abi.View(z[f"{tag}_bodies"].view(abi.BODY_DTYPE),
                              z[f"{tag}_fixed"].view(abi.BODY_DTYPE),
                              z[f"{tag}_contacts"].view(abi.CONTACT_DTYPE),
                              z[f"{tag}_joints"].view(abi.JOINT_DTYPE),
                              z["contact_color_counts"], z["joint_color_counts"]))
    params = abi.WorldParams.from_buffer_copy(z["params"].tobytes())
    return views[0], views[1], params, float(z["dt"][0])


if __name__ == "__main__":
    main()
