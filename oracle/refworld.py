"""TEST INFRASTRUCTURE (the oracle), never the product.

Python bindings for the two checkers built by oracle/Makefile:

  RefWorld  the reference engine's own physics (oracle/_ref/libnphref.so, compiled from the
            reference's sources) driven white-box: scene building, its stages one by one,
            and conversion of its world to and from the solver-stage view.
  port32 / port64 / port_graph_color
            this project's CPU restatement of the solver stage (oracle/_build/
            liboracle_port.so): FP32 (bit-exact with the reference) and FP64 (the error
            baseline), and the sequential first-fit colouring.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this module.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

from nepheline_b200 import abi

HERE = Path(__file__).resolve().parent
REF_LIB = HERE / "_ref" / "libnphref.so"
PORT_LIB = HERE / "_build" / "liboracle_port.so"

_u32 = ctypes.c_uint32
_f32 = ctypes.c_float
_vp = ctypes.c_void_p
_ref = None
_port = None


def ref_available() -> bool:
    return REF_LIB.exists()


def _ref_lib():
    global _ref
    if _ref is None:
        lib = ctypes.CDLL(str(REF_LIB))
        sig = {
            "nphref_world_create": (_vp, [ctypes.POINTER(abi.WorldParams), _u32, _u32]),
            "nphref_world_destroy": (None, [_vp]),
            "nphref_worker_count": (_u32, [_vp]),
            "nphref_force_participants": (None, [_vp, _u32]),
            "nphref_add_body": (_u32, [_vp, _u32, _vp, _vp, _vp, _vp, _u32, _vp, _f32, _f32,
                                       _f32, _u32]),
            "nphref_set_mass": (None, [_vp, _u32, _f32, _vp, _vp]),
            "nphref_add_shapeless_bodies": (_u32, [_vp, _u32, _vp, _vp]),
            "nphref_add_joints": (_u32, [_vp, _u32, _vp]),
            "nphref_inject_contacts": (_u32, [_vp, _u32, _vp]),
            "nphref_collide": (ctypes.c_int, [_vp]),
            "nphref_solve": (ctypes.c_int, [_vp, _f32]),
            "nphref_hit_events": (_u32, [_vp, _u32, _vp, _vp, _vp]),
            "nphref_set_hit_threshold": (None, [_vp, _f32]),
            "nphref_finish": (ctypes.c_int, [_vp]),
            "nphref_step": (ctypes.c_int, [_vp, _f32]),
            "nphref_hash": (ctypes.c_uint64, [_vp]),
            "nphref_last_solve_ms": (ctypes.c_double, [_vp]),
            "nphref_body_count": (_u32, [_vp]),
            "nphref_body_state": (None, [_vp, _u32, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
            "nphref_constraint_count": (_u32, [_vp]),
            "nphref_constraints": (None, [_vp, _vp, _vp, _vp, _vp, _vp]),
            "nphref_body_slots": (_u32, [_vp]),
            "nphref_view_sizes": (None, [_vp, _vp, _vp, _vp, _vp]),
            "nphref_export": (ctypes.c_int, [_vp, ctypes.POINTER(abi.WorldView)]),
            "nphref_import": (ctypes.c_int, [_vp, ctypes.POINTER(abi.WorldView), _f32]),
            "nphref_stats": (None, [_vp, _vp, _vp, _vp, _vp, _vp]),
            "nphref_set_velocity": (None, [_vp, _u32, _vp, _vp]),
            "nphref_collide_pairs": (None, [_vp, _vp, _vp, _vp, _vp, _u32, _vp]),
            "nphref_merge_islands": (ctypes.c_int, [_vp]),
            "nphref_sleep_islands": (ctypes.c_int, [_vp]),
            "nphref_island_view": (_u32, [_vp, _vp, _vp, _vp, _u32]),
            "nphref_island_state": (None, [_vp, _u32, _vp, _vp]),
            "nphref_awake_creation_ids": (None, [_vp, _vp]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _ref = lib
    return _ref


def _port_lib():
    global _port
    if _port is None:
        lib = ctypes.CDLL(str(PORT_LIB))
        lib.nph_port32_solve.restype = ctypes.c_int
        lib.nph_port32_solve.argtypes = [ctypes.POINTER(abi.WorldParams), _f32,
                                         ctypes.POINTER(abi.WorldView)]
        lib.nph_port64_solve.restype = ctypes.c_int
        lib.nph_port64_solve.argtypes = [ctypes.POINTER(abi.WorldParams), _f32,
                                         ctypes.POINTER(abi.WorldView), _vp]
        lib.nph_port32_converge.restype = ctypes.c_int
        lib.nph_port32_converge.argtypes = [ctypes.POINTER(abi.WorldParams), _f32,
                                            ctypes.POINTER(abi.WorldView), _vp, ctypes.c_double,
                                            ctypes.c_uint, ctypes.c_double, _vp, _vp, _vp, _vp]
        lib.nph_port_warm_update.restype = ctypes.c_int
        lib.nph_port_warm_update.argtypes = [_vp, _vp, ctypes.c_uint, _vp]
        lib.nph_port_graph_color.restype = ctypes.c_int
        lib.nph_port_graph_color.argtypes = [_vp, _vp, _vp, _u32, _u32, _vp, _vp]
        _port = lib
    return _port


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


class RefWorld:
    """A reference world (engine/physics) built and stepped through the harness."""

    def __init__(self, params: abi.WorldParams | None = None, enable_sleep: bool = False,
                 workers: int = 0):
        """workers: 0 no job system; n > 0 a job system of n workers; -1 the reference's
        default (logical cores - 1)."""
        self.params = params if params is not None else abi.WorldParams.default()
        lib = _ref_lib()
        w = abi.NULL if workers < 0 else workers
        self._h = lib.nphref_world_create(ctypes.byref(self.params), int(enable_sleep), w)
        if not self._h:
            raise RuntimeError("reference world creation failed")
        self.lib = lib

    def close(self):
        if self._h:
            self.lib.nphref_world_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def workers(self) -> int:
        return int(self.lib.nphref_worker_count(self._h))

    def force_participants(self, n: int):
        self.lib.nphref_force_participants(self._h, n)

    # -- scene building -------------------------------------------------------------
    def add_body(self, type_, position, rotation=(0, 0, 0, 1), velocity=(0, 0, 0),
                 angular_velocity=(0, 0, 0), shape=0, dims=(0, 0, 0), density=1000.0,
                 friction=0.6, restitution=0.0, gyroscopic=True, enable_sleep=True,
                 bullet=False, hit_events=False) -> int:
        pos = np.asarray(position, np.float64)
        rot = np.asarray(rotation, np.float32)
        v = np.asarray(velocity, np.float32)
        w = np.asarray(angular_velocity, np.float32)
        d = np.asarray(dims, np.float32)
        flags = ((1 if gyroscopic else 0) | (2 if enable_sleep else 0) | (4 if bullet else 0)
                 | (8 if hit_events else 0))
        idx = self.lib.nphref_add_body(self._h, type_, _p(pos), _p(rot), _p(v), _p(w), shape,
                                       _p(d), density, friction, restitution, flags)
        if idx == abi.NULL:
            raise RuntimeError("reference body creation failed")
        return int(idx)

    def add_box(self, position, half=(0.5, 0.5, 0.5), type_=abi.BODY_DYNAMIC, **kw) -> int:
        return self.add_body(type_, position, shape=1, dims=half, **kw)

    def add_sphere(self, position, radius, type_=abi.BODY_DYNAMIC, **kw) -> int:
        return self.add_body(type_, position, shape=2, dims=(radius, 0, 0), **kw)

    def add_capsule(self, position, half_height, radius, type_=abi.BODY_DYNAMIC, **kw) -> int:
        return self.add_body(type_, position, shape=3, dims=(half_height, radius, 0), **kw)

    def add_ground(self, top=0.0, friction=0.6) -> int:
        """A static slab whose top face is y = top (test_world_support.h:64-68)."""
        return self.add_box((0.0, top - 1.0, 0.0), half=(50.0, 1.0, 50.0),
                            type_=abi.BODY_STATIC, friction=friction)

    def add_shapeless_bodies(self, records: np.ndarray, mass: np.ndarray) -> int:
        records = np.ascontiguousarray(records, abi.BODY_DTYPE)
        mass = np.ascontiguousarray(mass, np.float32)
        first = self.lib.nphref_add_shapeless_bodies(self._h, len(records), _p(records), _p(mass))
        if first == abi.NULL:
            raise RuntimeError("reference body creation failed")
        return int(first)

    def add_joints(self, records: np.ndarray):
        records = np.ascontiguousarray(records, abi.JOINT_DTYPE)
        if len(records) and self.lib.nphref_add_joints(self._h, len(records), _p(records)) == abi.NULL:
            raise RuntimeError("reference joint creation failed")

    def inject_contacts(self, records: np.ndarray):
        records = np.ascontiguousarray(records, abi.CONTACT_DTYPE)
        if len(records) and self.lib.nphref_inject_contacts(self._h, len(records),
                                                            _p(records)) == abi.NULL:
            raise RuntimeError("reference contact injection failed")

    # -- stages -----------------------------------------------------------------------
    def collide(self):
        r = self.lib.nphref_collide(self._h)
        if r != 0:
            raise RuntimeError(f"reference collide failed: {r}")

    def hit_events(self):
        """The last solve's hit events (solver.c:919-960): approach speeds, world points (f64)
        and normals, in the reference's order."""
        n = int(self.lib.nphref_hit_events(self._h, 0, None, None, None))
        speed = np.zeros(max(n, 1), np.float32)
        point = np.zeros((max(n, 1), 3), np.float64)
        normal = np.zeros((max(n, 1), 3), np.float32)
        self.lib.nphref_hit_events(self._h, n, speed.ctypes.data, point.ctypes.data, normal.ctypes.data)
        return speed[:n], point[:n], normal[:n]

    def set_hit_threshold(self, speed: float) -> None:
        self.lib.nphref_set_hit_threshold(self._h, speed)

    def solve(self, dt: float) -> float:
        r = self.lib.nphref_solve(self._h, dt)
        if r != 0:
            raise RuntimeError(f"reference phys_solve failed: {r}")
        return 0.0

    def finish(self):
        r = self.lib.nphref_finish(self._h)
        if r != 0:
            raise RuntimeError(f"reference island stage failed: {r}")

    def merge_islands(self):
        r = self.lib.nphref_merge_islands(self._h)
        if r != 0:
            raise RuntimeError(f"reference island merge failed: {r}")

    def sleep_islands(self):
        r = self.lib.nphref_sleep_islands(self._h)
        if r != 0:
            raise RuntimeError(f"reference sleep and split failed: {r}")

    def island_view(self, awake_bodies: int):
        """(island_of per awake body, island record ids, constraint_remove_count per awake island)."""
        cap = max(awake_bodies, 1)
        island_of = np.zeros(cap, np.uint32)
        ids = np.zeros(cap, np.uint32)
        removed = np.zeros(cap, np.uint32)
        n = self.lib.nphref_island_view(self._h, _p(island_of), _p(ids), _p(removed), cap)
        return island_of[:awake_bodies], ids[:n], removed[:n]

    def island_state(self, island: int):
        removed, awake = ctypes.c_uint32(), ctypes.c_uint32()
        self.lib.nphref_island_state(self._h, island, ctypes.byref(removed), ctypes.byref(awake))
        return int(removed.value), bool(awake.value)

    def awake_creation_ids(self, awake_bodies: int) -> np.ndarray:
        out = np.zeros(max(awake_bodies, 1), np.uint32)
        self.lib.nphref_awake_creation_ids(self._h, _p(out))
        return out[:awake_bodies]

    def step(self, dt: float):
        r = self.lib.nphref_step(self._h, dt)
        if r != 0:
            raise RuntimeError(f"reference world step failed: {r}")

    def hash(self) -> int:
        return int(self.lib.nphref_hash(self._h))

    @property
    def last_solve_ms(self) -> float:
        return float(self.lib.nphref_last_solve_ms(self._h))

    def body_state(self, body: int) -> dict:
        c = np.zeros(3, np.float64)
        o = np.zeros(3, np.float64)
        q = np.zeros(4, np.float32)
        v = np.zeros(3, np.float32)
        w = np.zeros(3, np.float32)
        st = ctypes.c_float()
        fl = ctypes.c_uint32()
        self.lib.nphref_body_state(self._h, body, _p(c), _p(o), _p(q), _p(v), _p(w),
                                   ctypes.addressof(st), ctypes.addressof(fl))
        return {"center": c, "origin": o, "rotation": q, "v": v, "w": w,
                "sleep_time": st.value, "flags": fl.value}

    def stats(self) -> dict:
        vals = [ctypes.c_uint32() for _ in range(5)]
        self.lib.nphref_stats(self._h, *[ctypes.addressof(x) for x in vals])
        keys = ["touching", "points", "colors_used", "overflow", "awake"]
        return {k: int(x.value) for k, x in zip(keys, vals)}

    # -- the colouring ----------------------------------------------------------------
    def constraints(self) -> dict:
        n = int(self.lib.nphref_constraint_count(self._h))
        a = np.zeros(n, np.uint32)
        b = np.zeros(n, np.uint32)
        d = np.zeros(n, np.uint8)
        c = np.zeros(n, np.uint32)
        s = np.zeros(n, np.uint32)
        if n:
            self.lib.nphref_constraints(self._h, _p(a), _p(b), _p(d), _p(c), _p(s))
        return {"body_a": a, "body_b": b, "dynamic_bits": d, "color": c, "slot": s,
                "body_slots": int(self.lib.nphref_body_slots(self._h))}

    # -- world <-> view ---------------------------------------------------------------
    def export_view(self) -> abi.View:
        sizes = [ctypes.c_uint32() for _ in range(4)]
        self.lib.nphref_view_sizes(self._h, *[ctypes.addressof(x) for x in sizes])
        nb, nf, nc, nj = (int(x.value) for x in sizes)
        view = abi.View(np.zeros(nb, abi.BODY_DTYPE), np.zeros(nf, abi.BODY_DTYPE),
                        np.zeros(nc, abi.CONTACT_DTYPE), np.zeros(nj, abi.JOINT_DTYPE),
                        np.zeros(abi.COLOR_SLOTS, np.uint32), np.zeros(abi.COLOR_SLOTS, np.uint32))
        cv = view.c_view()
        r = self.lib.nphref_export(self._h, ctypes.byref(cv))
        if r != 0:
            raise RuntimeError("reference export found bodies outside the first mapping")
        view.contact_color_counts[:] = np.frombuffer(cv.contact_color_counts, np.uint32)
        view.joint_color_counts[:] = np.frombuffer(cv.joint_color_counts, np.uint32)
        return view

    def import_view(self, view: abi.View, dt: float):
        cv = view.c_view()
        r = self.lib.nphref_import(self._h, ctypes.byref(cv), dt)
        if r != 0:
            raise RuntimeError(f"reference import failed: {r}")


# ------------------------------------------------------------------------------------
# The CPU restatement
# ------------------------------------------------------------------------------------

def port32(view: abi.View, params: abi.WorldParams, dt: float) -> abi.View:
    """FP32 solve of a copy of `view` (the reference's arithmetic, one manifold at a time)."""
    out = view.copy()
    cv = out.c_view()
    r = _port_lib().nph_port32_solve(ctypes.byref(params), dt, ctypes.byref(cv))
    if r != 0:
        raise RuntimeError(f"port32 failed: {abi.RESULT_NAMES.get(r, r)}")
    return out


def port32_result(view: abi.View, params: abi.WorldParams, dt: float) -> int:
    """The result code of an FP32 solve of a copy of `view`."""
    work = view.copy()  # kept alive across the call: the C view points into its arrays
    cv = work.c_view()
    return int(_port_lib().nph_port32_solve(ctypes.byref(params), dt, ctypes.byref(cv)))


def port64(view: abi.View, params: abi.WorldParams, dt: float) -> dict:
    """FP64 re-run of the same step: the error baseline. Returns float64 arrays."""
    nb, nc, nj = len(view.bodies), len(view.contacts), len(view.joints)
    out = {
        "linear_velocity": np.zeros((nb, 3)), "angular_velocity": np.zeros((nb, 3)),
        "rotation": np.zeros((nb, 4)), "center": np.zeros((nb, 3)),
        "normal_impulse": np.zeros((nc, 4)), "max_normal_impulse": np.zeros((nc, 4)),
        "tangent_impulse": np.zeros((nc, 4, 3)), "relative_velocity": np.zeros((nc, 4)),
        "joint_linear_impulse": np.zeros((nj, 3)), "joint_angular_impulse": np.zeros((nj, 3)),
    }
    order = ["linear_velocity", "angular_velocity", "rotation", "center", "normal_impulse",
             "max_normal_impulse", "tangent_impulse", "relative_velocity",
             "joint_linear_impulse", "joint_angular_impulse"]
    ptrs = (ctypes.c_void_p * len(order))(*[out[k].ctypes.data for k in order])
    cv = view.c_view()
    r = _port_lib().nph_port64_solve(ctypes.byref(params), dt, ctypes.byref(cv), ptrs)
    if r != 0:
        raise RuntimeError(f"port64 failed: {abi.RESULT_NAMES.get(r, r)}")
    return out


def port_graph_color(body_a, body_b, dynamic_bits, body_slots) -> tuple[np.ndarray, np.ndarray]:
    a = np.ascontiguousarray(body_a, np.uint32)
    b = np.ascontiguousarray(body_b, np.uint32)
    d = np.ascontiguousarray(dynamic_bits, np.uint8)
    n = len(a)
    color = np.zeros(n, np.uint32)
    slot = np.zeros(n, np.uint32)
    r = _port_lib().nph_port_graph_color(_p(a), _p(b), _p(d), n, body_slots, _p(color), _p(slot))
    if r != 0:
        raise RuntimeError("port colouring failed")
    return color, slot


def scene_world(sc, params=None, workers: int = 0):
    """A solver scene in the reference: its bodies (then its fixed bodies, as static bodies,
    at the indices after them) created shapeless, joints made, manifolds injected in insertion
    order (coloured by the reference's phys_graph_add)."""
    w = RefWorld(params or abi.WorldParams.default(), enable_sleep=False, workers=workers)
    bodies, mass = sc.bodies, sc.mass
    if sc.fixed is not None and len(sc.fixed):
        bodies = np.concatenate([bodies, sc.fixed])
        mass = np.concatenate([mass, np.zeros(len(sc.fixed), np.float32)])
    w.add_shapeless_bodies(bodies, mass)
    w.add_joints(sc.joints)
    w.inject_contacts(sc.contacts)
    return w


def lattice_world(dims, seed: int = 0, joint_fraction: float = 0.1, params=None, workers: int = 0):
    """The synthetic constraint graph in the reference: shapeless bodies created, joints made,
    manifolds injected in insertion order (coloured by the reference's phys_graph_add)."""
    from nepheline_b200 import scenes
    sc = scenes.lattice_graph(dims, seed=seed, joint_fraction=joint_fraction)
    w = RefWorld(params or abi.WorldParams.default(), enable_sleep=False, workers=workers)
    w.add_shapeless_bodies(sc.bodies, sc.mass)
    w.add_joints(sc.joints)
    w.inject_contacts(sc.contacts)
    return w, sc


def port32_converge(view, params, dt: float, init=None, tol: float = 1e-4,
                    max_passes: int = 2000, ref: float = 0.0) -> dict:
    """The residual-driven mode restated on the CPU (FP32 solver, residual in double): the
    checker of nph_gpu_world_converge. `init`: 12 floats per manifold, the starting impulses
    of cold point slots."""
    lib = _port_lib()
    cv = view.c_view()
    res = np.zeros(max_passes + 1, np.float64)
    passes = ctypes.c_uint()
    cold = ctypes.c_uint()
    imp = np.zeros(12 * max(len(view.contacts), 1), np.float32)
    ini = None if init is None else np.ascontiguousarray(init, np.float32).reshape(-1)
    rc = lib.nph_port32_converge(ctypes.byref(params), dt, ctypes.byref(cv),
                                 None if ini is None else _p(ini), tol, max_passes, ref,
                                 _p(res), ctypes.byref(passes), ctypes.byref(cold), _p(imp))
    if rc != abi.OK:
        raise RuntimeError(f"port converge failed: {rc}")
    return {"passes": passes.value, "cold_points": cold.value,
            "residuals": res[: passes.value + 1].copy(),
            "impulses": imp[: 12 * len(view.contacts)].reshape(-1, 4, 3)}


def port_warm_update(old_contacts: np.ndarray, fresh_contacts: np.ndarray) -> np.ndarray:
    """The contact update's warm start restated on the CPU, contact by contact."""
    old_contacts = np.ascontiguousarray(old_contacts, abi.CONTACT_DTYPE)
    fresh_contacts = np.ascontiguousarray(fresh_contacts, abi.CONTACT_DTYPE)
    assert len(old_contacts) == len(fresh_contacts)
    out = np.zeros_like(fresh_contacts)
    rc = _port_lib().nph_port_warm_update(_p(old_contacts), _p(fresh_contacts), len(out), _p(out))
    if rc != abi.OK:
        raise RuntimeError(f"port warm update failed: {rc}")
    return out


def ref_collide(a, pose_a, b, pose_b, speculative) -> np.ndarray:
    """The reference's nph_physics_collide for each pair (oracle/_ref)."""
    a = np.ascontiguousarray(a, abi.SHAPE_DTYPE)
    b = np.ascontiguousarray(b, abi.SHAPE_DTYPE)
    pa = np.ascontiguousarray(pose_a, abi.POSE_DTYPE)
    pb = np.ascontiguousarray(pose_b, abi.POSE_DTYPE)
    sp = np.ascontiguousarray(speculative, np.float32)
    out = np.zeros(len(a), abi.MANIFOLD_DTYPE)
    _ref_lib().nphref_collide_pairs(_p(a), _p(pa), _p(b), _p(pb), _p(sp), len(a), _p(out))
    return out
