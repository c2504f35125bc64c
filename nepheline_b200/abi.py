"""Record layouts of include/nepheline_b200.h as numpy dtypes and ctypes structures.

The world view's arrays are numpy structured arrays with exactly the C structs' layout,
so a view built here is passed to the C ABI without copying. `check_layout` compares the
sizes with the ones the shared library reports.
"""
from __future__ import annotations

import ctypes

import numpy as np

NULL = 0xFFFFFFFF
MAX_POINTS = 4
COLORS = 24
DYNAMIC_COLORS = 20
OVERFLOW = 24
COLOR_SLOTS = 25

OK = 0
OUT_OF_MEMORY = 1
INVALID_ARGUMENT = 2
TOO_LARGE = 7
UNSUPPORTED = 8
DEVICE_LOST = 17
INVALID_STATE = 18
UNKNOWN = 19
RESULT_NAMES = {
    OK: "OK", OUT_OF_MEMORY: "OUT_OF_MEMORY", INVALID_ARGUMENT: "INVALID_ARGUMENT",
    TOO_LARGE: "TOO_LARGE", UNSUPPORTED: "UNSUPPORTED", DEVICE_LOST: "DEVICE_LOST", INVALID_STATE: "INVALID_STATE",
    UNKNOWN: "UNKNOWN",
}

BODY_STATIC = 0
BODY_KINEMATIC = 1
BODY_DYNAMIC = 2
BODY_ENABLE_SLEEP = 1 << 1
BODY_GYROSCOPIC = 1 << 2
BODY_BULLET = 1 << 5
CONTACT_HIT_EVENTS = 1 << 2
CONTACT_HIT = 1 << 4
CONSTRAINT_A_DYNAMIC = 1
CONSTRAINT_B_DYNAMIC = 2
CONSTRAINT_JOINT = 4
JOINT_BALL = 0
JOINT_HINGE = 1
JOINT_FIXED = 2
JOINT_SLIDER = 3
JOINT_DISTANCE = 4
JOINT_D6 = 5
AXIS_LOCKED, AXIS_LIMITED, AXIS_FREE = 0, 1, 2
D6_AXES = 6
ROW_LOCK, ROW_UPPER, ROW_MOTOR, ROW_SPRING = 0, 1, 2, 3
JOINT_BLOCK_ROTATION = 1 << 11
JOINT_BLOCK_SWING = 1 << 12
JOINT_BLOCK_POINT = 1 << 13
SOLVER_SOFT_STEP = 0
SOLVER_TGS = 1

BODY_DTYPE = np.dtype([
    ("center", "<f8", 3), ("origin", "<f8", 3), ("rotation", "<f4", 4),
    ("local_center", "<f4", 3), ("linear_velocity", "<f4", 3), ("angular_velocity", "<f4", 3),
    ("force", "<f4", 3), ("torque", "<f4", 3), ("inertia", "<f4", 9), ("inv_inertia", "<f4", 9),
    ("inv_mass", "<f4"), ("linear_damping", "<f4"), ("angular_damping", "<f4"),
    ("gravity_scale", "<f4"), ("sleep_threshold", "<f4"), ("sleep_time", "<f4"),
    ("max_extent", "<f4"), ("type", "<u4"), ("flags", "<u4"), ("locks", "<u4"), ("pad", "<u4"),
], align=True)

POINT_DTYPE = np.dtype([
    ("anchor_a", "<f4", 3), ("anchor_b", "<f4", 3), ("separation", "<f4"),
    ("normal_impulse", "<f4"), ("max_normal_impulse", "<f4"), ("tangent_impulse", "<f4", 3),
    ("relative_velocity", "<f4"), ("id", "<u4"),
], align=True)

CONTACT_DTYPE = np.dtype([
    ("body_a", "<u4"), ("body_b", "<u4"), ("flags", "<u4"), ("point_count", "<u4"),
    ("normal", "<f4", 3), ("friction", "<f4"), ("restitution", "<f4"), ("pad", "<u4", 3),
    ("points", POINT_DTYPE, MAX_POINTS),
], align=True)

# The settings union: ball, hinge, slider, distance and 6-DOF fields overlay the same 240 bytes.
_BALL = [("enable_swing_limit", "<u4", 0), ("swing_y", "<f4", 4), ("swing_z", "<f4", 8),
         ("enable_twist_limit", "<u4", 12), ("twist_lower", "<f4", 16),
         ("twist_upper", "<f4", 20), ("friction_torque", "<f4", 24)]
_HINGE = [("enable_limit", "<u4", 0), ("lower", "<f4", 4), ("upper", "<f4", 8),
          ("enable_motor", "<u4", 12), ("motor_speed", "<f4", 16),
          ("max_motor_torque", "<f4", 20), ("enable_spring", "<u4", 24),
          ("spring_hertz", "<f4", 28), ("spring_damping_ratio", "<f4", 32),
          ("spring_target", "<f4", 36)]
_SLIDER = [("enable_limit", "<u4", 0), ("lower", "<f4", 4), ("upper", "<f4", 8),
           ("enable_motor", "<u4", 12), ("motor_speed", "<f4", 16),
           ("max_motor_force", "<f4", 20), ("enable_spring", "<u4", 24),
           ("spring_hertz", "<f4", 28), ("spring_damping_ratio", "<f4", 32),
           ("spring_target", "<f4", 36)]
_DISTANCE = [("length", "<f4", 0), ("enable_limit", "<u4", 4), ("min_length", "<f4", 8),
             ("max_length", "<f4", 12), ("enable_spring", "<u4", 16), ("spring_hertz", "<f4", 20),
             ("spring_damping_ratio", "<f4", 24), ("enable_motor", "<u4", 28),
             ("motor_speed", "<f4", 32), ("max_motor_force", "<f4", 36)]
D6_AXIS_DTYPE = np.dtype([
    ("motion", "<u4"), ("lower", "<f4"), ("upper", "<f4"), ("enable_motor", "<u4"),
    ("motor_speed", "<f4"), ("max_motor_force", "<f4"), ("enable_spring", "<u4"),
    ("spring_hertz", "<f4"), ("spring_damping_ratio", "<f4"), ("spring_target", "<f4"),
])
_SETTINGS_BASE = 72
_IMPULSES = 312


def _joint_dtype() -> np.dtype:
    names, formats, offsets = [], [], []

    def add(name, fmt, off):
        names.append(name)
        formats.append(fmt)
        offsets.append(off)

    add("type", "<u4", 0)
    add("body_a", "<u4", 4)
    add("body_b", "<u4", 8)
    add("flags", "<u4", 12)
    add("frame_a_position", ("<f4", 3), 16)
    add("frame_a_rotation", ("<f4", 4), 28)
    add("frame_b_position", ("<f4", 3), 44)
    add("frame_b_rotation", ("<f4", 4), 56)
    add("settings", ("<u4", 60), _SETTINGS_BASE)
    for prefix, fields in (("ball_", _BALL), ("hinge_", _HINGE), ("slider_", _SLIDER),
                           ("distance_", _DISTANCE)):
        for name, fmt, off in fields:
            add(prefix + name, fmt, _SETTINGS_BASE + off)
    add("d6_axes", (D6_AXIS_DTYPE, D6_AXES), _SETTINGS_BASE)
    add("linear_impulse", ("<f4", 3), _IMPULSES)
    add("angular_impulse", ("<f4", 3), _IMPULSES + 12)
    add("friction_impulse", ("<f4", 3), _IMPULSES + 24)
    add("lower_impulse", "<f4", _IMPULSES + 36)
    add("upper_impulse", "<f4", _IMPULSES + 40)
    add("swing_impulse", "<f4", _IMPULSES + 44)
    add("motor_impulse", "<f4", _IMPULSES + 48)
    add("spring_impulse", "<f4", _IMPULSES + 52)
    add("axis_impulse", ("<f4", (D6_AXES, 4)), _IMPULSES + 56)
    return np.dtype({"names": names, "formats": formats, "offsets": offsets, "itemsize": 464})


JOINT_DTYPE = _joint_dtype()


class WorldParams(ctypes.Structure):
    """NphGpuWorldParams: the world settings the solver stage reads (world.h:104-143)."""

    _fields_ = [
        ("gravity", ctypes.c_float * 3), ("solver", ctypes.c_uint32),
        ("substeps", ctypes.c_uint32), ("contact_hertz", ctypes.c_float),
        ("contact_damping_ratio", ctypes.c_float), ("contact_push_max_velocity", ctypes.c_float),
        ("restitution_threshold", ctypes.c_float), ("max_linear_speed", ctypes.c_float),
        ("joint_hertz", ctypes.c_float), ("joint_damping_ratio", ctypes.c_float),
        ("enable_continuous", ctypes.c_uint32),
    ]

    @classmethod
    def default(cls, **overrides) -> "WorldParams":
        """The reference's defaults (world.c:85-104), continuous collision off."""
        p = cls()
        p.gravity[:] = (0.0, -9.81, 0.0)
        p.solver = SOLVER_SOFT_STEP
        p.substeps = 4
        p.contact_hertz = 0.0
        p.contact_damping_ratio = 10.0
        p.contact_push_max_velocity = 3.0
        p.restitution_threshold = 1.0
        p.max_linear_speed = 400.0
        p.joint_hertz = 0.0
        p.joint_damping_ratio = 2.0
        p.enable_continuous = 0
        for k, v in overrides.items():
            if k == "gravity":
                p.gravity[:] = v
            else:
                setattr(p, k, v)
        return p


class WorldView(ctypes.Structure):
    """NphGpuWorldView: pointers into numpy record arrays, updated in place by a solve."""

    _fields_ = [
        ("bodies", ctypes.c_void_p), ("body_count", ctypes.c_uint32),
        ("fixed_count", ctypes.c_uint32), ("fixed_bodies", ctypes.c_void_p),
        ("contacts", ctypes.c_void_p), ("contact_count", ctypes.c_uint32),
        ("joint_count", ctypes.c_uint32), ("joints", ctypes.c_void_p),
        ("contact_color_counts", ctypes.c_uint32 * COLOR_SLOTS),
        ("joint_color_counts", ctypes.c_uint32 * COLOR_SLOTS),
    ]


def _world_view_dtype() -> np.dtype:
    """A numpy record with NphGpuWorldView's layout, so that a batch's views fill one array."""
    names, formats, offsets = [], [], []
    for name, ctype in WorldView._fields_:
        names.append(name)
        offsets.append(getattr(WorldView, name).offset)
        if ctype is ctypes.c_void_p:
            formats.append(np.uint64)
        elif ctype is ctypes.c_uint32:
            formats.append(np.uint32)
        else:
            formats.append((np.uint32, (COLOR_SLOTS,)))
    return np.dtype({"names": names, "formats": formats, "offsets": offsets,
                     "itemsize": ctypes.sizeof(WorldView)})


WORLD_VIEW_DTYPE = _world_view_dtype()


class StepStats(ctypes.Structure):
    _fields_ = [
        ("colors_used", ctypes.c_uint32), ("overflow_contacts", ctypes.c_uint32),
        ("overflow_joints", ctypes.c_uint32), ("launches", ctypes.c_uint32),
        ("device_ms", ctypes.c_float), ("upload_ms", ctypes.c_float),
        ("download_ms", ctypes.c_float), ("error_word", ctypes.c_uint32),
    ]


class KernelTime(ctypes.Structure):
    """NphGpuKernelTime: one kind of kernel in a profiled step."""

    _fields_ = [
        ("name", ctypes.c_char * 32), ("launches", ctypes.c_uint32), ("pad", ctypes.c_uint32),
        ("units", ctypes.c_uint64), ("total_ms", ctypes.c_double),
        ("algorithmic_bytes", ctypes.c_double),
    ]


BATCH_SHARED_NONE, BATCH_SHARED_SMALL, BATCH_SHARED_LARGE = 0, 1, 2
BATCH_PERSISTENT, BATCH_MERGED = 0, 1
START_PLAIN, START_LEARNED, START_GATED = 0, 1, 2
# Pass configurations (csrc/solver.cu kPassConfigs) of the lean staged form, a colour a launch,
# and of the dependency-driven form, a pass a launch.
PASS_CONFIGS_LEAN = range(10, 15)
PASS_CONFIGS_FLOW = range(19, 22)

# The learned warm start's network and point slots (nepheline_b200.h).
MLP_INPUTS, MLP_HIDDEN, MLP_OUTPUTS = 16, 64, 3
MLP_PARAMS = (MLP_HIDDEN * MLP_INPUTS + MLP_HIDDEN + 2 * (MLP_HIDDEN * MLP_HIDDEN + MLP_HIDDEN)
              + MLP_OUTPUTS * MLP_HIDDEN + MLP_OUTPUTS)
POINT_NONE, POINT_WARM, POINT_COLD = 0, 1, 2


class ConvergeStats(ctypes.Structure):
    _fields_ = [("passes", ctypes.c_uint32), ("converged", ctypes.c_uint32),
                ("cold_points", ctypes.c_uint32), ("predicted_points", ctypes.c_uint32),
                ("initial_residual", ctypes.c_float), ("final_residual", ctypes.c_float),
                ("reference_residual", ctypes.c_float), ("ms", ctypes.c_float),
                ("fell_back", ctypes.c_uint32)]


class BatchTuning(ctypes.Structure):
    _fields_ = [("config", ctypes.c_uint32), ("threads", ctypes.c_uint32),
                ("shared_velocities", ctypes.c_uint32), ("items_per_thread", ctypes.c_uint32),
                ("packing", ctypes.c_uint32), ("ms_per_step", ctypes.c_float),
                ("persistent_ms_per_step", ctypes.c_float), ("merged_ms_per_step", ctypes.c_float)]


class BatchInfo(ctypes.Structure):
    _fields_ = [("worlds", ctypes.c_uint32), ("config", ctypes.c_uint32),
                ("bodies", ctypes.c_uint64), ("manifolds", ctypes.c_uint64),
                ("joints", ctypes.c_uint64), ("threads", ctypes.c_uint32),
                ("shared_velocities", ctypes.c_uint32), ("blocks_per_sm", ctypes.c_uint32),
                ("items_per_thread", ctypes.c_uint32), ("warp_worlds", ctypes.c_uint32),
                ("block_worlds", ctypes.c_uint32), ("packing", ctypes.c_uint32),
                ("launches_per_step", ctypes.c_uint32)]


class SolverDesc(ctypes.Structure):
    _fields_ = [
        ("device", ctypes.c_int32), ("stream", ctypes.c_void_p), ("use_graph", ctypes.c_uint32),
        ("body_capacity", ctypes.c_uint32), ("contact_capacity", ctypes.c_uint32),
        ("joint_capacity", ctypes.c_uint32),
    ]


def _ptr(a: np.ndarray | None) -> int | None:
    if a is None or len(a) == 0:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


class View:
    """A world view: the solver stage's records as numpy arrays plus the colour tables.

    bodies:  awake bodies (BODY_DTYPE), solver order
    fixed:   bodies without a solver slot (BODY_DTYPE), read only
    contacts: CONTACT_DTYPE in colour order (colours 0..23, then the overflow)
    joints:  JOINT_DTYPE in colour order
    contact_color_counts / joint_color_counts: 25 counts each
    """

    def __init__(self, bodies, fixed, contacts, joints, contact_color_counts,
                 joint_color_counts):
        self.bodies = np.ascontiguousarray(bodies, dtype=BODY_DTYPE)
        self.fixed = np.ascontiguousarray(fixed if fixed is not None else
                                          np.zeros(0, BODY_DTYPE), dtype=BODY_DTYPE)
        self.contacts = np.ascontiguousarray(contacts, dtype=CONTACT_DTYPE)
        self.joints = np.ascontiguousarray(joints if joints is not None else
                                           np.zeros(0, JOINT_DTYPE), dtype=JOINT_DTYPE)
        self.contact_color_counts = np.asarray(contact_color_counts, dtype=np.uint32).copy()
        self.joint_color_counts = np.asarray(joint_color_counts, dtype=np.uint32).copy()
        assert self.contact_color_counts.shape == (COLOR_SLOTS,)
        assert self.joint_color_counts.shape == (COLOR_SLOTS,)

    def copy(self) -> "View":
        return View(self.bodies.copy(), self.fixed.copy(), self.contacts.copy(),
                    self.joints.copy(), self.contact_color_counts, self.joint_color_counts)

    def c_view(self) -> WorldView:
        v = WorldView()
        v.bodies = _ptr(self.bodies)
        v.body_count = len(self.bodies)
        v.fixed_bodies = _ptr(self.fixed)
        v.fixed_count = len(self.fixed)
        v.contacts = _ptr(self.contacts)
        v.contact_count = len(self.contacts)
        v.joints = _ptr(self.joints)
        v.joint_count = len(self.joints)
        v.contact_color_counts[:] = [int(x) for x in self.contact_color_counts]
        v.joint_color_counts[:] = [int(x) for x in self.joint_color_counts]
        return v

    def addresses(self) -> tuple:
        """(address, count) of the bodies, fixed bodies, manifolds and joints: address 0 for
        an empty array. Kept while the view holds the same array objects."""
        key = (self.bodies, self.fixed, self.contacts, self.joints)
        cached = self.__dict__.get("_addresses")
        if cached is None or any(x is not y for x, y in zip(cached[0], key)):
            rec = []
            for arr in key:
                assert arr.flags["C_CONTIGUOUS"]
                rec += [arr.ctypes.data if len(arr) else 0, len(arr)]
            cached = (key, tuple(rec))
            self._addresses = cached
        return cached[1]

    @property
    def colors_used(self) -> int:
        return int(np.count_nonzero((self.contact_color_counts[:COLORS] > 0)
                                    | (self.joint_color_counts[:COLORS] > 0)))

    @property
    def manifold_points(self) -> int:
        return int(self.contacts["point_count"].sum())


# The packed drop-in's records (nph_gpu_phys_solve_packed): the fields the stage reads, and the
# fields it writes.
BODY_INPUT_DTYPE = np.dtype([
    ("center", "<f8", 3), ("rotation", "<f4", 4), ("local_center", "<f4", 3),
    ("linear_velocity", "<f4", 3), ("angular_velocity", "<f4", 3), ("force", "<f4", 3),
    ("torque", "<f4", 3), ("inertia", "<f4", 9), ("inv_inertia", "<f4", 9), ("inv_mass", "<f4"),
    ("linear_damping", "<f4"), ("angular_damping", "<f4"), ("gravity_scale", "<f4"),
    ("sleep_threshold", "<f4"), ("sleep_time", "<f4"), ("max_extent", "<f4"), ("type", "<u4"),
    ("flags", "<u4"), ("locks", "<u4"), ("pad", "<u4"),
], align=True)
POINT_INPUT_DTYPE = np.dtype([
    ("anchor_a", "<f4", 3), ("anchor_b", "<f4", 3), ("separation", "<f4"),
    ("normal_impulse", "<f4"), ("tangent_impulse", "<f4", 3), ("id", "<u4"),
])
CONTACT_INPUT_DTYPE = np.dtype([
    ("body_a", "<u4"), ("body_b", "<u4"), ("flags", "<u4"), ("point_count", "<u4"),
    ("normal", "<f4", 3), ("friction", "<f4"), ("restitution", "<f4"),
    ("points", POINT_INPUT_DTYPE, MAX_POINTS),
])
BODY_OUTPUT_DTYPE = np.dtype([
    ("center", "<f8", 3), ("origin", "<f8", 3), ("rotation", "<f4", 4),
    ("linear_velocity", "<f4", 3), ("angular_velocity", "<f4", 3), ("sleep_time", "<f4"),
    ("pad", "<u4"),
], align=True)
POINT_OUTPUT_DTYPE = np.dtype([
    ("normal_impulse", "<f4"), ("max_normal_impulse", "<f4"), ("tangent_impulse", "<f4", 3),
    ("relative_velocity", "<f4"),
])
CONTACT_OUTPUT_DTYPE = np.dtype([("flags", "<u4"), ("points", POINT_OUTPUT_DTYPE, MAX_POINTS)])
JOINT_OUTPUT_DTYPE = np.dtype([
    ("linear_impulse", "<f4", 3), ("angular_impulse", "<f4", 3), ("friction_impulse", "<f4", 3),
    ("lower_impulse", "<f4"), ("upper_impulse", "<f4"), ("swing_impulse", "<f4"),
    ("motor_impulse", "<f4"), ("spring_impulse", "<f4"), ("axis_impulse", "<f4", (D6_AXES, 4)),
    ("flags", "<u4"),
])


class PackedInput(ctypes.Structure):
    """NphGpuPackedInput."""

    _fields_ = [
        ("bodies", ctypes.c_void_p), ("body_count", ctypes.c_uint32),
        ("fixed_count", ctypes.c_uint32), ("fixed_bodies", ctypes.c_void_p),
        ("contacts", ctypes.c_void_p), ("contact_count", ctypes.c_uint32),
        ("joint_count", ctypes.c_uint32), ("joints", ctypes.c_void_p),
        ("contact_color_counts", ctypes.c_uint32 * COLOR_SLOTS),
        ("joint_color_counts", ctypes.c_uint32 * COLOR_SLOTS),
    ]


class PackedOutput(ctypes.Structure):
    """NphGpuPackedOutput."""

    _fields_ = [("bodies", ctypes.c_void_p), ("contacts", ctypes.c_void_p),
                ("joints", ctypes.c_void_p)]


class Packed:
    """A view's packed records: the stage's inputs gathered from the whole records, and the
    output arrays a packed solve fills (`alloc` makes the arrays, e.g. in page-locked memory)."""

    def __init__(self, view: "View", alloc=None):
        alloc = alloc or (lambda n, dt: np.zeros(n, dt))
        self.bodies = alloc(len(view.bodies), BODY_INPUT_DTYPE)
        self.contacts = alloc(len(view.contacts), CONTACT_INPUT_DTYPE)
        self.fixed = alloc(len(view.fixed), BODY_DTYPE)
        self.fixed[...] = view.fixed
        self.joints = alloc(len(view.joints), JOINT_DTYPE)
        self.counts = (view.contact_color_counts.copy(), view.joint_color_counts.copy())
        self.out_bodies = alloc(len(view.bodies), BODY_OUTPUT_DTYPE)
        self.out_contacts = alloc(len(view.contacts), CONTACT_OUTPUT_DTYPE)
        self.out_joints = alloc(len(view.joints), JOINT_OUTPUT_DTYPE)
        self.gather(view)

    def gather(self, view: "View") -> None:
        for f in BODY_INPUT_DTYPE.names:
            if f != "pad":
                self.bodies[f] = view.bodies[f]
        for f in ("body_a", "body_b", "flags", "point_count", "normal", "friction", "restitution"):
            self.contacts[f] = view.contacts[f]
        for f in POINT_INPUT_DTYPE.names:
            self.contacts["points"][f] = view.contacts["points"][f]
        self.joints[...] = view.joints

    def scatter(self, view: "View") -> None:
        """The outputs into the whole records, as a whole-record solve leaves them."""
        for f in ("center", "origin", "rotation", "linear_velocity", "angular_velocity", "sleep_time"):
            view.bodies[f] = self.out_bodies[f]
        view.bodies["force"] = 0.0
        view.bodies["torque"] = 0.0
        view.contacts["flags"] = self.out_contacts["flags"]
        for f in POINT_OUTPUT_DTYPE.names:
            view.contacts["points"][f] = self.out_contacts["points"][f]
        for f in JOINT_OUTPUT_DTYPE.names:
            view.joints[f] = self.out_joints[f]

    def c_input(self) -> PackedInput:
        c = PackedInput()
        c.bodies = _ptr(self.bodies)
        c.body_count = len(self.bodies)
        c.fixed_bodies = _ptr(self.fixed)
        c.fixed_count = len(self.fixed)
        c.contacts = _ptr(self.contacts)
        c.contact_count = len(self.contacts)
        c.joints = _ptr(self.joints)
        c.joint_count = len(self.joints)
        c.contact_color_counts[:] = [int(x) for x in self.counts[0]]
        c.joint_color_counts[:] = [int(x) for x in self.counts[1]]
        return c

    def c_output(self) -> PackedOutput:
        c = PackedOutput()
        c.bodies = _ptr(self.out_bodies)
        c.contacts = _ptr(self.out_contacts)
        c.joints = _ptr(self.out_joints)
        return c

    def input_bytes(self) -> int:
        return self.bodies.nbytes + self.contacts.nbytes + self.joints.nbytes + self.fixed.nbytes

    def output_bytes(self) -> int:
        return self.out_bodies.nbytes + self.out_contacts.nbytes + self.out_joints.nbytes


def layout_sizes() -> dict:
    return {"body": BODY_DTYPE.itemsize, "point": POINT_DTYPE.itemsize,
            "contact": CONTACT_DTYPE.itemsize, "joint": JOINT_DTYPE.itemsize,
            "params": ctypes.sizeof(WorldParams), "view": ctypes.sizeof(WorldView),
            "body_input": BODY_INPUT_DTYPE.itemsize, "contact_input": CONTACT_INPUT_DTYPE.itemsize,
            "body_output": BODY_OUTPUT_DTYPE.itemsize,
            "contact_output": CONTACT_OUTPUT_DTYPE.itemsize,
            "joint_output": JOINT_OUTPUT_DTYPE.itemsize,
            "packed_input": ctypes.sizeof(PackedInput), "packed_output": ctypes.sizeof(PackedOutput)}


def views_array(views: list) -> np.ndarray:
    """The NphGpuWorldView array of a batch's views (at least one record), filled a column at
    a time: a batch of thousands of worlds costs milliseconds, not a ctypes record each."""
    n = len(views)
    out = np.zeros(max(n, 1), WORLD_VIEW_DTYPE)
    if n == 0:
        return out
    rec = np.array([v.addresses() for v in views], dtype=np.uint64).reshape(n, 8)
    for k, name in enumerate(("bodies", "body_count", "fixed_bodies", "fixed_count", "contacts",
                              "contact_count", "joints", "joint_count")):
        out[name][:n] = rec[:, k]
    out["contact_color_counts"][:n] = np.stack([v.contact_color_counts for v in views])
    out["joint_color_counts"][:n] = np.stack([v.joint_color_counts for v in views])
    return out


def pack_views(views: list, alloc=None) -> list:
    """The same worlds with their records as consecutive slices of one array per record kind
    (bodies, fixed bodies, manifolds, joints), so that a batch copies each kind with one
    transfer. `alloc(nbytes)` gives the backing uint8 arrays (page-locked memory, say);
    the default is plain numpy memory. The returned views keep the arrays alive."""
    alloc = alloc or (lambda nbytes: np.empty(nbytes, np.uint8))

    def packed(field, dtype):
        total = sum(len(getattr(v, field)) for v in views)
        raw = alloc(max(total, 1) * dtype.itemsize)
        arr = raw[: total * dtype.itemsize].view(dtype)
        out, first = [], 0
        for v in views:
            src = getattr(v, field)
            arr[first:first + len(src)] = src
            out.append(arr[first:first + len(src)])
            first += len(src)
        return out, raw

    bodies, rb = packed("bodies", BODY_DTYPE)
    fixed, rf = packed("fixed", BODY_DTYPE)
    contacts, rc = packed("contacts", CONTACT_DTYPE)
    joints, rj = packed("joints", JOINT_DTYPE)
    out = []
    for i, v in enumerate(views):
        p = View(bodies[i], fixed[i], contacts[i], joints[i], v.contact_color_counts,
                 v.joint_color_counts)
        p._keep = (rb, rf, rc, rj)
        out.append(p)
    return out


# The narrow phase's records (nepheline_b200.h).
SHAPE_SPHERE, SHAPE_CAPSULE, SHAPE_BOX = 0, 1, 2
SHAPE_DTYPE = np.dtype([("type", "<u4"), ("dims", "<f4", 3)], align=True)
HIT_EVENT_DTYPE = np.dtype([("contact", "<u4"), ("point", "<u4"), ("approach_speed", "<f4"),
                            ("world", "<u4")])


def hit_points(view: "View", events: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """The world points and normals of hit events, from the view the step wrote back: body A's
    centre plus the point's anchor_a, each component a double sum (nph_dvec3_add_vec3), and the
    manifold's normal."""
    c = view.contacts[events["contact"]]
    a = c["body_a"].astype(np.int64)
    n = len(view.bodies)
    centers = np.empty((len(c), 3), np.float64)
    own = a < n
    centers[own] = view.bodies["center"][a[own]]
    centers[~own] = view.fixed["center"][a[~own] - n]
    anchor = c["points"]["anchor_a"][np.arange(len(c)), events["point"]]
    return centers + anchor.astype(np.float64), c["normal"].copy()


POSE_DTYPE = np.dtype([("position", "<f4", 3), ("rotation", "<f4", 4)], align=True)
MANIFOLD_POINT_DTYPE = np.dtype([("point", "<f4", 3), ("separation", "<f4"), ("id", "<u4")],
                                align=True)
MANIFOLD_DTYPE = np.dtype([("normal", "<f4", 3), ("point_count", "<u4"),
                           ("points", MANIFOLD_POINT_DTYPE, MAX_POINTS)], align=True)
