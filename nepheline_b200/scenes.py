"""Seeded synthetic workloads for the solver stage, as world-view records.

`lattice_graph` is the synthetic constraint graph the solver is benchmarked on (a lattice
of unit boxes at 1 m spacing, one 4-point manifold per neighbour pair, an extra 10 % of the
pairs jointed; 128 x 128 x 64 is the 1,048,576-body configuration), at any size. It returns the bodies, and the
constraints in their insertion order (joints, then contacts, each in lexicographic pair
order: x-axis pairs, then y, then z), with body fields that are body indices. The same
scene feeds the reference solver (bodies created and manifolds injected in that order)
and the device solver (coloured, then laid out in colour order by `to_view`).

Mass properties follow the reference's arithmetic for a body whose mass is set
explicitly: inv_mass = 1 / mass, and the inverse inertia by the adjugate
(engine/math/src/mat.c:14-29), in FP32, so a view built here equals the one the
reference exports for the same scene.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import abi

F32 = np.float32


def mat3_inverse_f32(m: np.ndarray) -> np.ndarray:
    """nph_mat3_inverse (mat.c:14-29) in FP32 for (n, 9) column-major matrices."""
    m = m.astype(F32).reshape(-1, 3, 3)  # [n, col, row]
    c0, c1, c2 = m[:, 0], m[:, 1], m[:, 2]

    def cross(a, b):
        return np.stack([a[:, 1] * b[:, 2] - a[:, 2] * b[:, 1],
                         a[:, 2] * b[:, 0] - a[:, 0] * b[:, 2],
                         a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0]], axis=1)

    r0, r1, r2 = cross(c1, c2), cross(c2, c0), cross(c0, c1)
    det = (c0[:, 0] * r0[:, 0] + c0[:, 1] * r0[:, 1]) + c0[:, 2] * r0[:, 2]
    inv = F32(1.0) / det
    rows = np.stack([r0 * inv[:, None], r1 * inv[:, None], r2 * inv[:, None]], axis=1)  # [n,row,k]
    return np.ascontiguousarray(np.transpose(rows, (0, 2, 1))).reshape(-1, 9).astype(F32)


def body_records(n: int) -> np.ndarray:
    """Dynamic bodies at rest with the reference's body defaults (body.c:12-24)."""
    b = np.zeros(n, abi.BODY_DTYPE)
    b["rotation"][:, 3] = 1.0
    b["gravity_scale"] = 1.0
    b["sleep_threshold"] = 0.05
    b["type"] = abi.BODY_DYNAMIC
    # Awake (bit 0), sleep enabled, gyroscopic, mass set explicitly (bit 3): the flags the
    # reference's body has after nph_physics_body_set_mass_data (world_internal.h:59-69).
    b["flags"] = 1 | abi.BODY_ENABLE_SLEEP | abi.BODY_GYROSCOPIC | (1 << 3)
    return b


def set_mass(b: np.ndarray, mass: np.ndarray, inertia: np.ndarray) -> None:
    """The explicit-mass branch of phys_body_update_mass (body.c:391-445)."""
    mass = mass.astype(F32)
    b["inv_mass"] = F32(1.0) / mass
    b["inertia"] = inertia.astype(F32)
    b["inv_inertia"] = mat3_inverse_f32(inertia)


def _tilted(axis: int, max_deg: float, rng: np.random.Generator, count: int) -> np.ndarray:
    """Unit vectors within `max_deg` of a lattice axis, as FP32."""
    e = np.zeros((count, 3))
    e[:, axis] = 1.0
    u = np.zeros((count, 3))
    u[:, (axis + 1) % 3] = 1.0
    v = np.zeros((count, 3))
    v[:, (axis + 2) % 3] = 1.0
    phi = rng.uniform(0.0, 2.0 * np.pi, count)
    theta = np.radians(rng.uniform(0.0, max_deg, count))
    d = np.cos(phi)[:, None] * u + np.sin(phi)[:, None] * v
    n = np.cos(theta)[:, None] * e + np.sin(theta)[:, None] * d
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    return n.astype(F32)


@dataclass
class SolverScene:
    """Bodies and constraints in insertion order; body fields are body indices."""

    bodies: np.ndarray       # BODY_DTYPE, all awake, in index order
    mass: np.ndarray         # float32 per body (the reference's explicit mass)
    joints: np.ndarray       # JOINT_DTYPE, insertion order
    contacts: np.ndarray     # CONTACT_DTYPE, insertion order (after the joints)
    fixed: np.ndarray | None = None  # BODY_DTYPE bodies without a solver slot

    @property
    def constraint_count(self) -> int:
        return len(self.joints) + len(self.contacts)

    def constraint_arrays(self) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        """Body indices and dynamic bits of every constraint, joints first (insertion order)."""
        a = np.concatenate([self.joints["body_a"], self.contacts["body_a"]]).astype(np.uint32)
        b = np.concatenate([self.joints["body_b"], self.contacts["body_b"]]).astype(np.uint32)
        nb = len(self.bodies)
        types = self.bodies["type"]
        if self.fixed is not None and len(self.fixed):
            types = np.concatenate([types, self.fixed["type"]])
        dyn = ((types[a] == abi.BODY_DYNAMIC).astype(np.uint8)
               | ((types[b] == abi.BODY_DYNAMIC).astype(np.uint8) << 1))
        dyn[:len(self.joints)] |= abi.CONSTRAINT_JOINT
        del nb
        return a, b, dyn

    def to_view(self, color: np.ndarray, slot: np.ndarray) -> abi.View:
        """Lays the constraints out in colour order (colours 0..23, then the overflow), each
        colour's list in slot order, from a colouring of the insertion order."""
        nj = len(self.joints)
        jc, js = color[:nj], slot[:nj]
        cc, cs = color[nj:], slot[nj:]
        jcounts = np.bincount(jc, minlength=abi.COLOR_SLOTS).astype(np.uint32)
        ccounts = np.bincount(cc, minlength=abi.COLOR_SLOTS).astype(np.uint32)
        jfirst = np.concatenate([[0], np.cumsum(jcounts, dtype=np.int64)[:-1]]).astype(np.int64)
        cfirst = np.concatenate([[0], np.cumsum(ccounts, dtype=np.int64)[:-1]]).astype(np.int64)
        joints = np.empty_like(self.joints)
        joints[jfirst[jc] + js] = self.joints
        contacts = np.empty_like(self.contacts)
        contacts[cfirst[cc] + cs] = self.contacts
        return abi.View(self.bodies.copy(), self.fixed, contacts, joints, ccounts, jcounts)


def lattice_graph(edge: int | tuple[int, int, int] = 128, seed: int = 0,
                  joint_fraction: float = 0.1, max_tilt_deg: float = 5.0,
                  max_penetration: float = 0.02) -> SolverScene:
    """The synthetic constraint graph: a lattice of unit boxes at 1 m spacing, `edge` bodies
    along each axis (or (nx, ny, nz)).

    Mass log-uniform in 0.1-100 kg, unit-box inertia scaled by mass (m/6, isotropic). Each
    6-neighbour pair carries one 4-point manifold: normal the lattice axis tilted by up to
    `max_tilt_deg`, points at the shared face's corners (+-0.25 m), penetration uniform in
    0-`max_penetration` per point, friction uniform in 0.2-1.0, restitution 0. An extra
    `joint_fraction` of the pairs carry a ball or a hinge joint (half each) at the face
    centre. Bodies start at rest with zero warm-start impulses.
    """
    rng = np.random.default_rng(seed)
    nx, ny, nz = (edge, edge, edge) if isinstance(edge, int) else tuple(edge)
    nb = nx * ny * nz
    idx = np.arange(nb, dtype=np.int64)
    x = idx % nx
    y = (idx // nx) % ny
    z = idx // (nx * ny)
    bodies = body_records(nb)
    bodies["center"][:, 0] = x
    bodies["center"][:, 1] = y
    bodies["center"][:, 2] = z
    bodies["origin"] = bodies["center"]
    mass = np.exp(rng.uniform(np.log(0.1), np.log(100.0), nb)).astype(F32)
    inertia = np.zeros((nb, 9), F32)
    diag = mass * F32(1.0 / 6.0)
    inertia[:, 0] = diag
    inertia[:, 4] = diag
    inertia[:, 8] = diag
    set_mass(bodies, mass, inertia)

    pairs_a, pairs_b, axes = [], [], []
    coords = (x, y, z)
    dims = (nx, ny, nz)
    strides = (1, nx, nx * ny)
    for axis in range(3):
        sel = idx[coords[axis] < dims[axis] - 1]
        pairs_a.append(sel)
        pairs_b.append(sel + strides[axis])
        axes.append(np.full(len(sel), axis, np.int64))
    pa = np.concatenate(pairs_a)
    pb = np.concatenate(pairs_b)
    pax = np.concatenate(axes)
    npairs = len(pa)

    contacts = np.zeros(npairs, abi.CONTACT_DTYPE)
    contacts["body_a"] = pa
    contacts["body_b"] = pb
    contacts["point_count"] = 4
    contacts["friction"] = rng.uniform(0.2, 1.0, npairs).astype(F32)
    normals = np.zeros((npairs, 3), F32)
    for axis in range(3):
        m = pax == axis
        normals[m] = _tilted(axis, max_tilt_deg, rng, int(m.sum()))
    contacts["normal"] = normals
    pen = rng.uniform(0.0, max_penetration, (npairs, 4)).astype(F32)
    e = np.eye(3, dtype=F32)
    corners = np.array([[-1, -1], [1, -1], [1, 1], [-1, 1]], F32) * F32(0.25)
    anchor_a = np.zeros((npairs, 4, 3), F32)
    anchor_b = np.zeros((npairs, 4, 3), F32)
    for axis in range(3):
        m = pax == axis
        ea, eu, ev = e[axis], e[(axis + 1) % 3], e[(axis + 2) % 3]
        for k in range(4):
            pt = F32(0.5) * ea + corners[k, 0] * eu + corners[k, 1] * ev
            anchor_a[m, k] = pt
            anchor_b[m, k] = pt - ea
    pts = contacts["points"]
    pts["anchor_a"] = anchor_a
    pts["anchor_b"] = anchor_b
    pts["separation"] = -pen
    pts["id"] = np.arange(4, dtype=np.uint32)[None, :]

    jsel = np.sort(rng.choice(npairs, int(round(joint_fraction * npairs)), replace=False))
    joints = np.zeros(len(jsel), abi.JOINT_DTYPE)
    joints["type"] = np.where(rng.random(len(jsel)) < 0.5, abi.JOINT_BALL, abi.JOINT_HINGE)
    joints["body_a"] = pa[jsel]
    joints["body_b"] = pb[jsel]
    half = np.zeros((len(jsel), 3), F32)
    half[np.arange(len(jsel)), pax[jsel]] = 0.5
    joints["frame_a_position"] = half
    joints["frame_b_position"] = -half
    joints["frame_a_rotation"][:, 3] = 1.0
    joints["frame_b_rotation"][:, 3] = 1.0
    return SolverScene(bodies=bodies, mass=mass, joints=joints, contacts=contacts)


def host_color(scene: SolverScene) -> tuple[np.ndarray, np.ndarray]:
    """Sequential first-fit colouring of the scene's insertion order on the host, with the
    same rule as the device colouring (graph_pick_color, island.c:34-56). Vectorised over
    nothing: used for small scenes and as a fallback-free cross-check in tests."""
    a, b, dyn = scene.constraint_arrays()
    nbits = len(scene.bodies) + (0 if scene.fixed is None else len(scene.fixed))
    used = np.zeros((abi.COLORS, nbits), bool)
    color = np.zeros(len(a), np.uint32)
    slot = np.zeros(len(a), np.uint32)
    lens = np.zeros((2, abi.COLOR_SLOTS), np.uint32)  # contact lists, joint lists
    for i in range(len(a)):
        da, db = dyn[i] & 1, dyn[i] & 2
        c = abi.OVERFLOW
        if da and db:
            for k in range(abi.DYNAMIC_COLORS):
                if not used[k, a[i]] and not used[k, b[i]]:
                    c = k
                    break
        else:
            body = a[i] if da else b[i]
            for k in range(1, abi.COLORS):
                if not used[k, body]:
                    c = k
                    break
        if c != abi.OVERFLOW:
            if da:
                used[c, a[i]] = True
            if db:
                used[c, b[i]] = True
        kind = 1 if dyn[i] & abi.CONSTRAINT_JOINT else 0
        color[i] = c
        slot[i] = lens[kind, c]
        lens[kind, c] += 1
    return color, slot
