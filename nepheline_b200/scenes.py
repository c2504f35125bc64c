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


# ---------------------------------------------------------------------------------------
# Batched worlds: box pyramids, sphere piles and capsule chains on hinges
# ---------------------------------------------------------------------------------------

_DENSITY = 1000.0


def _ground() -> np.ndarray:
    g = np.zeros(1, abi.BODY_DTYPE)
    g["rotation"][:, 3] = 1.0
    g["type"] = abi.BODY_STATIC
    g["center"][:, 1] = -1.0
    g["origin"][:, 1] = -1.0
    return g


class _WorldBuilder:
    """Bodies resting on a ground (the world's one fixed body, index n), with their manifolds
    and joints in insertion order; all shapes' contacts computed analytically at rest."""

    def __init__(self, rng):
        self.rng = rng
        self.centers: list = []
        self.mass: list = []
        self.inertia: list = []
        self.extent: list = []
        self.contacts: list = []
        self.joints: list = []
        self.x = 0.0  # next free x on the ground

    def body(self, center, mass, inertia_diag, extent) -> int:
        self.centers.append(center)
        self.mass.append(mass)
        self.inertia.append(inertia_diag)
        self.extent.append(extent)
        return len(self.centers) - 1

    GROUND = -1  # resolved to the fixed body's index at the end

    def pyramid(self, rows: int):
        """Unit boxes, row r holding rows - r boxes at 1.05 m spacing."""
        m = _DENSITY
        ids = {}
        for r in range(rows):
            cnt = rows - r
            for j in range(cnt):
                x = self.x + (j - (cnt - 1) / 2) * 1.05
                ids[(r, j)] = self.body((x, 0.5 + r - 0.005 * r, 0.0), m, (m / 6,) * 3, 0.866)
        half = 0.5
        for r in range(rows):
            cnt = rows - r
            for j in range(cnt):
                b = ids[(r, j)]
                if r == 0:
                    corners_b = [(-half, -half, -half), (half, -half, -half), (half, -half, half),
                                 (-half, -half, half)]
                    cx, cy, cz = self.centers[b]
                    # A is the ground (centre y = -1): anchors from its centre.
                    pa = [(cx + p[0], cy + p[1] + 1.0, cz + p[2]) for p in corners_b]
                    self.contacts.append((self.GROUND, b, (0, 1, 0), pa, corners_b, -0.005, 0.6))
                else:
                    for dj in (0, 1):
                        a = ids[(r - 1, j + dj)]
                        ax = self.centers[a][0]
                        bx = self.centers[b][0]
                        lo = max(ax, bx) - half + abs(ax - bx) * 0.0
                        x0, x1 = max(ax - half, bx - half), min(ax + half, bx + half)
                        dy = self.centers[b][1] - self.centers[a][1]
                        pts_world = [(x0, -half), (x1, -half), (x1, half), (x0, half)]
                        pa = [(px - ax, half, pz) for px, pz in pts_world]
                        pb = [(px - bx, half - dy, pz) for px, pz in pts_world]
                        self.contacts.append((a, b, (0, 1, 0), pa, pb, -0.005, 0.6))
        self.x += rows * 1.05 + 2.0

    def pile(self, columns: int, height: int):
        """Spheres of radius 0.5 stacked in columns (one-point manifolds)."""
        r = 0.5
        m = _DENSITY * 4.0 / 3.0 * np.pi * r ** 3
        for c in range(columns):
            x = self.x + c * 1.1
            prev = None
            for h in range(height):
                y = r + h * (2 * r - 0.004)
                b = self.body((x, y, 0.0), m, (0.4 * m * r * r,) * 3, r)
                if prev is None:
                    self.contacts.append((self.GROUND, b, (0, 1, 0), [(x, 1.0 + y - r, 0.0)],
                                          [(0.0, -r, 0.0)], -0.002, 0.5, 0.2))
                else:
                    self.contacts.append((prev, b, (0, 1, 0), [(0.0, r, 0.0)], [(0.0, -r, 0.0)],
                                          -0.004, 0.5, 0.2))
                prev = b
        self.x += columns * 1.1 + 2.0

    def chain(self, links: int):
        """Capsules (radius 0.25, 1 m long) lying along x on hinges about z at their ends."""
        rad, half_len = 0.25, 0.25
        m = _DENSITY * (np.pi * rad * rad * 2 * half_len + 4.0 / 3.0 * np.pi * rad ** 3)
        ix = m * (0.5 * rad * rad)
        iy = m * (0.25 * rad * rad + (2 * half_len + rad) ** 2 / 12.0)
        prev = None
        for k in range(links):
            x = self.x + 0.5 + k * 1.0
            b = self.body((x, rad - 0.002, 0.0), m, (ix, iy, iy), 0.5)
            cx, cy, cz = self.centers[b]
            pb = [(-half_len, -rad, 0.0), (half_len, -rad, 0.0)]
            pa = [(cx + p[0], cy + p[1] + 1.0, cz) for p in pb]
            self.contacts.append((self.GROUND, b, (0, 1, 0), pa, pb, -0.002, 0.7))
            if prev is not None:
                j = np.zeros(1, abi.JOINT_DTYPE)
                j["type"] = abi.JOINT_HINGE
                j["body_a"] = prev
                j["body_b"] = b
                j["frame_a_position"] = (0.5, 0.0, 0.0)
                j["frame_b_position"] = (-0.5, 0.0, 0.0)
                s = np.sqrt(0.5)
                j["frame_a_rotation"] = (0.0, -s, 0.0, s)  # frame X along world z
                j["frame_b_rotation"] = (0.0, -s, 0.0, s)
                self.joints.append(j)
            prev = b
        self.x += links * 1.0 + 2.0

    def scene(self) -> "SolverScene":
        n = len(self.centers)
        bodies = body_records(n)
        bodies["center"] = np.asarray(self.centers, np.float64)
        bodies["origin"] = bodies["center"]
        mass = np.asarray(self.mass, np.float32)
        inertia = np.zeros((n, 9), np.float32)
        diag = np.asarray(self.inertia, np.float32)
        inertia[:, 0], inertia[:, 4], inertia[:, 8] = diag[:, 0], diag[:, 1], diag[:, 2]
        set_mass(bodies, mass, inertia)
        bodies["max_extent"] = np.asarray(self.extent, np.float32)
        m = len(self.contacts)
        contacts = np.zeros(m, abi.CONTACT_DTYPE)
        if m:
            a = np.array([c[0] for c in self.contacts], np.int64)
            contacts["body_a"] = np.where(a == self.GROUND, n, a)
            contacts["body_b"] = [c[1] for c in self.contacts]
            contacts["normal"] = np.array([c[2] for c in self.contacts], np.float32)
            counts = np.array([len(c[3]) for c in self.contacts], np.uint32)
            contacts["point_count"] = counts
            contacts["friction"] = [c[6] for c in self.contacts]
            contacts["restitution"] = [c[7] if len(c) > 7 else 0.0 for c in self.contacts]
            pa = np.zeros((m, 4, 3), np.float32)
            pb = np.zeros((m, 4, 3), np.float32)
            sep = np.zeros((m, 4), np.float32)
            for i, c in enumerate(self.contacts):
                k = len(c[3])
                pa[i, :k] = c[3]
                pb[i, :k] = c[4]
                sep[i, :k] = c[5]
            pts = contacts["points"]
            pts["anchor_a"] = pa
            pts["anchor_b"] = pb
            pts["separation"] = sep
            pts["id"] = np.arange(4, dtype=np.uint32)[None, :]
        joints = np.concatenate(self.joints) if self.joints else np.zeros(0, abi.JOINT_DTYPE)
        return SolverScene(bodies=bodies, mass=mass, joints=joints, contacts=contacts,
                           fixed=_ground())


def mixed_world(bodies: int, seed: int) -> SolverScene:
    """One world of about `bodies` bodies: a seeded mix of box pyramids, sphere piles and
    capsule chains on hinges, resting on a ground."""
    rng = np.random.default_rng(seed)
    wb = _WorldBuilder(rng)
    share = rng.dirichlet((1.0, 1.0, 1.0))
    want = [int(round(bodies * s)) for s in share]
    while sum(want) < bodies:
        want[int(rng.integers(0, 3))] += 1
    # Pyramids: rows with rows (rows + 1) / 2 <= the share.
    left = want[0]
    while left >= 3:
        rows = int(min(20, max(2, np.floor((np.sqrt(8 * left + 1) - 1) / 2))))
        wb.pyramid(rows)
        left -= rows * (rows + 1) // 2
    left += want[1]
    while left >= 1:
        h = int(min(left, rng.integers(1, 8)))
        cols = max(1, min(left // h, int(rng.integers(1, 16))))
        wb.pile(cols, h)
        left -= cols * h
    left = want[2]
    while left >= 2:
        links = int(min(left, rng.integers(2, 40)))
        wb.chain(links)
        left -= links
    if not wb.centers:
        wb.pile(1, 1)
    return wb.scene()


def color_scenes(solver, scs: list) -> list:
    """Colours many disjoint scenes in one device call and lays each out as its own view:
    disjoint worlds colour as they would alone, and each world's list slots are its own."""
    offs = np.cumsum([0] + [len(s.bodies) + (0 if s.fixed is None else len(s.fixed)) for s in scs])
    aa, bb, dd, world, kind = [], [], [], [], []
    for w, s in enumerate(scs):
        a, b, d = s.constraint_arrays()
        aa.append(a + offs[w])
        bb.append(b + offs[w])
        dd.append(d)
        world.append(np.full(len(a), w, np.int64))
    a = np.concatenate(aa).astype(np.uint32)
    b = np.concatenate(bb).astype(np.uint32)
    d = np.concatenate(dd).astype(np.uint8)
    world = np.concatenate(world)
    color, _ = solver.graph_color(a, b, d, int(offs[-1]))
    # Slots per (world, kind, colour) in insertion order.
    key = (world * 2 + (d >> 2 & 1)) * abi.COLOR_SLOTS + color
    order = np.argsort(key, kind="stable")
    sorted_key = key[order]
    starts = np.r_[0, np.flatnonzero(np.diff(sorted_key)) + 1]
    rank = np.arange(len(key)) - np.repeat(starts, np.diff(np.r_[starts, len(key)]))
    slot = np.empty(len(key), np.uint32)
    slot[order] = rank
    views = []
    first = 0
    for s in scs:
        cnt = s.constraint_count
        views.append(s.to_view(color[first:first + cnt], slot[first:first + cnt]))
        first += cnt
    return views


def batched_sizes(count: int = 4096, seed: int = 0, min_bodies: int = 8,
                  max_bodies: int = 4096) -> np.ndarray:
    """Body counts of the batch's worlds, log-uniform in [min_bodies, max_bodies]."""
    rng = np.random.default_rng(seed)
    return np.round(np.exp(rng.uniform(np.log(min_bodies), np.log(max_bodies), count))).astype(int)


def batched_worlds(count: int = 4096, seed: int = 0, min_bodies: int = 8,
                   max_bodies: int = 4096, shard: int = 0, shards: int = 1) -> list:
    """`count` worlds with body counts log-uniform in [min_bodies, max_bodies]; with `shards`
    > 1 only the worlds i with i % shards == shard (each world is the same whichever shard
    builds it)."""
    sizes = batched_sizes(count, seed, min_bodies, max_bodies)
    return [mixed_world(int(sizes[i]), seed * 1_000_003 + i) for i in range(shard, count, shards)]


# ---- collapsing box piles (the learned warm start's workload) ---------------------------

def _rect_corners(c: np.ndarray, half: np.ndarray, yaw: np.ndarray) -> np.ndarray:
    """Corners (n, 4, 2) in the ground plane (x, z) of rectangles centred at c (n, 2) with
    half extents (n, 2) turned by yaw about the vertical axis, counter-clockwise."""
    s = np.array([[-1, -1], [1, -1], [1, 1], [-1, 1]], np.float64)
    local = s[None, :, :] * half[:, None, :]
    cy, sy = np.cos(yaw)[:, None], np.sin(yaw)[:, None]
    # A turn by yaw about +y maps (x, z) to (x cos + z sin, -x sin + z cos).
    x = local[:, :, 0] * cy + local[:, :, 1] * sy
    z = -local[:, :, 0] * sy + local[:, :, 1] * cy
    return np.stack([x, z], axis=2) + c[:, None, :]


def _inside(p: np.ndarray, rect: np.ndarray) -> np.ndarray:
    """Whether points p (n, k, 2) lie in the convex quads rect (n, 4, 2)."""
    ok = np.ones(p.shape[:2], bool)
    for e in range(4):
        a = rect[:, e][:, None, :]
        b = rect[:, (e + 1) % 4][:, None, :]
        cr = (b[..., 0] - a[..., 0]) * (p[..., 1] - a[..., 1]) - (b[..., 1] - a[..., 1]) * (p[..., 0] - a[..., 0])
        ok &= cr >= -1e-9
    return ok


def _overlap_points(ra: np.ndarray, rb: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Up to four points spanning the overlap of quads ra and rb (n, 4, 2): the overlap's
    vertices (corners of each inside the other, edge crossings), reduced as a manifold is: the
    vertex furthest along a fixed direction, the one furthest from it, then the furthest on
    each side of the line through both. Returns points (n, 4, 2) and their count (n,)."""
    n = len(ra)
    cand = [rb, ra]
    ok = [_inside(rb, ra), _inside(ra, rb)]
    for i in range(4):
        p0, p1 = ra[:, i], ra[:, (i + 1) % 4]
        for j in range(4):
            q0, q1 = rb[:, j], rb[:, (j + 1) % 4]
            d1, d2 = p1 - p0, q1 - q0
            den = d1[:, 0] * d2[:, 1] - d1[:, 1] * d2[:, 0]
            w = q0 - p0
            safe = np.where(np.abs(den) > 1e-12, den, 1.0)
            t = (w[:, 0] * d2[:, 1] - w[:, 1] * d2[:, 0]) / safe
            u = (w[:, 0] * d1[:, 1] - w[:, 1] * d1[:, 0]) / safe
            hit = (np.abs(den) > 1e-12) & (t >= 0) & (t <= 1) & (u >= 0) & (u <= 1)
            cand.append((p0 + t[:, None] * d1)[:, None, :])
            ok.append(hit[:, None])
    pts = np.concatenate(cand, axis=1)
    valid = np.concatenate(ok, axis=1)
    big = 1e30
    rows = np.arange(n)
    # 1: furthest along a fixed direction; 2: furthest from it.
    d = np.array([0.8, 0.6])
    i0 = np.argmax(np.where(valid, pts @ d, -big), axis=1)
    p0 = pts[rows, i0]
    dist = np.where(valid, np.sum((pts - p0[:, None, :]) ** 2, axis=2), -big)
    i1 = np.argmax(dist, axis=1)
    p1 = pts[rows, i1]
    e = p1 - p0
    area = e[:, None, 0] * (pts[..., 1] - p0[:, None, 1]) - e[:, None, 1] * (pts[..., 0] - p0[:, None, 0])
    i2 = np.argmax(np.where(valid, area, -big), axis=1)
    i3 = np.argmin(np.where(valid, area, big), axis=1)
    a2 = area[rows, i2]
    a3 = area[rows, i3]
    out = np.stack([p0, p1, pts[rows, i2], pts[rows, i3]], axis=1)
    tol = 1e-6
    has1 = dist[rows, i1] > tol
    has2 = a2 > tol
    has3 = a3 < -tol
    count = 1 + has1.astype(int) + (has1 & has2).astype(int) + (has1 & has3).astype(int)
    # Pack the points present to the front.
    order = np.stack([np.zeros(n, bool) | True, has1, has1 & has2, has1 & has3], axis=1)
    packed = np.zeros_like(out)
    for r in range(n):
        packed[r, : count[r]] = out[r][order[r]]
    return packed, count


def box_pile_world(boxes: int, seed: int, dt: float = 1.0 / 60.0, substeps: int = 4,
                   gravity: float = 9.81, max_height: int = 8,
                   new_share: float | None = None) -> SolverScene:
    """A collapsing box pile: `boxes` boxes (half extents uniform in 0.2-1.0 m, density
    1000 kg/m^3, friction 0.6, each turned by a seeded angle about the vertical) stacked in
    columns of 1-8 on a fixed ground, every box resting on the one below through the
    overlap of their faces (up to 4 points, penetration uniform in 0-1 cm). The pile is
    collapsing: every box moves a little, the columns' top boxes have just been dropped onto
    them (approach speed uniform in 0.5-3 m/s), and a seeded share of the other contacts has
    just formed. Contacts that persisted carry the impulses of the column's resting load
    (the weight above times g h, shared by the points); the new ones start at zero.
    `max_height` caps the columns (1: every box on the ground); `new_share` fixes the share of
    new contacts (default: seeded, uniform in 0.1-0.5, plus every dropped box's)."""
    rng = np.random.default_rng(seed)
    h = dt / substeps
    heights = []
    left = boxes
    while left > 0:
        k = int(min(left, rng.integers(1, max_height + 1)))
        heights.append(k)
        left -= k
    cols = len(heights)
    side = int(np.ceil(np.sqrt(cols)))
    half = rng.uniform(0.2, 1.0, (boxes, 3))
    yaw = rng.uniform(0.0, 2.0 * np.pi, boxes)
    pen = rng.uniform(0.0, 0.01, boxes)
    share = rng.uniform(0.1, 0.5) if new_share is None else new_share
    center = np.zeros((boxes, 3))
    below = np.full(boxes, -1, np.int64)  # the box each rests on (-1: the ground)
    top = np.zeros(boxes, bool)
    level = np.zeros(boxes, np.int64)
    i = 0
    for c, k in enumerate(heights):
        base = np.array([(c % side) * 3.4, (c // side) * 3.4])
        y = 0.0
        for lev in range(k):
            if lev == 0:
                xz = base
                y_bottom = 0.0 - pen[i]
            else:
                j = i - 1
                reach = 0.5 * min(half[j, 0], half[j, 2], half[i, 0], half[i, 2])
                xz = center[j, [0, 2]] + rng.uniform(-reach, reach, 2)
                y_bottom = y - pen[i]
                below[i] = j
            center[i] = (xz[0], y_bottom + half[i, 1], xz[1])
            y = center[i, 1] + half[i, 1]
            level[i] = lev
            i += 1
        top[i - 1] = k > 1
    mass = (_DENSITY * 8.0 * half[:, 0] * half[:, 1] * half[:, 2]).astype(F32)
    inertia = np.zeros((boxes, 9), F32)
    inertia[:, 0] = mass / 3.0 * (half[:, 1] ** 2 + half[:, 2] ** 2)
    inertia[:, 4] = mass / 3.0 * (half[:, 0] ** 2 + half[:, 2] ** 2)
    inertia[:, 8] = mass / 3.0 * (half[:, 0] ** 2 + half[:, 1] ** 2)
    bodies = body_records(boxes)
    set_mass(bodies, mass, inertia)
    bodies["center"] = center
    bodies["origin"] = center
    bodies["rotation"][:, 1] = np.sin(0.5 * yaw)
    bodies["rotation"][:, 3] = np.cos(0.5 * yaw)
    bodies["max_extent"] = np.linalg.norm(half, axis=1)
    v = rng.normal(0.0, 0.05, (boxes, 3))
    w = rng.normal(0.0, 0.1, (boxes, 3))
    v[top, 1] = -rng.uniform(0.5, 3.0, int(top.sum()))
    v[top, 0] += rng.normal(0.0, 0.3, int(top.sum()))
    v[top, 2] += rng.normal(0.0, 0.3, int(top.sum()))
    w[top] += rng.normal(0.0, 0.5, (int(top.sum()), 3))
    bodies["linear_velocity"] = v.astype(F32)
    bodies["angular_velocity"] = w.astype(F32)
    # Contacts: one per box with what is below it (A below, B the box), normal +y.
    fixed = _ground()
    ground = boxes  # the fixed body's index
    on_box = below >= 0
    lower = np.where(on_box, below, 0)
    rect_b = _rect_corners(center[:, [0, 2]], half[:, [0, 2]], yaw)
    rect_a = np.where(on_box[:, None, None],
                      _rect_corners(center[lower][:, [0, 2]], half[lower][:, [0, 2]], yaw[lower]),
                      _rect_corners(center[:, [0, 2]], half[:, [0, 2]] * 3.0, yaw))
    pts, count = _overlap_points(rect_a, rect_b)
    contacts = np.zeros(boxes, abi.CONTACT_DTYPE)
    contacts["body_a"] = np.where(on_box, below, ground)
    contacts["body_b"] = np.arange(boxes)
    contacts["point_count"] = count
    contacts["friction"] = 0.6
    contacts["normal"] = (0.0, 1.0, 0.0)
    a_center = np.where(on_box[:, None], center[lower], np.array([0.0, -1.0, 0.0]))
    y_plane = center[:, 1] - half[:, 1] + pen  # the top face of what is below
    # The load each contact carries at rest: the box and every box above it in its column.
    load = mass.astype(np.float64).copy()
    for b in range(boxes - 1, -1, -1):
        if below[b] >= 0:
            load[below[b]] += load[b]
    new = (top & (new_share is None)) | (rng.random(boxes) < share)
    for k in range(4):
        live = k < count
        p = np.stack([pts[:, k, 0], y_plane, pts[:, k, 1]], axis=1)
        cp = contacts["points"][:, k]
        cp["anchor_a"] = np.where(live[:, None], p - a_center, 0.0).astype(F32)
        cp["anchor_b"] = np.where(live[:, None], p - center, 0.0).astype(F32)
        cp["separation"] = np.where(live, -pen, 0.0).astype(F32)
        cp["id"] = k
        rest = load * gravity * h / np.maximum(count, 1)
        cp["normal_impulse"] = np.where(live & ~new, rest, 0.0).astype(F32)
    return SolverScene(bodies=bodies, mass=mass, joints=np.zeros(0, abi.JOINT_DTYPE),
                       contacts=contacts, fixed=fixed)


def merge_scenes(scs: list) -> SolverScene:
    """Disjoint worlds as one: bodies and contacts concatenated in order, each world's fixed
    bodies after all bodies (a body index below the total body count is an awake body, the
    fixed body k of world w is index total + w's first fixed + k)."""
    nb = [len(s.bodies) for s in scs]
    nf = [0 if s.fixed is None else len(s.fixed) for s in scs]
    total = int(sum(nb))
    boff = np.concatenate([[0], np.cumsum(nb)[:-1]]).astype(np.int64)
    foff = np.concatenate([[0], np.cumsum(nf)[:-1]]).astype(np.int64)

    def remap(idx, w):
        idx = idx.astype(np.int64)
        own = idx < nb[w]
        return np.where(own, idx + boff[w], idx - nb[w] + total + foff[w]).astype(np.uint32)

    cs, js = [], []
    for w, s in enumerate(scs):
        c = s.contacts.copy()
        c["body_a"] = remap(c["body_a"], w)
        c["body_b"] = remap(c["body_b"], w)
        cs.append(c)
        j = s.joints.copy()
        if len(j):
            j["body_a"] = remap(j["body_a"], w)
            j["body_b"] = remap(j["body_b"], w)
        js.append(j)
    fixed = [s.fixed for s in scs if s.fixed is not None and len(s.fixed)]
    return SolverScene(bodies=np.concatenate([s.bodies for s in scs]),
                       mass=np.concatenate([s.mass for s in scs]),
                       joints=np.concatenate(js) if js else np.zeros(0, abi.JOINT_DTYPE),
                       contacts=np.concatenate(cs),
                       fixed=np.concatenate(fixed) if fixed else None)


def box_pile_batch(worlds: int = 256, seed: int = 0, min_boxes: int = 500,
                   max_boxes: int = 5000) -> list:
    """`worlds` collapsing box piles with box counts uniform in [min_boxes, max_boxes]."""
    rng = np.random.default_rng(seed)
    sizes = rng.integers(min_boxes, max_boxes + 1, worlds)
    return [box_pile_world(int(n), seed * 1_000_003 + i) for i, n in enumerate(sizes)]


# ---------------------------------------------------------------------------------------
# Narrow-phase pairs
# ---------------------------------------------------------------------------------------

def _unit_quats(rng, n):
    q = rng.normal(size=(n, 4))
    return q / np.linalg.norm(q, axis=1, keepdims=True)


def _quat_mul(x, y):
    x1, y1, z1, w1 = x.T
    x2, y2, z2, w2 = y.T
    return np.stack([w1 * x2 + x1 * w2 + y1 * z2 - z1 * y2, w1 * y2 - x1 * z2 + y1 * w2 + z1 * x2,
                     w1 * z2 + x1 * y2 - y1 * x2 + z1 * w2, w1 * w2 - x1 * x2 - y1 * y2 - z1 * z2], 1)


def _quat_rotate(q, v):
    u, w = q[:, :3], q[:, 3:4]
    t = 2.0 * np.cross(u, v)
    return v + w * t + np.cross(u, t)


def narrow_pairs(n: int, seed: int = 0):
    """Pairs for the narrow phase in the proportions of the piles, pours and chains the solver
    steps, near or in contact, as the contact update hands them over (poses relative to the
    first body, speculative distance per pair): 60 % box on box (one resting on the other,
    tilted a little, sunk up to 2 cm or up to 3 cm apart), 15 % sphere on sphere, 10 % sphere on
    a box, 10 % capsule on a box, 5 % capsule on capsule. Returns (a, pose_a, b, pose_b,
    speculative) as SHAPE_DTYPE / POSE_DTYPE / float32 arrays."""
    rng = np.random.default_rng(seed)
    a = np.zeros(n, abi.SHAPE_DTYPE)
    b = np.zeros(n, abi.SHAPE_DTYPE)
    pa = np.zeros(n, abi.POSE_DTYPE)
    pb = np.zeros(n, abi.POSE_DTYPE)
    kind = rng.choice(5, size=n, p=[0.60, 0.15, 0.10, 0.10, 0.05])
    qa = _unit_quats(rng, n)
    half_a = rng.uniform(0.2, 1.0, (n, 3))
    half_b = rng.uniform(0.2, 1.0, (n, 3))
    radius_a = rng.uniform(0.1, 0.6, n)
    radius_b = rng.uniform(0.1, 0.6, n)
    core = rng.uniform(0.1, 0.8, n)
    gap = rng.uniform(-0.02, 0.03, n)
    tilt = rng.normal(0.0, 0.02, (n, 4))
    tilt[:, 3] = 1.0
    tilt /= np.linalg.norm(tilt, axis=1, keepdims=True)
    across = rng.uniform(-0.5, 0.5, (n, 2))
    off = np.zeros((n, 3))
    off[:, 0], off[:, 2] = across[:, 0], across[:, 1]
    qb = _quat_mul(qa, tilt)
    box_b = kind == 0
    a["type"][box_b], b["type"][box_b] = abi.SHAPE_BOX, abi.SHAPE_BOX
    a["dims"][box_b], b["dims"][box_b] = half_a[box_b], half_b[box_b]
    off[box_b, 1] = half_a[box_b, 1] + half_b[box_b, 1] + gap[box_b]
    sph = kind == 1
    a["type"][sph], b["type"][sph] = abi.SHAPE_SPHERE, abi.SHAPE_SPHERE
    a["dims"][sph, 0], b["dims"][sph, 0] = radius_a[sph], radius_b[sph]
    off[sph, 0] = off[sph, 2] = 0.0
    off[sph, 1] = radius_a[sph] + radius_b[sph] + gap[sph]
    sb = kind == 2
    a["type"][sb], b["type"][sb] = abi.SHAPE_BOX, abi.SHAPE_SPHERE
    a["dims"][sb], b["dims"][sb, 0] = half_a[sb], radius_b[sb]
    off[sb, 1] = half_a[sb, 1] + radius_b[sb] + gap[sb]
    cb = kind == 3
    a["type"][cb], b["type"][cb] = abi.SHAPE_BOX, abi.SHAPE_CAPSULE
    a["dims"][cb] = half_a[cb]
    b["dims"][cb, 0], b["dims"][cb, 1] = core[cb], radius_b[cb]
    # A capsule lying on the face: its core along the box's x, then tilted.
    lie = np.tile(np.array([0.0, 0.0, np.sqrt(0.5), np.sqrt(0.5)]), (int(cb.sum()), 1))
    qb[cb] = _quat_mul(qb[cb], lie)
    off[cb, 1] = half_a[cb, 1] + radius_b[cb] + gap[cb]
    cc = kind == 4
    a["type"][cc], b["type"][cc] = abi.SHAPE_CAPSULE, abi.SHAPE_CAPSULE
    a["dims"][cc, 0], a["dims"][cc, 1] = core[cc], radius_a[cc]
    b["dims"][cc, 0], b["dims"][cc, 1] = core[cc], radius_b[cc]
    qb[cc] = _unit_quats(rng, int(cc.sum()))
    off[cc, 1] = radius_a[cc] + radius_b[cc] + gap[cc]
    pa["rotation"] = qa.astype(np.float32)
    pb["rotation"] = qb.astype(np.float32)
    pb["position"] = _quat_rotate(qa, off).astype(np.float32)
    spec = np.full(n, 0.04, np.float32)
    return a, pa, b, pb, spec
