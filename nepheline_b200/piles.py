"""Collapsing box piles stepped by the library's own stages: the learned warm start's workload.

Worlds of boxes (half extents uniform in 0.2-1.0 m, density 1000 kg/m^3, friction 0.6,
restitution 0) dropped from seeded random orientations in layers above a ground slab; the
worlds lie far apart and never touch. Every step runs, for all worlds at once:

  broad phase     nph_gpu_broad_phase over the boxes' bounds grown by the AABB margin (0.1 m,
                  the reference's proxy fattening, types.h:56), and each box against its world's
                  ground when its grown bounds reach the ground's top;
  narrow phase    nph_gpu_collide on every pair, poses relative to body A's centre
                  (phys_contact_update, contact.c:525-532) and the pair's speculative distance
                  (phys_pair_speculative, contact.c:485-511);
  contact update  the manifolds with points become contact records (anchor_a the point,
                  anchor_b the point less B's centre from A's, contact.c:540-552; friction
                  sqrt(f_a f_b) and restitution max(e_a, e_b), phys_pair_surface,
                  world_internal.h:181-194), warm-started from last step's record of the same
                  pair on the device (nph_gpu_warm_start_contacts: by feature id, then by
                  place); a pair new this step starts cold (contact.c:547-565);
  colouring       nph_gpu_graph_color over the contacts in their order: pairs that persisted in
                  last step's order, then the new pairs;
  solve           nph_gpu_phys_solve, the plain start or a network attached to the solver.

The reference's broad phase keeps pairs in AABB trees with fattened proxies and its constraint
graph colours incrementally (island.c:77-104); these piles are the library's own simulation
of the same scenes, not a copy of the reference's trajectory.
"""
from __future__ import annotations

import numpy as np

from . import abi, scenes
from .solver import broad_phase, collide, warm_start_contacts

F32 = np.float32
LINEAR_SLOP = 0.005          # NPH_PHYSICS_LINEAR_SLOP, types.h:38
SPECULATIVE = 4.0 * LINEAR_SLOP  # NPH_PHYSICS_SPECULATIVE_DISTANCE, types.h:52
AABB_MARGIN = 0.1            # NPH_PHYSICS_AABB_MARGIN, types.h:56
FRICTION = 0.6               # the shape default (shape.h:83)
GROUND_HALF = (60.0, 1.0, 60.0)
WORLD_SPACING = 300.0        # between world centres: worlds never meet
DROP_SPACING = 3.7           # between drop sites: no two boxes start in contact
CELL = 2.0 * (float(np.sqrt(3.0)) + AABB_MARGIN) + 0.01  # no grown box is wider


def _rotations(q: np.ndarray) -> np.ndarray:
    """Rotation matrices (n, 3, 3) of unit quaternions (x, y, z, w), in double."""
    x, y, z, w = (q[:, i].astype(np.float64) for i in range(4))
    return np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], 1),
        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], 1),
        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], 1)], 1)


def pile_sizes(worlds: int, seed: int, min_boxes: int = 500, max_boxes: int = 5000) -> np.ndarray:
    return np.random.default_rng(seed).integers(min_boxes, max_boxes + 1, worlds)


class Piles:
    """`sizes[w]` boxes per world, dropped; stepped by `step`."""

    def __init__(self, sizes, seed: int):
        rng = np.random.default_rng(seed)
        sizes = np.asarray(sizes, np.int64)
        self.worlds = len(sizes)
        n = int(sizes.sum())
        self.n = n
        self.world = np.repeat(np.arange(self.worlds), sizes).astype(np.uint32)
        side = int(np.ceil(np.sqrt(self.worlds)))
        origin = np.stack([(np.arange(self.worlds) % side) * WORLD_SPACING, np.zeros(self.worlds),
                           (np.arange(self.worlds) // side) * WORLD_SPACING], 1)
        self.half = rng.uniform(0.2, 1.0, (n, 3))
        centers = np.zeros((n, 3))
        first = 0
        for w, k in enumerate(sizes):
            per_layer = int(np.ceil(np.sqrt(k / 6.0))) ** 2  # about six layers
            row = int(np.sqrt(per_layer))
            i = np.arange(k)
            layer, site = i // per_layer, i % per_layer
            xz = (np.stack([site % row, site // row], 1) - (row - 1) / 2.0) * DROP_SPACING
            centers[first:first + k, 0] = origin[w, 0] + xz[:, 0] + rng.uniform(-0.2, 0.2, k)
            centers[first:first + k, 1] = 2.0 + DROP_SPACING * layer
            centers[first:first + k, 2] = origin[w, 2] + xz[:, 1] + rng.uniform(-0.2, 0.2, k)
            first += k
        q = rng.normal(size=(n, 4))
        q /= np.linalg.norm(q, axis=1, keepdims=True)
        mass = (1000.0 * 8.0 * self.half.prod(axis=1)).astype(F32)
        inertia = np.zeros((n, 9), F32)
        h2 = self.half ** 2
        inertia[:, 0] = mass / 3.0 * (h2[:, 1] + h2[:, 2])
        inertia[:, 4] = mass / 3.0 * (h2[:, 0] + h2[:, 2])
        inertia[:, 8] = mass / 3.0 * (h2[:, 0] + h2[:, 1])
        b = scenes.body_records(n)
        scenes.set_mass(b, mass, inertia)
        b["center"] = centers
        b["origin"] = centers
        b["rotation"] = q.astype(F32)
        b["max_extent"] = np.linalg.norm(self.half, axis=1).astype(F32)
        b["flags"] &= ~np.uint32(abi.BODY_ENABLE_SLEEP)  # the piles run with sleep off
        self.bodies = b
        g = np.zeros(self.worlds, abi.BODY_DTYPE)
        g["rotation"][:, 3] = 1.0
        g["type"] = abi.BODY_STATIC
        g["center"] = origin + np.array([0.0, -GROUND_HALF[1], 0.0])
        g["origin"] = g["center"]
        self.grounds = g
        self.shape_half = self.half.astype(F32)
        # Last step's contacts: pair keys (a << 32 | b, view indices) in insertion order, and the
        # records the solve left them.
        self.keys = np.zeros(0, np.uint64)
        self.records = np.zeros(0, abi.CONTACT_DTYPE)
        self.steps = 0

    # ---- the stages --------------------------------------------------------------------

    def _pairs(self):
        """(a, b) view indices of the pairs to collide: box pairs from the broad phase, then each
        box with its world's ground."""
        b = self.bodies
        rot = _rotations(b["rotation"])
        ext = np.einsum("nij,nj->ni", np.abs(rot), self.half) + AABB_MARGIN
        lo = b["center"] - ext
        hi = b["center"] + ext
        pa, pb = broad_phase(lo.astype(F32), hi.astype(F32), self.world, CELL)
        on_ground = np.flatnonzero(lo[:, 1] <= AABB_MARGIN)
        ga = on_ground.astype(np.uint32)
        gb = (self.n + self.world[on_ground]).astype(np.uint32)
        return np.concatenate([pa, ga]), np.concatenate([pb, gb])

    def _speculative(self, a, b, dt):
        """phys_pair_speculative (contact.c:485-511), per pair."""
        allb = np.concatenate([self.bodies, self.grounds])
        va, vb = allb["linear_velocity"][a].astype(F32), allb["linear_velocity"][b].astype(F32)
        wa, wb = allb["angular_velocity"][a].astype(F32), allb["angular_velocity"][b].astype(F32)
        ea, eb = allb["max_extent"][a].astype(F32), allb["max_extent"][b].astype(F32)
        dv = vb - va
        room = F32((SPECULATIVE - LINEAR_SLOP) / max(dt, 1e-9))
        slow = F32(3.0) * ((dv * dv).sum(1) + (wa * wa).sum(1) * ea * ea + (wb * wb).sum(1) * eb * eb) <= room * room
        closing = F32(dt) * (np.linalg.norm(dv, axis=1) + np.linalg.norm(wa, axis=1) * ea
                             + np.linalg.norm(wb, axis=1) * eb)
        reach = closing + F32(LINEAR_SLOP)
        out = np.where(slow | ~(reach > SPECULATIVE), F32(SPECULATIVE), np.minimum(reach, F32(AABB_MARGIN)))
        return out.astype(F32)

    def _manifolds(self, a, b, dt):
        allb = np.concatenate([self.bodies, self.grounds])
        n = len(a)
        sa = np.zeros(n, abi.SHAPE_DTYPE)
        sb = np.zeros(n, abi.SHAPE_DTYPE)
        sa["type"] = abi.SHAPE_BOX
        sb["type"] = abi.SHAPE_BOX
        sa["dims"] = self.shape_half[a]
        ground = b >= self.n
        dims_b = np.empty((n, 3), F32)
        dims_b[~ground] = self.shape_half[b[~ground]]
        dims_b[ground] = GROUND_HALF
        sb["dims"] = dims_b
        pa = np.zeros(n, abi.POSE_DTYPE)
        pb = np.zeros(n, abi.POSE_DTYPE)
        pa["rotation"] = allb["rotation"][a]
        pb["rotation"] = allb["rotation"][b]
        ab = (allb["center"][b] - allb["center"][a]).astype(F32)  # nph_dvec3_relative
        pb["position"] = ab
        m = collide(sa, pa, sb, pb, self._speculative(a, b, dt))
        return m, ab

    def update_contacts(self, dt: float):
        """This step's contacts in insertion order (pairs that persisted first, in last step's
        order), warm-started; returns (records, keys)."""
        a, b = self._pairs()
        m, ab = self._manifolds(a, b, dt)
        touching = m["point_count"] > 0
        a, b, m, ab = a[touching], b[touching], m[touching], ab[touching]
        keys = (a.astype(np.uint64) << np.uint64(32)) | b.astype(np.uint64)
        fresh = np.zeros(len(a), abi.CONTACT_DTYPE)
        fresh["body_a"] = a
        fresh["body_b"] = b
        fresh["point_count"] = m["point_count"]
        fresh["normal"] = m["normal"]
        fresh["friction"] = np.sqrt(F32(FRICTION) * F32(FRICTION))
        fresh["restitution"] = 0.0
        pts = fresh["points"]
        pts["anchor_a"] = m["points"]["point"]
        pts["anchor_b"] = m["points"]["point"] - ab[:, None, :]
        live = np.arange(abi.MAX_POINTS)[None, :] < m["point_count"][:, None]
        pts["anchor_b"] = np.where(live[..., None], pts["anchor_b"], 0.0)
        pts["separation"] = m["points"]["separation"]
        pts["id"] = m["points"]["id"]
        # Last step's record of each pair (a new pair: its bodies, no points, flags clear).
        old = np.zeros(len(a), abi.CONTACT_DTYPE)
        old["body_a"] = a
        old["body_b"] = b
        if len(self.keys):
            order = np.argsort(self.keys, kind="stable")
            at = np.searchsorted(self.keys[order], keys)
            at = np.minimum(at, len(self.keys) - 1)
            found = self.keys[order][at] == keys
            prev = order[at]
            old[found] = self.records[prev[found]]
            rank = np.where(found, prev, len(self.keys) + np.arange(len(keys)))
        else:
            found = np.zeros(len(keys), bool)
            rank = np.arange(len(keys))
        contacts = warm_start_contacts(old, fresh)
        # Insertion order: persisted pairs in last step's order, then the new ones in key order
        # (the keys come sorted from the broad phase, the ground pairs after the box pairs).
        order = np.argsort(rank, kind="stable")
        return contacts[order], keys[order], int((~found).sum())

    def view(self, solver, dt: float):
        """This step's solver input: the contacts updated and coloured, the view laid out in
        colour order. Returns (view, permutation from insertion order to view order, keys)."""
        contacts, keys, new = self.update_contacts(dt)
        self._new = new
        sc = scenes.SolverScene(bodies=self.bodies, mass=np.zeros(self.n, F32),
                                joints=np.zeros(0, abi.JOINT_DTYPE), contacts=contacts,
                                fixed=self.grounds)
        a, b, d = sc.constraint_arrays()
        color, slot = solver.graph_color(a, b, d, self.n + self.worlds)
        view = sc.to_view(color, slot)
        ccounts = np.bincount(color, minlength=abi.COLOR_SLOTS).astype(np.int64)
        first = np.concatenate([[0], np.cumsum(ccounts)[:-1]])
        where = first[color] + slot  # each contact's place in the view
        return view, where, keys

    def finish(self, view, where, keys):
        """The solved view's bodies and contacts become the world's (for the next step)."""
        self.bodies = view.bodies.copy()
        self.records = view.contacts[where]
        self.keys = keys
        self.steps += 1

    def step(self, solver, params, dt: float):
        view, where, keys = self.view(solver, dt)
        solver.phys_solve(view, params, dt)
        self.finish(view, where, keys)
        return view
