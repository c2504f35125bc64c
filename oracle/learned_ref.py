"""TEST INFRASTRUCTURE (the oracle), never the product.

The learned warm start restated in numpy, the checker of the device's kernels:

  features()        the 16 per-point features, impulse scales and point kinds of a world view
                    at the step's start (nph_gpu_world_features), in float64
  Mlp               the 16 -> 64 -> 64 -> 64 -> 3 ReLU network in float64, with the device's
                    bf16 roundings at the same places (inputs, weights, hidden activations,
                    and on the backward pass the output error and each layer's dZ as tensor-core
                    operands) or without any (the FP64 reference of the same function)
  adam()            Adam (Kingma and Ba, 2015) as the device's optimiser step
  initial_impulses() the warm-start impulses the device writes for cold points from the
                    network's outputs (normal max(y0, 0) x scale, friction y1, y2 x scale,
                    scaled back onto the friction cone), in float32 as the device

There is no counterpart in the reference (its new contact points start at zero impulse,
engine/physics/src/contact.c:547-565): parity for this part is against this restatement, and
the network's use is judged by the plain solver's residual.
"""
from __future__ import annotations

import numpy as np

from nepheline_b200 import abi

IN, HID, OUT = abi.MLP_INPUTS, abi.MLP_HIDDEN, abi.MLP_OUTPUTS


# ---- features --------------------------------------------------------------------------

def perpendicular(n: np.ndarray) -> np.ndarray:
    """vec.h:460-469: n x (the axis of n's smallest component), normalised."""
    a = np.abs(n)
    axis = np.zeros_like(n)
    ix = (a[:, 0] <= a[:, 1]) & (a[:, 0] <= a[:, 2])
    iy = ~ix & (a[:, 1] <= a[:, 2])
    iz = ~ix & ~iy
    axis[ix, 0] = 1.0
    axis[iy, 1] = 1.0
    axis[iz, 2] = 1.0
    c = np.cross(n, axis)
    return c / np.linalg.norm(c, axis=1, keepdims=True)


def quat_matrix(q: np.ndarray) -> np.ndarray:
    """Rotation matrices of unit quaternions (x, y, z, w)."""
    x, y, z, w = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    r = np.empty((len(q), 3, 3))
    r[:, 0, 0] = 1 - 2 * (y * y + z * z)
    r[:, 0, 1] = 2 * (x * y - w * z)
    r[:, 0, 2] = 2 * (x * z + w * y)
    r[:, 1, 0] = 2 * (x * y + w * z)
    r[:, 1, 1] = 1 - 2 * (x * x + z * z)
    r[:, 1, 2] = 2 * (y * z - w * x)
    r[:, 2, 0] = 2 * (x * z - w * y)
    r[:, 2, 1] = 2 * (y * z + w * x)
    r[:, 2, 2] = 1 - 2 * (x * x + y * y)
    return r


def features(view: abi.View, params: abi.WorldParams, dt: float):
    """Per point slot 4 g + k: features (16), scale g h / kn and kind, as nph_gpu_world_features
    defines them (bodies without locks)."""
    n = len(view.bodies)
    m = len(view.contacts)
    b = view.bodies
    assert not np.any(b["locks"]), "the restatement covers bodies without locks"
    dyn = b["type"] == abi.BODY_DYNAMIC
    rot = quat_matrix(b["rotation"].astype(np.float64))
    # The record's nine floats are the matrix's columns.
    inv_local = b["inv_inertia"].astype(np.float64).reshape(-1, 3, 3).transpose(0, 2, 1)
    inv_world = np.einsum("nij,njk,nlk->nil", rot, inv_local, rot)
    inv_world[~dyn] = 0.0
    inv_mass = np.where(dyn, b["inv_mass"].astype(np.float64), 0.0)
    vel = b["linear_velocity"].astype(np.float64)
    ang = b["angular_velocity"].astype(np.float64)

    def side(idx):
        inside = idx < n
        j = np.where(inside, idx, 0)
        v = np.where(inside[:, None], vel[j], 0.0)
        w = np.where(inside[:, None], ang[j], 0.0)
        im = np.where(inside, inv_mass[j], 0.0)
        ii = np.where(inside[:, None, None], inv_world[j], 0.0)
        d = np.where(inside, dyn[j], False)
        return v, w, im, ii, d

    c = view.contacts
    va, wa, ma, ia, da = side(c["body_a"].astype(np.int64))
    vb, wb, mb, ib, db = side(c["body_b"].astype(np.int64))
    nrm = c["normal"].astype(np.float64)
    t1 = perpendicular(nrm)
    t2 = np.cross(nrm, t1)
    grav = np.array(params.gravity[:], np.float64)
    gl = np.linalg.norm(grav)
    g = gl if gl > 0 else 1.0
    gdir = grav / gl if gl > 0 else np.zeros(3)
    h = dt / params.substeps
    feat = np.zeros((m, 4, IN))
    scale = np.zeros((m, 4))
    kind = np.zeros((m, 4), np.uint32)
    pc = c["point_count"].astype(np.int64)
    for k in range(4):
        live = k < pc
        p = c["points"][:, k]
        ra = p["anchor_a"].astype(np.float64)
        rb = p["anchor_b"].astype(np.float64)
        rxa = np.cross(ra, nrm)
        rxb = np.cross(rb, nrm)
        ang_a = np.einsum("ni,nij,nj->n", rxa, ia, rxa)
        ang_b = np.einsum("ni,nij,nj->n", rxb, ib, rxb)
        kn = ma + mb + ang_a + ang_b
        inv_kn = np.where(kn > 0, 1.0 / np.where(kn > 0, kn, 1.0), 0.0)

        def kt(u, v_):
            return (np.einsum("ni,nij,nj->n", np.cross(ra, u), ia, np.cross(ra, v_))
                    + np.einsum("ni,nij,nj->n", np.cross(rb, u), ib, np.cross(rb, v_)))

        k11 = ma + mb + kt(t1, t1)
        k22 = ma + mb + kt(t2, t2)
        k12 = kt(t1, t2)
        det = k11 * k22 - k12 * k12
        t00 = np.where(det > 0, k22 / np.where(det > 0, det, 1.0), 0.0)
        dv = (vb + np.cross(wb, rb)) - (va + np.cross(wa, ra))
        f = feat[:, k]
        f[:, 0] = np.einsum("ni,ni->n", dv, nrm) / (g * h)
        f[:, 1] = np.einsum("ni,ni->n", dv, t1) / (g * h)
        f[:, 2] = np.einsum("ni,ni->n", dv, t2) / (g * h)
        f[:, 3:6] = nrm
        f[:, 6] = p["separation"].astype(np.float64) * 50.0
        f[:, 7] = ma * inv_kn
        f[:, 8] = mb * inv_kn
        f[:, 9] = ang_a * inv_kn
        f[:, 10] = ang_b * inv_kn
        f[:, 11] = pc * 0.25
        f[:, 12] = c["friction"]
        f[:, 13] = -(nrm @ gdir)
        f[:, 14] = np.where(da & db, 0.0, 1.0)
        f[:, 15] = t00 * kn
        f[~live] = 0.0
        scale[:, k] = np.where(live, g * h * inv_kn, 0.0)
        cold = (p["normal_impulse"] == 0) & np.all(p["tangent_impulse"] == 0, axis=1)
        kind[:, k] = np.where(live, np.where(cold, abi.POINT_COLD, abi.POINT_WARM), abi.POINT_NONE)
    return feat.reshape(-1, IN), scale.reshape(-1), kind.reshape(-1)


def initial_impulses(pred: np.ndarray, scale: np.ndarray, friction: np.ndarray) -> np.ndarray:
    """The cold points' starting impulses (normal, t1, t2) from network outputs, in float32
    with the device's operations: normal max(y0, 0) x scale, friction (y1, y2) x scale scaled
    back onto the cone mu x normal when outside it."""
    f32 = np.float32
    pred = np.asarray(pred, f32)
    sc = np.asarray(scale, f32)
    ln = np.maximum(pred[:, 0], f32(0)) * sc
    l1 = pred[:, 1] * sc
    l2 = pred[:, 2] * sc
    limit = np.asarray(friction, f32) * ln
    length = np.sqrt(l1 * l1 + l2 * l2)
    out = length > limit
    r = np.where(length > 0, limit / np.where(length > 0, length, f32(1)), f32(0)).astype(f32)
    l1 = np.where(out, l1 * r, l1)
    l2 = np.where(out, l2 * r, l2)
    return np.stack([ln, l1, l2], axis=1).astype(f32)


# ---- the network -----------------------------------------------------------------------

def bf16(x: np.ndarray) -> np.ndarray:
    """Rounds to bfloat16 (round to nearest, ties to even) through float32; float64 out."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(params: np.ndarray):
    """The parameter vector's W1, b1, W2, b2, W3, b3, W4, b4 (weights [out][in])."""
    p = np.asarray(params, np.float64)
    shapes = [(HID, IN), (HID,), (HID, HID), (HID,), (HID, HID), (HID,), (OUT, HID), (OUT,)]
    out, i = [], 0
    for s in shapes:
        size = int(np.prod(s))
        out.append(p[i:i + size].reshape(s))
        i += size
    assert i == len(p)
    return out


def pack(parts) -> np.ndarray:
    return np.concatenate([np.asarray(a, np.float64).reshape(-1) for a in parts])


class Mlp:
    """The network as the device computes it (`rounded`: bf16 operands of every tensor-core
    product) or in plain float64."""

    def __init__(self, params: np.ndarray, rounded: bool = True):
        self.params = np.asarray(params, np.float64)
        self.r = bf16 if rounded else (lambda a: np.asarray(a, np.float64))

    def _weights(self):
        w1, b1, w2, b2, w3, b3, w4, b4 = unpack(self.params)
        r = self.r
        return r(w1), b1, r(w2), b2, r(w3), b3, r(w4), b4

    def forward(self, x: np.ndarray):
        w1, b1, w2, b2, w3, b3, w4, b4 = self._weights()
        r = self.r
        h0 = r(x)
        z1 = h0 @ w1.T + b1
        h1 = r(np.maximum(z1, 0.0))
        z2 = h1 @ w2.T + b2
        h2 = r(np.maximum(z2, 0.0))
        z3 = h2 @ w3.T + b3
        h3 = r(np.maximum(z3, 0.0))
        y = h3 @ w4.T + b4
        return y, (h0, z1, h1, z2, h2, z3, h3)

    def predict(self, x: np.ndarray) -> np.ndarray:
        return self.forward(x)[0]

    def gradients(self, x: np.ndarray, t: np.ndarray):
        """The gradient of the mean over samples of the squared error summed over outputs, and
        that loss."""
        w1, b1, w2, b2, w3, b3, w4, b4 = self._weights()
        r = self.r
        y, (h0, z1, h1, z2, h2, z3, h3) = self.forward(x)
        count = len(x)
        e = y - np.asarray(t, np.float64)
        loss = float(np.sum(e * e) / count)
        dy = 2.0 * e / count
        dyr = r(dy)
        gw4 = dyr.T @ h3
        gb4 = dy.sum(0)
        dz3 = (dyr @ w4) * (z3 > 0)
        dz3r = r(dz3)
        gw3 = dz3r.T @ h2
        gb3 = dz3.sum(0)
        dz2 = (dz3r @ w3) * (z2 > 0)
        dz2r = r(dz2)
        gw2 = dz2r.T @ h1
        gb2 = dz2.sum(0)
        dz1 = (dz2r @ w2) * (z1 > 0)
        dz1r = r(dz1)
        gw1 = dz1r.T @ h0
        gb1 = dz1.sum(0)
        return pack([gw1, gb1, gw2, gb2, gw3, gb3, gw4, gb4]), loss


def adam(params, grad, m, v, step: int, lr: float, beta1=0.9, beta2=0.999, eps=1e-8):
    """One Adam step (Kingma and Ba, 2015); returns the new parameters and moments."""
    m = beta1 * m + (1 - beta1) * grad
    v = beta2 * v + (1 - beta2) * grad * grad
    c1 = 1 - beta1 ** step
    c2 = 1 - beta2 ** step
    return params - lr * (m / c1) / (np.sqrt(v / c2) + eps), m, v
