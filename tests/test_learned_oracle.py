"""The learned warm start's CPU restatement, pinned on its own (CPU only): the network's
backward pass against central differences, its bf16 roundings against plain float64, the
features against first principles on a hand-built contact, and the residual-driven mode's
restatement (oracle/port_impl.h) on a batch world."""
from __future__ import annotations

import numpy as np

from nepheline_b200 import abi, scenes

DT = 1.0 / 60.0


def small_net(seed=0):
    from oracle.learned_ref import pack
    rng = np.random.default_rng(seed)
    parts = [rng.normal(0, 0.4, (64, 16)), rng.normal(0, 0.1, 64), rng.normal(0, 0.2, (64, 64)),
             rng.normal(0, 0.1, 64), rng.normal(0, 0.2, (64, 64)), rng.normal(0, 0.1, 64),
             rng.normal(0, 0.2, (3, 64)), rng.normal(0, 0.1, 3)]
    return pack(parts)


def test_backward_pass_matches_central_differences():
    from oracle.learned_ref import Mlp
    rng = np.random.default_rng(1)
    w = small_net()
    x = rng.normal(0, 1, (24, 16))
    t = rng.normal(0, 1, (24, 3))
    g, loss = Mlp(w, rounded=False).gradients(x, t)
    eps = 1e-6
    for i in rng.choice(len(w), 200, replace=False):
        wp, wm = w.copy(), w.copy()
        wp[i] += eps
        wm[i] -= eps
        fd = (Mlp(wp, rounded=False).gradients(x, t)[1]
              - Mlp(wm, rounded=False).gradients(x, t)[1]) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])
    assert loss > 0


def test_bf16_rounding_is_round_to_nearest_even():
    from oracle.learned_ref import bf16
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, -2.5, 3.1415927],
                 np.float32)
    got = bf16(x)
    assert got[0] == 1.0
    assert got[1] == 1.0               # a tie rounds to the even mantissa
    assert got[2] == 1.0 + 2 ** -6     # ... and up when that is the even one
    assert got[3] == 1.0
    assert got[4] == -2.5
    assert abs(got[5] - 3.140625) < 1e-7


def test_rounded_network_stays_near_float64():
    from oracle.learned_ref import Mlp
    rng = np.random.default_rng(2)
    w = small_net(3)
    x = rng.normal(0, 1, (256, 16))
    t = rng.normal(0, 1, (256, 3))
    y_r = Mlp(w, rounded=True).predict(x)
    y_f = Mlp(w, rounded=False).predict(x)
    assert np.linalg.norm(y_r - y_f) / np.linalg.norm(y_f) < 2e-2
    g_r, _ = Mlp(w, rounded=True).gradients(x, t)
    g_f, _ = Mlp(w, rounded=False).gradients(x, t)
    assert np.linalg.norm(g_r - g_f) / np.linalg.norm(g_f) < 5e-2


def box_on_ground_view(vy=-0.3):
    """One unit box (1 kg) resting on the fixed ground through 4 cold points."""
    bodies = scenes.body_records(1)
    mass = np.array([1.0], np.float32)
    inertia = np.zeros((1, 9), np.float32)
    inertia[:, [0, 4, 8]] = 1.0 / 6.0
    scenes.set_mass(bodies, mass, inertia)
    bodies["linear_velocity"][0] = (0.0, vy, 0.0)
    fixed = scenes._ground()
    c = np.zeros(1, abi.CONTACT_DTYPE)
    c["body_a"] = 1  # the ground
    c["body_b"] = 0
    c["point_count"] = 4
    c["friction"] = 0.6
    c["normal"] = (0.0, 1.0, 0.0)
    corners = np.array([[-0.5, -0.5], [0.5, -0.5], [0.5, 0.5], [-0.5, 0.5]], np.float32)
    for k in range(4):
        c["points"]["anchor_b"][0, k] = (corners[k, 0], -0.5, corners[k, 1])
        c["points"]["anchor_a"][0, k] = (corners[k, 0], 1.0, corners[k, 1])
        c["points"]["separation"][0, k] = -0.01
    counts = np.zeros(abi.COLOR_SLOTS, np.uint32)
    counts[1] = 1
    return abi.View(bodies, fixed, c, np.zeros(0, abi.JOINT_DTYPE), counts,
                    np.zeros(abi.COLOR_SLOTS, np.uint32))


def test_features_of_a_box_resting_on_the_ground():
    """Its features follow from first principles: |rB x n|^2 = 0.5 and an inverse inertia of
    6 give an angular term 3, so kn = 1 + 3."""
    from oracle.learned_ref import features
    params = abi.WorldParams.default()
    f, scale, kind = features(box_on_ground_view(), params, DT)
    h = DT / params.substeps
    g = 9.81
    assert list(kind) == [abi.POINT_COLD] * 4
    assert np.allclose(f[:, 0], -0.3 / (g * h))
    assert np.allclose(f[:, 3:6], [0.0, 1.0, 0.0])
    assert np.allclose(f[:, 6], -0.5)
    assert np.allclose(f[:, 7], 0.0) and np.allclose(f[:, 8], 0.25)
    assert np.allclose(f[:, 9], 0.0) and np.allclose(f[:, 10], 0.75)
    assert np.allclose(f[:, 11], 1.0) and np.allclose(f[:, 12], 0.6)
    assert np.allclose(f[:, 13], 1.0) and np.allclose(f[:, 14], 1.0)
    assert np.allclose(scale, g * h / 4.0)


def test_initial_impulses_stay_in_the_friction_cone():
    from oracle.learned_ref import initial_impulses
    pred = np.array([[1.0, 0.1, 0.0], [-1.0, 0.5, 0.5], [2.0, 3.0, 4.0]], np.float32)
    out = initial_impulses(pred, np.full(3, 0.5, np.float32), np.full(3, 0.6, np.float32))
    assert np.allclose(out[0], [0.5, 0.05, 0.0])
    assert np.allclose(out[1], [0.0, 0.0, 0.0])
    assert np.isclose(np.hypot(out[2, 1], out[2, 2]), 0.6 * 1.0)


def test_port_converge_reduces_the_residual_to_tolerance(ref_lib):
    """The restatement of the residual-driven mode on a batch world: the residual falls to the
    tolerance, every point starts cold, and starting at the converged impulses takes far fewer
    passes."""
    from oracle.refworld import port32_converge
    params = abi.WorldParams.default()
    sc = scenes.mixed_world(200, 4)
    c, s = scenes.host_color(sc)
    v = sc.to_view(c, s)
    r = port32_converge(v, params, DT, tol=1e-3, max_passes=4000)
    assert r["passes"] > 0
    assert r["residuals"][-1] <= 1e-3 * r["residuals"][0]
    assert r["cold_points"] == int(np.sum(v.contacts["point_count"]))
    again = port32_converge(v, params, DT, init=r["impulses"].reshape(-1), tol=1e-3,
                            max_passes=4000, ref=r["residuals"][0])
    assert again["passes"] < r["passes"] // 4
