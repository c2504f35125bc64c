"""The learned warm start on the device against its CPU restatement (oracle/learned_ref.py,
oracle/port_impl.h): the network's forward pass, gradients and Adam steps, the per-point
features, the cold points' starting impulses, and the residual-driven mode, plain and
learned."""
from __future__ import annotations

import numpy as np
import pytest

from nepheline_b200 import abi, scenes

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0

# The network: the device and the restatement make the same bf16 roundings; they differ by
# the FP32 accumulation order of the tensor-core products (and a rare bf16 tie it moves).
FORWARD_TOL = 1e-3
GRADIENT_TOL = 1e-3
# The features: FP32 on the device against FP64, relative to each feature's own scale.
FEATURE_TOL = 1e-4
# The residual: a float sum of squares on the device (block partial sums, atomics) against
# a double sum on the host, over the same bit-identical velocities and impulses.
RESIDUAL_TOL = 1e-4


def net_inputs(rng, count):
    x = rng.normal(0, 1, (count, abi.MLP_INPUTS)).astype(np.float32)
    t = rng.normal(0, 0.5, (count, abi.MLP_OUTPUTS)).astype(np.float32)
    return x, t


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30))


def test_forward_matches_the_restatement():
    from nepheline_b200.solver import Mlp
    from oracle.learned_ref import Mlp as RefMlp
    rng = np.random.default_rng(0)
    net = Mlp(seed=3)
    for count in (1, 15, 16, 17, 1000, 70001):
        x, _ = net_inputs(rng, count)
        y = net.predict(x)
        want = RefMlp(net.get_weights()).predict(x)
        assert rel(y, want) < FORWARD_TOL, count
    net.close()


def test_gradients_match_the_restatement():
    from nepheline_b200.solver import Mlp
    from oracle.learned_ref import Mlp as RefMlp
    rng = np.random.default_rng(1)
    net = Mlp(seed=5)
    w = net.get_weights()
    for count in (16, 33, 4096, 50000):
        x, t = net_inputs(rng, count)
        g, loss = net.gradients(x, t)
        want, want_loss = RefMlp(w).gradients(x, t)
        assert rel(g, want) < GRADIENT_TOL, count
        assert abs(loss - want_loss) <= 1e-4 * want_loss
        # Against the float64 network without roundings: the bf16 operands' own error.
        exact, _ = RefMlp(w, rounded=False).gradients(x, t)
        assert rel(g, exact) < 5e-2
    net.close()


def test_adam_steps_match_the_restatement():
    """Full-batch steps (every step sees every sample, so the shuffled order does not matter)."""
    from nepheline_b200.solver import Mlp
    from oracle.learned_ref import Mlp as RefMlp, adam
    rng = np.random.default_rng(2)
    net = Mlp(seed=7)
    w0 = net.get_weights().astype(np.float64)
    x, t = net_inputs(rng, 2048)
    lr, steps = 1e-3, 6
    net.train(x, t, epochs=steps, batch=len(x), lr=lr, seed=1)
    w = w0.copy()
    m = np.zeros_like(w)
    v = np.zeros_like(w)
    for k in range(1, steps + 1):
        g, _ = RefMlp(w.astype(np.float32)).gradients(x, t)
        w, m, v = adam(w, g, m, v, k, lr)
    got = net.get_weights()
    assert rel(got - w0, w - w0) < 1e-2
    net.close()


def test_training_reduces_the_loss_on_a_smooth_target():
    from nepheline_b200.solver import Mlp
    rng = np.random.default_rng(3)
    x = rng.uniform(-1, 1, (20000, abi.MLP_INPUTS)).astype(np.float32)
    t = np.stack([np.sin(x[:, 0]) + x[:, 1] ** 2, x[:, 2] * x[:, 3], np.cos(x[:, 4])], 1)
    net = Mlp(seed=1)
    _, before = net.gradients(x, t)
    after = net.train(x, t.astype(np.float32), epochs=30, batch=256, lr=2e-3, seed=4)
    assert after < 0.05 * before
    net.close()


def moving_world(bodies=300, seed=4, warm_fraction=0.5):
    """A batch world with seeded velocities and a share of its points warm (non-zero)."""
    rng = np.random.default_rng(seed)
    sc = scenes.mixed_world(bodies, seed)
    sc.bodies["linear_velocity"] = rng.normal(0, 0.5, (len(sc.bodies), 3)).astype(np.float32)
    sc.bodies["angular_velocity"] = rng.normal(0, 0.5, (len(sc.bodies), 3)).astype(np.float32)
    pts = sc.contacts["points"]
    warm = rng.random(pts.shape) < warm_fraction
    pts["normal_impulse"] = np.where(warm, rng.uniform(0.0, 0.05, pts.shape), 0.0)
    c, s = scenes.host_color(sc)
    return sc.to_view(c, s)


def test_features_match_the_restatement(solver):
    from oracle.learned_ref import features
    params = abi.WorldParams.default()
    view = moving_world()
    solver.upload(view)
    f, scale, kind = solver.features(params, DT)
    want_f, want_s, want_k = features(view, params, DT)
    assert np.array_equal(kind, want_k)
    col = np.maximum(1.0, np.abs(want_f).max(axis=0))
    assert np.all(np.abs(f - want_f) <= FEATURE_TOL * col)
    assert np.all(np.abs(scale - want_s) <= FEATURE_TOL * np.abs(want_s).max())


def test_plain_converge_matches_the_restatement(solver):
    """The passes are the relax pass, bit for bit: at the same pass count the impulses are
    equal; the residuals agree to the sum's rounding."""
    from oracle.refworld import port32_converge
    params = abi.WorldParams.default()
    view = moving_world(seed=6)
    solver.upload(view)
    dev = solver.converge(params, DT, tolerance=1e-4, max_passes=3000, impulses=True)
    ref = port32_converge(view, params, DT, tol=1e-4, max_passes=3000)
    assert dev["cold_points"] == ref["cold_points"]
    assert abs(dev["passes"] - ref["passes"]) <= 1
    n = min(len(dev["residuals"]), len(ref["residuals"]))
    assert np.allclose(dev["residuals"][:n], ref["residuals"][:n], rtol=RESIDUAL_TOL, atol=0)
    same = port32_converge(view, params, DT, tol=1e-30, max_passes=dev["passes"])
    assert np.array_equal(dev["impulses"], same["impulses"])


def test_learned_converge_matches_the_restatement(solver):
    """An untrained network starts the cold points: the device's starting impulses are the
    restatement's from the same predictions, and the passes agree bit for bit."""
    from nepheline_b200.solver import Mlp
    from oracle.learned_ref import initial_impulses
    from oracle.refworld import port32_converge
    params = abi.WorldParams.default()
    view = moving_world(seed=8)
    net = Mlp(seed=11)
    solver.upload(view)
    f, scale, kind = solver.features(params, DT)
    cold = kind == abi.POINT_COLD
    pred = net.predict(f[cold])
    init = np.zeros((len(kind), 3), np.float32)
    friction = np.repeat(view.contacts["friction"], 4)
    init[cold] = initial_impulses(pred, scale[cold], friction[cold])
    solver.set_warm_start_model(net)
    try:
        dev = solver.converge(params, DT, learned=True, tolerance=1e-4, max_passes=3000,
                              impulses=True)
    finally:
        solver.set_warm_start_model(None)
    assert dev["predicted_points"] == dev["cold_points"] == int(cold.sum())
    ref = port32_converge(view, params, DT, init=init.reshape(-1), tol=1e-4, max_passes=3000)
    assert abs(dev["passes"] - ref["passes"]) <= 1
    n = min(len(dev["residuals"]), len(ref["residuals"]))
    assert np.allclose(dev["residuals"][:n], ref["residuals"][:n], rtol=RESIDUAL_TOL, atol=0)
    same = port32_converge(view, params, DT, init=init.reshape(-1), tol=1e-30,
                           max_passes=dev["passes"])
    assert np.array_equal(dev["impulses"], same["impulses"])
    net.close()


def gated_against_plain_and_learned(solver, net, view, params, tol=1e-4, max_passes=3000):
    """The gated start beside the plain and the network's own start on one world: the gate
    keeps the network's start exactly when its initial residual is no larger than the plain
    start's, and the run it keeps is that start's run, bit for bit. Given no reference, the
    gated start runs the plain start first and judges by its residual the same way."""
    solver.upload(view)
    plain = solver.converge(params, DT, tolerance=tol, max_passes=max_passes, impulses=True)
    ref = float(plain["reference_residual"])
    solver.set_warm_start_model(net)
    try:
        learned = solver.converge(params, DT, learned=abi.START_LEARNED, tolerance=tol,
                                  max_passes=max_passes, reference_residual=ref, impulses=True)
        gated = solver.converge(params, DT, learned=abi.START_GATED, tolerance=tol,
                                max_passes=max_passes, reference_residual=ref, impulses=True)
        alone = solver.converge(params, DT, learned=abi.START_GATED, tolerance=tol,
                                max_passes=max_passes, impulses=True)
    finally:
        solver.set_warm_start_model(None)
    keep = learned["initial_residual"] <= ref
    want = learned if keep else plain
    for run in (gated, alone):
        assert run["fell_back"] == (0 if keep else 1)
        assert run["passes"] == want["passes"] and run["converged"] == want["converged"]
        assert np.array_equal(run["residuals"], want["residuals"])
        assert np.array_equal(run["impulses"], want["impulses"])
        assert run["predicted_points"] == (learned["predicted_points"] if keep else 0)
        assert run["reference_residual"] == ref
    assert plain["fell_back"] == learned["fell_back"] == 0
    return keep


def test_gated_start_falls_back_to_the_plain_start(solver):
    """A network whose starts push every new contact far too hard (an untrained network whose
    normal output's bias, the last layer's first bias, is set to 50 impulse scales): the gate
    sees the larger residual and the plain start runs."""
    from nepheline_b200.solver import Mlp
    params = abi.WorldParams.default()
    net = Mlp(seed=11)
    w = net.get_weights()
    w[-abi.MLP_OUTPUTS] = 50.0
    net.set_weights(w)
    try:
        assert not gated_against_plain_and_learned(solver, net, moving_world(seed=8), params)
    finally:
        net.close()


def test_attached_model_changes_only_cold_points(solver):
    """With every point warm, a step with a network attached is the plain step bit for bit; with
    cold points it differs; detached, the plain step again."""
    from nepheline_b200.solver import Mlp
    from oracle.refworld import port32
    params = abi.WorldParams.default()
    net = Mlp(seed=2)
    warm = moving_world(seed=9, warm_fraction=1.1)
    cold = moving_world(seed=9, warm_fraction=0.3)
    solver.set_warm_start_model(net)
    try:
        a = warm.copy()
        solver.phys_solve(a, params, DT)
        b = cold.copy()
        solver.phys_solve(b, params, DT)
    finally:
        solver.set_warm_start_model(None)
    assert a.bodies.tobytes() == port32(warm, params, DT).bodies.tobytes()
    assert b.bodies.tobytes() != port32(cold, params, DT).bodies.tobytes()
    c = cold.copy()
    solver.phys_solve(c, params, DT)
    assert c.bodies.tobytes() == port32(cold, params, DT).bodies.tobytes()
    net.close()


def ground_drop(seed, boxes=300):
    """Boxes falling onto the ground at up to 2 m/s, every contact new this step."""
    rng = np.random.default_rng(seed)
    sc = scenes.box_pile_world(boxes, seed, max_height=1, new_share=1.0)
    sc.bodies["linear_velocity"][:, 1] -= rng.uniform(0.0, 2.0, boxes).astype(np.float32)
    c, s = scenes.host_color(sc)
    return sc.to_view(c, s)


def test_trained_network_gains_over_the_zero_start(solver):
    """Trained on the device on eight worlds' converged impulses, the network starts two held-out
    worlds' new contacts: their initial residual falls well below the zero start's, and the
    plain solver needs fewer passes to reach 1e-3 of it."""
    from nepheline_b200 import learned
    from nepheline_b200.solver import Mlp
    params = abi.WorldParams.default()
    xs, ts = [], []
    for seed in range(8):
        x, t, _ = learned.samples(solver, ground_drop(seed), params, DT, tolerance=1e-5,
                                  max_passes=500)
        xs.append(x)
        ts.append(t)
    net = Mlp(seed=0)
    fit = learned.train(net, np.concatenate(xs), np.concatenate(ts), epochs=60, batch=512,
                        lr=1e-3, seed=2)
    assert fit["loss_after"] < 0.5 * fit["loss_zero_start"]
    plain = learned_total = 0
    for seed in (100, 101):
        cmp = learned.compare(solver, net, ground_drop(seed), params, DT, tolerances=(1e-2, 1e-3),
                              max_passes=500)
        assert cmp["predicted_points"] == cmp["cold_points"] > 0
        assert cmp["learned_initial_over_plain"] < 0.5
        plain += cmp["tolerances"]["0.001"]["plain"]
        learned_total += cmp["tolerances"]["0.001"]["learned"]
        # The gate keeps this network's start.
        assert gated_against_plain_and_learned(solver, net, ground_drop(seed), params, tol=1e-3,
                                               max_passes=500)
    assert learned_total < plain
    net.close()
