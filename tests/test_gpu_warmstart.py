"""Learned warm start: the GPU forward/backward kernels against the CPU
restatement (oracle/mlp_oracle.py), training, and the gain in density-loop
iterations at an unchanged tolerance."""
import numpy as np
import pytest

from mlp_oracle import NIN, NPARAM, gradient as orc_gradient, predict as orc_predict

pytestmark = pytest.mark.gpu


def _net(seed=0):
    from graphics_b200.warmstart import WarmStartNet
    return WarmStartNet(device=0, dataset_cap=200_000, seed=seed)


def _random_state(rng):
    w = rng.normal(0, 0.25, NPARAM).astype(np.float32)
    norm = np.concatenate([rng.normal(0, 0.5, NIN), rng.uniform(0.5, 2, NIN), [0.2, 1.5]]).astype(np.float32)
    return w, norm


def test_mlp_forward_matches_oracle():
    rng = np.random.default_rng(1)
    net = _net()
    w, norm = _random_state(rng)
    net.set_params(w)
    net.set_norm(norm)
    X = rng.normal(0, 1, (1000, NIN)).astype(np.float32)
    yg = net.predict(X)
    yo = orc_predict(w, norm.astype(np.float64), X)
    assert np.max(np.abs(yg - yo)) <= 2e-3 * np.max(np.abs(yo)) + 1e-5


@pytest.mark.parametrize("n", [128, 300])
def test_mlp_gradient_matches_oracle(n):
    rng = np.random.default_rng(n)
    net = _net()
    w, norm = _random_state(rng)
    net.set_params(w)
    net.set_norm(norm)
    X = rng.normal(0, 1, (n, NIN)).astype(np.float32)
    t = rng.normal(0, 1, n).astype(np.float32)
    gg, lg = net.gradient(X, t)
    go, lo = orc_gradient(w, norm.astype(np.float64), X, t)
    scale = np.max(np.abs(go))
    assert abs(lg - lo) <= 1e-3 * lo + 1e-6
    assert np.max(np.abs(gg - go)) <= 5e-3 * scale, np.max(np.abs(gg - go)) / scale
    # per block of parameters too (W1, b1, W2, b2, W3, b3 all exercised)
    for a, b in ((0, 1024), (1024, 1088), (1088, 5184), (5184, 5248), (5248, 5312), (5312, 5313)):
        assert np.max(np.abs(gg[a:b] - go[a:b])) <= 5e-3 * max(np.max(np.abs(go[a:b])), 1e-3 * scale)


def test_training_reduces_loss():
    rng = np.random.default_rng(3)
    net = _net(seed=5)
    X = rng.normal(0, 1, (40_000, NIN)).astype(np.float32)
    y = (np.sin(X[:, 0]) + 0.5 * X[:, 1] ** 2 - X[:, 2] * X[:, 3]).astype(np.float32)
    net.set_dataset(X, y)
    net.fit_normalisation()
    losses = net.train(epochs=8, batch=1024, lr=3e-3)
    assert losses[-1] < 0.2 * losses[0], losses


def test_training_is_deterministic():
    """Per-tile gradients summed in a fixed order (no float atomics): two
    trainings from the same seed and data give bit-identical weights and
    losses."""
    rng = np.random.default_rng(4)
    X = rng.normal(0, 1, (20_000, NIN)).astype(np.float32)
    y = (np.cos(X[:, 0]) - X[:, 1] * X[:, 4]).astype(np.float32)
    out = []
    for _ in range(2):
        net = _net(seed=9)
        net.set_dataset(X, y)
        net.fit_normalisation()
        losses = net.train(epochs=3, batch=2048, lr=3e-3)
        out.append((np.asarray(losses), net.params()))
        net.close()
    np.testing.assert_array_equal(out[0][0], out[1][0])
    np.testing.assert_array_equal(out[0][1], out[1][1])


def test_recording_is_deterministic():
    """Dataset recording from a plain run: the samples land in particle
    order, so two recordings of the same run are identical."""
    from graphics_b200.scene import dam_break
    from graphics_b200.sph import scene_to_gpu
    from graphics_b200.warmstart import attach
    kw = dict(cfl=1, cfl_factor=0.4, dt_max=2e-3, dt=2e-3, nu=1e-3, df_div_goal_abs=0.0, df_div_goal_rel=1e-3)
    data = []
    for _ in range(2):
        net = _net(seed=2)
        g = scene_to_gpu(dam_break((16, 16, 16), 0.01, (0.6, 0.6, 0.4), seed=3), **kw)
        attach(g, net, 2, 7)
        g.step("dfsph", 5)
        data.append(net.dataset())
        g.close()
        net.close()
    assert len(data[0][1]) > 0
    np.testing.assert_array_equal(data[0][0], data[1][0])
    np.testing.assert_array_equal(data[0][1], data[1][1])


def test_warm_start_saves_iterations_at_same_tolerance():
    """Trained on plain runs of two jitter seeds, applied to a third: the
    density loop reaches the same 0.01% goal in fewer iterations."""
    from graphics_b200.scene import dam_break
    from graphics_b200.sph import scene_to_gpu
    from graphics_b200.warmstart import attach, train_for_scenes

    kw = dict(cfl=1, cfl_factor=0.4, dt_max=2e-3, dt=2e-3, nu=1e-3, df_density_goal=1e-4, df_density_max_iter=1000,
              df_div_goal_abs=0.0, df_div_goal_rel=1e-3, df_div_max_iter=100)

    def make(seed):
        return dam_break((24, 48, 24), 0.01, (1.0, 1.2, 0.5), seed=seed)

    net, losses = train_for_scenes(make, seeds=[1, 2], settle=60, record_steps=60, every=2, epochs=20,
                                   dataset_cap=2_000_000, **kw)
    assert losses[-1] < losses[0]
    its = {}
    for mode in (2, 1):
        g = scene_to_gpu(make(0), **kw)
        attach(g, net, 2, 1000000)  # keeps the step history, records almost nothing
        g.step("dfsph", 80)
        attach(g, net, mode, 1000000)
        st = g.step("dfsph", 30)
        its[mode] = st["total_iter_density"]
        assert st["err_density"] <= 1e-4 and not (st["status"] & 1)
        g.close()
    assert its[1] < its[2], its


def test_scene_inference_kernel_matches_oracle():
    """The in-step inference kernel (register-fragment MLP over the
    normalised BF16 features) against the FP64 oracle on the same inputs."""
    from graphics_b200.scene import small_dam_break
    from graphics_b200.sph import scene_to_gpu
    from graphics_b200.warmstart import attach
    rng = np.random.default_rng(7)
    net = _net()
    w, norm = _random_state(rng)
    net.set_params(w)
    net.set_norm(norm)
    g = scene_to_gpu(small_dam_break((16, 16, 16), 0.025, seed=3), dt=1e-3, ws_scale=1.0)
    attach(g, net, 1)
    g.step("dfsph", 2)
    xn = g.get("ws_features")
    kw = g.get("kappa_warm")
    ident = np.concatenate([np.zeros(NIN), np.ones(NIN), norm[2 * NIN:]]).astype(np.float64)
    ko = np.maximum(orc_predict(w, ident, xn.astype(np.float32)), 0.0)
    assert xn.shape == (g.n_fluid, NIN) and np.all(np.isfinite(xn))
    assert np.max(np.abs(kw - ko)) <= 2e-3 * np.max(np.abs(ko)) + 1e-5
    g.close()
