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


def _bf16(x):
    a = np.asarray(x, np.float32).copy().view(np.uint32)
    a = (a + (((a >> 16) & 1) + np.uint32(0x7FFF))) & np.uint32(0xFFFF0000)
    return a.view(np.float32).astype(np.float64)


def test_feature_gather_matches_cpu_restatement():
    """The warm-start feature gather (k_ws_features) against a CPU
    restatement of its 16 features from the same state: the neighbour lists,
    densities, alpha and non-pressure accelerations of the CPU oracle from
    the GPU's state after one warm-start step, the velocities and the
    per-particle history (the last step's stiffness sum, predicted error and
    divergence term) of the GPU.  The GPU hands the features over as the
    network's BF16 inputs (identity normalisation here), so they agree to
    BF16 rounding."""
    from graphics_b200.scene import small_dam_break
    from graphics_b200.sph import scene_to_gpu
    from helpers import COMMON
    from oracle import make_scene_oracle
    from graphics_b200.warmstart import attach
    rng = np.random.default_rng(11)
    net = _net()
    w, _ = _random_state(rng)
    net.set_params(w * np.float32(0.2))
    net.set_norm(np.concatenate([np.zeros(NIN), np.ones(NIN), [0.0, 1.0]]).astype(np.float32))
    sc = small_dam_break((14, 14, 14), 0.025, seed=4)
    kw = dict(cfl=0, dt=1e-3, dt_max=2e-3, nu=1e-3, ws_scale=1.0)
    g = scene_to_gpu(sc, **kw)
    attach(g, net, 1)
    g.step("dfsph", 1)
    pos, vel, hist = (g.get(f).astype(np.float64) for f in ("position", "velocity", "ws_hist"))
    g.step("dfsph", 1)
    feat = g.get("ws_features").astype(np.float64)
    g.close()
    # the CPU side of the second step's features, from the state after the first
    p = dict(COMMON)
    p.update(kw)
    o = make_scene_oracle(sc, **{k: v for k, v in p.items() if k != "ws_scale"})
    o.set("position", pos)
    o.set("velocity", vel)
    o.set_frame(0)
    for stg in ("neighbourSearch", "updateSolidPartWeight", "DF_constantDensitySolverFirst", "DF_forceExceptPressure"):
        o.stage(stg)
    cnt, t, idx, _ = o.neighbours()
    rho, alpha, a_adv, a1 = o.get("density"), o.get("DFalpha"), o.get("acce_adv"), o.get("DFalpha1")
    vol = o.get_solid("volume")
    o.close()
    d, dt, rho0 = sc.d, kw["dt"], sc.rho0
    m_f = rho0 * d ** 3
    va = vel + a_adv * dt
    live = np.arange(t.shape[1])[None, :] < cnt[:, None]
    bnd = t > 0
    j = np.where(live, idx, 0)
    bpos = sc.boundary_pos.astype(np.float64)
    xj = np.where(bnd[..., None], bpos[np.where(bnd, j, 0)], pos[np.where(bnd, 0, j)])
    vj = np.where(bnd[..., None], 0.0, va[np.where(bnd, 0, j)])
    mj = np.where(bnd, rho0 * vol[np.where(bnd, j, 0)], m_f)
    xij = pos[:, None, :] - xj
    r = np.linalg.norm(xij, axis=2)
    r = np.where(live, r, 1.0)
    q = r / d
    sig = 1.0 / (np.pi * d ** 3)
    dw = np.where(q <= 1, sig / d * (-3 * q + 2.25 * q * q), -sig / d * 0.75 * (2 - q) ** 2)
    grad = (mj * dw / r)[..., None] * xij
    acc = np.where(live, np.einsum("nkc,nkc->nk", grad, va[:, None, :] - vj), 0.0).sum(1)
    nb = (live & bnd).sum(1)
    nfl = (live & ~bnd).sum(1)
    kp = np.where(live & ~bnd, hist[np.where(bnd, 0, j), 0], 0.0).sum(1)
    # alpha of an interior particle of the ideal lattice (the feature's scale)
    ii = np.array([(a, b, c) for a in range(-2, 3) for b in range(-2, 3) for c in range(-2, 3)], np.float64)
    rr = d * np.linalg.norm(ii, axis=1)
    rr = rr[(rr > 0) & (rr < 2 * d)]
    qq = rr / d
    W = lambda x: np.where(x <= 1, sig * (1 - 1.5 * x * x + 0.75 * x ** 3), sig * 0.25 * (2 - x) ** 3)
    Wg = np.where(qq <= 1, sig / d * (3 * qq - 2.25 * qq * qq), sig / d * 0.75 * (2 - qq) ** 2)
    alpha_ref = m_f * (W(0.0) + W(qq).sum()) / ((m_f * Wg) ** 2).sum()
    divt = dt * acc / rho0 * 100
    pred = (np.maximum(rho + acc * dt, rho0) - rho0) / rho0 * 100
    x = np.stack([cnt / 32, (rho - rho0) / rho0 * 100, divt, pred, 0.1 * hist[:, 0], hist[:, 1], hist[:, 2],
                  np.linalg.norm(vel, axis=1) * dt / d, np.linalg.norm(a_adv, axis=1) * dt * dt / d,
                  np.where(cnt > 0, nb / np.maximum(cnt, 1), 0), np.log(np.maximum(alpha, 1e-30) / alpha_ref),
                  np.where(nfl > 0, 0.1 * kp / np.maximum(nfl, 1), 0), np.full(len(cnt), dt / kw["dt_max"]),
                  np.linalg.norm(a1, axis=1) * d / rho0, vel[:, 1] * dt / d, np.ones(len(cnt))], axis=1)
    # two BF16 steps of the value, plus 0.2 % of the feature's range for the
    # FP32 sums behind the differences rho - rho0 and the divergence term
    ref = _bf16(x)
    scale = np.abs(x).max(0) + 1e-12
    excess = np.abs(feat - ref) - (2.0 ** -7 * np.abs(ref) + 2e-3 * scale)
    assert np.all(excess <= 0), excess.max(0)
    assert np.abs(x[:, 4]).max() > 0 and np.abs(x[:, 11]).max() > 0  # the history features are exercised


@pytest.mark.parametrize("graphs", [1, 0])
def test_fused_features_inference_identical_to_separate(graphs):
    # k_ws_features_infer (features gathered and the network run in one
    # kernel, packed-pair GELU) against k_ws_features + k_ws_infer
    from graphics_b200.scene import small_dam_break
    from graphics_b200.sph import GpuScene, params_for_scene
    from graphics_b200.warmstart import attach
    rng = np.random.default_rng(11)
    net = _net(seed=2)
    w, norm = _random_state(rng)
    net.set_params(0.2 * w)
    norm[-1] = 50.0
    net.set_norm(norm)
    sc = small_dam_break((14, 14, 14), r=0.025, seed=5)
    out = []
    for fused in (1, 0):
        g = GpuScene(params_for_scene(sc, dt=1e-3, nu=1e-3), sc.n_fluid, device=0)
        g.set_boundary(sc.boundary_pos)
        g.add_fluid(sc.fluid_pos, sc.fluid_vel, rho0=sc.rho0)
        g.debug_set("use_graphs", graphs)
        g.debug_set("fuse_ws", fused)
        g.step("dfsph", 2)
        attach(g, net, 1)
        its = [g.step("dfsph", 1)["iter_density"] for _ in range(3)]
        out.append((g.get("kappa_warm"), g.get("position"), its))
        g.close()
    assert np.any(out[0][0] > 0)
    np.testing.assert_array_equal(out[0][0], out[1][0])
    np.testing.assert_array_equal(out[0][1], out[1][1])
    assert out[0][2] == out[1][2]
