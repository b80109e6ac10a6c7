"""A batch of independent DFSPH scenes (sphgpu_batch_*) against the same
scenes run one at a time through the single-scene path: each scene keeps its
own CFL step and its own loop convergence, so iteration counts must be equal
and the states must agree (the per-particle arithmetic is the same code)."""
import numpy as np
import pytest

from graphics_b200.scene import config_batched_dfsph, small_dam_break
from graphics_b200.sph import batch_to_gpu, scene_to_gpu

pytestmark = pytest.mark.gpu

KW = dict(cfl=1, cfl_factor=0.4, dt_max=2e-3, dt=2e-3, nu=1e-3, df_density_goal=1e-4, df_density_max_iter=200,
          df_div_goal_abs=0.0, df_div_goal_rel=1e-3, df_div_max_iter=100)


def _scenes():
    return [small_dam_break((8, 8, 8), 0.025, seed=1), small_dam_break((14, 10, 6), 0.025, seed=2),
            small_dam_break((10, 16, 12), 0.025, seed=3)]


def test_batch_matches_single_scenes():
    scenes = _scenes()
    b = batch_to_gpu(scenes, **KW)
    for k, sc in enumerate(scenes):
        assert b.scene_range(k)[1] == sc.n_fluid
    steps = 6
    b.step("dfsph", steps)
    bst = b.scene_stats()
    for k, sc in enumerate(scenes):
        g = scene_to_gpu(sc, **KW)
        st = g.step("dfsph", steps)
        assert bst[k]["total_iter_density"] == st["total_iter_density"], k
        assert bst[k]["total_iter_divergence"] == st["total_iter_divergence"], k
        assert abs(bst[k]["dt"] - st["dt"]) <= 1e-12 * st["dt"]
        for f in ("position", "velocity"):
            a, ref = b.get_scene(f, k), g.get(f)
            assert a.shape == ref.shape
            assert np.max(np.abs(a - ref)) <= 1e-6 * max(np.max(np.abs(ref)), 1e-6), (k, f)
        g.close()
    b.close()


@pytest.mark.parametrize("graphs", [1, 0])
def test_batch_fused_divergence_sweep_identical_to_separate(graphs):
    # the list build's fused first divergence sweep in a batch (per-scene dt,
    # per-scene decisions) against the separate sweep A launch
    out = []
    for fused in (1, 0):
        b = batch_to_gpu(_scenes(), **KW)
        b.debug_set("use_graphs", graphs)
        b.debug_set("fuse_div", fused)
        b.step("dfsph", 5)
        its = [(s["total_iter_divergence"], s["total_iter_density"]) for s in b.scene_stats()]
        out.append((b.get("position"), b.get("velocity"), b.get("DFkappaV"), its))
        b.close()
    for a, c in zip(out[0][:3], out[1][:3]):
        np.testing.assert_array_equal(a, c)
    assert out[0][3] == out[1][3]


def test_batch_scenes_converge_independently():
    """Scenes of different sizes need different iteration counts: each
    stops at its own goal (the loop runs while any scene is active)."""
    scenes = config_batched_dfsph(nscenes=6, seed=3, n_min=2e3, n_max=2e4)
    b = batch_to_gpu(scenes, **KW)
    b.step("dfsph", 20)
    st = b.scene_stats()
    for s in st:
        assert s["err_density"] <= 1e-4 and not (s["status"] & 1)
    its = [s["iter_density"] for s in st]
    assert len(set(its)) > 1 or len(its) == 1, its
    n = sum(b.scene_range(k)[1] for k in range(len(scenes)))
    assert n == b.n_fluid
    b.close()


def test_autotune_picks_block_sizes_and_keeps_results():
    """The autotuner times 64/128/256 threads per block and keeps a valid
    choice; stepping with it gives the same iteration counts and states as
    the default block sizes (the per-particle arithmetic does not depend on
    the block size)."""
    sc = small_dam_break((16, 16, 16), 0.025, seed=4)
    g1, g2 = scene_to_gpu(sc, **KW), scene_to_gpu(sc, **KW)
    rep = g1.autotune("dfsph", 1)
    assert set(rep["chosen"]) == {"forces", "sweep_a", "sweep_b", "build"}
    assert all(v in (64, 128, 256) for v in rep["chosen"].values())
    # every kernel class was timed at every candidate (the list build under
    # either of its DFSPH names, with or without the fused divergence sweep)
    for cand in rep["candidates"].values():
        assert all(0 < t < 1e6 for t in cand.values()), cand
    g2.step("dfsph", 3)  # g1 advanced 3 steps while tuning
    s1, s2 = g1.step("dfsph", 4), g2.step("dfsph", 4)
    assert s1["total_iter_density"] == s2["total_iter_density"]
    assert np.max(np.abs(g1.get("position") - g2.get("position"))) <= 1e-5
    g1.close()
    g2.close()


def test_batch_scenes_match_oracle_from_shared_state():
    """Every scene of a batch against the CPU oracle (the restatement pinned
    to the reference): before each step the oracle takes the scene's state
    from the batch, then both run one DFSPH step with the scene's own CFL
    step and loop convergence.  The loops stop at a tolerance, so the step
    is compared by what it decides and what it conserves: the CFL dt,
    iteration counts (within one: the FP64 error sums can land on either
    side of the goal), the mean density error, the kinetic energy and the
    positions."""
    from helpers import COMMON
    from oracle import make_scene_oracle
    scenes = _scenes() + config_batched_dfsph(nscenes=2, seed=5, n_min=5e3, n_max=2e4, r=0.025)
    b = batch_to_gpu(scenes, **KW)
    p = dict(COMMON)
    p.update(KW)
    orc = [make_scene_oracle(sc, **p) for sc in scenes]
    for step in range(3):
        for k, o in enumerate(orc):
            o.set("position", b.get_scene("position", k).astype(np.float64))
            o.set("velocity", b.get_scene("velocity", k).astype(np.float64))
            o.set_frame(0)
        b.step("dfsph", 1)
        bst = b.scene_stats()
        for k, o in enumerate(orc):
            o.stage("df_step")
            it, err, dt, _ = o.stats()
            st = bst[k]
            assert abs(st["dt"] - dt) <= 1e-6 * dt, (step, k)
            assert abs(st["iter_density"] - it[0]) <= 1, (step, k, st["iter_density"], it[0])
            assert abs(st["iter_divergence"] - it[1]) <= 1, (step, k, st["iter_divergence"], it[1])
            rg, ro = b.get_scene("density", k).astype(np.float64), o.get("density")
            vg, vo = b.get_scene("velocity", k).astype(np.float64), o.get("velocity")
            assert abs(rg.mean() - ro.mean()) / 1000.0 < 1e-6, (step, k)
            ke_g, ke_o = np.sum(vg * vg), np.sum(vo * vo)
            assert abs(ke_g - ke_o) <= 1e-3 * ke_o, (step, k)
            assert np.abs(b.get_scene("position", k) - o.get("position")).max() < 1e-5, (step, k)
    for o in orc:
        o.close()
    b.close()
