"""Dynamic rigid solids on the GPU (through the C ABI) against the CPU
oracle: placement (updatePaticles) bit for bit, volumes to 1e-6, boundary
forces and their per-solid join within FP32 tolerances stated per test, and
coupled steps with the same host rigid-body world on both sides."""
import importlib.util
import os

import numpy as np
import pytest

from graphics_b200 import _lib
from graphics_b200.rigid import RigidWorld
from graphics_b200.sph import SphGpuError
from helpers import elem_rel, make_pair, rel_err

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _mg():
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLD, "make_golden.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


MG = _mg()
KW = dict(dt=1e-3, nu=1e-3, df_density_max_iter=1000)


def _pair(world=True, **kw):
    sc = MG.rigid_scene()
    args = dict(KW)
    args.update(kw)
    sc, g, o = make_pair(sc, **args)
    b = sc.meta["bodies"][0]
    wg, wo = MG.rigid_world(sc), MG.rigid_world(sc)
    g.set_solid_dynamic(1, b["inner"], wg.state(1))
    o.set_solid_dynamic(1, b["inner"], wo.state(1))
    if world:
        g.set_rigid_world(wg)
        o.set_rigid_world(wo)
    return sc, g, o, wg, wo


def _oracle_boundary(o, field):
    return np.concatenate([o.get_solid(field, 0), o.get_solid(field, 1)])


def test_placement_bit_exact_and_prepared_volumes():
    """updatePaticles (transform in the reference's float evaluation order)
    and the rigid velocity are bit-exact; kerSumFromSelf and the volumes of
    prepareSolidPartWeight agree to 1e-6."""
    sc, g, o, _, _ = _pair(world=False)
    nb = len(sc.meta["bodies"][0]["inner"])
    np.testing.assert_array_equal(g.get_boundary("position"), _oracle_boundary(o, "position").astype(np.float32))
    np.testing.assert_array_equal(g.get_boundary("velocity")[-nb:], o.get_solid("velocity", 1).astype(np.float32))
    assert np.abs(g.get_boundary("velocity")[:-nb]).max() == 0
    assert elem_rel(g.get_boundary("kerSumFromSelf"), _oracle_boundary(o, "kerSumFromSelf")) < 1e-6
    assert elem_rel(g.get_boundary("volume"), _oracle_boundary(o, "volume")) < 1e-6


def test_boundary_forces_of_one_density_solve():
    """After the neighbour search (volumes of updateSolidPartWeight to 1e-6)
    and DF_constantDensitySolverSecond: the body's per-particle forces within
    1e-4 of the largest, the joined force and torque within 1e-4 of the sum
    of the per-particle magnitudes (the GPU sums the iterations' stiffness
    before the gradient, the reference after; both are FP32)."""
    sc, g, o, wg, _ = _pair(world=False)
    g.stage("neighbourSearch")
    for st in ("neighbourSearch", "updateSolidPartWeight", "DF_constantDensitySolverFirst"):
        o.stage(st)
    assert elem_rel(g.get_boundary("volume"), _oracle_boundary(o, "volume")) < 1e-6
    sg = g.stage("DF_constantDensitySolverSecond")
    o.stage("DF_constantDensitySolverSecond")
    it, _, _, _ = o.stats()
    assert sg["iter_density"] == it[0]
    fo = o.get_solid("force", 1)
    fg = g.get_boundary("force")[-len(fo):]
    print("per-particle force rel err", rel_err(fg, fo), "max |f|", np.abs(fo).max())
    assert rel_err(fg, fo) < 1e-4
    com = wg.state(1)[16:19].astype(np.float64)
    F, T = g.get_solid_force(1)
    Fo, To = o.rigid_force_join(1, com)
    scale = np.abs(fo).sum()
    lever = np.abs(o.get_solid("position", 1) - com).max()
    print("join", F, Fo, T, To)
    assert np.abs(F - Fo).max() < 1e-4 * scale
    assert np.abs(T - To).max() < 1e-4 * scale * lever
    assert np.abs(Fo).max() > 100


def test_coupled_steps_follow_the_oracle():
    """Five DFSPH steps with the rigid-body world in the loop on each side:
    the forces handed over each step, the body's trajectory and the fluid."""
    sc, g, o, wg, wo = _pair()
    for k in range(5):
        st = g.step("dfsph", 1)
        o.stage("df_step")
        it, _, _, _ = o.stats()
        print(k, st["iter_density"], it[0], wg.log[-1][1], wo.log[-1][1])
        assert abs(st["iter_density"] - it[0]) <= 1
        F, Fo = wg.log[-1][1][0], wo.log[-1][1][0]
        assert np.abs(F - Fo).max() <= 1e-3 * max(np.abs(Fo).max(), 10.0), k
        assert wg.log[-1][0] == [1] and abs(wg.log[-1][3] - wo.log[-1][3]) < 1e-9
    sg, so = wg.state(1), wo.state(1)
    print("state diff", np.abs(sg - so).max())
    assert np.abs(sg[16:19] - so[16:19]).max() < 1e-5
    assert np.abs(sg[:16] - so[:16]).max() < 1e-4
    assert rel_err(g.get("position"), o.get("position"), scale=1.0) < 1e-5
    np.testing.assert_allclose(g.get_boundary("position"), _oracle_boundary(o, "position"), atol=1e-5)


def test_without_callback_the_body_keeps_its_state():
    """No rigid-body world: the body stays where its state puts it, the force
    of each step is still joined; a state set between steps moves the body
    at the next step's updateSolids point."""
    sc, g, o, wg, _ = _pair(world=False)
    p0 = g.get_boundary("position")
    g.step("dfsph", 2)
    np.testing.assert_array_equal(g.get_boundary("position"), p0)
    F, T = g.get_solid_force(1)
    assert np.all(np.isfinite(F)) and np.abs(F).max() > 0
    s = wg.state(1).copy()
    s[13] += 0.01  # origin y
    s[17] += 0.01  # centre of mass y
    g.set_solid_state(1, s)
    np.testing.assert_array_equal(g.get_solid_state(1), s)
    g.step("dfsph", 1)
    p1 = g.get_boundary("position")
    nb = len(sc.meta["bodies"][0]["inner"])
    np.testing.assert_array_equal(p1[:-nb], p0[:-nb])
    assert np.abs(p1[-nb:, 1] - p0[-nb:, 1] - 0.01).max() < 1e-6


def test_graph_and_host_driven_steps_identical():
    out = []
    for graphs in (1, 0):
        sc, g, o, wg, _ = _pair()
        g.debug_set("use_graphs", graphs)
        g.step("dfsph", 3)
        out.append((g.get("position"), g.get_boundary("position"), np.array([f for _, f, _, _ in wg.log])))
        g.close()
    for a, b in zip(*out):
        np.testing.assert_array_equal(a, b)


def test_callback_failure_is_reported():
    sc, g, o, _, _ = _pair(world=False)

    class Failing(RigidWorld):
        def step(self, ids, force, torque, dt):
            raise RuntimeError("world failed")

    w = Failing()
    g.set_rigid_world(w)
    with pytest.raises(SphGpuError) as e:
        g.step("dfsph", 1)
    assert e.value.code == _lib.EINVAL
    g.set_rigid_world(None)
    g.step("dfsph", 1)


def test_body_leaving_the_grid_is_reported():
    """A state that puts the body outside the grid: the particles go to the
    dead cell (no cell scan reaches them), the step reports
    SPHGPU_EOUT_OF_DOMAIN with status bit 64."""
    sc, g, o, wg, _ = _pair(world=False)
    s = wg.state(1).copy()
    s[12] += 50.0
    s[16] += 50.0
    g.set_solid_state(1, s)
    with pytest.raises(SphGpuError) as e:
        g.step("dfsph", 1, allow_maxiter=True)
    assert e.value.code == _lib.EOUT_OF_DOMAIN


def test_other_solvers_refuse_dynamic_solids(tmp_path):
    sc, g, o, _, _ = _pair(world=False)
    for solver in ("wcsph", "pcisph", "iisph_m", "iisph"):
        with pytest.raises(SphGpuError) as e:
            g.step(solver, 1)
        assert e.value.code == _lib.ENOTIMPL
    with pytest.raises(SphGpuError):
        g.save_snapshot(tmp_path / "scene.snap")
