"""GPU path (through the C ABI) against the CPU oracle on the same seeded
inputs.  Integer/index results (cell ids, neighbour sets and their order) must
be bit-exact; FP32 fields must agree within RTOL = 1e-5 relative (per element
for densities/alpha, relative to the field's max magnitude for vectors and
for fields that cross zero)."""
import numpy as np
import pytest

from graphics_b200.scene import small_dam_break, dam_break
from helpers import elem_rel, make_pair, rel_err

pytestmark = pytest.mark.gpu
RTOL = 1e-5


def _ns(g, o):
    g.stage("neighbourSearch")
    o.stage("neighbourSearch")
    o.stage("updateSolidPartWeight")
    o.stage("DF_constantDensitySolverFirst")


@pytest.mark.parametrize("n,seed", [((12, 12, 12), 7), ((20, 25, 16), 1)])
def test_neighbour_sets_and_cells_bit_exact(n, seed):
    sc, g, o = make_pair(small_dam_break(n, r=0.025, seed=seed))
    _ns(g, o)
    np.testing.assert_array_equal(g.cells(), o.cells())
    gc, gt, gi = g.neighbours()
    oc, ot, oi, _ = o.neighbours()
    np.testing.assert_array_equal(gc, oc)
    m = np.arange(gt.shape[1])[None, :] < gc[:, None]
    np.testing.assert_array_equal(gt[m], ot[m])
    np.testing.assert_array_equal(gi[m], oi[m])
    assert elem_rel(g.get_boundary("volume"), o.get_solid("volume")) < 1e-6


def test_first_density_alpha():
    sc, g, o = make_pair()
    _ns(g, o)
    assert elem_rel(g.get("density"), o.get("density")) < RTOL
    assert elem_rel(g.get("DFalpha"), o.get("DFalpha")) < RTOL


def test_neighbour_cap_overflow_matches_oracle():
    """A small cap truncates lists exactly where the reference's does."""
    sc, g, o = make_pair(cap=20)
    _ns(g, o)
    gc, gt, gi = g.neighbours()
    oc, ot, oi, _ = o.neighbours()
    np.testing.assert_array_equal(gc, oc)
    m = np.arange(gt.shape[1])[None, :] < gc[:, None]
    np.testing.assert_array_equal(gi[m], oi[m])
    st = g.stage("neighbourSearch")
    assert st["neighbour_overflow"] > 0 and (st["status"] & 8)


def test_forces_except_pressure():
    sc, g, o = make_pair()
    # give the particles a shared random velocity field so viscosity acts
    rng = np.random.default_rng(0)
    v = rng.normal(0, 0.5, size=(sc.n_fluid, 3)).astype(np.float32)
    g.set("velocity", v)
    o.set("velocity", v.astype(np.float64))
    _ns(g, o)
    g.stage("DF_forceExceptPressure")
    o.stage("DF_forceExceptPressure")
    assert rel_err(g.get("acce_adv"), o.get("acce_adv")) < RTOL


def test_constant_density_solver_from_shared_state():
    sc, g, o = make_pair()
    _ns(g, o)
    sg = g.stage("DF_constantDensitySolverSecond")
    o.stage("DF_constantDensitySolverSecond")
    it, err, _, _ = o.stats()
    assert sg["iter_density"] == it[0]
    assert abs(sg["err_density"] - err[0]) < 1e-7
    dadv = o.get("density_adv")
    assert elem_rel(g.get("density_adv"), dadv) < RTOL
    # kappa = (rho_adv - rho0)/dt^2 * alpha cancels catastrophically; it must
    # agree to what a 1e-5 relative change of rho_adv moves it by
    bound = RTOL * dadv * o.get("DFalpha") / 1e-3 ** 2
    assert np.all(np.abs(g.get("DFkappa") - o.get("DFkappa")) <= bound)
    assert rel_err(g.get("velocity"), o.get("velocity")) < RTOL
    assert rel_err(g.get("position"), o.get("position"), scale=1.0) < 1e-6


def test_divergence_free_solver_from_shared_state():
    sc, g, o = make_pair()
    rng = np.random.default_rng(1)
    v = rng.normal(0, 0.3, size=(sc.n_fluid, 3)).astype(np.float32)
    g.set("velocity", v)
    o.set("velocity", v.astype(np.float64))
    o.set("vel_adv", v.astype(np.float64))
    _ns(g, o)
    sg = g.stage("DF_divergenceFreeSolver")
    o.stage("DF_divergenceFreeSolver")
    it, err, _, _ = o.stats()
    assert sg["iter_divergence"] == it[1]
    assert rel_err(g.get("velocity"), o.get("velocity")) < RTOL
    assert rel_err(g.get("divergenceDeviation"), o.get("divergenceDeviation")) < 1e-4


@pytest.mark.parametrize("cfl", [0, 1])
def test_dfsph_steps_from_shared_state(cfl):
    """Each step starts both paths from the same state (the GPU's), then
    compares -- the state after the step, and the non-pressure acceleration
    and rho_adv, which the step computes before its re-sort.  When the FP64 error sums of the two paths land on different
    sides of the goal, the iteration counts differ by one and the fields are
    compared at the size of one Jacobi correction instead."""
    sc, g, o = make_pair(cfl=cfl)
    same = 0
    for k in range(4):
        o.set("position", g.get("position").astype(np.float64))
        o.set("velocity", g.get("velocity").astype(np.float64))
        o.set_frame(0)  # re-run neighbour search + rho/alpha from the shared state
        st = g.step("dfsph", 1)
        o.stage("df_step")
        it, err, dt, _ = o.stats()
        assert abs(st["dt"] - dt) <= 1e-6 * dt
        assert abs(st["iter_density"] - it[0]) <= 1, (k, st["iter_density"], it[0])
        tol = RTOL if (st["iter_density"] == it[0] and st["iter_divergence"] == it[1]) else 1e-4
        same += tol == RTOL
        assert elem_rel(g.get("density"), o.get("density")) < tol, k
        assert rel_err(g.get("velocity"), o.get("velocity")) < tol * 10, k
        assert rel_err(g.get("position"), o.get("position"), scale=1.0) < 1e-6, k
        # written before the step's re-sort, read back in reference order
        assert rel_err(g.get("acce_adv"), o.get("acce_adv")) < RTOL, k
        assert elem_rel(g.get("density_adv"), o.get("density_adv")) < tol, k
    assert same >= 3


def test_long_run_statistics():
    """Trajectories diverge chaotically; long runs are compared by mean density
    error and kinetic energy."""
    from graphics_b200.scene import dam_break
    sc = dam_break((24, 24, 24), 0.01, (4.0, 2.0, 2.0), seed=5)
    _, g, o = make_pair(sc, cfl=1, dt=5e-3, df_div_goal_abs=0.0, df_div_goal_rel=1e-3, df_div_max_iter=100)
    eg, eo = [], []
    for _ in range(30):
        g.step("dfsph", 1)
        o.stage("df_step")
        for path, acc in ((g, eg), (o, eo)):
            v = np.asarray(path.get("velocity"), np.float64)
            rho = np.asarray(path.get("density"), np.float64)
            acc.append((np.mean(rho / 1000.0 - 1.0), 0.5 * np.sum(v * v)))
    eg, eo = np.array(eg), np.array(eo)
    assert np.max(np.abs(eg[:, 0] - eo[:, 0])) < 1e-3
    assert np.max(np.abs(eg[:, 1] - eo[:, 1]) / np.max(eo[:, 1])) < 0.02


def test_graph_and_host_loops_identical_and_deterministic():
    out = []
    for graphs in (1, 0, 1):
        sc, g, o = make_pair()
        g.debug_set("use_graphs", graphs)
        g.step("dfsph", 4)
        out.append((g.get("position"), g.get("velocity"), g.get("density")))
    for a, b in zip(out[0], out[1]):
        np.testing.assert_array_equal(a, b)
    for a, b in zip(out[0], out[2]):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("graphs", [1, 0])
def test_fused_divergence_sweep_identical_to_separate(graphs):
    # the list build's fused first divergence sweep (build mode 4) against the
    # separate k_df_div_a launch, on a dam break that settles over the steps
    # (several divergence iterations in the first ones)
    out = []
    for fused in (1, 0):
        sc, g, o = make_pair(scene=small_dam_break((16, 16, 16), r=0.025, seed=3), cfl=1)
        g.debug_set("use_graphs", graphs)
        g.debug_set("fuse_div", fused)
        its = [g.step("dfsph", 1)["iter_divergence"] for _ in range(6)]
        out.append((g.get("position"), g.get("velocity"), g.get("density"), g.get("DFkappaV"), its))
    for a, b in zip(out[0][:4], out[1][:4]):
        np.testing.assert_array_equal(a, b)
    assert out[0][4] == out[1][4]


def test_wcsph_graph_and_host_steps_identical():
    """The WCSPH step as one CUDA graph per step and launched from the host
    give the same state bit for bit."""
    out = []
    for graphs in (1, 0):
        sc, g, o = make_pair(visc_alpha=0.01, boundary_visc=0.01, dt=2.5e-4, soundSpeed_cs=18.708287)
        g.debug_set("use_graphs", graphs)
        g.step("wcsph", 6)
        out.append((g.get("position"), g.get("velocity"), g.get("density"), g.get("acceleration")))
    for a, b in zip(out[0], out[1]):
        np.testing.assert_array_equal(a, b)


def test_wcsph_pressure_force_and_steps():
    kw = dict(dt=2.5e-4, soundSpeed_cs=18.708287)
    sc, g, o = make_pair(visc_alpha=0.01, boundary_visc=0.01, **kw)
    g.stage("wc_computePressure")
    o.stage("neighbourSearch")
    o.stage("updateSolidPartWeight")
    o.stage("wc_computePressure")
    assert elem_rel(g.get("density"), o.get("density")) < RTOL
    assert rel_err(g.get("presure"), o.get("presure")) < 1e-4
    g.stage("wc_computeForce")
    o.stage("wc_computeForce")
    assert rel_err(g.get("acceleration"), o.get("acceleration")) < 1e-4
    sc, g, o = make_pair(visc_alpha=0.01, boundary_visc=0.01, **kw)
    for _ in range(3):
        g.step("wcsph", 1)
        o.stage("wc_step")
    assert elem_rel(g.get("density"), o.get("density")) < 1e-4
    assert rel_err(g.get("position"), o.get("position"), scale=1.0) < 1e-6


@pytest.mark.parametrize("surf", [0, 1])
def test_wcsph_lanes_match_one_thread_per_particle(surf):
    """The small-scene WCSPH kernels (4 threads per particle: list build
    with density and pressure, force pass) against one thread per particle
    on the same scene: the neighbour lists bit for bit, densities, pressures
    and accelerations to rounding, and the trajectory over steps."""
    kw = dict(dt=2.5e-4, soundSpeed_cs=18.708287)
    if surf:
        kw.update(th_h=0.1, th_r=0.5, th_bt=0.3)
    out = []
    for lanes in (1, 4):
        sc, g, o = make_pair(visc_alpha=0.01, boundary_visc=0.01, **kw)
        g.debug_set("wc_lanes", lanes)
        g.stage("wc_computePressure")
        lists = g.neighbours()
        fields = [g.get("density"), g.get("presure")]
        g.stage("wc_computeForce")
        fields.append(g.get("acceleration"))
        for _ in range(20):
            g.step("wcsph", 1)
        fields.append(g.get("position"))
        out.append((lists, fields))
    (c1, t1, i1), (c4, t4, i4) = out[0][0], out[1][0]
    np.testing.assert_array_equal(c1, c4)
    m = np.arange(t1.shape[1])[None, :] < c1[:, None]
    np.testing.assert_array_equal(t1[m], t4[m])
    np.testing.assert_array_equal(i1[m], i4[m])
    f1, f4 = out[0][1], out[1][1]
    assert elem_rel(f1[0], f4[0]) < 1e-6
    assert rel_err(f1[1], f4[1]) < 1e-4
    assert rel_err(f1[2], f4[2]) < 1e-5
    assert rel_err(f1[3], f4[3], scale=1.0) < 1e-6


def test_wcsph_surface_tension_and_adhesion():
    """m_TH.h / r / bt set (the reference's demo values): the surface
    normal, cohesion, curvature and adhesion terms against the oracle's
    force pass (itself bit-exact with the reference's), then steps."""
    sc = small_dam_break((12, 12, 12), r=0.025, seed=7)
    kw = dict(dt=2.5e-4, soundSpeed_cs=18.708287, th_h=sc.smooth_radius, th_r=0.2, th_bt=1.0)
    sc, g, o = make_pair(sc, visc_alpha=0.01, boundary_visc=0.01, **kw)
    g.stage("wc_computePressure")
    for st in ("neighbourSearch", "updateSolidPartWeight", "wc_computePressure"):
        o.stage(st)
    assert elem_rel(g.get("density"), o.get("density")) < RTOL
    g.stage("wc_computeForce")
    o.stage("wc_computeForce")
    assert rel_err(g.get("acceleration"), o.get("acceleration")) < 1e-4
    sc, g, o = make_pair(sc, visc_alpha=0.01, boundary_visc=0.01, **kw)
    for _ in range(3):
        g.step("wcsph", 1)
        o.stage("wc_step")
    assert elem_rel(g.get("density"), o.get("density")) < 1e-4
    assert rel_err(g.get("position"), o.get("position"), scale=1.0) < 1e-6


def test_out_of_domain_particles_removed_with_status():
    sc = small_dam_break((8, 8, 8), r=0.025, seed=2)
    sc.fluid_pos[0] = np.array(sc.space_max) + 1.0  # outside
    sc2, g, o = make_pair(sc)
    st = g.step("dfsph", 1)
    assert st["status"] & 16
    assert g.n_fluid == sc.n_fluid - 1


def test_nan_particle_reported():
    from graphics_b200._lib import ENAN, SphGpuError
    sc = small_dam_break((8, 8, 8), r=0.025, seed=2)
    sc.fluid_vel[5] = np.nan
    sc2, g, o = make_pair(sc)
    with pytest.raises(SphGpuError) as e:
        g.step("dfsph", 2)
    assert e.value.code == ENAN


def test_no_boundary_scene():
    sc = small_dam_break((8, 8, 8), r=0.025, seed=2)
    sc.boundary_pos = np.zeros((0, 3), np.float32)
    sc2, g, o = make_pair(sc)
    _ns(g, o)
    gc, gt, gi = g.neighbours()
    oc, ot, oi, _ = o.neighbours()
    np.testing.assert_array_equal(gc, oc)
    assert elem_rel(g.get("density"), o.get("density")) < RTOL


def test_larger_scene_density_error_property():
    """27k-particle dam break, CFL steps: every step's density loop ends at or
    below the goal (or reports the cap), no particle is lost or non-finite."""
    sc = dam_break((30, 30, 30), 0.025, (3.0, 1.6, 1.6), seed=0)
    _, g, o = make_pair(sc, cfl=1, df_div_goal_abs=0.0, df_div_goal_rel=1e-3, df_div_max_iter=100)
    for _ in range(10):
        st = g.step("dfsph", 1)
        assert (st["err_density"] <= 1e-4) or (st["status"] & 1)
        assert st["n_fluid"] == sc.n_fluid
    assert np.isfinite(g.get("position")).all()


def test_step_host_matches_device_steps():
    """sphgpu_step_host (host buffers in and out) against the same steps on
    the device state: handing back the previous output (lists still valid,
    no new search), changing only velocities, and moving one particle
    (positions staged and searched again) all give the device path's
    result bit for bit."""
    sc, g, o = make_pair(cfl=1)
    sc2, ref, o2 = make_pair(cfl=1)
    g.step("dfsph", 2)
    ref.step("dfsph", 2)
    pos, vel = g.get("position"), g.get("velocity")
    po, vo = np.empty_like(pos), np.empty_like(vel)
    for k in range(3):
        if k == 1:
            vel = vel * np.float32(0.5)
            ref.set("velocity", vel)
        if k == 2:
            pos = pos.copy()
            pos[7] += np.float32(0.001)
            ref.set("position", pos)
        g.step_host("dfsph", pos, vel, po, vo)
        ref.step("dfsph", 1)
        np.testing.assert_array_equal(po, ref.get("position"))
        np.testing.assert_array_equal(vo, ref.get("velocity"))
        pos, vel = po.copy(), vo.copy()


def test_step_host_speculative_with_warm_start_in_place():
    """The speculative host step (part 1 runs while the inputs are copied in
    and checked) with the learned warm start attached and the output arrays
    the input arrays: handed-back state, changed velocities and a moved
    particle each give the device path's step bit for bit, and so does the
    same sequence with the speculation off."""
    from graphics_b200 import _lib
    from graphics_b200.warmstart import WarmStartNet, attach
    net = WarmStartNet(device=0, dataset_cap=1024, seed=4)
    rng = np.random.default_rng(4)
    net.set_params(rng.normal(0, 0.05, _lib.MLP_NPARAM).astype(np.float32))
    net.set_norm(np.concatenate([np.zeros(16), np.ones(16), [0.0, 50.0]]).astype(np.float32))
    runs = []
    for spec in (1, 0):
        sc, g, o = make_pair(cfl=1)
        sc2, ref, o2 = make_pair(cfl=1)
        g.debug_set("speculative_host_step", spec)
        for x in (g, ref):
            x.step("dfsph", 2)
            attach(x, net, 1)
            x.step("dfsph", 1)
        pos, vel = g.get("position"), g.get("velocity")
        out = []
        for k in range(4):
            if k == 1:
                vel *= np.float32(0.5)
                ref.set("velocity", vel)
            if k == 3:
                pos[11] += np.float32(0.001)
                ref.set("position", pos)
            g.step_host("dfsph", pos, vel, pos, vel)  # in place
            ref.step("dfsph", 1)
            np.testing.assert_array_equal(pos, ref.get("position"))
            np.testing.assert_array_equal(vel, ref.get("velocity"))
            np.testing.assert_array_equal(g.get("kappa_warm"), ref.get("kappa_warm"))
            out.append((pos.copy(), vel.copy()))
        runs.append(out)
    for a, b in zip(runs[0], runs[1]):
        np.testing.assert_array_equal(a[0], b[0])
        np.testing.assert_array_equal(a[1], b[1])


def test_step_host_removal_during_step():
    """A host-buffer step whose integration carries particles out of the
    domain: the positions copied out while the step runs include them, so
    the outputs are read again after the step -- the survivors, in
    reference order, bit for bit as the device path gives them."""
    sc, g, o = make_pair(cfl=0, dt=1e-3)
    sc2, ref, o2 = make_pair(cfl=0, dt=1e-3)
    g.step("dfsph", 2)
    ref.step("dfsph", 2)
    pos, vel = g.get("position"), g.get("velocity")
    vel = vel.copy()
    vel[5] = (1.0e4, 0.0, 0.0)
    ref.set("velocity", vel)
    po, vo = np.zeros_like(pos), np.zeros_like(vel)
    st = g.step_host("dfsph", pos, vel, po, vo)
    ref.step("dfsph", 1)
    m = ref.n_fluid  # the fast particle's neighbours may follow it out
    assert m < len(pos) and g.n_fluid == m and st["removed"] == len(pos) - m
    np.testing.assert_array_equal(po[:m], ref.get("position"))
    np.testing.assert_array_equal(vo[:m], ref.get("velocity"))
