"""The DFSPH vorticity options on the GPU (through the C ABI) against the
reference's own DFSPH (compiled from its sources, oracle/_ref) from the same
state: the vectors each option computes (TRRV omega and dOmega, the
micropolar angular velocity, the stream function's n0, delta and psi) and
the velocities they leave, within FP32 tolerances stated per test."""
import os

import numpy as np
import pytest

from graphics_b200.scene import small_dam_break
from graphics_b200.sph import scene_to_gpu
from helpers import rel_err
from oracle import make_scene_oracle

pytestmark = pytest.mark.gpu
REF = os.path.exists(os.path.join(os.path.dirname(__file__), "..", "oracle", "_ref", "libref_dfsph.so"))
needs_ref = pytest.mark.skipif(not REF, reason="compiled reference not built")
OPT = dict(alpha=0.5, zeta=0.2, nu_t=0.02)


def _scene():
    sc = small_dam_break((12, 12, 12), 0.025, seed=5)
    c = sc.fluid_pos.mean(0)
    d = sc.fluid_pos - c
    sc.fluid_vel = (np.stack([-d[:, 1], d[:, 0], 0.3 * d[:, 0]], 1) * 4.0).astype(np.float32)  # a swirl
    return sc


def _pair(mode):
    sc = _scene()
    kw = dict(dt=1e-3, nu=1e-3, soundSpeed_cs=100.0)
    g = scene_to_gpu(sc, enable_vortex=mode, vort_alpha=OPT["alpha"], vort_zeta=OPT["zeta"], vort_nu_t=OPT["nu_t"],
                     df_density_goal=1e-4, df_density_max_iter=1000, df_div_goal_abs=2.5, df_div_max_iter=30, **kw)
    o = make_scene_oracle(sc, kind="reference", solver="dfsph", enable_vortex=mode, **OPT, **kw)
    g.stage("neighbourSearch")
    for st in ("neighbourSearch", "updateSolidPartWeight", "DF_constantDensitySolverFirst"):
        o.stage(st)
    return sc, g, o


@needs_ref
def test_trrv_vectors_and_step():
    """TRRV (enable_vortex = 1): omega = curl v and dOmega to 1e-4 of their
    maxima; positions after DF_constantDensitySolverSecond to 1e-6 m."""
    sc, g, o = _pair(1)
    g.stage("DF_constantDensitySolverSecond")
    o.stage("DF_constantDensitySolverSecond")
    e1, e2 = rel_err(g.get("omega"), o.get("omega")), rel_err(g.get("dOmega"), o.get("dOmega"))
    print("omega", e1, "dOmega", e2, np.abs(o.get("omega")).max())
    assert e1 < 1e-4 and e2 < 1e-4 and np.abs(o.get("omega")).max() > 1.0
    assert rel_err(g.get("position"), o.get("position"), scale=1.0) < 1e-6


@needs_ref
def test_micropolar_angular_velocity_and_step():
    """Micropolar (enable_vortex = 2): the updated angular velocity to 1e-4
    of its maximum, over two Second stages (the angular velocity is carried
    through the sort); positions to 1e-6 m."""
    sc, g, o = _pair(2)
    for k in range(2):
        g.stage("DF_constantDensitySolverSecond")
        o.stage("DF_constantDensitySolverSecond")
        e = rel_err(g.get("angular_velocity"), o.get("angular_velocity"))
        print(k, "angular velocity", e, np.abs(o.get("angular_velocity")).max())
        assert e < 1e-4
        assert rel_err(g.get("position"), o.get("position"), scale=1.0) < 1e-6
        g.stage("neighbourSearch")
        o.set("position", g.get("position").astype(np.float64))
        o.set("velocity", g.get("velocity").astype(np.float64))
        for st in ("neighbourSearch", "updateSolidPartWeight", "DF_constantDensitySolverFirst"):
            o.stage(st)
    assert np.abs(o.get("angular_velocity")).max() > 0


@needs_ref
def test_stream_function_correction():
    """Stream function (enable_vortex = 3): n0 after Second; after the
    neighbour search and the divergence loop from the same state, delta,
    psi and the corrected velocity, each to 1e-4 of its maximum."""
    sc, g, o = _pair(3)
    g.stage("DF_constantDensitySolverSecond")
    o.stage("DF_constantDensitySolverSecond")
    e0 = rel_err(g.get("n0Vorticity"), o.get("n0Vorticity"))
    print("n0", e0)
    assert e0 < 1e-4
    g.stage("neighbourSearch")
    o.set("position", g.get("position").astype(np.float64))
    o.set("velocity", g.get("velocity").astype(np.float64))
    o.set("vel_adv", g.get("velocity").astype(np.float64))
    o.set("n0Vorticity", g.get("n0Vorticity").astype(np.float64))
    for st in ("neighbourSearch", "updateSolidPartWeight", "DF_constantDensitySolverFirst"):
        o.stage(st)
    sg = g.stage("DF_divergenceFreeSolver")
    o.stage("DF_divergenceFreeSolver")
    ed, ep = rel_err(g.get("deltaVorticity"), o.get("deltaVorticity")), rel_err(g.get("psi"), o.get("psi"))
    ev = rel_err(g.get("velocity"), o.get("velocity"))
    print("delta", ed, "psi", ep, "velocity", ev, "div iterations", sg["iter_divergence"],
          np.abs(o.get("deltaVorticity")).max())
    assert ed < 1e-4 and ep < 1e-4 and ev < 1e-4
    assert np.abs(o.get("psi")).max() > 0


def test_options_run_full_steps():
    """Each option through full graph steps: finite, and different from the
    plain method."""
    out = {}
    for mode in (0, 1, 2, 3):
        sc = _scene()
        g = scene_to_gpu(sc, enable_vortex=mode, vort_alpha=OPT["alpha"], vort_zeta=OPT["zeta"],
                         vort_nu_t=OPT["nu_t"], dt=1e-3, nu=1e-3)
        g.step("dfsph", 5)
        out[mode] = g.get("velocity")
        assert np.isfinite(out[mode]).all()
        g.close()
    for mode in (1, 2, 3):
        assert np.abs(out[mode] - out[0]).max() > 1e-6
