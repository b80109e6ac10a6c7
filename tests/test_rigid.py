"""Dynamic rigid solids on the CPU: the restatement (oracle/sph_oracle.c)
pinned against the reference's own DFSPH + rigidForceJoin + updatePaticles
(golden fixture rigid_dfsph.npz, and the compiled reference directly when it
is built here), and the host rigid-body world."""
import importlib.util
import os

import numpy as np
import pytest

from graphics_b200.rigid import RigidBody, RigidWorld, state_array, state_struct
from oracle import make_scene_oracle

GOLD = os.path.join(os.path.dirname(__file__), "golden")
REF = os.path.exists(os.path.join(os.path.dirname(__file__), "..", "oracle", "_ref", "libref_dfsph.so"))


def _mg():
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLD, "make_golden.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def _run(kind, steps):
    mg = _mg()
    sc = mg.rigid_scene()
    o = make_scene_oracle(sc, kind=kind, solver="dfsph", **mg.RIGID_KW)
    if kind == "reference":
        o.set_threads(1)
    w = mg.rigid_world(sc)
    b = sc.meta["bodies"][0]
    o.set_solid_dynamic(b["solid_id"], b["inner"], w.state(b["solid_id"]))
    o.set_rigid_world(w)
    for _ in range(steps):
        o.stage("df_step" if kind == "port" else "runOneStep")
    assert o.rigid_error() == 0
    return o, w


def test_restatement_matches_rigid_golden():
    """Five coupled steps: the force and torque handed to the rigid-body world
    every step, the body's state and particles, the volumes of walls and
    body, and the fluid reproduce the reference bit for bit."""
    g = np.load(os.path.join(GOLD, "rigid_dfsph.npz"))
    o, w = _run("port", len(g["dt"]))
    np.testing.assert_array_equal(np.array([f for _, f, _, _ in w.log])[:, 0], g["force"])
    np.testing.assert_array_equal(np.array([t for _, _, t, _ in w.log])[:, 0], g["torque"])
    np.testing.assert_array_equal(np.array([d for *_, d in w.log]), g["dt"])
    np.testing.assert_array_equal(w.state(1), g["state"])
    np.testing.assert_array_equal(o.get_solid("position", 1).astype(np.float32), g["body_position"])
    np.testing.assert_array_equal(o.get_solid("velocity", 1).astype(np.float32), g["body_velocity"])
    np.testing.assert_array_equal(o.get_solid("volume", 0).astype(np.float32), g["wall_volume"])
    np.testing.assert_array_equal(o.get_solid("volume", 1).astype(np.float32), g["body_volume"])
    np.testing.assert_array_equal(o.get("position").astype(np.float32), g["position"])
    np.testing.assert_array_equal(o.get("velocity").astype(np.float32), g["velocity"])
    # the fixture is not a trivial one: the box is pushed and turned
    assert np.abs(g["force"]).max() > 100 and np.abs(g["torque"]).max() > 1


@pytest.mark.skipif(not REF, reason="compiled reference not built here")
def test_restatement_matches_reference_per_particle_forces():
    """Boundary forces per particle after DF_constantDensitySolverSecond, for
    the walls (static: the reference accumulates forces on every solid) and
    the body, against the reference run with one thread."""
    mg = _mg()
    sc = mg.rigid_scene()
    out = []
    for kind in ("port", "reference"):
        o = make_scene_oracle(sc, kind=kind, solver="dfsph", **mg.RIGID_KW)
        if kind == "reference":
            o.set_threads(1)
        w = mg.rigid_world(sc)
        b = sc.meta["bodies"][0]
        o.set_solid_dynamic(1, b["inner"], w.state(1))
        for st in ("neighbourSearch", "updateSolidPartWeight", "DF_constantDensitySolverFirst",
                   "DF_constantDensitySolverSecond"):
            o.stage(st)
        com = w.state(1)[16:19].astype(np.float64)
        out.append((o.get_solid("force", 0), o.get_solid("force", 1), o.rigid_force_join(1, com)))
        o.close()
    (a0, a1, (fa, ta)), (b0, b1, (fb, tb)) = out
    np.testing.assert_array_equal(a0, b0)
    np.testing.assert_array_equal(a1, b1)
    np.testing.assert_array_equal(fa, fb)
    np.testing.assert_array_equal(ta, tb)
    assert np.abs(a0).max() > 0 and np.abs(a1).max() > 0


def test_rigid_world_free_fall_and_spin():
    """Semi-implicit Euler: v += g dt, x += v dt; a torque-free spin about a
    principal axis keeps its rate and turns the transform about that axis."""
    w = RigidWorld(gravity=(0.0, -9.81, 0.0))
    w.add(3, RigidBody.box(500.0, (0.1, 0.2, 0.3), (0.0, 1.0, 0.0), w=(0.0, 0.0, 2.0)))
    dt, n = 1e-3, 100
    for _ in range(n):
        w.step([3], np.zeros(3), np.zeros(3), dt)
    s = w.state(3)
    vy = -9.81 * dt * n
    yy = 1.0 - 9.81 * dt * dt * n * (n + 1) / 2
    assert abs(s[20] - vy) < 1e-5 and abs(s[17] - yy) < 1e-5
    assert abs(s[24] - 2.0) < 1e-6
    ang = np.arctan2(s[1], s[0])  # first column = rotated x axis
    assert abs(ang - 2.0 * dt * n) < 1e-3
    # OpenGL layout: origin in [12:15], last row (0, 0, 0, 1)
    np.testing.assert_allclose(s[12:15], s[16:19])
    assert s[3] == 0 and s[7] == 0 and s[11] == 0 and s[15] == 1


def test_rigid_world_force_and_torque_response():
    w = RigidWorld(gravity=(0.0, 0.0, 0.0))
    b = w.add(1, RigidBody.box(1000.0, (0.1, 0.1, 0.1), (0.0, 0.0, 0.0)))
    w.step([1], [8.0, 0.0, 0.0], [0.0, 0.0, 0.0], 0.5)
    assert abs(w.state(1)[19] - 8.0 / b.mass * 0.5) < 1e-6
    w2 = RigidWorld(gravity=(0.0, 0.0, 0.0))
    b2 = w2.add(1, RigidBody.box(1000.0, (0.1, 0.1, 0.1), (0.0, 0.0, 0.0)))
    w2.step([1], [0.0, 0.0, 0.0], [0.0, 0.0, 0.3], 0.5)
    assert abs(w2.state(1)[24] - 0.3 / b2.inertia[2] * 0.5) < 1e-4


def test_state_struct_round_trip():
    s = np.arange(25, dtype=np.float32) * 0.5
    np.testing.assert_array_equal(state_array(state_struct(s)), s)
