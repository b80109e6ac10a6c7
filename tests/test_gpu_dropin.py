"""The C++ drop-in (include/sphgpu_solver.hpp): for each of the reference's
solver classes (DFSPH, IISph, WcSph, PciSph, IISph_M), a scene class derived
from it (compiled from the reference's sources by oracle/build_ref.py into
oracle/_ref/dropin_<solver>) switched to the GPU by changing its base class
to GpuSolver<Class, SPHGPU_...>.  Stepped with the reference's runOneStep(),
it must give the states the GPU path gives through the Python mirror for the
same scene and parameters, bit for bit."""
import os
import struct
import subprocess

import numpy as np
import pytest

from graphics_b200.scene import small_dam_break
from graphics_b200.sph import scene_to_gpu

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")


def _write(path, sc, steps, kw):
    p = [sc.spacing_r, sc.smooth_radius, kw["dt"], 0.0, -9.81, 0.0, *sc.space_min, *sc.space_max,
         kw["soundSpeed_cs"], kw["nu"], sc.rho0, 0.0, 0.0, sc.d, kw["df_density_goal"], kw["df_div_goal_rel"],
         kw["densityErro_eta"], kw.get("th_h", 0.0), kw.get("th_r", 0.0), kw.get("th_bt", 0.0)]
    with open(path, "wb") as f:
        f.write(struct.pack("3i", sc.n_fluid, len(sc.boundary_pos), steps))
        f.write(np.asarray(p, np.float32).tobytes())
        f.write(np.ascontiguousarray(sc.fluid_pos, np.float32).tobytes())
        f.write(np.ascontiguousarray(sc.fluid_vel, np.float32).tobytes())
        f.write(np.ascontiguousarray(sc.boundary_pos, np.float32).tobytes())


def _read(path):
    b = open(path, "rb").read()
    n, frame, iters = struct.unpack("3i", b[:12])
    a = np.frombuffer(b[12:], np.float32)
    return n, frame, iters, a[:3 * n].reshape(n, 3), a[3 * n:6 * n].reshape(n, 3), a[6 * n:7 * n]


def _settled_column():
    """The settled column of tests/golden/settled_column.npz as one phase
    (the pressure-projection solvers start from a settled state)."""
    import importlib.util
    from graphics_b200.scene import Scene
    gold = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "make_golden.py")
    spec = importlib.util.spec_from_file_location("make_golden", gold)
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    col = mg.column_scene(rho=(1000.0, 1000.0))
    kw = dict(col.__dict__)
    kw.update(phase=None, rho0_phases=(1000.0,))
    return Scene(**kw)


@pytest.mark.parametrize("solver,dt,cs", [("dfsph", 1e-3, 100.0), ("iisph", 2.5e-4, 100.0),
                                          ("wcsph", 2.5e-4, 18.708287), ("pcisph", 1e-3, 20.0),
                                          ("iisph_m", 1e-3, 20.0)])
def test_cpp_dropin_subclass_matches_gpu_path(tmp_path, solver, dt, cs):
    exe = os.path.join(REF, "dropin_" + solver)
    if not os.path.exists(exe):
        pytest.skip("drop-in check not built (needs the reference sources)")
    sc = small_dam_break((12, 12, 12), 0.025, seed=5) if solver in ("dfsph", "iisph") else _settled_column()
    kw = dict(dt=dt, soundSpeed_cs=cs, nu=1e-3, df_density_goal=1e-4, df_div_goal_rel=1e-3, densityErro_eta=0.01)
    steps = 5
    _write(tmp_path / "in.bin", sc, steps, kw)
    r = subprocess.run([exe, str(tmp_path / "in.bin"), str(tmp_path / "out.bin")], cwd=tmp_path,
                       capture_output=True, timeout=300)
    assert r.returncode == 0, r.stderr.decode()[-2000:]
    n, frame, iters, x, v, rho = _read(tmp_path / "out.bin")
    assert frame == steps and n <= sc.n_fluid
    if solver != "wcsph":
        assert iters >= 2 * steps
    g = scene_to_gpu(sc, df_div_goal_abs=0.0, df_div_max_iter=100, **kw)
    g.step(solver, steps)
    assert g.n_fluid == n
    assert np.array_equal(g.get("position"), x)
    assert np.array_equal(g.get("velocity"), v)
    assert np.array_equal(g.get("sphDensity" if solver == "iisph" else "density"), rho)
    g.close()


def test_cpp_dropin_wcsph_surface_terms(tmp_path):
    """WcSph with m_TH.h / r / bt set in the scene (surface tension and
    adhesion): the drop-in reads them from m_TH like the reference does."""
    exe = os.path.join(REF, "dropin_wcsph")
    if not os.path.exists(exe):
        pytest.skip("drop-in check not built (needs the reference sources)")
    sc = _settled_column()
    kw = dict(dt=2.5e-4, soundSpeed_cs=18.708287, nu=1e-3, df_density_goal=1e-4, df_div_goal_rel=1e-3,
              densityErro_eta=0.01, th_h=sc.smooth_radius, th_r=0.2, th_bt=1.0)
    steps = 5
    _write(tmp_path / "in.bin", sc, steps, kw)
    r = subprocess.run([exe, str(tmp_path / "in.bin"), str(tmp_path / "out.bin")], cwd=tmp_path,
                       capture_output=True, timeout=300)
    assert r.returncode == 0, r.stderr.decode()[-2000:]
    n, frame, _, x, v, rho = _read(tmp_path / "out.bin")
    g = scene_to_gpu(sc, df_div_goal_abs=0.0, df_div_max_iter=100, **kw)
    g.step("wcsph", steps)
    assert frame == steps and g.n_fluid == n
    assert np.array_equal(g.get("position"), x)
    assert np.array_equal(g.get("velocity"), v)
    assert np.array_equal(g.get("density"), rho)
    plain = scene_to_gpu(sc, df_div_goal_abs=0.0, df_div_max_iter=100, **dict(kw, th_h=0.0, th_r=0.0, th_bt=0.0))
    plain.step("wcsph", steps)
    assert not np.array_equal(plain.get("velocity"), v)
    plain.close()
    g.close()


class _PrescribedWorld:
    """A body in prescribed motion (translation + rotation about z through
    the centre of mass), as the drop-in scene's gpuRigidStep advances it:
    the same double arithmetic (math.sin/cos, the C library's) and float
    rounding, so both sides hand the library identical states."""

    def __init__(self, com0, lin, wz):
        self.com0, self.lin, self.wz = [float(x) for x in com0], [float(x) for x in lin], float(wz)
        self.t = 0.0
        self.log = []

    def state(self, _sid=1):
        import math
        a = self.wz * self.t
        c, s = math.cos(a), math.sin(a)
        st = np.zeros(25, np.float32)
        st[0], st[1], st[4], st[5], st[10], st[15] = c, s, -s, c, 1.0, 1.0
        for k in range(3):
            x = np.float32(self.com0[k] + self.lin[k] * self.t)
            st[12 + k] = st[16 + k] = x
            st[19 + k] = self.lin[k]
        st[24] = self.wz
        return st

    def step(self, ids, force, torque, dt):
        self.log.append((np.array(force, np.float64), np.array(torque, np.float64)))
        self.t += dt

    def gpu_callback(self):
        from graphics_b200.rigid import RigidWorld
        return RigidWorld.gpu_callback(self)


def test_cpp_dropin_dynamic_solid_matches_gpu_path(tmp_path):
    """A DFSPH scene with a dynamic rigid solid (SphSolid(dynamic=true)) in
    the C++ drop-in: upload of innerPositions and state, the rigid-body world
    behind gpuRigidStep every step, the solid's particles written back into
    m_Solids -- bit for bit what the Python path gives with the same world."""
    exe = os.path.join(REF, "dropin_dfsph")
    if not os.path.exists(exe):
        pytest.skip("drop-in check not built (needs the reference sources)")
    from graphics_b200.scene import floating_box
    sc = floating_box((16, 8, 16), 0.025, (0.8, 0.8, 0.8), (0.1, 0.1, 0.1), (0.4, 0.38, 0.4), seed=3)
    sid = sc.meta["solid_id"]
    body = sc.meta["bodies"][0]
    walls = sc.boundary_pos[sid == 0]
    com0, lin, wz = np.float32(body["center"]), np.float32([0.0, -0.1, 0.05]), np.float32(0.8)
    kw = dict(dt=1e-3, soundSpeed_cs=100.0, nu=1e-3, df_density_goal=1e-4, df_div_goal_rel=1e-3, densityErro_eta=0.01)
    steps = 5
    wsc = type(sc)(**{**sc.__dict__, "boundary_pos": walls, "meta": {}})
    _write(tmp_path / "in.bin", wsc, steps, kw)
    with open(tmp_path / "in.bin", "ab") as f:
        f.write(struct.pack("i", len(body["inner"])))
        f.write(np.ascontiguousarray(body["inner"], np.float32).tobytes())
        f.write(np.concatenate([com0, lin, [wz]]).astype(np.float32).tobytes())
    r = subprocess.run([exe, str(tmp_path / "in.bin"), str(tmp_path / "out.bin")], cwd=tmp_path,
                       capture_output=True, timeout=300)
    assert r.returncode == 0, r.stderr.decode()[-2000:]
    n, frame, iters, x, v, rho = _read(tmp_path / "out.bin")
    raw = open(tmp_path / "out.bin", "rb").read()[12 + 28 * n:]
    nb = len(body["inner"])
    bx = np.frombuffer(raw[:12 * nb], np.float32).reshape(nb, 3)
    ft = np.frombuffer(raw[12 * nb:12 * nb + 48], np.float64)
    g = scene_to_gpu(sc, df_div_goal_abs=0.0, df_div_max_iter=100, **kw)
    w = _PrescribedWorld(com0, lin, wz)
    g.set_solid_dynamic(1, body["inner"], w.state())
    g.set_rigid_world(w)
    g.step("dfsph", steps)
    assert frame == steps and g.n_fluid == n
    assert np.array_equal(g.get("position"), x)
    assert np.array_equal(g.get("velocity"), v)
    assert np.array_equal(g.get("density"), rho)
    assert np.array_equal(g.get_boundary("position")[-nb:], bx)
    assert np.array_equal(np.concatenate(w.log[-1]).ravel(), ft)
    assert np.abs(ft).max() > 0
    g.close()
