"""The C++ drop-in (include/sphgpu_solver.hpp): a scene class derived from
the reference's own DFSPH (or IISph) class (compiled from its sources by
oracle/build_ref.py into oracle/_ref/dropin_dfsph, dropin_iisph) switched to
the GPU by changing its base class to GpuSolver<DFSPH, SPHGPU_DFSPH> (or
GpuSolver<IISph, SPHGPU_IISPH>).  Stepped with the reference's runOneStep(),
it must give the states the GPU path gives through the Python mirror for the
same scene and parameters."""
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
         kw["soundSpeed_cs"], kw["nu"], sc.rho0, 0.0, 0.0, sc.d, kw["df_density_goal"], kw["df_div_goal_rel"], 0.0]
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


@pytest.mark.parametrize("solver,dt", [("dfsph", 1e-3), ("iisph", 2.5e-4)])
def test_cpp_dropin_subclass_matches_gpu_path(tmp_path, solver, dt):
    exe = os.path.join(REF, "dropin_" + solver)
    if not os.path.exists(exe):
        pytest.skip("drop-in check not built (needs the reference sources)")
    sc = small_dam_break((12, 12, 12), 0.025, seed=5)
    kw = dict(dt=dt, soundSpeed_cs=100.0, nu=1e-3, df_density_goal=1e-4, df_div_goal_rel=1e-3)
    steps = 5
    _write(tmp_path / "in.bin", sc, steps, kw)
    r = subprocess.run([exe, str(tmp_path / "in.bin"), str(tmp_path / "out.bin")], cwd=tmp_path,
                       capture_output=True, timeout=300)
    assert r.returncode == 0, r.stderr.decode()[-2000:]
    n, frame, iters, x, v, rho = _read(tmp_path / "out.bin")
    assert frame == steps and n <= sc.n_fluid and iters >= 2 * steps
    g = scene_to_gpu(sc, df_div_goal_abs=0.0, df_div_max_iter=100, **kw)
    st = g.step(solver, steps)
    assert g.n_fluid == n
    assert np.array_equal(g.get("position"), x)
    assert np.array_equal(g.get("velocity"), v)
    assert np.array_equal(g.get("sphDensity" if solver == "iisph" else "density"), rho)
    g.close()
