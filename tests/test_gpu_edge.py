"""Edge cases through the C ABI, for every solver: a scene whose particles
all leave the domain (removed, as SphBase::updateFluids does,
SphBase.cpp:393-401) keeps stepping with no particles, and a lone particle
(no neighbours: density below rest, so no pressure) falls freely."""
import numpy as np
import pytest

from graphics_b200.scene import small_dam_break
from graphics_b200.sph import GpuScene, params_for_scene

pytestmark = pytest.mark.gpu
SOLVERS = ["dfsph", "wcsph", "pcisph", "iisph_m", "iisph"]
KW = dict(dt=1e-3, soundSpeed_cs=20.0, nu=0.0, cfl=0)


def _scene(pos, vel, solver):
    sc = small_dam_break((4, 4, 4), r=0.025, seed=1)
    g = GpuScene(params_for_scene(sc, max_neighbours=48, **KW), len(pos))
    g.set_boundary(sc.boundary_pos)
    g.add_fluid(pos, vel, rho0=1000.0)
    return sc, g


@pytest.mark.parametrize("solver", SOLVERS)
def test_all_particles_leave_then_steps_continue(solver):
    sc = small_dam_break((4, 4, 4), r=0.025, seed=1)
    pos = (np.array(sc.space_max, np.float32) + 0.5 + 0.01 * np.arange(8, dtype=np.float32)[:, None]).astype(np.float32)
    _, g = _scene(pos, np.zeros_like(pos), solver)
    st = g.step(solver, 1)
    assert st["status"] & 16
    assert g.n_fluid == 0
    st = g.step(solver, 3)
    assert g.n_fluid == 0
    assert st["status"] & ~16 & 0xff == 0
    g.close()


@pytest.mark.parametrize("solver", SOLVERS)
def test_lone_particle_falls_freely(solver):
    sc = small_dam_break((4, 4, 4), r=0.025, seed=1)
    mid = (np.array(sc.space_min) + np.array(sc.space_max)) / 2
    pos = np.array([[mid[0], sc.space_max[1] - 0.2, mid[2]]], np.float32)
    _, g = _scene(pos, np.zeros_like(pos), solver)
    steps = 5
    g.step(solver, steps)
    v = g.get("velocity")[0]
    x = g.get("position")[0]
    # Euler-Cromer in float: v += g dt; x += v dt
    vy, y = np.float32(0), np.float32(pos[0, 1])
    for _ in range(steps):
        vy = np.float32(vy + np.float32(np.float32(-9.81) * np.float32(KW["dt"])))
        y = np.float32(y + np.float32(vy * np.float32(KW["dt"])))
    assert abs(v[0]) == 0 and abs(v[2]) == 0
    assert abs(v[1] - vy) <= 1e-6 * abs(vy)
    assert abs(x[1] - y) <= 1e-6
    assert x[0] == pos[0, 0] and x[2] == pos[0, 2]
    g.close()
