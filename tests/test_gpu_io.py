"""Output and restart on the GPU path: .pos files in the reference's format
(write_fluid_particles, fUtility.h:254-303) and snapshots that resume a run
bit for bit (DFSPH with CFL steps, PCISPH, IISph with two phases, DFSPH with
the learned warm start attached)."""
import importlib.util
import os

import numpy as np
import pytest

from graphics_b200.scene import small_dam_break
from graphics_b200.sph import GpuScene, scene_to_gpu

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _column():
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLD, "make_golden.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m.column_scene(), m.II_KW


def _parse_reference_pos(path):
    """The reference's layout read independently: four text lines, then
    float32 records."""
    with open(path, "rb") as f:
        lines = [f.readline().decode() for _ in range(4)]
        body = np.frombuffer(f.read(), np.float32)
    n = int(lines[3].split()[0])
    frame = int(lines[2].split()[0])
    idx = int(lines[2].rsplit(":", 1)[1])
    return lines, n, frame, idx, body


def test_write_pos_per_phase(tmp_path):
    sc, kw = _column()
    g = scene_to_gpu(sc, **kw)
    g.step("iisph", 2)
    x, v = g.get("position"), g.get("velocity")
    rho = g.get("sphDensity")
    ph = g.get("phase").astype(int)
    for phase in (0, 1):
        path = tmp_path / ("f%d.pos" % phase)
        n = g.write_pos(path, phase, ("position", "velocity", "density"), "run.log")
        lines, m, frame, idx, body = _parse_reference_pos(path)
        sel = ph == phase
        assert n == m == int(sel.sum()) and frame == 2 and idx == phase
        assert lines[0] == 'for parameters and scene info, please refer to "run.log"\n'
        assert lines[1] == "components writed: < position  velocity  density >\n"
        rec = body.reshape(m, 7)
        np.testing.assert_array_equal(rec[:, 0:3], x[sel])
        np.testing.assert_array_equal(rec[:, 3:6], v[sel])
        np.testing.assert_array_equal(rec[:, 6], rho[sel])
    # the reference's default: position only
    g.write_pos(tmp_path / "p.pos", 0)
    lines, m, _, _, body = _parse_reference_pos(tmp_path / "p.pos")
    assert lines[1] == "components writed: < position >\n" and body.size == 3 * m
    g.close()


def _resume_case(g, solver, k, m, tmp_path, attach=None):
    g.step(solver, k)
    g.save_snapshot(tmp_path / "s.snap")
    g.step(solver, m)
    a = (g.get("position"), g.get("velocity"))
    g.close()
    h = GpuScene.load_snapshot(tmp_path / "s.snap")
    if attach:
        attach(h)
    h.step(solver, m)
    b = (h.get("position"), h.get("velocity"))
    h.close()
    return a, b


@pytest.mark.parametrize("case", ["dfsph_cfl", "pcisph", "iisph_two_phases"])
def test_snapshot_resumes_bit_for_bit(tmp_path, case):
    if case == "dfsph_cfl":
        sc = small_dam_break((12, 12, 12), 0.025, seed=3)
        g = scene_to_gpu(sc, dt=1e-3, cfl=1, cfl_factor=0.4, dt_max=2e-3, nu=1e-3, df_div_goal_abs=0.0)
        solver = "dfsph"
    else:
        sc, kw = _column()
        kw = dict(kw)
        if case == "pcisph":
            kw.update(densityErro_eta=5e-3, pci_min_iter=3, pci_max_iter=50)
        g = scene_to_gpu(sc, **kw)
        solver = "pcisph" if case == "pcisph" else "iisph"
    a, b = _resume_case(g, solver, 4, 5, tmp_path)
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])


def test_snapshot_keeps_warm_start_history(tmp_path):
    """The per-particle history the warm start reads travels in the
    snapshot; the network is attached again to the loaded scene."""
    from graphics_b200 import _lib
    from graphics_b200.warmstart import WarmStartNet, attach
    net = WarmStartNet(device=0, dataset_cap=1024, seed=3)
    rng = np.random.default_rng(3)
    net.set_params(rng.normal(0, 0.05, _lib.MLP_NPARAM).astype(np.float32))
    net.set_norm(np.concatenate([np.zeros(16), np.ones(16), [0.0, 1.0]]).astype(np.float32))
    sc = small_dam_break((12, 12, 12), 0.025, seed=4)
    g = scene_to_gpu(sc, dt=1e-3, nu=1e-3, df_div_goal_abs=0.0)
    attach(g, net, 1)
    a, b = _resume_case(g, "dfsph", 3, 4, tmp_path, attach=lambda h: attach(h, net, 1))
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])
    net.close()
