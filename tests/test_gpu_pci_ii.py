"""PCISPH and IISPH_M on the GPU (through the C ABI) against the CPU oracle,
from the settled two-phase column of tests/golden/settled_column.npz (rest
densities 1000 below, 3000 above).

The oracle is the restatement pinned bit for bit to the reference's
PciSph / IISph_M (tests/test_oracle.py).  For IISPH_M it runs the relaxed
Jacobi sweep (every particle reads the previous iterate), which is what the
GPU computes; the reference's own sweep races on p_l (IISph_M.cpp:320-348).
Fields must agree within RTOL = 1e-5: per element for densities, relative to
the field's largest magnitude for vectors.  Pressures and what follows from
them (pressure accelerations, velocities) come out of rho - rho0, which
cancels in FP32: for those the GPU must be as close to the float oracle as
the float oracle is to its own FP64 build (within a factor 2), or within
RTOL."""
import importlib.util
import os

import numpy as np
import pytest

from helpers import elem_rel, make_pair, rel_err

pytestmark = pytest.mark.gpu
RTOL = 1e-5
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _golden():
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLD, "make_golden.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


MG = _golden()


def _pair(**kw):
    p = dict(MG.II_KW)
    p.update(kw)
    return make_pair(MG.column_scene(), visc_alpha=MG.MULTI_VISC["visc_alpha"],
                     boundary_visc=MG.MULTI_VISC["solid_visc"], **p)


def _o(o, f):
    return np.concatenate([o.get(f, k) for k in range(o.nfluid_phases)])


def _f64(**kw):
    from helpers import COMMON
    from oracle import make_scene_oracle
    p = dict(COMMON)
    p.update(MG.II_KW)
    p.update(kw)
    return make_scene_oracle(MG.column_scene(), f64=True, visc_alpha=MG.MULTI_VISC["visc_alpha"],
                             solid_visc=MG.MULTI_VISC["solid_visc"], **p)


def _close_as_float(g, o, od, field):
    """max|gpu - f32| <= max(RTOL, 2 max|f32 - f64|), relative to max|f32|."""
    a, b, c = g.get(field).astype(np.float64), _o(o, field), _o(od, field)
    scale = max(np.abs(b).max(), 1e-30)
    d_gpu = np.abs(a - b).max() / scale
    d_f64 = np.abs(b - c).max() / scale
    assert d_gpu <= max(RTOL, 2 * d_f64), (field, d_gpu, d_f64)


def test_pcisph_step_fixed_iterations():
    """One step with the iteration count pinned (5), so the comparison does
    not depend on where the max-error test falls."""
    kw = dict(densityErro_eta=5e-3, pci_min_iter=5, pci_max_iter=5)
    sc, g, o = _pair(**kw)
    od = _f64(**kw)
    st = g.step("pcisph", 1)
    o.stage("pci_step")
    od.stage("pci_step")
    assert st["iter_density"] == 5 == o.stats()[0][2]
    rho = _o(o, "density")
    assert elem_rel(g.get("density"), rho) < RTOL
    # p = sum over the iterations of delta * max(rho* - rho0, 0): the
    # subtraction cancels, so p is also held to what RTOL on rho* allows
    dp = np.abs(g.get("presure") - _o(o, "presure")).max()
    assert dp <= 5 * o.pci_delta() * RTOL * rho.max()
    for f in ("presure", "acceleration", "velocity"):
        _close_as_float(g, o, od, f)
    assert rel_err(g.get("position"), _o(o, "position")) < 1e-6


def test_pcisph_steps_reference_loop():
    """Three steps with the reference's loop (max error < 0.5 %, 3..50
    iterations): same iteration counts, fields close."""
    sc, g, o = _pair(densityErro_eta=5e-3, pci_min_iter=3, pci_max_iter=50)
    for _ in range(3):
        st = g.step("pcisph", 1)
        o.stage("pci_step")
        assert abs(st["iter_density"] - o.stats()[0][2]) <= 1
    assert elem_rel(g.get("density"), _o(o, "density")) < 1e-4
    assert rel_err(g.get("velocity"), _o(o, "velocity")) < 1e-3


@pytest.mark.parametrize("compat", [0, 3])
def test_iisph_step(compat):
    """One IISPH_M step (both phases solved in turn)."""
    kw = dict(ii_compat=compat, ii_min_iter=2, ii_max_iter=100, ii_eta_rel=1e-3)
    sc, g, o = _pair(**kw)
    od = _f64(**kw)
    st = g.step("iisph_m", 1)
    o.stage("ii_step")
    od.stage("ii_step")
    assert st["iter_density"] == o.stats()[0][3]
    assert elem_rel(g.get("density"), _o(o, "density")) < RTOL
    assert rel_err(g.get("aii"), _o(o, "aii")) < RTOL
    assert rel_err(g.get("dii"), _o(o, "dii")) < RTOL
    assert elem_rel(g.get("rho_adv"), _o(o, "rho_adv")) < RTOL
    for f in ("presure", "acce_presure", "velocity"):
        _close_as_float(g, o, od, f)
    assert rel_err(g.get("position"), _o(o, "position")) < 1e-6


def test_iisph_second_step_reads_previous_phase_state():
    """The second step's phase-0 solve reads phase 1's state of the first
    step (carried through the GPU's reorder)."""
    sc, g, o = _pair(ii_compat=0)
    od = _f64(ii_compat=0)
    for _ in range(2):
        st = g.step("iisph_m", 1)
        o.stage("ii_step")
        od.stage("ii_step")
        assert st["iter_density"] == o.stats()[0][3]
    assert elem_rel(g.get("density"), _o(o, "density")) < RTOL
    for f in ("presure", "velocity", "dii", "sum_dijpj"):
        _close_as_float(g, o, od, f)


def test_pci_ii_long_run_statistics():
    """Several steps: mean density and kinetic energy agree.  (The heavy
    phase on top is unstable under the reference's IISPH_M formulation: from
    about step 11 its velocities grow to O(100) m/s in the oracle as on the
    GPU, and the two trajectories part; the IISPH_M run stops at 10.)"""
    for solver, stage, kw, steps in (
            ("pcisph", "pci_step", dict(densityErro_eta=5e-3, pci_min_iter=3, pci_max_iter=50), 20),
            ("iisph_m", "ii_step", dict(ii_compat=0), 10)):
        sc, g, o = _pair(**kw)
        for _ in range(steps):
            g.step(solver, 1)
            o.stage(stage)
        gr, orr = g.get("density"), _o(o, "density")
        assert abs(gr.mean() - orr.mean()) / orr.mean() < 1e-5, solver
        ke_g = float((g.get("velocity").astype(np.float64) ** 2).sum())
        ke_o = float((_o(o, "velocity") ** 2).sum())
        assert abs(ke_g - ke_o) / max(ke_o, 1e-12) < 1e-3, solver
