#!/usr/bin/env python3
"""Generate the golden fixtures from the reference's own solver code.

Runs the reference (compiled from its sources by oracle/build_ref.py into
oracle/_ref/) on small seeded scenes and records its outputs:
  ns_dfsph.npz      neighbour lists (PartIdx t, i; dis), cells, boundary
                    volumes, rho and alpha after neighbourSearch +
                    updateSolidPartWeight + DF_constantDensitySolverFirst
  step_dfsph.npz    state after 3 DFSPH runOneStep() calls (reference
                    bookkeeping: float error sums, goals 1e-4 / 2.5)
  step_wcsph.npz    state after 3 WcSph runOneStep() calls
  settled_column.npz  input state for the PCISPH / IISPH_M fixtures: a
                    10 x 20 x 10 column after 300 DFSPH steps of the CPU
                    restatement (a raw lattice next to the walls starts
                    ~8 % over rest density in the corners; PCISPH and IISPH
                    resolve that in one step and blow up, so they start
                    from a settled state)
  step_pcisph.npz   PciSph::sphStep x 3 from the settled column, two phases
                    (rest densities 1000 below, 3000 above)
  step_iisphm.npz   IISph_M::sphStep x 3 from the same state, run with one
                    OpenMP thread (the reference's pressure loop races on
                    p_l and on its error sums, IISph_M.cpp:320-350)
  step_iisph.npz    IISph::sphStep x 3 (volume form) from the same state and
                    phases, one OpenMP thread (its error sums run under
                    `omp critical` in thread order, IISph.cpp:785,1437),
                    with the boundary particles' own loop state
  rigid_dfsph.npz   DFSPH runOneStep x 5 with a dynamic rigid box in a
                    tank (rigid_scene), one OpenMP thread (the boundary
                    forces are summed without synchronisation inside the
                    parallel loops, DFSPH.cpp:689,1357): the force and torque
                    handed to the rigid-body world each step, the body's
                    final state, particle positions and volumes
Run in the build container (the reference tree must be present):
    python tests/golden/make_golden.py            # all fixtures
    python tests/golden/make_golden.py step_iisph # one of them
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from graphics_b200.rigid import RigidBody, RigidWorld  # noqa: E402
from graphics_b200.scene import Scene, floating_box, rayleigh_taylor, small_dam_break  # noqa: E402
from oracle import make_scene_oracle  # noqa: E402

SCENE = dict(n=(12, 12, 12), r=0.025, seed=7)
DF_KW = dict(float_err=1, df_density_max_iter=1000000, nu=1e-3, dt=1e-3)
WC_KW = dict(dt=2.5e-4, soundSpeed_cs=18.708287, nu=0.0)


COLUMN = dict(counts=(10, 20, 10), r=0.025, box=(0.5, 1.25, 0.5), seed=1)
PCI_KW = dict(dt=1e-3, densityErro_eta=5e-3, pci_min_iter=3, pci_max_iter=50, soundSpeed_cs=20.0, nu=1e-3)
II_KW = dict(dt=1e-3, nu=1e-3, soundSpeed_cs=20.0)
MULTI_VISC = dict(visc_alpha=0.02, solid_visc=0.01)


def scene():
    return small_dam_break(SCENE["n"], r=SCENE["r"], seed=SCENE["seed"])


def column_scene(state=None, rho=(1000.0, 3000.0)):
    """The column of settled_column.npz: walls of rayleigh_taylor(COLUMN),
    fluid state from the fixture, phase 1 above the median height."""
    sc = rayleigh_taylor(COLUMN["counts"], COLUMN["r"], COLUMN["box"], seed=COLUMN["seed"])
    if state is None:
        state = np.load(os.path.join(HERE, "settled_column.npz"))
    pos, vel = state["position"], state["velocity"]
    kw = dict(sc.__dict__)
    kw.update(fluid_pos=pos.astype(np.float32), fluid_vel=vel.astype(np.float32),
              phase=(pos[:, 1] > np.median(pos[:, 1])).astype(np.int32), rho0_phases=list(rho))
    return Scene(**kw)


def make_settled_column():
    sc = rayleigh_taylor(COLUMN["counts"], COLUMN["r"], COLUMN["box"], seed=COLUMN["seed"], rho_heavy=1000.0)
    sc.phase = None
    o = make_scene_oracle(sc, kind="port", dt=1e-3, nu=1e-3, df_div_goal_abs=0.0, df_div_goal_rel=1e-3,
                          df_div_max_iter=100, **MULTI_VISC)
    for _ in range(300):
        o.stage("df_step")
    assert o.n_fluid() == sc.n_fluid
    st = dict(position=o.get("position").astype(np.float32), velocity=o.get("velocity").astype(np.float32))
    np.savez_compressed(os.path.join(HERE, "settled_column.npz"), **st)
    o.close()
    return st


MULTI_FIELDS = ("position", "velocity", "density", "presure")
IV_FIELDS = ("position", "velocity", "sphDensity", "VF_gamma", "VF_sphVolume", "VF_alpha", "VF_kappa",
             "VF_kappaV", "VF_advectionVolume", "acce_presure")
IV_SOLID_FIELDS = ("VF_gamma", "VF_sphVolume", "VF_alpha", "VF_kappa", "VF_kappaV")


# a 0.2 m box of density 500 pushed down and spun, half in the fluid of a
# 0.8 m tank (1,940 fluid particles, 3,904 wall and 98 body particles)
RIGID = dict(counts=(16, 8, 16), r=0.025, box=(0.8, 0.8, 0.8), half=(0.1, 0.1, 0.1), center=(0.4, 0.38, 0.4),
             seed=3, density=500.0, q=(np.cos(0.02), 0.6 * np.sin(0.02), 0.0, 0.8 * np.sin(0.02)),
             v=(0.0, -0.2, 0.05), w=(0.5, 0.0, 0.3))
RIGID_KW = dict(float_err=1, df_density_max_iter=1000000, nu=1e-3, dt=1e-3)
RIGID_STEPS = 5


def rigid_scene():
    c = RIGID
    return floating_box(c["counts"], c["r"], c["box"], c["half"], c["center"], seed=c["seed"])


def rigid_world(sc):
    """The rigid-body world holding the scene's box (solid 1)."""
    c, b = RIGID, sc.meta["bodies"][0]
    w = RigidWorld()
    w.add(b["solid_id"], RigidBody.box(c["density"], b["half"], b["center"], q=c["q"], v=c["v"], w=c["w"]))
    return w


def make_rigid_dfsph():
    sc = rigid_scene()
    o = make_scene_oracle(sc, kind="reference", solver="dfsph", **RIGID_KW)
    o.set_threads(1)
    w = rigid_world(sc)
    b = sc.meta["bodies"][0]
    o.set_solid_dynamic(b["solid_id"], b["inner"], w.state(b["solid_id"]))
    o.set_rigid_world(w)
    for _ in range(RIGID_STEPS):
        o.stage("runOneStep")
    assert o.rigid_error() == 0
    out = dict(force=np.array([f for _, f, _, _ in w.log])[:, 0], torque=np.array([t for _, _, t, _ in w.log])[:, 0],
               dt=np.array([d for *_, d in w.log]), state=w.state(b["solid_id"]),
               body_position=o.get_solid("position", 1).astype(np.float32),
               body_velocity=o.get_solid("velocity", 1).astype(np.float32),
               wall_volume=o.get_solid("volume", 0).astype(np.float32),
               body_volume=o.get_solid("volume", 1).astype(np.float32),
               position=o.get("position").astype(np.float32), velocity=o.get("velocity").astype(np.float32))
    np.savez_compressed(os.path.join(HERE, "rigid_dfsph.npz"), **out)
    o.close()


def make_step_iisph():
    col = column_scene()
    o = make_scene_oracle(col, kind="reference", solver="iisph", **MULTI_VISC, **II_KW)
    o.set_threads(1)
    for _ in range(3):
        o.stage("runOneStep")
    out = {"%s_%d" % (f, k): o.get(f, k).astype(np.float32) for k in range(2) for f in IV_FIELDS}
    out.update({"solid_%s" % f: o.get_solid(f).astype(np.float32) for f in IV_SOLID_FIELDS})
    np.savez_compressed(os.path.join(HERE, "step_iisph.npz"), **out)
    o.close()


def main():
    if len(sys.argv) > 1:
        for name in sys.argv[1:]:
            globals()["make_" + name]()
        return
    sc = scene()
    o = make_scene_oracle(sc, kind="reference", solver="dfsph", **DF_KW)
    o.stage("neighbourSearch")
    o.stage("updateSolidPartWeight")
    o.stage("DF_constantDensitySolverFirst")
    c, t, i, dis = o.neighbours()
    m = np.arange(t.shape[1])[None, :] < c[:, None]
    np.savez_compressed(os.path.join(HERE, "ns_dfsph.npz"), counts=c, t=t[m].astype(np.int8),
                        i=i[m].astype(np.int32), dis=dis[m].astype(np.float32), cells=o.cells(),
                        volume=o.get_solid("volume").astype(np.float32),
                        density=o.get("density").astype(np.float32), alpha=o.get("DFalpha").astype(np.float32))
    o.close()

    o = make_scene_oracle(sc, kind="reference", solver="dfsph", **DF_KW)
    for _ in range(3):
        o.stage("runOneStep")
    np.savez_compressed(os.path.join(HERE, "step_dfsph.npz"),
                        **{f: o.get(f).astype(np.float32) for f in
                           ("position", "velocity", "density", "DFalpha", "DFkappa", "DFkappaV",
                            "density_adv", "divergenceDeviation")})
    o.close()

    o = make_scene_oracle(sc, kind="reference", solver="wcsph", visc_alpha=0.01, solid_visc=0.01, **WC_KW)
    for _ in range(3):
        o.stage("runOneStep")
    np.savez_compressed(os.path.join(HERE, "step_wcsph.npz"),
                        **{f: o.get(f).astype(np.float32) for f in
                           ("position", "velocity", "density", "presure", "acceleration")})
    o.close()
    state = make_settled_column()
    col = column_scene(state)
    o = make_scene_oracle(col, kind="reference", solver="pcisph", **MULTI_VISC, **PCI_KW)
    for _ in range(3):
        o.stage("runOneStep")
    np.savez_compressed(os.path.join(HERE, "step_pcisph.npz"),
                        **{"%s_%d" % (f, k): o.get(f, k).astype(np.float32)
                           for k in range(2) for f in MULTI_FIELDS + ("acceleration", "acce_pressure")})
    o.close()

    o = make_scene_oracle(col, kind="reference", solver="iisphm", **MULTI_VISC, **II_KW)
    o.set_threads(1)
    for _ in range(3):
        o.stage("runOneStep")
    np.savez_compressed(os.path.join(HERE, "step_iisphm.npz"),
                        **{"%s_%d" % (f, k): o.get(f, k).astype(np.float32)
                           for k in range(2)
                           for f in MULTI_FIELDS + ("dii", "aii", "rho_adv", "sum_dijpj", "acce_presure")})
    o.close()
    make_step_iisph()
    make_rigid_dfsph()
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main()
