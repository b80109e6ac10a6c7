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
Run in the build container (the reference tree must be present):
    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from graphics_b200.scene import small_dam_break  # noqa: E402
from oracle import make_scene_oracle  # noqa: E402

SCENE = dict(n=(12, 12, 12), r=0.025, seed=7)
DF_KW = dict(float_err=1, df_density_max_iter=1000000, nu=1e-3, dt=1e-3)
WC_KW = dict(dt=2.5e-4, soundSpeed_cs=18.708287, nu=0.0)


def scene():
    return small_dam_break(SCENE["n"], r=SCENE["r"], seed=SCENE["seed"])


def main():
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
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main()
