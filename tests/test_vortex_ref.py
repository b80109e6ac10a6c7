"""The reference's DFSPH vorticity options (m_TH.enable_vortex,
DFSPH.cpp:233-553, 913-1022) run in the oracle build of the reference: the
checker of the GPU's options (tests/test_gpu_vortex.py).  Each option runs,
stays finite and changes the flow."""
import os

import numpy as np
import pytest

from graphics_b200.scene import small_dam_break
from oracle import make_scene_oracle

REF = os.path.exists(os.path.join(os.path.dirname(__file__), "..", "oracle", "_ref", "libref_dfsph.so"))


@pytest.mark.skipif(not REF, reason="compiled reference not built here")
def test_reference_vorticity_options_run():
    out = {}
    for mode in (0, 1, 2, 3):
        sc = small_dam_break((10, 10, 10), 0.025, seed=5)
        d = sc.fluid_pos - sc.fluid_pos.mean(0)
        sc.fluid_vel = (np.stack([-d[:, 1], d[:, 0], 0.3 * d[:, 0]], 1) * 4.0).astype(np.float32)
        o = make_scene_oracle(sc, kind="reference", solver="dfsph", enable_vortex=mode, alpha=0.5, zeta=0.2,
                              nu_t=0.02, dt=1e-3, nu=1e-3)
        for _ in range(2):
            o.stage("runOneStep")
        out[mode] = o.get("velocity")
        assert np.isfinite(out[mode]).all()
        if mode == 1:
            assert np.abs(o.get("omega")).max() > 0
        if mode == 2:
            assert np.abs(o.get("angular_velocity")).max() > 0
        o.close()
    for mode in (1, 2, 3):
        assert np.abs(out[mode] - out[0]).max() > 1e-6
