"""sphgpu_cfl_dt_noalloc (static device scratch, no allocation) against the
CFL step that sphgpu_step computes for the same velocities.  Collected last
so that it also runs after every other GPU test in one process."""
import ctypes

import numpy as np
import pytest

from graphics_b200 import _lib
from helpers import make_pair

pytestmark = pytest.mark.gpu

CFL = dict(cfl=1, cfl_factor=0.4, dt_max=5e-3, dt_min=1e-6)


def _noalloc(vel_dev, n, stride, d):
    import torch
    lib = _lib.load()
    dt = torch.zeros(1, dtype=torch.float32, device="cuda")
    vm = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = lib.sphgpu_cfl_dt_noalloc(ctypes.c_void_p(vel_dev.data_ptr()), n, stride, CFL["cfl_factor"], d,
                                   CFL["dt_max"], CFL["dt_min"], ctypes.c_void_p(dt.data_ptr()),
                                   ctypes.c_void_p(vm.data_ptr()),
                                   ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0
    torch.cuda.synchronize()
    return float(dt.item()), float(vm.item())


@pytest.mark.parametrize("stride", [3, 4])
def test_noalloc_cfl_matches_step(stride):
    import torch
    sc, g, o = make_pair(**CFL)
    rng = np.random.default_rng(3)
    v = rng.normal(0, 2.0, size=(sc.n_fluid, 3)).astype(np.float32)
    g.set("velocity", v)
    st = g.step("dfsph", 1)  # its dt is the CFL step of these velocities
    vmax = float(np.sqrt((v.astype(np.float64) ** 2).sum(1)).max())
    vs = np.concatenate([v, rng.normal(size=(len(v), 1)).astype(np.float32)], 1) if stride == 4 else v
    vd = torch.from_numpy(np.ascontiguousarray(vs)).cuda()
    for _ in range(2):  # two calls in a row: the scratch's ticket is reset
        dt, vm = _noalloc(vd, len(v), stride, sc.d)
        assert dt == np.float32(st["dt"])
        assert abs(vm - vmax) <= 1e-12 * vmax


def test_noalloc_rejects_oversize():
    lib = _lib.load()
    rc = lib.sphgpu_cfl_dt_noalloc(ctypes.c_void_p(1), _lib.NOALLOC_MAX_N + 1, 3, 0.4, 0.02, 5e-3, 1e-6,
                                   ctypes.c_void_p(1), None, None)
    assert rc == _lib.EINVAL
