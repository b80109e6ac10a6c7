"""sphgpu_cfl_dt_noalloc (static device scratch, no allocation) against the
CFL step that sphgpu_step computes for the same velocities, and against an
FP64 NumPy max-norm with the same clamp on inputs that span many blocks.
Collected last so that it also runs after every other GPU test in one
process."""
import ctypes

import numpy as np
import pytest

from graphics_b200 import _lib
from helpers import make_pair

pytestmark = pytest.mark.gpu

CFL = dict(cfl=1, cfl_factor=0.4, dt_max=5e-3, dt_min=1e-6)
PER_BLOCK = 2048  # velocities per block of the kernel


class _Outs:
    """Device outputs allocated once, so repeated calls allocate nothing."""

    def __init__(self):
        import torch
        self.dt = torch.zeros(1, dtype=torch.float32, device="cuda")
        self.vm = torch.zeros(1, dtype=torch.float64, device="cuda")


def _noalloc(vel_dev, n, stride, d, outs=None):
    import torch
    lib = _lib.load()
    o = outs or _Outs()
    ptr = vel_dev.data_ptr() if vel_dev is not None else 0
    rc = lib.sphgpu_cfl_dt_noalloc(ctypes.c_void_p(ptr), n, stride, CFL["cfl_factor"], d, CFL["dt_max"],
                                   CFL["dt_min"], ctypes.c_void_p(o.dt.data_ptr()), ctypes.c_void_p(o.vm.data_ptr()),
                                   ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0
    torch.cuda.synchronize()
    return float(o.dt.item()), float(o.vm.item())


def _expected(v, d):
    vmax = float(np.sqrt((v[:, :3].astype(np.float64) ** 2).sum(1)).max()) if len(v) else 0.0
    dt = CFL["cfl_factor"] * d / vmax if vmax > 0 else CFL["dt_max"]
    return float(np.float32(min(max(dt, CFL["dt_min"]), CFL["dt_max"]))), vmax


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


@pytest.mark.parametrize("n", [1_000_003, _lib.NOALLOC_MAX_N])
def test_noalloc_many_blocks(n):
    """Hundreds to 4096 blocks (a partial last block at 1,000,003; every
    block full at the maximum): the per-block partials, the last-block
    ticket and its reset, called twice in a row with different inputs."""
    import torch
    d = 0.02
    rng = np.random.default_rng(n)
    outs = _Outs()
    for call in range(2):
        v = rng.normal(0, 1.0 + call, size=(n, 3)).astype(np.float32)
        v[rng.integers(n)] *= 40.0  # one fast particle anywhere decides dt
        vd = torch.from_numpy(v).cuda()
        dt, vm = _noalloc(vd, n, 3, d, outs)
        dt_ref, vm_ref = _expected(v, d)
        assert abs(vm - vm_ref) <= 1e-12 * vm_ref
        assert abs(dt - dt_ref) <= 1e-6 * dt_ref
        del vd
    assert n // PER_BLOCK >= 488


def test_noalloc_empty():
    """n = 0: no velocity, so vmax = 0 and dt = dt_max."""
    dt, vm = _noalloc(None, 0, 3, 0.02)
    assert vm == 0.0
    assert dt == np.float32(CFL["dt_max"])


def test_noalloc_non_finite():
    """A NaN (or infinite) component anywhere makes vmax and dt NaN, and the
    next call with finite velocities is correct again."""
    import torch
    n, d = 300_000, 0.02
    rng = np.random.default_rng(7)
    v = rng.normal(0, 1.0, size=(n, 3)).astype(np.float32)
    outs = _Outs()
    for bad in (np.nan, np.inf):
        w = v.copy()
        w[123_457, 1] = bad
        dt, vm = _noalloc(torch.from_numpy(w).cuda(), n, 3, d, outs)
        assert np.isnan(vm) and np.isnan(dt)
    dt, vm = _noalloc(torch.from_numpy(v).cuda(), n, 3, d, outs)
    dt_ref, vm_ref = _expected(v, d)
    assert abs(vm - vm_ref) <= 1e-12 * vm_ref
    assert abs(dt - dt_ref) <= 1e-6 * dt_ref


def test_noalloc_allocates_nothing():
    """Device free memory is unchanged over many calls after the first."""
    import torch
    n = 500_000
    v = torch.from_numpy(np.random.default_rng(1).normal(size=(n, 3)).astype(np.float32)).cuda()
    outs = _Outs()
    _noalloc(v, n, 3, 0.02, outs)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(50):
        _noalloc(v, n, 3, 0.02, outs)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0


def test_noalloc_rejects_oversize():
    lib = _lib.load()
    rc = lib.sphgpu_cfl_dt_noalloc(ctypes.c_void_p(1), _lib.NOALLOC_MAX_N + 1, 3, 0.4, 0.02, 5e-3, 1e-6,
                                   ctypes.c_void_p(1), None, None)
    assert rc == _lib.EINVAL
