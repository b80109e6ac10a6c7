"""The C-ABI library loads and exports every symbol include/sphgpu.h declares
(no compute calls: this runs without a GPU)."""
import ctypes
import os
import re

from graphics_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "sphgpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(sphgpu_[a-z_0-9]+)\s*\(", src)))


def test_library_exports_all_declared_symbols():
    lib = _lib.load()
    names = declared_symbols()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(_lib.SIGNATURES), "ctypes signatures out of sync with the header"


def test_params_default_and_struct_sizes():
    lib = _lib.load()
    p = _lib.SphParams()
    assert lib.sphgpu_params_default(ctypes.byref(p)) == 0
    assert p.max_neighbours == 48 and p.df_density_min_iter == 2 and abs(p.df_div_goal_abs - 2.5) < 1e-12
    # fields after the DFSPH controls: a layout mismatch of the ctypes mirror
    # would read other fields' bytes here
    assert p.ii_max_iter == 100 and abs(p.ws_scale - 1.0) < 1e-7
    assert (p.iv_cv_min_iter, p.iv_cv_max_iter, p.iv_div_min_iter, p.iv_div_max_iter) == (3, 100, 2, 50)
    assert abs(p.iv_kvisc - 0.1) < 1e-7 and abs(p.iv_cv_goal - 1e-4) < 1e-10 and abs(p.iv_div_goal - 1e-3) < 1e-9
    assert lib.sphgpu_abi_version() == 3


def test_create_without_gpu_fails_loudly():
    import torch
    if torch.cuda.is_available():
        return
    lib = _lib.load()
    p = _lib.SphParams()
    lib.sphgpu_params_default(ctypes.byref(p))
    h = ctypes.c_void_p()
    rc = lib.sphgpu_create(ctypes.byref(p), 0, 1000, ctypes.byref(h))
    assert rc < 0 and not h.value
