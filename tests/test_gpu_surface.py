"""Surface reconstruction on the GPU (through the C ABI) against the
reference's own surface_field / marchingCubes (oracle/_ref/libref_surface.so)
and the restated marching cubes (oracle/mc_table.py)."""
import os

import numpy as np
import pytest

import mc_table as mt
from graphics_b200.scene import lattice_block
from helpers import closed_and_oriented

pytestmark = pytest.mark.gpu
REF = os.path.exists(os.path.join(os.path.dirname(__file__), "..", "oracle", "_ref", "libref_surface.so"))
needs_ref = pytest.mark.skipif(not REF, reason="compiled reference not built")
# the radii of every reference call in the process (function-local statics)
R_P, R_H = 0.01, 0.02


def blob(n=(12, 12, 12), seed=1):
    return lattice_block(n, R_P, lo=(0.1, 0.1, 0.1), jitter=0.1, seed=seed)


def _pair(pos, cell=R_P / 2):
    from oracle import RefSurface
    from graphics_b200.surface import surface_field
    p64 = pos.astype(np.float64)
    mn, mx = p64.min(0), p64.max(0)
    rs = RefSurface(mn, mx, R_P, R_H, cell)
    sf = surface_field()
    sf.surface_setup(mn, mx, R_P, R_H, cell)
    np.testing.assert_array_equal(sf.get_grid_num(), rs.grid_num)
    np.testing.assert_array_equal(sf.get_grid_min(), rs.grid_min)
    assert sf.get_cell_size() == rs.cell
    return rs, sf


@needs_ref
def test_isotropic_field_matches_reference():
    pos = blob()
    rs, sf = _pair(pos)
    fr = rs.field(pos.astype(np.float64), aniso=False)
    sf.surface_isotro(pos)
    fg = sf.get_field()
    err = np.abs(fg - fr).max() / np.abs(fr).max()
    print("isotropic field max rel err", err)
    assert err < 1e-5
    assert np.count_nonzero(fr) == np.count_nonzero(fg)


@needs_ref
def test_anisotropic_field_matches_reference():
    """FP32 neighbour sums and covariance on the GPU (FP64 eigen-solve), FP64
    in the reference: nodes to 1e-4 of the field's maximum."""
    pos = blob()
    rs, sf = _pair(pos)
    fr = rs.field(pos.astype(np.float64), aniso=True)
    sf.surface_aniso(pos)
    fg = sf.get_field()
    err = np.abs(fg - fr).max() / np.abs(fr).max()
    print("anisotropic field max rel err", err, "nonzero", np.count_nonzero(fr), np.count_nonzero(fg))
    assert err < 1e-4


@needs_ref
@pytest.mark.parametrize("ref_rows", [False, True])
def test_gpu_marching_cubes_is_the_restatement(ref_rows):
    """On the reference's anisotropic field: the GPU's triangles equal the
    restated marching cubes' bit for bit (same table, same order)."""
    pos = blob()
    rs, sf = _pair(pos)
    f = rs.field(pos.astype(np.float64), aniso=True)
    sf.set_field(f)
    g = sf.mesh(0.5, ref_rows=ref_rows)
    c = mt.marching_cubes(f, tuple(rs.grid_num), rs.grid_min.astype(np.float32), np.float32(rs.cell), 0.5,
                          ref_rows=ref_rows)
    assert len(g) > 1000
    np.testing.assert_array_equal(g, c)


@needs_ref
def test_gpu_marching_cubes_vertices_are_the_references():
    """With the reference's row pairing: per cube the same triangle count and
    the same vertices as the reference's marchingCubes, bit for bit."""
    from oracle import RefSurface
    pos = blob(seed=2)
    rs, sf = _pair(pos)
    f = rs.field(pos.astype(np.float64), aniso=True)
    sf.set_field(f)
    g = sf.mesh(0.5, ref_rows=True)
    ref = RefSurface.marching_cubes(0.5, f, rs.grid_min.astype(np.float32), rs.grid_num, np.float32(rs.cell))
    _, counts = mt.marching_cubes(f, tuple(rs.grid_num), rs.grid_min.astype(np.float32), np.float32(rs.cell), 0.5,
                                  ref_rows=True, per_cube=True)
    assert len(g) == len(ref)
    k = 0
    for _, m in counts:
        assert np.array_equal(np.unique(g[k:k + m].reshape(-1, 3), axis=0), np.unique(ref[k:k + m].reshape(-1, 3), axis=0))
        k += m


def test_gpu_mesh_of_a_sphere_is_closed():
    from graphics_b200.surface import surface_field
    sf = surface_field()
    sf.surface_setup((0, 0, 0), (1, 1, 1), R_P, R_H, 1.0 / 32)
    num = sf.get_grid_num()
    mn = sf.get_grid_min()
    z, y, x = np.meshgrid(*[mn[a] + np.arange(num[a]) * sf.get_cell_size() for a in (2, 1, 0)], indexing="ij")
    f = np.sqrt((x - 0.5) ** 2 + (y - 0.5) ** 2 + (z - 0.5) ** 2).astype(np.float32)
    sf.set_field(f)
    tris = sf.mesh(0.3).astype(np.float64)
    assert closed_and_oriented(tris, 1e-6)
    vol = np.einsum("ij,ij->i", tris[:, 0], np.cross(tris[:, 1], tris[:, 2])).sum() / 6.0
    assert abs(abs(vol) - 4 / 3 * np.pi * 0.3 ** 3) < 0.02 * 4 / 3 * np.pi * 0.3 ** 3


def test_isotropic_field_integral():
    """Each particle's kernel integrates to its volume r_p^3: the field summed
    over the nodes times cell^3 is n r_p^3 (to the quadrature error)."""
    from graphics_b200.surface import surface_field
    pos = lattice_block((40, 40, 40), R_P, lo=(0.0, 0.0, 0.0), jitter=0.2, seed=3)
    sf = surface_field()
    sf.surface_setup(pos.min(0), pos.max(0), R_P, R_H, R_P / 4)
    sf.surface_isotro(pos)
    tot = sf.get_field().astype(np.float64).sum() * sf.get_cell_size() ** 3
    assert abs(tot - len(pos) * R_P ** 3) < 0.01 * len(pos) * R_P ** 3
    sf.surface_aniso(pos)
    assert np.isfinite(sf.get_field()).all()


def test_cpp_dropin_matches_python_path(tmp_path):
    """include/sphgpu_surface.hpp driven as the reconstruction driver drives
    surface_field and marchingCubes (tests/cpp/surface_dropin_main.cpp): the
    same field and triangles as the Python mirror, bit for bit."""
    import struct
    import subprocess
    from graphics_b200.surface import surface_field
    from helpers import build_surface_dropin
    exe = build_surface_dropin(tmp_path)
    pos = blob(seed=4).astype(np.float32)
    with open(tmp_path / "in.bin", "wb") as f:
        f.write(struct.pack("i", len(pos)) + pos.tobytes())
    r = subprocess.run([exe, str(tmp_path / "in.bin"), str(tmp_path / "f.bin"), str(tmp_path / "t.bin")],
                       capture_output=True, timeout=300)
    assert r.returncode == 0, r.stderr.decode()[-2000:]
    raw = open(tmp_path / "f.bin", "rb").read()
    num = np.frombuffer(raw[:12], np.int32)
    field = np.frombuffer(raw[12:], np.float32)
    tris = np.fromfile(tmp_path / "t.bin", np.float32).reshape(-1, 3, 3)
    sf = surface_field()
    p64 = pos.astype(np.float64)
    sf.surface_setup(p64.min(0), p64.max(0), 0.01, 0.02, 0.005)
    np.testing.assert_array_equal(sf.get_grid_num(), num)
    sf.surface_aniso(pos)
    np.testing.assert_array_equal(sf.get_field().ravel(), field)
    g = sf.mesh(0.5)
    assert len(g) > 100
    np.testing.assert_array_equal(g, tris)
    sf.close()
