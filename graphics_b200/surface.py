"""Surface reconstruction on the GPU: the host-side mirror of the
reference's surface_field class (surface_field.h:34-80) and its
marchingCubes function (marching_cubes.h:16-17), as its driver re.c uses
them (surface_setup, surface_aniso / surface_isotro, get_field /
get_grid_min / get_grid_num / get_cell_size, marchingCubes).

    sf = surface_field()
    sf.surface_setup(space_min, space_max, r_p, r_h, r_p / 4)
    sf.surface_aniso(positions)                 # (n, 3)
    tris = marchingCubes(0.5, sf)              # (T, 3, 3) float32
"""
import ctypes as C

import numpy as np

from . import _lib
from ._lib import SphGpuError


class surface_field:
    """GPU surface_field: the scalar field lives on the device."""

    def __init__(self, device=0):
        self.lib = _lib.load()
        self.h = None
        self.device = device

    def close(self):
        if self.h:
            self.lib.sphgpu_surface_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _err(self):
        buf = C.create_string_buffer(512)
        self.lib.sphgpu_surface_last_error(self.h, buf, 512)
        return buf.value.decode(errors="replace")

    def surface_setup(self, min3, max3, r_p, r_h, cell_size):
        self.close()
        mn = (C.c_double * 3)(*[float(x) for x in min3])
        mx = (C.c_double * 3)(*[float(x) for x in max3])
        h = C.c_void_p()
        rc = self.lib.sphgpu_surface_create(mn, mx, float(r_p), float(r_h), float(cell_size), int(self.device),
                                            C.byref(h))
        if rc:
            raise SphGpuError(rc, "sphgpu_surface_create failed")
        self.h = h
        g = (C.c_double * 3)()
        n = (C.c_int * 3)()
        c = C.c_double()
        self.lib.sphgpu_surface_grid(self.h, g, n, C.byref(c))
        self.grid_min, self.grid_num, self.cell_size = np.array(g[:]), np.array(n[:], np.int64), c.value

    def _field(self, aniso, position, on_device=False, n=None):
        if on_device:
            ptr, cnt = position, int(n)
        else:
            pos = np.ascontiguousarray(position, dtype=np.float32).reshape(-1, 3)
            self._keep = pos
            ptr, cnt = pos.ctypes.data, len(pos)
        rc = self.lib.sphgpu_surface_field(self.h, int(aniso), ptr, cnt, int(bool(on_device)))
        if rc and rc != _lib.EOUT_OF_DOMAIN:
            raise SphGpuError(rc, self._err())
        return rc

    def surface_isotro(self, position, **kw):
        return self._field(0, position, **kw)

    def surface_aniso(self, position, **kw):
        return self._field(1, position, **kw)

    def get_field(self):
        out = np.empty(int(np.prod(self.grid_num)), dtype=np.float32)
        rc = self.lib.sphgpu_surface_get_field(self.h, out.ctypes.data_as(C.POINTER(C.c_float)))
        if rc:
            raise SphGpuError(rc, self._err())
        return out

    def set_field(self, field):
        f = np.ascontiguousarray(field, dtype=np.float32).ravel()
        rc = self.lib.sphgpu_surface_set_field(self.h, f.ctypes.data_as(C.POINTER(C.c_float)))
        if rc:
            raise SphGpuError(rc, self._err())

    def get_grid_min(self):
        return self.grid_min

    def get_grid_num(self):
        return self.grid_num

    def get_cell_size(self):
        return self.cell_size

    def stats(self):
        """(tile-particle pairs of the last field, tiles, kernel launches so far)."""
        pairs, tiles, kern = C.c_longlong(), C.c_int(), C.c_longlong()
        self.lib.sphgpu_surface_stats(self.h, C.byref(pairs), C.byref(tiles), C.byref(kern))
        return pairs.value, tiles.value, kern.value

    def mesh(self, iso, ref_rows=False):
        """marchingCubes over the device field: (T, 3, 3) float32."""
        n = self.lib.sphgpu_surface_mesh(self.h, float(iso), int(bool(ref_rows)), None, 0)
        if n < 0:
            raise SphGpuError(n, self._err())
        out = np.empty((max(n, 1), 3, 3), dtype=np.float32)
        m = self.lib.sphgpu_surface_mesh(self.h, float(iso), int(bool(ref_rows)),
                                         out.ctypes.data_as(C.POINTER(C.c_float)), n)
        if m < 0:
            raise SphGpuError(m, self._err())
        return out[:m]


def marchingCubes(iso, sf, ref_rows=False):
    """marchingCubes(result, iso, sf.get_field(), ...) (marching_cubes.cpp:
    45-120) on the field held by `sf`."""
    return sf.mesh(iso, ref_rows)


def mc_table():
    """The library's marching-cubes case table: (ntri[256], tri[256, 16])."""
    lib = _lib.load()
    n = np.zeros(256, np.int32)
    t = np.zeros(256 * 16, np.int8)
    lib.sphgpu_mc_table(n.ctypes.data_as(C.POINTER(C.c_int)), t.ctypes.data_as(C.POINTER(C.c_byte)))
    return n, t.reshape(256, 16)
