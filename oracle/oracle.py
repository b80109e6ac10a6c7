"""ctypes front end for the CPU oracles (TEST INFRASTRUCTURE ONLY).

Two back ends share one interface:
  * "port"      -- oracle/sph_oracle.c, the C restatement of the reference's
                   SPH hot path (liboracle.so float, liboracle_f64.so double);
  * "reference" -- the reference's own solver sources compiled by
                   oracle/build_ref.py (oracle/_ref/libref_<solver>[_f64].so).

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use this
module, and only as the checker or the timed CPU baseline.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
LOG_DIR = os.path.join(REF_DIR, "logs")

_dbl3 = C.c_double * 3


class RefParams(C.Structure):
    """Mirror of RefParams in refshim/ref_harness.cpp (m_TH fields)."""
    _fields_ = [("spacing_r", C.c_double), ("smoothRadius_h", C.c_double), ("dt", C.c_double),
                ("gravity", _dbl3), ("densityErro_eta", C.c_double), ("soundSpeed_cs", C.c_double),
                ("nu", C.c_double), ("th_h", C.c_double), ("th_r", C.c_double), ("th_bt", C.c_double),
                ("spaceMin", _dbl3), ("spaceMax", _dbl3)]


class RefParamsV(C.Structure):
    """RefParams of the reference harness (RefParams + the vorticity
    options; the restatement's OrcParams starts with the first part)."""
    _fields_ = RefParams._fields_ + [("enable_vortex", C.c_int), ("alpha", C.c_double), ("zeta", C.c_double),
                                     ("nu_t", C.c_double)]


class OrcParams(C.Structure):
    """Mirror of OrcParams in sph_oracle.c."""
    _fields_ = RefParams._fields_ + [
        ("cap", C.c_int), ("float_err", C.c_int),
        ("df_density_goal", C.c_double), ("df_density_min_iter", C.c_int), ("df_density_max_iter", C.c_int),
        ("df_div_goal_abs", C.c_double), ("df_div_goal_rel", C.c_double),
        ("df_div_min_iter", C.c_int), ("df_div_max_iter", C.c_int),
        ("cfl", C.c_int), ("cfl_factor", C.c_double), ("dt_max", C.c_double), ("dt_min", C.c_double),
        ("wc_gamma", C.c_double),
        ("pci_eta", C.c_double), ("pci_min_iter", C.c_int), ("pci_max_iter", C.c_int),
        ("ii_omega", C.c_double), ("ii_eta_rel", C.c_double), ("ii_min_iter", C.c_int), ("ii_max_iter", C.c_int),
        ("ii_compat", C.c_int),
        ("iv_kvisc", C.c_double), ("iv_kvisc_b", C.c_double), ("iv_cv_goal", C.c_double),
        ("iv_div_goal", C.c_double), ("iv_cv_min_iter", C.c_int), ("iv_cv_max_iter", C.c_int),
        ("iv_div_min_iter", C.c_int), ("iv_div_max_iter", C.c_int)]


def build():
    """Build the restatement (always) and the reference (when its sources are
    present in this container)."""
    subprocess.check_call(["make", "-s", "-C", HERE])
    subprocess.check_call(["python3", os.path.join(HERE, "build_ref.py")])


def default_params(scene=None, **kw):
    """Parameters shared by both back ends, defaulting to the reference's
    DFSPH conventions (see graphics_b200.scene for the geometry mapping)."""
    p = dict(spacing_r=0.05, smoothRadius_h=0.1, dt=2.5e-4, gravity=(0.0, -9.81, 0.0),
             densityErro_eta=0.01, soundSpeed_cs=100.0, nu=1e-3, th_h=0.0, th_r=0.0, th_bt=0.0,
             spaceMin=(0.0, 0.0, 0.0), spaceMax=(1.0, 1.0, 1.0),
             cap=48, float_err=0, df_density_goal=1e-4, df_density_min_iter=2, df_density_max_iter=100,
             df_div_goal_abs=2.5, df_div_goal_rel=1e-3, df_div_min_iter=1, df_div_max_iter=30,
             cfl=0, cfl_factor=0.4, dt_max=5e-3, dt_min=1e-6, wc_gamma=7.0,
             pci_eta=0.01, pci_min_iter=3, pci_max_iter=10,
             ii_omega=0.5, ii_eta_rel=1e-3, ii_min_iter=2, ii_max_iter=100, ii_compat=0,
             iv_kvisc=0.1, iv_kvisc_b=0.1, iv_cv_goal=1e-4, iv_div_goal=1e-3, iv_cv_min_iter=3,
             iv_cv_max_iter=100, iv_div_min_iter=2, iv_div_max_iter=50)
    if scene is not None:
        p.update(spacing_r=scene.spacing_r, smoothRadius_h=scene.smooth_radius,
                 spaceMin=scene.space_min, spaceMax=scene.space_max)
    p.update(kw)
    return p


def _fill(struct, p):
    s = struct()
    for name, _ in struct._fields_:
        if name in p:
            v = p[name]
            if isinstance(v, (tuple, list, np.ndarray)):
                getattr(s, name)[:] = [float(x) for x in v]
            else:
                setattr(s, name, v)
    return s


class Oracle:
    """One scene in either back end.

    kind:  "port" (restatement) or "reference" (compiled reference)
    solver: for "reference": dfsph | dfsph_capped | wcsph | pcisph | iisphm | iisph
    f64:   double-precision build
    """

    _libs = {}

    def __init__(self, params, kind="port", solver="dfsph", f64=False):
        self.kind, self.solver, self.f64 = kind, solver, f64
        self.p = dict(params)
        self.lib = self._load(kind, solver, f64)
        if kind == "port":
            self._ps = _fill(OrcParams, self.p)
            self.h = self.lib.orc_create(C.byref(self._ps))
            self.cap = int(self.p.get("cap", 48))
        else:
            os.makedirs(LOG_DIR, exist_ok=True)
            self._ps = _fill(RefParamsV, self.p)
            self.h = self.lib.ref_create(C.byref(self._ps), LOG_DIR.encode())
            self.cap = 48
            if self.h and solver == "pcisph":
                self.lib.ref_set_iter_limits(self.h, int(self.p.get("pci_min_iter", 3)),
                                             int(self.p.get("pci_max_iter", 10)))
        if not self.h:
            raise RuntimeError("oracle creation failed")
        self.nfluid_phases = 0

    @classmethod
    def _load(cls, kind, solver, f64):
        if kind == "port":
            name = os.path.join(HERE, "liboracle_f64.so" if f64 else "liboracle.so")
            pre = "orc_"
        else:
            name = os.path.join(REF_DIR, "libref_%s%s.so" % (solver, "_f64" if f64 else ""))
            pre = "ref_"
        if name in cls._libs:
            return cls._libs[name]
        if not os.path.exists(name):
            raise FileNotFoundError(name + " (run `make -C oracle` / oracle/build_ref.py)")
        lib = C.CDLL(name)
        vp, ip, dp, cp, i, d = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double), C.c_char_p, C.c_int, C.c_double
        llp = C.POINTER(C.c_longlong)
        sig = {
            "create": (vp, [vp] if kind == "port" else [vp, cp]),
            "destroy": (None, [vp]),
            "add_solid": (i, [vp, i, dp, d, d, d, i]),
            "add_fluid": (i, [vp, i, dp, dp, d, d, d, d]),
            "num_fluid": (i, [vp, i]),
            "num_solid": (i, [vp, i]),
            "stage": (i, [vp, cp]),
            "get": (i, [vp, i, cp, dp]),
            "set": (i, [vp, i, cp, dp]),
            "get_solid": (i, [vp, i, cp, dp]),
            "neighbours": (i, [vp, i, i, ip, ip, ip, dp]),
            "cells": (i, [vp, i, i, llp]),
            "grid_info": (None, [vp, dp, dp, llp]),
            "set_dt": (None, [vp, d]),
            "set_frame": (None, [vp, i]),
            "kernel": (d, [vp, i, d]),
            "threads": (i, []),
        }
        for k, (res, args) in sig.items():
            f = getattr(lib, pre + k)
            f.restype, f.argtypes = res, args
        if kind == "port":
            lib.orc_error_counts.argtypes = [vp, llp, llp]
            lib.orc_stats.argtypes = [vp, ip, dp, dp, ip]
            lib.orc_set_solid.argtypes = [vp, i, cp, dp]
            lib.orc_set_solid.restype = i
            lib.orc_pci_delta.argtypes = [vp]
            lib.orc_pci_delta.restype = d
            lib.orc_vf_stats.argtypes = [vp, ip, dp]
            lib.orc_vf_stats.restype = None
        else:
            lib.ref_error_counts.argtypes = [vp, ip, ip]
            lib.ref_frame.restype = i
            lib.ref_frame.argtypes = [vp]
            lib.ref_set_iter_limits.restype = i
            lib.ref_set_iter_limits.argtypes = [vp, i, i]
            lib.ref_set_threads.restype = None
            lib.ref_set_threads.argtypes = [i]
            lib.ref_vf_iters.restype = i
            lib.ref_vf_iters.argtypes = [vp, ip, ip]
            lib.ref_set_solid.restype = i
            lib.ref_set_solid.argtypes = [vp, i, cp, dp]
        cls._libs[name] = lib
        return lib

    def _f(self, name):
        return getattr(self.lib, ("orc_" if self.kind == "port" else "ref_") + name)

    def close(self):
        if self.h:
            self._f("destroy")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _dp(a):
        return a.ctypes.data_as(C.POINTER(C.c_double))

    def add_solid(self, pos, d, visc_alpha=0.0, rho0=1000.0, prepare=True):
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        return self._f("add_solid")(self.h, len(pos), self._dp(pos), float(d), float(visc_alpha), float(rho0),
                                    int(prepare))

    def add_fluid(self, pos, vel=None, d=0.05, rho0=1000.0, visc_alpha=0.0, tension=0.0):
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        vel = None if vel is None else np.ascontiguousarray(vel, dtype=np.float64)
        k = self._f("add_fluid")(self.h, len(pos), self._dp(pos), None if vel is None else self._dp(vel),
                                 float(d), float(rho0), float(visc_alpha), float(tension))
        self.nfluid_phases = k + 1
        return k

    def n_fluid(self, k=0):
        return self._f("num_fluid")(self.h, k)

    def n_solid(self, k=0):
        return self._f("num_solid")(self.h, k)

    def stage(self, name):
        rc = self._f("stage")(self.h, name.encode())
        if rc != 0:
            raise ValueError("unknown stage %s for %s/%s" % (name, self.kind, self.solver))

    def get(self, field, k=0):
        n = self.n_fluid(k)
        out = np.zeros(3 * n + 3, dtype=np.float64)
        if self._f("get")(self.h, k, field.encode(), self._dp(out)) != 0:
            raise KeyError(field)
        vec = field in ("position", "velocity", "vel_adv", "acce_adv", "acceleration", "DFalpha1", "n",
                        "pos_prediction", "acce_pressure", "dii", "sum_dijpj", "advectionVelocity",
                        "acce_presure", "advectionAcceleration", "DF_alpha1", "VF_alpha1", "omega",
                        "angular_velocity", "dOmega", "n0Vorticity", "deltaVorticity", "psi", "vorticity")
        return out[:3 * n].reshape(n, 3) if vec else out[:n]

    def set(self, field, values, k=0):
        v = np.ascontiguousarray(values, dtype=np.float64).ravel()
        if self._f("set")(self.h, k, field.encode(), self._dp(v)) != 0:
            raise KeyError(field)

    def get_solid(self, field, k=0):
        n = self.n_solid(k)
        out = np.zeros(3 * n + 3, dtype=np.float64)
        if self._f("get_solid")(self.h, k, field.encode(), self._dp(out)) != 0:
            raise KeyError(field)
        vec = field in ("position", "velocity", "force", "singleVelocity")
        return out[:3 * n].reshape(n, 3) if vec else out[:n]

    def neighbours(self, kind=0, k=0):
        """(counts[n], t[n,cap], i[n,cap], dis[n,cap]) in list order."""
        n = self.n_fluid(k) if kind == 0 else self.n_solid(k)
        cap = self.cap
        counts = np.zeros(n + 1, dtype=np.int32)
        t = np.zeros(n * cap + 1, dtype=np.int32)
        i = np.zeros(n * cap + 1, dtype=np.int32)
        dis = np.zeros(n * cap + 1, dtype=np.float64)
        ip = C.POINTER(C.c_int)
        self._f("neighbours")(self.h, kind, k, counts.ctypes.data_as(ip), t.ctypes.data_as(ip),
                              i.ctypes.data_as(ip), self._dp(dis))
        return counts[:n], t[:n * cap].reshape(n, cap), i[:n * cap].reshape(n, cap), dis[:n * cap].reshape(n, cap)

    def cells(self, kind=0, k=0):
        n = self.n_fluid(k) if kind == 0 else self.n_solid(k)
        out = np.zeros(n + 1, dtype=np.int64)
        self._f("cells")(self.h, kind, k, out.ctypes.data_as(C.POINTER(C.c_longlong)))
        return out[:n]

    def grid_info(self):
        mn = np.zeros(3)
        dv = np.zeros(1)
        num = np.zeros(3, dtype=np.int64)
        self._f("grid_info")(self.h, self._dp(mn), self._dp(dv), num.ctypes.data_as(C.POINTER(C.c_longlong)))
        return mn, float(dv[0]), num

    def set_dt(self, dt):
        self._f("set_dt")(self.h, float(dt))

    def set_frame(self, f):
        self._f("set_frame")(self.h, int(f))

    def kernel(self, r, grad=False):
        return self._f("kernel")(self.h, int(grad), float(r))

    def error_counts(self):
        if self.kind == "port":
            a, b = C.c_longlong(), C.c_longlong()
        else:
            a, b = C.c_int(), C.c_int()
        self._f("error_counts")(self.h, C.byref(a), C.byref(b))
        return a.value, b.value

    def stats(self):
        """(iters[4], errs[4], dt, frame) of the last step (port only)."""
        it = (C.c_int * 4)()
        er = (C.c_double * 4)()
        dt = C.c_double()
        fr = C.c_int()
        self.lib.orc_stats(self.h, it, er, C.byref(dt), C.byref(fr))
        return list(it), list(er), dt.value, fr.value

    def threads(self):
        return self._f("threads")()

    def pci_delta(self):
        """PCISPH delta / dt^2 of the last pci_updateDelta (port only)."""
        return float(self.lib.orc_pci_delta(self.h))

    def vf_iters(self):
        """IISph: (divergence-free, constant-volume) iterations.  Reference
        build: m_TH.dF_iteration / cV_iteration accumulated since the last
        call (each loop adds its iterations - 1; read and reset).  Port: the
        iterations of the last loops, summed over phases."""
        if self.kind == "port":
            return self.vf_stats()[0]
        a, b = C.c_int(), C.c_int()
        self.lib.ref_vf_iters(self.h, C.byref(a), C.byref(b))
        return a.value, b.value

    def df_iters(self):
        """Reference "dfsph_capped" build: (density, divergence) loop
        iterations summed since the last call (read and reset)."""
        a, b = C.c_int(), C.c_int()
        if self.lib.ref_df_iters(C.byref(a), C.byref(b)) != 0:
            raise RuntimeError("iteration counts exist in the dfsph_capped reference build only")
        return a.value, b.value

    def vf_stats(self):
        """Port only: ((it_div, it_cv), (err_div, err_cv)) of the last IISph loops."""
        it = (C.c_int * 2)()
        er = (C.c_double * 2)()
        self.lib.orc_vf_stats(self.h, it, er)
        return (it[0], it[1]), (er[0], er[1])

    def set_solid(self, field, values, k=0):
        v = np.ascontiguousarray(values, dtype=np.float64).ravel()
        if self._f("set_solid")(self.h, k, field.encode(), self._dp(v)) != 0:
            raise KeyError(field)

    def set_threads(self, n):
        """OpenMP threads of the compiled reference (process-wide)."""
        self.lib.ref_set_threads(int(n))

    # -- dynamic rigid solids (SphWithBullet::updateSolids with a host world) --
    def _rigid_sigs(self):
        vp, dp, i = C.c_void_p, C.POINTER(C.c_double), C.c_int
        pre = "orc_" if self.kind == "port" else "ref_"
        for name, res, args in (("set_solid_dynamic", i, [vp, i, dp, dp]),
                                ("set_rigid_callback", None, [vp, vp, vp]),
                                ("rigid_force_join", i, [vp, i, dp, dp, dp]),
                                ("rigid_error", i, [vp])):
            f = getattr(self.lib, pre + name)
            f.restype, f.argtypes = res, args

    def set_solid_dynamic(self, k, inner, state):
        """Solid k becomes a dynamic rigid body: body-frame positions inner
        (n, 3), 25-value state (transform[16], com, v, w)."""
        self._rigid_sigs()
        inner = np.ascontiguousarray(inner, dtype=np.float64)
        st = np.ascontiguousarray(state, dtype=np.float64)
        if self._f("set_solid_dynamic")(self.h, int(k), self._dp(inner), self._dp(st)) != 0:
            raise ValueError("set_solid_dynamic")

    def set_rigid_world(self, world):
        """Drive the dynamic solids with a graphics_b200.rigid.RigidWorld."""
        self._rigid_sigs()
        self._rigid_cb = world.double_callback()
        self._f("set_rigid_callback")(self.h, C.cast(self._rigid_cb, C.c_void_p), None)

    def rigid_force_join(self, k, com):
        self._rigid_sigs()
        c = np.ascontiguousarray(com, dtype=np.float64)
        f, t = np.zeros(3), np.zeros(3)
        self._f("rigid_force_join")(self.h, int(k), self._dp(c), self._dp(f), self._dp(t))
        return f, t

    def rigid_error(self):
        self._rigid_sigs()
        return self._f("rigid_error")(self.h)


def make_scene_oracle(scene, kind="port", solver="dfsph", f64=False, visc_alpha=0.0, solid_visc=0.0, **kw):
    """Oracle holding `scene` (graphics_b200.scene.Scene): the walls are added
    first as static rigid solids (one, or one per scene.meta["solid_id"]
    value; their volumes come from boundary neighbours only), then one fluid
    phase per rest density."""
    p = default_params(scene, **kw)
    o = Oracle(p, kind=kind, solver=solver, f64=f64)
    sid = scene.meta.get("solid_id")
    if sid is None:
        o.add_solid(scene.boundary_pos, scene.d, visc_alpha=solid_visc, rho0=scene.rho0, prepare=True)
    else:
        # one solid per id, in id order (each addSolid prepares all solids)
        for k in range(int(sid.max()) + 1):
            o.add_solid(scene.boundary_pos[sid == k], scene.d, visc_alpha=solid_visc, rho0=scene.rho0, prepare=True)
    if scene.phase is None:
        o.add_fluid(scene.fluid_pos, scene.fluid_vel, d=scene.d, rho0=scene.rho0, visc_alpha=visc_alpha)
    else:
        for ph, rho in enumerate(scene.rho0_phases):
            m = scene.phase == ph
            o.add_fluid(scene.fluid_pos[m], scene.fluid_vel[m], d=scene.d, rho0=rho, visc_alpha=visc_alpha)
    return o


class RefSurface:
    """The reference's surface_field and marchingCubes compiled from its
    sources (oracle/_ref/libref_surface.so; TNT/JAMA replaced by the stand-in
    refshim/jama_svd.h).  The reference keeps its spline constants in
    function-local statics (surface_field.cpp:237-241, 255): one radius per
    process.  surface_aniso prints a progress line every 1 % of the particles
    and divides by n / 100, so it needs at least 100 particles."""

    _lib = None

    @classmethod
    def load(cls):
        if cls._lib is None:
            name = os.path.join(REF_DIR, "libref_surface.so")
            if not os.path.exists(name):
                raise FileNotFoundError(name + " (run oracle/build_ref.py)")
            lib = C.CDLL(name)
            dp, fp, ip = C.POINTER(C.c_double), C.POINTER(C.c_float), C.POINTER(C.c_int)
            lib.rsf_create.restype = C.c_void_p
            lib.rsf_create.argtypes = [dp, dp, C.c_double, C.c_double, C.c_double]
            lib.rsf_destroy.argtypes = [C.c_void_p]
            lib.rsf_grid.argtypes = [C.c_void_p, dp, ip, dp]
            lib.rsf_field.restype = C.c_longlong
            lib.rsf_field.argtypes = [C.c_void_p, C.c_int, dp, C.c_int, fp]
            lib.rsf_marching_cubes.restype = C.c_longlong
            lib.rsf_marching_cubes.argtypes = [C.c_float, fp, fp, ip, C.c_float, fp, C.c_longlong]
            cls._lib = lib
        return cls._lib

    def __init__(self, mn, mx, r_p, r_h, cell):
        lib = self.load()
        dp = C.POINTER(C.c_double)
        a = np.asarray(mn, np.float64)
        b = np.asarray(mx, np.float64)
        self.h = lib.rsf_create(a.ctypes.data_as(dp), b.ctypes.data_as(dp), r_p, r_h, cell)
        g = np.zeros(3)
        n = np.zeros(3, np.int32)
        c = C.c_double()
        lib.rsf_grid(self.h, g.ctypes.data_as(dp), n.ctypes.data_as(C.POINTER(C.c_int)), C.byref(c))
        self.grid_min, self.grid_num, self.cell = g, n, c.value

    def field(self, positions, aniso=True):
        lib = self.load()
        p = np.ascontiguousarray(positions, np.float64)
        out = np.zeros(int(np.prod(self.grid_num)), np.float32)
        lib.rsf_field(self.h, int(aniso), p.ctypes.data_as(C.POINTER(C.c_double)), len(p),
                      out.ctypes.data_as(C.POINTER(C.c_float)))
        return out

    @classmethod
    def marching_cubes(cls, iso, field, grid_min, grid_num, cell, max_tris=None):
        lib = cls.load()
        f = np.ascontiguousarray(field, np.float32)
        mn = np.asarray(grid_min, np.float32)
        res = np.asarray(grid_num, np.int32)
        fp = C.POINTER(C.c_float)
        n = lib.rsf_marching_cubes(float(iso), f.ctypes.data_as(fp), mn.ctypes.data_as(fp),
                                   res.ctypes.data_as(C.POINTER(C.c_int)), float(cell), None, 0)
        out = np.zeros((max(n, 1), 3, 3), np.float32)
        lib.rsf_marching_cubes(float(iso), f.ctypes.data_as(fp), mn.ctypes.data_as(fp),
                               res.ctypes.data_as(C.POINTER(C.c_int)), float(cell), out.ctypes.data_as(fp), n)
        return out[:n]

    def close(self):
        if self.h:
            self.load().rsf_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
