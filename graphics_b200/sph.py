"""Host-side mirror of the reference's SPH solver interface, over the C ABI.

Reference interface (Artemisaturn/GRAPHICS, Source/):
  * SphBase (SphBase.h:373-802): pure virtual setupScene()/stepEvent()/
    sphStep(), runOneStep() (SphBase.cpp:348-354), m_TH thresholds
    (SphBase.h:546-583), m_EC error counters (SphBase.h:586-592), getters
    (SphBase.h:493-541), neighbourSearch() (SphBase.h:673).
  * Scene building of SphWithIO: addFluidCuboid (SphWithIO.cpp:149-194),
    addRigidCuboid (SphWithIO.cpp:642-659).
  * Solvers: WcSph, PciSph, IISph_M, DFSPH, each overriding sphStep().

A user subclasses a solver and fills setupScene(), exactly as the reference's
scenes do (Demo-mySPH.h:17-126); sphStep() then runs on the GPU.  Particle
arrays are exposed as numpy arrays in the reference's particle order.

`GpuScene` is the thin object wrapper over one sphgpu handle; the solver
classes use it and tests/bench use it directly.
"""
import ctypes as C
import os

import numpy as np

from . import _lib
from ._lib import SphParams, SphStepStats, SphGpuError

SOLVERS = {"wcsph": _lib.WCSPH, "pcisph": _lib.PCISPH, "iisph_m": _lib.IISPH_M, "dfsph": _lib.DFSPH,
           "iisph": _lib.IISPH}

VEC_FIELDS = ("position", "velocity", "vel_adv", "acce_adv", "acceleration", "ws_hist", "acce_pressure",
              "pos_prediction", "dii", "sum_dijpj", "ii_vel_adv", "acce_presure", "advectionAcceleration",
              "advectionVelocity", "omega", "dOmega", "angular_velocity", "n0Vorticity", "deltaVorticity", "psi")


def _fptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def default_params():
    p = SphParams()
    rc = _lib.load().sphgpu_params_default(C.byref(p))
    if rc:
        raise SphGpuError(rc, "params_default")
    return p


def params_for_scene(scene, **kw):
    """SphParams for a graphics_b200.scene.Scene: spacing_r = d = 2r,
    smoothRadius_h = 2d, particle diameter d; keyword overrides by field name."""
    p = default_params()
    p.spacing_r = scene.spacing_r
    p.smoothRadius_h = scene.smooth_radius
    p.particle_d = scene.d
    p.gravity[:] = [0.0, -9.81, 0.0]
    p.spaceMin[:] = list(scene.space_min)
    p.spaceMax[:] = list(scene.space_max)
    set_params(p, **kw)
    return p


def set_params(p, **kw):
    for k, v in kw.items():
        if not hasattr(p, k):
            raise AttributeError("SphParams has no field " + k)
        if isinstance(v, (tuple, list, np.ndarray)):
            getattr(p, k)[:] = [float(x) for x in v]
        else:
            setattr(p, k, v)
    return p


class GpuScene:
    """One SPH scene resident on a GPU (one sphgpu handle)."""

    def __init__(self, params, max_fluid, device=0):
        self.lib = _lib.load()
        self.params = params
        h = C.c_void_p()
        rc = self.lib.sphgpu_create(C.byref(params), int(device), int(max_fluid), C.byref(h))
        if rc:
            raise SphGpuError(rc, "sphgpu_create failed (is a CUDA device present?)")
        self.h = h
        self.nb = 0

    # -- lifetime --
    def close(self):
        if getattr(self, "h", None):
            self.lib.sphgpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _err(self):
        buf = C.create_string_buffer(1024)
        self.lib.sphgpu_last_error(self.h, buf, 1024)
        return buf.value.decode(errors="replace")

    def _check(self, rc, what, allow=()):
        if rc < 0 and rc not in allow:
            raise SphGpuError(rc, "%s: %s" % (what, self._err()))
        return rc

    # -- scene --
    def set_params(self, params):
        self.params = params
        self._check(self.lib.sphgpu_set_params(self.h, C.byref(params)), "set_params")

    def set_boundary(self, pos, solid_id=None, volume=None):
        pos = np.ascontiguousarray(pos, dtype=np.float32)
        sid = None if solid_id is None else np.ascontiguousarray(solid_id, dtype=np.int32)
        vol = None if volume is None else np.ascontiguousarray(volume, dtype=np.float32)
        rc = self.lib.sphgpu_set_boundary(self.h, len(pos), _fptr(pos),
                                          None if sid is None else sid.ctypes.data_as(C.POINTER(C.c_int)),
                                          None if vol is None else _fptr(vol))
        self._check(rc, "set_boundary")
        self.nb = len(pos)

    def add_fluid(self, pos, vel=None, rho0=1000.0, visc_alpha=0.0):
        pos = np.ascontiguousarray(pos, dtype=np.float32)
        vel = None if vel is None else np.ascontiguousarray(vel, dtype=np.float32)
        return self._check(self.lib.sphgpu_add_fluid(self.h, len(pos), _fptr(pos),
                                                     None if vel is None else _fptr(vel), float(rho0),
                                                     float(visc_alpha)), "add_fluid")

    @property
    def n_fluid(self):
        return self._check(self.lib.sphgpu_num_fluid(self.h), "num_fluid")

    # -- stepping --
    def step(self, solver="dfsph", nsteps=1, allow_maxiter=True):
        st = SphStepStats()
        rc = self.lib.sphgpu_step(self.h, SOLVERS.get(solver, solver), int(nsteps), C.byref(st))
        self._check(rc, "step", allow=(_lib.EMAXITER,) if allow_maxiter else ())
        d = st.as_dict()
        d["rc"] = rc
        return d

    def step_async(self, solver="dfsph", nsteps=1):
        self._check(self.lib.sphgpu_step_async(self.h, SOLVERS.get(solver, solver), int(nsteps)), "step_async")

    def synchronize(self, allow_maxiter=True):
        st = SphStepStats()
        rc = self.lib.sphgpu_synchronize(self.h, C.byref(st))
        self._check(rc, "synchronize", allow=(_lib.EMAXITER,) if allow_maxiter else ())
        d = st.as_dict()
        d["rc"] = rc
        return d

    def step_host(self, solver, pos, vel, pos_out, vel_out):
        st = SphStepStats()
        rc = self.lib.sphgpu_step_host(self.h, SOLVERS.get(solver, solver), _fptr(pos), _fptr(vel),
                                       _fptr(pos_out), _fptr(vel_out), C.byref(st))
        self._check(rc, "step_host", allow=(_lib.EMAXITER,))
        return st.as_dict()

    def stage(self, name):
        st = SphStepStats()
        rc = self.lib.sphgpu_stage(self.h, name.encode(), C.byref(st))
        self._check(rc, "stage " + name, allow=(_lib.EMAXITER,))
        d = st.as_dict()
        d["rc"] = rc
        return d

    # -- fields --
    def get(self, field):
        n = self.n_fluid
        comps = 3 if field in VEC_FIELDS else (_lib.MLP_IN if field == "ws_features" else 1)
        out = np.zeros(max(n, 1) * comps, dtype=np.float32)
        m = self._check(self.lib.sphgpu_get_fluid(self.h, field.encode(), _fptr(out)), "get " + field)
        return out[:m * comps].reshape(m, comps) if comps > 1 else out[:m]

    def set(self, field, values):
        v = np.ascontiguousarray(values, dtype=np.float32).ravel()
        self._check(self.lib.sphgpu_set_fluid(self.h, field.encode(), _fptr(v)), "set " + field)

    # -- output and restart --
    def write_pos(self, path, phase=0, components=("position",), log_name=""):
        """The reference's .pos file of one fluid phase (sphgpu_write_pos)."""
        rc = self.lib.sphgpu_write_pos(self.h, os.fspath(path).encode(), int(phase), " ".join(components).encode(),
                                       log_name.encode())
        return self._check(rc, "write_pos")

    def save_snapshot(self, path):
        """Checkpoint of the scene (sphgpu_save_snapshot)."""
        self._check(self.lib.sphgpu_save_snapshot(self.h, os.fspath(path).encode()), "save_snapshot")

    @classmethod
    def load_snapshot(cls, path, device=0):
        """A new scene continuing a saved one (sphgpu_load_snapshot)."""
        lib = _lib.load()
        h = C.c_void_p()
        rc = lib.sphgpu_load_snapshot(os.fspath(path).encode(), int(device), C.byref(h))
        if rc:
            raise SphGpuError(rc, "sphgpu_load_snapshot failed")
        g = cls.__new__(cls)
        g.lib, g.h = lib, h
        with open(path, "rb") as f:
            f.read(8)
            hdr = np.frombuffer(f.read(32), np.int32)
            p = _lib.SphParams()
            C.memmove(C.byref(p), f.read(C.sizeof(p)), C.sizeof(p))
        g.params, g.nb = p, int(hdr[3])
        return g

    # -- dynamic rigid solids --
    def set_solid_dynamic(self, solid_id, inner, state):
        """Make solid `solid_id` a dynamic rigid body with body-frame
        particle positions `inner` and a 25-value initial state
        (sphgpu_set_solid_dynamic)."""
        from .rigid import state_struct
        inner = np.ascontiguousarray(inner, dtype=np.float32)
        st = state_struct(state)
        self._check(self.lib.sphgpu_set_solid_dynamic(self.h, int(solid_id), _fptr(inner), C.byref(st)),
                    "set_solid_dynamic")

    def set_rigid_world(self, world):
        """Drive the dynamic solids with `world` (graphics_b200.rigid.RigidWorld
        or any object with its gpu_callback()); None removes it."""
        self._rigid_cb = None if world is None else world.gpu_callback()
        fn = self._rigid_cb if self._rigid_cb is not None else _lib.RIGID_FN()
        self._check(self.lib.sphgpu_set_rigid_callback(self.h, fn, None), "set_rigid_callback")

    def set_solid_state(self, solid_id, state):
        from .rigid import state_struct
        st = state_struct(state)
        self._check(self.lib.sphgpu_set_solid_state(self.h, int(solid_id), C.byref(st)), "set_solid_state")

    def get_solid_state(self, solid_id):
        from .rigid import state_array
        st = _lib.SphRigidState()
        self._check(self.lib.sphgpu_get_solid_state(self.h, int(solid_id), C.byref(st)), "get_solid_state")
        return state_array(st)

    def get_solid_force(self, solid_id):
        """(force[3], torque[3]) of the last DFSPH step (rigidForceJoin)."""
        f = (C.c_double * 3)()
        t = (C.c_double * 3)()
        self._check(self.lib.sphgpu_get_solid_force(self.h, int(solid_id), f, t), "get_solid_force")
        return np.array(f[:]), np.array(t[:])

    def get_boundary(self, field):
        comps = 3 if field in ("position", "velocity", "force") else 1
        out = np.zeros(max(self.nb, 1) * comps, dtype=np.float32)
        m = self._check(self.lib.sphgpu_get_boundary(self.h, field.encode(), _fptr(out)), "get_boundary")
        return out[:m * comps].reshape(m, comps) if comps > 1 else out[:m]

    def neighbours(self):
        """(counts[n], t[n,cap], i[n,cap]) in the reference's PartIdx encoding."""
        n = self.n_fluid
        cap = int(self.params.max_neighbours)
        counts = np.zeros(max(n, 1), dtype=np.int32)
        t = np.zeros(max(n, 1) * cap, dtype=np.int32)
        i = np.zeros(max(n, 1) * cap, dtype=np.int32)
        ip = C.POINTER(C.c_int)
        self._check(self.lib.sphgpu_get_neighbours(self.h, counts.ctypes.data_as(ip), t.ctypes.data_as(ip),
                                                   i.ctypes.data_as(ip)), "get_neighbours")
        return counts[:n], t[:n * cap].reshape(n, cap), i[:n * cap].reshape(n, cap)

    def cells(self):
        out = np.zeros(max(self.n_fluid, 1), dtype=np.int64)
        m = self._check(self.lib.sphgpu_get_cells(self.h, out.ctypes.data_as(C.POINTER(C.c_longlong))), "cells")
        return out[:m]

    # -- profiling --
    def autotune(self, solver="dfsph", steps=3):
        """Pick block sizes per kernel class by measurement (sphgpu_autotune);
        advances the scene by 3 * steps steps.  Returns the JSON report."""
        import json
        buf = C.create_string_buffer(4096)
        self._check(self.lib.sphgpu_autotune(self.h, SOLVERS.get(solver, solver), int(steps), buf, 4096), "autotune")
        return json.loads(buf.value.decode())

    def profile(self, on=True):
        self._check(self.lib.sphgpu_profile(self.h, int(on)), "profile")

    def profile_read(self):
        cap, nl = 64, 64
        names = C.create_string_buffer(cap * nl)
        ms = (C.c_double * cap)()
        la = (C.c_int * cap)()
        k = self.lib.sphgpu_profile_read(self.h, names, nl, ms, la, cap)
        raw = names.raw
        out = {}
        for j in range(k):
            nm = raw[j * nl:(j + 1) * nl].split(b"\0", 1)[0].decode()
            out[nm] = (ms[j], la[j])
        return out

    def debug_set(self, key, value):
        self._check(self.lib.sphgpu_debug_set(self.h, key.encode(), int(value)), "debug_set " + key)


class GpuBatch(GpuScene):
    """Many independent DFSPH scenes in one handle (sphgpu_batch_*): one
    set of arrays, per-scene boxes, CFL steps and loop convergence."""

    def __init__(self, params, space_min, space_max, max_fluid, device=0):
        self.lib = _lib.load()
        self.params = params
        smin = np.ascontiguousarray(space_min, dtype=np.float32).reshape(-1, 3)
        smax = np.ascontiguousarray(space_max, dtype=np.float32).reshape(-1, 3)
        self.nscenes = len(smin)
        h = C.c_void_p()
        rc = self.lib.sphgpu_batch_create(C.byref(params), self.nscenes, _fptr(smin), _fptr(smax), int(device),
                                          int(max_fluid), C.byref(h))
        if rc:
            raise SphGpuError(rc, "sphgpu_batch_create failed (is a CUDA device present?)")
        self.h = h
        self.nb = 0

    def set_boundary(self, pos, scene):
        pos = np.ascontiguousarray(pos, dtype=np.float32)
        sc = np.ascontiguousarray(scene, dtype=np.int32)
        self._check(self.lib.sphgpu_batch_set_boundary(self.h, len(pos), _fptr(pos),
                                                       sc.ctypes.data_as(C.POINTER(C.c_int))), "batch_set_boundary")
        self.nb = len(pos)

    def add_fluid(self, pos, vel, scene, rho0=1000.0, visc_alpha=0.0):
        pos = np.ascontiguousarray(pos, dtype=np.float32)
        vel = np.ascontiguousarray(vel, dtype=np.float32)
        sc = np.ascontiguousarray(scene, dtype=np.int32)
        return self._check(self.lib.sphgpu_batch_add_fluid(self.h, len(pos), _fptr(pos), _fptr(vel),
                                                           sc.ctypes.data_as(C.POINTER(C.c_int)), float(rho0),
                                                           float(visc_alpha)), "batch_add_fluid")

    def scene_stats(self):
        out = (SphStepStats * self.nscenes)()
        m = self._check(self.lib.sphgpu_batch_stats(self.h, out, self.nscenes), "batch_stats")
        return [out[i].as_dict() for i in range(m)]

    def scene_range(self, k):
        a, b = C.c_int(), C.c_int()
        self._check(self.lib.sphgpu_batch_scene_range(self.h, int(k), C.byref(a), C.byref(b)), "batch_scene_range")
        return a.value, b.value

    def get_scene(self, field, k):
        a, n = self.scene_range(k)
        return self.get(field)[a:a + n]


def batch_to_gpu(scenes, device=0, max_fluid=None, **params):
    """GpuBatch holding a list of graphics_b200.scene.Scene (one phase each,
    same particle size and rest density), walls as each scene's static solid."""
    p = params_for_scene(scenes[0], **params)
    smin = np.array([sc.space_min for sc in scenes], np.float32)
    smax = np.array([sc.space_max for sc in scenes], np.float32)
    n = sum(sc.n_fluid for sc in scenes)
    b = GpuBatch(p, smin, smax, max_fluid or n, device=device)
    b.set_boundary(np.concatenate([sc.boundary_pos for sc in scenes]),
                   np.concatenate([np.full(len(sc.boundary_pos), k, np.int32) for k, sc in enumerate(scenes)]))
    b.add_fluid(np.concatenate([sc.fluid_pos for sc in scenes]), np.concatenate([sc.fluid_vel for sc in scenes]),
                np.concatenate([np.full(sc.n_fluid, k, np.int32) for k, sc in enumerate(scenes)]),
                rho0=scenes[0].rho0)
    return b


def read_pos(path):
    """A .pos file in the reference's format (read_fluid_particles,
    fUtility.h:486-510): (records as an (n, floats per particle) float32
    array, component mask, frame number)."""
    lib = _lib.load()
    n = lib.sphgpu_read_pos(os.fspath(path).encode(), None, 0, None, 0, None)
    if n < 0:
        raise SphGpuError(int(n), "read_pos " + os.fspath(path))
    mask = C.create_string_buffer(256)
    frame = C.c_int()
    size = os.path.getsize(path)
    buf = np.zeros(max(size // 4, 1), np.float32)
    n = lib.sphgpu_read_pos(os.fspath(path).encode(), _fptr(buf), len(buf), mask, 256, C.byref(frame))
    if n < 0:
        raise SphGpuError(int(n), "read_pos " + os.fspath(path))
    per = 0
    m = mask.value.decode()
    for word, k in (("position", 3), ("velocity", 3), ("color", 4), ("density", 1), ("presure", 1),
                    ("acceleration", 3), ("dt", 1)):
        if word in m:
            per += k
    return buf[:n * per].reshape(n, per), m, frame.value


def scene_to_gpu(scene, device=0, max_fluid=None, **params):
    """GpuScene holding a graphics_b200.scene.Scene (walls as one static
    solid, or one per scene.meta["solid_id"] value)."""
    p = params_for_scene(scene, **params)
    g = GpuScene(p, max_fluid or scene.n_fluid, device=device)
    g.set_boundary(scene.boundary_pos, scene.meta.get("solid_id"))
    if scene.phase is None:
        g.add_fluid(scene.fluid_pos, scene.fluid_vel, rho0=scene.rho0)
    else:
        for ph, rho in enumerate(scene.rho0_phases):
            m = scene.phase == ph
            g.add_fluid(scene.fluid_pos[m], scene.fluid_vel[m], rho0=rho)
    return g


# ---------------------------------------------------------------------------
# Mirror of the reference's class hierarchy
# ---------------------------------------------------------------------------

class Thresholds:
    """m_TH (SphBase.h:546-583) with the defaults of SphBase::SphBase
    (SphBase.cpp:214-225)."""

    def __init__(self):
        self.spacing_r = 0.1
        self.smoothRadius_h = 0.2
        self.spaceMin = np.zeros(3)
        self.spaceMax = np.ones(3)
        self.dt = 0.001
        self.gravity_g = np.array([0.0, -9.8, 0.0])
        self.densityErro_eta = 0.01
        self.soundSpeed_cs = 100.0
        self.nu = 0.0
        self.frameNumber = 0
        self.systemTime = 0.0


class ErrorCount:
    """m_EC (SphBase.h:586-592)."""

    def __init__(self):
        self.zeroDis = 0
        self.tooManyNeigb = 0
        self.hashCodeOfPos = 0


class SphBase:
    """Base of the GPU solvers; subclass and implement setupScene()."""

    SOLVER = None

    def __init__(self, device=0):
        self.m_TH = Thresholds()
        self.m_EC = ErrorCount()
        self.device = device
        self.particle_d = None
        self.max_neighbours = 48
        self.solver_params = {}
        self._fluids = []   # [pos, vel, rho0, viscosity]
        self._solids = []   # [pos, viscosity]
        self._gpu = None
        self.last_stats = None

    # --- pure virtuals of the reference ---
    def setupScene(self):
        raise NotImplementedError

    def stepEvent(self):
        pass

    # --- SphBase::runOneStep, SphBase.cpp:348-354 ---
    def runOneStep(self):
        self.stepEvent()
        self.sphStep()
        self.m_TH.frameNumber += 1
        self.m_TH.systemTime += self.m_TH.dt

    def sphStep(self):
        g = self._ensure_gpu()
        st = g.step(self.SOLVER, 1)
        self._absorb(st)

    def _absorb(self, st):
        self.last_stats = st
        self.m_TH.dt = st["dt"]
        self.m_EC.zeroDis += st["zero_distance"]
        self.m_EC.tooManyNeigb += st["neighbour_overflow"]

    # --- scene building (SphWithIO) ---
    def addFluidCuboid(self, newFluid, fluidIdx, leftBottom, rightTop, d, restDensity=1000.0, viscosity=0.05,
                       tension=0.0):
        """Lattice of spacing d in [leftBottom, rightTop] as in
        SphWithIO::addFluidCuboid (SphWithIO.cpp:149-194): num = int((rt-lb)/d)
        intervals, num+1 points per axis, centred."""
        lb = np.asarray(leftBottom, dtype=np.float32)
        rt = np.asarray(rightTop, dtype=np.float32)
        d = np.float32(d)
        num = ((rt - lb) / d).astype(np.int32)
        pmin = lb + (rt - lb - num.astype(np.float32) * d) * np.float32(0.5)
        ii = [np.arange(num[a] + 1, dtype=np.float32) for a in range(3)]
        zz, yy, xx = np.meshgrid(ii[2], ii[1], ii[0], indexing="ij")
        pos = np.stack([pmin[0] + xx.ravel() * d, pmin[1] + yy.ravel() * d, pmin[2] + zz.ravel() * d], 1)
        self.m_TH.spaceMin = np.minimum(self.m_TH.spaceMin, lb)
        self.m_TH.spaceMax = np.maximum(self.m_TH.spaceMax, rt)
        self.particle_d = float(d)
        if newFluid or not self._fluids:
            self._fluids.append([pos.astype(np.float32), np.zeros_like(pos, dtype=np.float32), restDensity, viscosity])
        else:
            f = self._fluids[fluidIdx]
            f[0] = np.concatenate([f[0], pos.astype(np.float32)])
            f[1] = np.concatenate([f[1], np.zeros_like(pos, dtype=np.float32)])

    def addFluidParts(self, fluidIdx, positions, velocities=None, restDensity=1000.0, viscosity=0.0):
        pos = np.asarray(positions, dtype=np.float32)
        vel = np.zeros_like(pos) if velocities is None else np.asarray(velocities, dtype=np.float32)
        if fluidIdx >= len(self._fluids):
            self._fluids.append([pos, vel, restDensity, viscosity])
        else:
            f = self._fluids[fluidIdx]
            f[0] = np.concatenate([f[0], pos])
            f[1] = np.concatenate([f[1], vel])

    def addBoundaryParts(self, positions, viscosity=0.0):
        """A static rigid solid made of the given boundary particles."""
        self._solids.append([np.asarray(positions, dtype=np.float32), viscosity])

    # --- GPU scene ---
    def _params(self):
        p = default_params()
        d = self.particle_d if self.particle_d else self.m_TH.spacing_r
        set_params(p, spacing_r=self.m_TH.spacing_r, smoothRadius_h=self.m_TH.smoothRadius_h, particle_d=d,
                   dt=self.m_TH.dt, gravity=self.m_TH.gravity_g, spaceMin=self.m_TH.spaceMin,
                   spaceMax=self.m_TH.spaceMax, soundSpeed_cs=self.m_TH.soundSpeed_cs, nu=self.m_TH.nu,
                   densityErro_eta=self.m_TH.densityErro_eta, max_neighbours=self.max_neighbours)
        if self._solids:
            p.boundary_visc = float(self._solids[0][1])
        set_params(p, **self.solver_params)
        return p

    def _ensure_gpu(self):
        if self._gpu is None:
            n = sum(len(f[0]) for f in self._fluids)
            g = GpuScene(self._params(), max(n, 1), device=self.device)
            if self._solids:
                pos = np.concatenate([s[0] for s in self._solids])
                sid = np.concatenate([np.full(len(s[0]), k, np.int32) for k, s in enumerate(self._solids)])
                g.set_boundary(pos, sid)
            for pos, vel, rho0, visc in self._fluids:
                g.add_fluid(pos, vel, rho0=rho0, visc_alpha=visc)
            self._gpu = g
        return self._gpu

    def neighbourSearch(self):
        self._ensure_gpu().stage("neighbourSearch")

    # --- getters, SphBase.h:493-541 ---
    def getSpacing_r(self):
        return self.m_TH.spacing_r

    def getSmoothRadius_h(self):
        return self.m_TH.smoothRadius_h

    def getSpaceMin(self):
        return self.m_TH.spaceMin

    def getSpaceMax(self):
        return self.m_TH.spaceMax

    def getDt(self):
        return self.m_TH.dt

    def getGravity_g(self):
        return self.m_TH.gravity_g

    def getDensityErro_eta(self):
        return self.m_TH.densityErro_eta

    def getFrameNumber(self):
        return self.m_TH.frameNumber

    def getSystemTime(self):
        return self.m_TH.systemTime

    def getErrorCount(self):
        return self.m_EC.zeroDis + self.m_EC.tooManyNeigb

    def getErrorCountZeroDis(self):
        return self.m_EC.zeroDis

    def getErrorCountManyNeigb(self):
        return self.m_EC.tooManyNeigb

    def getNumFluids(self):
        return len(self._fluids)

    def getNumSolids(self):
        return len(self._solids)

    def getNumFluidParts(self):
        if self._gpu is not None:
            return self._gpu.n_fluid
        return sum(len(f[0]) for f in self._fluids)

    def getNumBounParts(self):
        return sum(len(s[0]) for s in self._solids)

    def getNumParts(self):
        return self.getNumFluidParts() + self.getNumBounParts()

    def getFluidParticles(self, i):
        """Fields of fluid phase i as numpy arrays (reference order)."""
        if self._gpu is None:
            pos, vel = self._fluids[i][0], self._fluids[i][1]
            return {"position": pos, "velocity": vel}
        g = self._gpu
        lo = sum(len(f[0]) for f in self._fluids[:i])
        hi = lo + len(self._fluids[i][0])
        out = {}
        for f in ("position", "velocity", "density"):
            out[f] = g.get(f)[lo:hi]
        return out

    def getBoundaryParticles(self, i):
        return {"position": self._solids[i][0]}


class WcSph(SphBase):
    """WCSPH (WcSph.h, WcSph.cpp): Tait EOS, artificial viscosity."""
    SOLVER = "wcsph"

    def __init__(self, device=0):
        super().__init__(device)
        self.m_DensityPower_gamma = 7.0
        self.m_TH.soundSpeed_cs = 100.0
        self.m_TH.dt = 0.4 * self.m_TH.spacing_r / self.m_TH.soundSpeed_cs  # WcSph.h:36

    def _params(self):
        p = super()._params()
        p.wc_gamma = self.m_DensityPower_gamma
        return p


class PciSph(SphBase):
    """PCISPH (PciSph.h, PciSph.cpp): predict-correct loop on the maximum
    density error, m_TH.densityErro_eta, between m_minIterations and
    m_maxIterations iterations (PciSph.h:35)."""
    SOLVER = "pcisph"

    def __init__(self, device=0):
        super().__init__(device)
        self.m_minIterations = 3
        self.m_maxIterations = 10

    def _params(self):
        p = super()._params()
        p.pci_min_iter = int(self.m_minIterations)
        p.pci_max_iter = int(self.m_maxIterations)
        return p


class IISph_M(SphBase):
    """IISPH, multiphase (IISph_M.h, IISph_M.cpp): relaxed Jacobi (omega 0.5)
    per phase to the average density error 0.001 rho0 (IISph_M.cpp:285).
    `ii_compat` selects the reference's loop bookkeeping / integration
    (see SphParams.ii_compat in include/sphgpu.h)."""
    SOLVER = "iisph_m"

    def __init__(self, device=0, ii_compat=0):
        super().__init__(device)
        self.ii_compat = ii_compat

    def _params(self):
        p = super()._params()
        p.ii_compat = int(self.ii_compat)
        return p


class IISph(SphBase):
    """IISph, the volume form (IISph.h, IISph.cpp): per-pair kernel h,
    boundary particles with their own divergence / volume error, a
    divergence-free loop (goal 1e-3 on mean(div) dt, 2..51 iterations) and a
    constant-volume loop (goal 1e-4 on the mean relative volume error,
    3..101 iterations), v += acce_presure dt (-DIISPH).  The particles'
    kinematic viscosity (FluidParticle / BoundaryParticle::kinematicViscosity,
    0.1) is `kinematicViscosity` / `boundaryKinematicViscosity`; the
    temperature update (m_TH.phaseTransition) is off, as in the reference's
    demo scene."""
    SOLVER = "iisph"

    def __init__(self, device=0):
        super().__init__(device)
        self.kinematicViscosity = 0.1
        self.boundaryKinematicViscosity = 0.1

    def _params(self):
        p = super()._params()
        p.iv_kvisc = float(self.kinematicViscosity)
        p.iv_kvisc_b = float(self.boundaryKinematicViscosity)
        return p


class DFSPH(SphBase):
    """DFSPH (DFSPH.h, DFSPH.cpp)."""
    SOLVER = "dfsph"
