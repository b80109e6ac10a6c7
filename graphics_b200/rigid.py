"""Host rigid-body world for dynamic solids.

The reference advances its dynamic solids with Bullet (SphWithBullet, built on
btSoftRigidDynamicsWorld, SphWithBullet.cpp:25-51): every DFSPH step hands
each dynamic rigid body the fluid's force and torque (applyCentralForce /
applyTorque), steps the world by dt (stepSimulation(dt, 1, dt)) and reads back
the body's OpenGL transform, centre of mass and velocities
(SphWithBullet.cpp:180-224, 302-317).  The library keeps that split: the
per-particle work runs on the device and a rigid-body world on the host
receives one force and torque per body and step and returns one state
(sphgpu_set_rigid_callback).  Bullet itself is not part of this build; a user
with Bullet passes a callback that drives it.  `RigidWorld` is a small world
of free rigid bodies with the same interface: gravity, semi-implicit Euler on
the linear and angular momentum, quaternion orientation -- enough for the
coupling to be exercised and checked, not a contact solver.

State layout everywhere: 25 values, transform[16] (column-major, [12:15] =
origin), center_of_mass[3], linear_velocity[3], angular_velocity[3].
"""
import ctypes as C

import numpy as np

from . import _lib


def _quat_to_matrix(q):
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                     [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                     [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])


def _quat_mul(a, b):
    aw, ax, ay, az = a
    bw, bx, by, bz = b
    return np.array([aw * bw - ax * bx - ay * by - az * bz, aw * bx + ax * bw + ay * bz - az * by,
                     aw * by - ax * bz + ay * bw + az * bx, aw * bz + ax * by - ay * bx + az * bw])


class RigidBody:
    """A free rigid body: mass, principal inertia (body frame), centre of
    mass, orientation quaternion (w, x, y, z), linear and angular velocity."""

    def __init__(self, mass, inertia, com, q=(1.0, 0.0, 0.0, 0.0), v=(0.0, 0.0, 0.0), w=(0.0, 0.0, 0.0)):
        self.mass = float(mass)
        self.inertia = np.asarray(inertia, dtype=np.float64).reshape(3)
        self.com = np.asarray(com, dtype=np.float64).copy()
        self.q = np.asarray(q, dtype=np.float64) / np.linalg.norm(q)
        self.v = np.asarray(v, dtype=np.float64).copy()
        self.w = np.asarray(w, dtype=np.float64).copy()

    @classmethod
    def box(cls, density, half, com, **kw):
        """Solid box of the given density and half extents."""
        a, b, c = (2.0 * float(h) for h in half)
        m = density * a * b * c
        return cls(m, (m * (b * b + c * c) / 12, m * (a * a + c * c) / 12, m * (a * a + b * b) / 12), com, **kw)

    def state(self):
        """The 25-value state (float32), as getOpenGLMatrix and the velocity
        getters give it."""
        R = _quat_to_matrix(self.q)
        t = np.zeros(16)
        t[0:3], t[4:7], t[8:11] = R[:, 0], R[:, 1], R[:, 2]
        t[12:15] = self.com
        t[15] = 1.0
        return np.concatenate([t, self.com, self.v, self.w]).astype(np.float32)

    def advance(self, force, torque, dt, gravity):
        R = _quat_to_matrix(self.q)
        self.v = self.v + (np.asarray(force, np.float64) / self.mass + gravity) * dt
        Iw = R @ np.diag(self.inertia) @ R.T
        L = Iw @ self.w
        self.w = self.w + np.linalg.solve(Iw, np.asarray(torque, np.float64) - np.cross(self.w, L)) * dt
        self.com = self.com + self.v * dt
        dq = 0.5 * _quat_mul(np.concatenate([[0.0], self.w]), self.q) * dt
        self.q = self.q + dq
        self.q /= np.linalg.norm(self.q)


class RigidWorld:
    """Rigid bodies keyed by solid id, advanced one step per call.

    `log` keeps (solid_ids, force, torque, dt) of every call, the numbers the
    fluid side handed over."""

    def __init__(self, gravity=(0.0, -9.81, 0.0)):
        self.gravity = np.asarray(gravity, dtype=np.float64)
        self.bodies = {}
        self.log = []

    def add(self, solid_id, body):
        self.bodies[int(solid_id)] = body
        return body

    def step(self, ids, force, torque, dt):
        force = np.asarray(force, dtype=np.float64).reshape(-1, 3)
        torque = np.asarray(torque, dtype=np.float64).reshape(-1, 3)
        self.log.append((list(ids), force.copy(), torque.copy(), float(dt)))
        for k, sid in enumerate(ids):
            self.bodies[int(sid)].advance(force[k], torque[k], float(dt), self.gravity)

    def state(self, solid_id):
        return self.bodies[int(solid_id)].state()

    # -- C callbacks --
    def gpu_callback(self):
        """A sphgpu_rigid_fn over this world (keep the returned object alive
        while the scene uses it)."""

        def fn(user, n, ids, force, torque, dt, states):
            try:
                sid = [ids[k] for k in range(n)]
                self.step(sid, np.ctypeslib.as_array(force, (3 * n,)), np.ctypeslib.as_array(torque, (3 * n,)), dt)
                for k in range(n):
                    st = self.state(sid[k])
                    C.memmove(C.byref(states[k]), st.ctypes.data, 25 * 4)
                return 0
            except Exception:  # a failure fails the step call
                return 1

        return _lib.RIGID_FN(fn)

    def double_callback(self):
        """The same world behind the oracles' callback, whose states are 25
        doubles per solid."""
        proto = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double),
                            C.POINTER(C.c_double), C.c_double, C.POINTER(C.c_double))

        def fn(user, n, ids, force, torque, dt, states):
            try:
                sid = [ids[k] for k in range(n)]
                self.step(sid, np.ctypeslib.as_array(force, (3 * n,)), np.ctypeslib.as_array(torque, (3 * n,)), dt)
                out = np.ctypeslib.as_array(states, (25 * n,))
                for k in range(n):
                    out[25 * k:25 * (k + 1)] = self.state(sid[k]).astype(np.float64)
                return 0
            except Exception:
                return 1

        return proto(fn)


def state_struct(state):
    """SphRigidState from a 25-value state."""
    s = _lib.SphRigidState()
    C.memmove(C.byref(s), np.ascontiguousarray(state, dtype=np.float32).ctypes.data, 25 * 4)
    return s


def state_array(s):
    """25-value float32 state from an SphRigidState."""
    out = np.zeros(25, dtype=np.float32)
    C.memmove(out.ctypes.data, C.byref(s), 25 * 4)
    return out
