"""ctypes binding of libsphgpu.so (the C ABI declared in include/sphgpu.h).

The library is built in-tree by graphics_b200/csrc/build.py.  There is no
fallback: if the library cannot be loaded, or no CUDA device is present when
a scene is created, the calls raise.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsphgpu.so")

OK, EINVAL, ENOMEM, ECUDA, EMAXITER, ENAN, ENEIGHBOUR_OVERFLOW, EOUT_OF_DOMAIN, ENOTIMPL = 0, -1, -2, -3, -4, -5, -6, -7, -8
WCSPH, PCISPH, IISPH_M, DFSPH, IISPH = 0, 1, 2, 3, 4
STATUS_MAXITER_DENSITY, STATUS_MAXITER_DIVERGENCE, STATUS_NAN = 1, 2, 4
STATUS_NEIGHBOUR_OVERFLOW, STATUS_OUT_OF_DOMAIN, STATUS_ZERO_DISTANCE = 8, 16, 32
STATUS_SOLID_OUTSIDE = 64

_f3 = C.c_float * 3


class SphParams(C.Structure):
    _fields_ = [("spacing_r", C.c_float), ("smoothRadius_h", C.c_float), ("particle_d", C.c_float),
                ("dt", C.c_float), ("gravity", _f3), ("spaceMin", _f3), ("spaceMax", _f3),
                ("soundSpeed_cs", C.c_float), ("nu", C.c_float), ("densityErro_eta", C.c_float),
                ("boundary_visc", C.c_float), ("max_neighbours", C.c_int),
                ("df_density_goal", C.c_double), ("df_density_min_iter", C.c_int),
                ("df_density_max_iter", C.c_int), ("df_div_goal_abs", C.c_double),
                ("df_div_goal_rel", C.c_double), ("df_div_min_iter", C.c_int), ("df_div_max_iter", C.c_int),
                ("cfl", C.c_int), ("cfl_factor", C.c_float), ("dt_max", C.c_float), ("dt_min", C.c_float),
                ("wc_gamma", C.c_float), ("pci_min_iter", C.c_int), ("pci_max_iter", C.c_int),
                ("ii_omega", C.c_float), ("ii_eta_rel", C.c_float), ("ii_min_iter", C.c_int),
                ("ii_max_iter", C.c_int), ("warm_start", C.c_int), ("ws_scale", C.c_float),
                ("ii_compat", C.c_int),
                ("iv_kvisc", C.c_float), ("iv_kvisc_b", C.c_float), ("iv_cv_goal", C.c_float),
                ("iv_div_goal", C.c_float), ("iv_cv_min_iter", C.c_int), ("iv_cv_max_iter", C.c_int),
                ("iv_div_min_iter", C.c_int), ("iv_div_max_iter", C.c_int),
                ("enable_vortex", C.c_int), ("vort_alpha", C.c_float), ("vort_zeta", C.c_float),
                ("vort_nu_t", C.c_float), ("th_h", C.c_float), ("th_r", C.c_float), ("th_bt", C.c_float),
                ("reserved", C.c_int * 5)]


class SphStepStats(C.Structure):
    _fields_ = [("n_fluid", C.c_int), ("iter_density", C.c_int), ("iter_divergence", C.c_int),
                ("removed", C.c_int), ("err_density", C.c_double), ("err_divergence", C.c_double),
                ("dt", C.c_double), ("status", C.c_uint32), ("neighbour_overflow", C.c_int),
                ("zero_distance", C.c_int), ("max_neighbours_seen", C.c_int), ("mean_neighbours", C.c_double),
                ("total_iter_density", C.c_int), ("total_iter_divergence", C.c_int), ("steps", C.c_int),
                ("reserved", C.c_int * 5)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


class SphRigidState(C.Structure):
    """A rigid body's state as Bullet reports it (OpenGL column-major
    transform, centre of mass, linear and angular velocity)."""
    _fields_ = [("transform", C.c_float * 16), ("center_of_mass", _f3), ("linear_velocity", _f3),
                ("angular_velocity", _f3)]


# int fn(void* user, int nsolids, const int* solid_ids, const double* force,
#        const double* torque, double dt, SphRigidState* states)
RIGID_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double),
                       C.POINTER(C.c_double), C.c_double, C.POINTER(SphRigidState))

# every symbol include/sphgpu.h declares, with (restype, argtypes)
_vp, _i, _f, _d = C.c_void_p, C.c_int, C.c_float, C.c_double
_fp, _ip, _cp = C.POINTER(C.c_float), C.POINTER(C.c_int), C.c_char_p
SIGNATURES = {
    "sphgpu_abi_version": (_i, []),
    "sphgpu_params_default": (_i, [C.POINTER(SphParams)]),
    "sphgpu_create": (_i, [C.POINTER(SphParams), _i, _i, C.POINTER(_vp)]),
    "sphgpu_destroy": (_i, [_vp]),
    "sphgpu_set_params": (_i, [_vp, C.POINTER(SphParams)]),
    "sphgpu_set_boundary": (_i, [_vp, _i, _fp, _ip, _fp]),
    "sphgpu_add_fluid": (_i, [_vp, _i, _fp, _fp, _f, _f]),
    "sphgpu_num_fluid": (_i, [_vp]),
    "sphgpu_step": (_i, [_vp, _i, _i, C.POINTER(SphStepStats)]),
    "sphgpu_step_async": (_i, [_vp, _i, _i]),
    "sphgpu_synchronize": (_i, [_vp, C.POINTER(SphStepStats)]),
    "sphgpu_step_host": (_i, [_vp, _i, _fp, _fp, _fp, _fp, C.POINTER(SphStepStats)]),
    "sphgpu_get_fluid": (_i, [_vp, _cp, _fp]),
    "sphgpu_set_fluid": (_i, [_vp, _cp, _fp]),
    "sphgpu_get_boundary": (_i, [_vp, _cp, _fp]),
    "sphgpu_stage": (_i, [_vp, _cp, C.POINTER(SphStepStats)]),
    "sphgpu_write_pos": (_i, [_vp, _cp, _i, _cp, _cp]),
    "sphgpu_read_pos": (C.c_longlong, [_cp, _fp, C.c_longlong, _cp, _i, _ip]),
    "sphgpu_save_snapshot": (_i, [_vp, _cp]),
    "sphgpu_load_snapshot": (_i, [_cp, _i, C.POINTER(_vp)]),
    "sphgpu_set_solid_dynamic": (_i, [_vp, _i, _fp, C.POINTER(SphRigidState)]),
    "sphgpu_set_rigid_callback": (_i, [_vp, RIGID_FN, _vp]),
    "sphgpu_set_solid_state": (_i, [_vp, _i, C.POINTER(SphRigidState)]),
    "sphgpu_get_solid_state": (_i, [_vp, _i, C.POINTER(SphRigidState)]),
    "sphgpu_get_solid_force": (_i, [_vp, _i, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "sphgpu_surface_create": (_i, [C.POINTER(C.c_double), C.POINTER(C.c_double), _d, _d, _d, _i, C.POINTER(_vp)]),
    "sphgpu_surface_destroy": (_i, [_vp]),
    "sphgpu_surface_grid": (_i, [_vp, C.POINTER(C.c_double), _ip, C.POINTER(C.c_double)]),
    "sphgpu_surface_field": (_i, [_vp, _i, _vp, _i, _i]),
    "sphgpu_surface_get_field": (_i, [_vp, _fp]),
    "sphgpu_surface_set_field": (_i, [_vp, _fp]),
    "sphgpu_surface_mesh": (C.c_longlong, [_vp, _f, _i, _fp, C.c_longlong]),
    "sphgpu_surface_stream": (_vp, [_vp]),
    "sphgpu_surface_last_error": (_i, [_vp, _cp, _i]),
    "sphgpu_surface_stats": (_i, [_vp, C.POINTER(C.c_longlong), _ip, C.POINTER(C.c_longlong)]),
    "sphgpu_mc_table": (_i, [_ip, C.POINTER(C.c_byte)]),
    "sphgpu_get_neighbours": (_i, [_vp, _ip, _ip, _ip]),
    "sphgpu_get_cells": (_i, [_vp, C.POINTER(C.c_longlong)]),
    "sphgpu_stream": (_vp, [_vp]),
    "sphgpu_profile": (_i, [_vp, _i]),
    "sphgpu_profile_read": (_i, [_vp, _cp, _i, C.POINTER(C.c_double), _ip, _i]),
    "sphgpu_last_error": (_i, [_vp, _cp, _i]),
    "sphgpu_mlp_create": (_i, [_i, _i, C.c_uint64, C.POINTER(_vp)]),
    "sphgpu_mlp_destroy": (_i, [_vp]),
    "sphgpu_mlp_set_params": (_i, [_vp, _fp]),
    "sphgpu_mlp_get_params": (_i, [_vp, _fp]),
    "sphgpu_mlp_set_norm": (_i, [_vp, _fp]),
    "sphgpu_mlp_get_norm": (_i, [_vp, _fp]),
    "sphgpu_mlp_dataset_size": (_i, [_vp]),
    "sphgpu_mlp_dataset_set": (_i, [_vp, _fp, _fp, _i]),
    "sphgpu_mlp_dataset_get": (_i, [_vp, _fp, _fp, _i]),
    "sphgpu_mlp_dataset_shuffle": (_i, [_vp, C.c_uint64]),
    "sphgpu_mlp_train": (_i, [_vp, _i, _i, _f, _fp]),
    "sphgpu_mlp_gradient": (_i, [_vp, _fp, _fp, _i, _fp, _fp]),
    "sphgpu_mlp_predict": (_i, [_vp, _fp, _fp, _i]),
    "sphgpu_attach_warm_start": (_i, [_vp, _vp, _i, _i]),
    "sphgpu_cfl_dt_noalloc": (_i, [_vp, _i, _i, _f, _f, _f, _f, _vp, _vp, _vp]),
    "sphgpu_autotune": (_i, [_vp, _i, _i, _cp, _i]),
    "sphgpu_batch_create": (_i, [C.POINTER(SphParams), _i, _fp, _fp, _i, _i, C.POINTER(_vp)]),
    "sphgpu_batch_num_scenes": (_i, [_vp]),
    "sphgpu_batch_set_boundary": (_i, [_vp, _i, _fp, _ip]),
    "sphgpu_batch_add_fluid": (_i, [_vp, _i, _fp, _fp, _ip, _f, _f]),
    "sphgpu_batch_stats": (_i, [_vp, C.POINTER(SphStepStats), _i]),
    "sphgpu_batch_scene_range": (_i, [_vp, _i, _ip, _ip]),
}
NOALLOC_MAX_N = 8388608
MLP_NPARAM = 5313
MLP_IN = 16
EXTRA = {"sphgpu_debug_set": (_i, [_vp, _cp, _i])}

_lib = None


def load():
    """Load libsphgpu.so (raises OSError if it is missing or unloadable)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError("libsphgpu.so not built (run graphics_b200/csrc/build.py): " + LIB_PATH)
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in {**SIGNATURES, **EXTRA}.items():
            f = getattr(lib, name)
            f.restype, f.argtypes = res, args
        _lib = lib
    return _lib


class SphGpuError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("sphgpu error %d: %s" % (code, msg))
        self.code = code
