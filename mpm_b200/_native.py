"""ctypes binding of libmpm_b200.so (the C ABI declared in include/mpm_gpu.h).

The library is built in-tree by ``mpm_b200.build``.  Loading fails loudly when
the library is missing: there is no CPU fallback on the product path.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libmpm_b200.so")

MPM_OK = 0
STATUS = {0: "MPM_OK", -1: "MPM_ERR_INVALID", -2: "MPM_ERR_CUDA", -3: "MPM_ERR_OUTSIDE",
          -4: "MPM_ERR_NONFINITE", -5: "MPM_ERR_TIMEOUT", -6: "MPM_ERR_ALLOC",
          -7: "MPM_ERR_UNSUPPORTED"}


class MPMError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


class Config(C.Structure):
    _fields_ = [("dim", C.c_int32), ("scheme", C.c_int32), ("velocity_update", C.c_int32),
                ("precision", C.c_int32), ("blending_ratio", C.c_double), ("dt", C.c_double),
                ("damping_factor", C.c_double), ("gravity", C.c_double * 3),
                ("gravity_ramping_time", C.c_double), ("locate_particles", C.c_int32),
                ("device", C.c_int32)]


class Particles(C.Structure):
    _fields_ = [(n, C.POINTER(C.c_double)) for n in (
        "x", "u", "v", "stress", "strain", "F", "volume", "mass", "density")] + [
        ("cell", C.POINTER(C.c_int64)), ("material", C.POINTER(C.c_int32)),
        ("svars", C.POINTER(C.c_double))]


# every symbol the header declares, with its ctypes signature
_vp = C.c_void_p
_pd = C.POINTER(C.c_double)
_pi64 = C.POINTER(C.c_int64)
_pi32 = C.POINTER(C.c_int32)
_psz = C.POINTER(C.c_size_t)
SIGNATURES = {
    "mpm_gpu_create": (C.c_int, [C.POINTER(Config), C.POINTER(_vp)]),
    "mpm_gpu_destroy": (C.c_int, [_vp]),
    "mpm_gpu_last_error": (C.c_char_p, [_vp]),
    "mpm_gpu_set_mesh": (C.c_int, [_vp, C.c_int64, _pd, C.c_int64, C.c_int32, _pi64]),
    "mpm_gpu_add_material": (C.c_int, [_vp, C.c_int32, C.c_char_p, C.c_char_p]),
    "mpm_gpu_add_velocity_constraints": (C.c_int, [_vp, C.c_int64, _pi64, _pi32, _pd]),
    "mpm_gpu_add_acceleration_constraints": (C.c_int, [_vp, C.c_int64, _pi64, _pi32, _pd]),
    "mpm_gpu_add_friction_constraints": (C.c_int, [_vp, C.c_int64, _pi64, _pi32, _pi32, _pd]),
    "mpm_gpu_add_particles": (C.c_int, [_vp, C.c_int64, _pd, C.c_int32]),
    "mpm_gpu_assign_particle_materials": (C.c_int, [_vp, C.c_int64, _pi64, C.c_int32]),
    "mpm_gpu_initialise": (C.c_int, [_vp]),
    "mpm_gpu_assign_particle_stresses": (C.c_int, [_vp, C.c_int64, _pd]),
    "mpm_gpu_add_particle_velocity_constraint": (C.c_int, [_vp, C.c_int64, _pi64, C.c_int32,
                                                           C.c_double]),
    "mpm_gpu_load_particles": (C.c_int, [_vp, C.c_int64, C.POINTER(Particles)]),
    "mpm_gpu_step": (C.c_int, [_vp, C.c_int64]),
    "mpm_gpu_step_timed": (C.c_int, [_vp, C.c_int64, _pd]),
    "mpm_gpu_set_launch_shape": (C.c_int, [_vp, C.c_int32, C.c_int32, C.c_int32]),
    "mpm_gpu_set_persistent": (C.c_int, [_vp, C.c_int32]),
    "mpm_gpu_get_persistent": (C.c_int, [_vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "mpm_gpu_host_alloc": (C.c_int, [C.c_size_t, C.POINTER(C.c_void_p)]),
    "mpm_gpu_host_free": (C.c_int, [C.c_void_p]),
    "mpm_gpu_get_launch_shape": (C.c_int, [_vp, C.POINTER(C.c_int32)]),
    "mpm_gpu_autotune": (C.c_int, [_vp, C.c_int64, C.c_char_p, C.c_size_t]),
    "mpm_gpu_set_profiling": (C.c_int, [_vp, C.c_int32]),
    "mpm_gpu_kernel_profile": (C.c_int, [_vp, C.c_int32, C.POINTER(C.c_char_p), _pd, _pi64]),
    "mpm_gpu_launch_count": (C.c_int64, [_vp]),
    "mpm_gpu_nparticles": (C.c_int64, [_vp]),
    "mpm_gpu_current_step": (C.c_int64, [_vp]),
    "mpm_gpu_read_particles": (C.c_int, [_vp, C.POINTER(Particles)]),
    "mpm_gpu_read_mapping_matrix": (C.c_int, [_vp, _pd]),
    "mpm_gpu_set_isoparametric": (C.c_int, [_vp, C.c_int32]),
    "mpm_gpu_set_nodal_euler_angles": (C.c_int, [_vp, C.c_int64, _pi64, _pd]),
    "mpm_gpu_load_mapping_matrix": (C.c_int, [_vp, _pd]),
    "mpm_gpu_write_pod": (C.c_int, [_vp, _vp, C.c_int64, _pi64, C.c_size_t, _psz, _psz,
                                    C.c_int32]),
    "mpm_gpu_load_pod": (C.c_int, [_vp, _vp, C.c_int64, C.c_size_t, _psz, _psz, C.c_int32]),
    "mpm_gpu_set_current_step": (C.c_int, [_vp, C.c_int64]),
    "mpm_gpu_adjoint_record": (C.c_int, [_vp, C.c_int64, C.c_int64, C.c_int32, _pi32, _pi32]),
    "mpm_gpu_adjoint_reverse": (C.c_int, [_vp, _pd, _pd, _pd, _pd, _pd, _pd]),
    "mpm_gpu_adjoint_run": (C.c_int, [_vp, C.c_int64, C.c_int64, C.c_int32, _pi32, _pi32, _pd,
                                      _pd, _pd]),
    "mpm_gpu_set_sensitivities": (C.c_int, [_vp, C.c_int32, _pi32, _pi32]),
    "mpm_gpu_read_sensitivities": (C.c_int, [_vp, C.c_int32, _pd]),
    "mpm_gpu_device_field": (C.c_int, [_vp, C.c_int32, C.POINTER(_vp), _pi64, _pi32]),
    "mpm_gpu_material_stress_batch": (C.c_int, [C.c_int32, C.c_int32, C.c_char_p, C.c_char_p,
                                                C.c_int64, _pd, _pd, _pd, _pd, _pd]),
    "mpm_gpu_material_stress_batch_noalloc": (C.c_int, [C.c_int32, C.c_int32, C.c_char_p,
                                                        C.c_char_p, C.c_int64, _pd, _pd, _pd,
                                                        _pd, _pd, C.c_char_p, C.c_int64]),
    "mpm_gpu_version": (C.c_char_p, []),
    "mpm_gpu_step_begin": (C.c_int, [_vp]),
    "mpm_gpu_step_end": (C.c_int, [_vp]),
    "mpm_gpu_halo_bytes": (C.c_int, [_vp, _pi64]),
    "mpm_gpu_halo_pack": (C.c_int, [_vp, C.c_int32, _vp]),
    "mpm_gpu_halo_unpack": (C.c_int, [_vp, C.c_int32, _vp]),
    "mpm_gpu_layer_count": (C.c_int, [_vp, C.c_int32, C.c_int32, _pi64, _pi64]),
    "mpm_gpu_write_hdf5": (C.c_int, [_vp, C.c_char_p]),
    "mpm_gpu_load_hdf5": (C.c_int, [_vp, C.c_char_p]),
    "mpm_h5_write_table": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int64, C.c_size_t, C.c_int32,
                                     C.POINTER(C.c_char_p), _psz, _pi32, _vp, C.c_int64]),
    "mpm_h5_read_table": (C.c_int, [C.c_char_p, _pi64, C.c_size_t, C.c_int32,
                                    C.POINTER(C.c_char_p), _psz, _pi32, _vp, C.c_int64,
                                    C.c_char_p, C.c_int64]),
}

_lib = None


def lib():
    """Load libmpm_b200.so; raise if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m mpm_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib
