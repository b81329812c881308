"""ctypes binding of libdemsph_b200.so (the C ABI declared in include/demsph.h).

The library is built in-tree by ``python -m this_studio_b200.build``.  There
is no fallback: importing the solvers without the built library raises.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libdemsph_b200.so")

OK = 0
ERR_INVALID = 1
ERR_SCENE = 2
ERR_OVERFLOW = 3
ERR_CUDA = 4
ERR_NOT_READY = 5
ERR_TIMEOUT = 6
ERR_ALLOC = 7
PRECISION_FP64 = 0
PRECISION_MIXED = 1

_d = C.POINTER(C.c_double)
_i = C.POINTER(C.c_int)
_l = C.POINTER(C.c_long)
_vp = C.c_void_p
_pvp = C.POINTER(C.c_void_p)
_int = C.c_int
_dbl = C.c_double
_long = C.c_long


class Double3(C.Structure):
    """CUDA's double3, passed by value."""
    _fields_ = [("x", C.c_double), ("y", C.c_double), ("z", C.c_double)]


class BallArrays(C.Structure):
    """demsph_ball_arrays: device pointers to the ball arrays in the
    reference's layout, filled by demsph_dem_hook_arrays."""
    _fields_ = [("position", C.c_void_p), ("velocity", C.c_void_p), ("angularVelocity", C.c_void_p),
                ("force", C.c_void_p), ("torque", C.c_void_p), ("radius", C.c_void_p),
                ("inverseMass", C.c_void_p), ("materialID", C.c_void_p), ("clumpID", C.c_void_p),
                ("n", C.c_long)]


# demsph_dem_hook_fn: void (*)(void* user, long iStep, double time)
HOOK_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_long, C.c_double)
_sz = C.c_size_t

# name -> argument types (all return int unless listed in _RESTYPE)
SIGNATURES = {
    "demsph_device_alloc": [_pvp, _sz, _vp],
    "demsph_device_free": [_vp, _vp],
    "demsph_memcpy": [_vp, _vp, _sz, _int, _vp],
    "demsph_dem_set_external_hook": [_vp, HOOK_FN, _vp],
    "demsph_dem_hook_arrays": [_vp, C.POINTER(BallArrays)],
    "demsph_dem_set_bonds": [_vp, _long, _i, _d, _d, _d, _d, _d, _d],
    "demsph_dem_diagnostics": [_vp, _d],
    "demsph_sph_diagnostics": [_vp, _d],
    "demsph_sph_set_uniform_kernels": [_vp, _int],
    "demsph_dem_snapshot": [_vp, _pvp],
    "demsph_dem_restore": [_vp, _vp],
    "demsph_dem_snapshot_destroy": [_vp],
    "demsph_sph_snapshot": [_vp, _pvp],
    "demsph_sph_restore": [_vp, _vp],
    "demsph_sph_snapshot_destroy": [_vp],
    "demsph_sph_uniform_kernels": [_vp, _i],
    "launchAddConstantForce": [_vp, _vp, _sz, _sz, _sz, _vp],
    "launchAddGlobalDampingForceTorque": [_vp, _vp, _vp, _vp, _dbl, _sz, _sz, _sz, _vp],
    "launchAddBuoyancyDrag": [_vp, _vp, _vp, _vp, _vp, _dbl, _dbl, Double3, Double3, _dbl, _sz, _sz, _sz, _vp],
    "demsph_last_error": [],
    "demsph_version": [],
    "demsph_kernel_launches": [],
    "demsph_retain_device_memory": [C.c_ulonglong],
    "demsph_dem_create": [_pvp, _vp],
    "demsph_dem_destroy": [_vp],
    "demsph_dem_set_hertzian_pair": [_vp, _int, _int] + [_dbl] * 8,
    "demsph_dem_set_linear_pair": [_vp, _int, _int] + [_dbl] * 11,
    "demsph_dem_set_bonded_pair": [_vp, _int, _int] + [_dbl] * 6,
    "demsph_dem_add_balls": [_vp, _long, _d, _d, _d, _d, _d, _i, _i, _int],
    "demsph_dem_add_clump": [_vp, _long, _d, _d, _d, _d, _d, _dbl, _d, _int],
    "demsph_dem_add_mesh_wall": [_vp, _long, _d, _long, _i, _i, _i, _d, _int],
    "demsph_dem_set_wall_motion": [_vp, _int, _d, _d],
    "demsph_dem_add_bonds": [_vp, _long, _i, _i, _d, _long],
    "demsph_dem_set_constant_force": [_vp, _long, _d, _dbl],
    "demsph_dem_set_global_damping": [_vp, _dbl],
    "demsph_dem_set_buoyancy_drag": [_vp, _dbl, _dbl, _d, _d, _dbl],
    "demsph_dem_initialize": [_vp, _d, _d, _d, _dbl, _int],
    "demsph_dem_step": [_vp, _long],
    "demsph_dem_neighbor_search": [_vp],
    "demsph_dem_eval_forces": [_vp, _dbl, _int, _dbl],
    "demsph_dem_num_balls": [_vp, _l],
    "demsph_dem_num_pairs": [_vp, _int, _l],
    "demsph_dem_num_bonds": [_vp, _l],
    "demsph_dem_num_clumps": [_vp, _l],
    "demsph_dem_step_index": [_vp, _l, _d],
    "demsph_dem_get_balls": [_vp, _d, _d, _d, _d, _d],
    "demsph_dem_set_balls": [_vp, _d, _d, _d],
    "demsph_dem_get_pairs": [_vp, _int, _i, _i, _d, _d, _d, _d, _d],
    "demsph_dem_import_springs": [_vp, _long, _i, _i, _d, _d, _d],
    "demsph_dem_import_wall_springs": [_vp, _long, _i, _i, _d, _d, _d],
    "demsph_dem_member_create": [_pvp, _vp],
    "demsph_dem_member_destroy": [_vp],
    "demsph_dem_member_add_balls": [_vp, _long, _d, _d, _d, _d, _d, _i, _int],
    "demsph_dem_member_add_clump": [_vp, _long, _d, _d, _d, _d, _d, _dbl, _d, _int],
    "demsph_dem_member_num_clumps": [_vp, C.POINTER(_long)],
    "demsph_dem_member_seal": [_vp],
    "demsph_dem_set_cell_factor": [_vp, _dbl],
    "demsph_sph_set_cell_factor": [_vp, _dbl],
    "demsph_sph_set_conditional_rebuild": [_vp, _int],
    "demsph_sph_conditional_rebuild": [_vp, _i, C.POINTER(_long)],
    "demsph_sph_set_list_headroom": [_vp, _dbl],
    "demsph_sph_list_capacity": [_vp, _i, _i],
    "demsph_dem_member_count": [_vp, _l],
    "demsph_dem_assemble_balls": [_vp, _int, _pvp, _d, _i],
    "demsph_dem_set_graphs": [_vp, _int],
    "demsph_dem_set_periodic": [_vp, _int, _int, _int],
    "demsph_dem_reserve": [_vp, _int, _int, _int],
    "demsph_dem_capacity": [_vp, _i, _i, _i],
    "demsph_dem_write_vtu": [_vp, C.c_char_p, _long, _int],
    "demsph_dem_copy_members": [_vp, _vp, _int, _i, _i, _i, _i, _d],
    "demsph_dem_copy_member_bodies": [_vp, _vp, _int, _i, _i, _i, _i, _i, _i, _d],
    "demsph_dem_get_bonds": [_vp, _i, _i, _i, _d, _d, _d, _d, _d, _d],
    "demsph_dem_get_clumps": [_vp, _d, _d, _d, _d],
    "demsph_dem_get_walls": [_vp, _d, _d, _d],
    "demsph_sph_create": [_pvp, _vp],
    "demsph_sph_destroy": [_vp],
    "demsph_sph_add": [_vp, _int, _long, _d, _d, _d, _d, _d, _d],
    "demsph_sph_initialize": [_vp, _d, _d, _d, _dbl, _int],
    "demsph_sph_step": [_vp, _long],
    "demsph_sph_synchronize": [_vp],
    "demsph_sph_neighbor_search": [_vp],
    "demsph_sph_eval_accel": [_vp],
    "demsph_sph_profile_steps": [_vp, _long, _d],
    "demsph_sph_tune": [_vp, _int, _i, _d],
    "demsph_sph_set_graphs": [_vp, _int],
    "demsph_sph_set_skin": [_vp, _dbl],
    "demsph_sph_tune_skin": [_vp, _int, _d, _d],
    "demsph_sph_skin_stats": [_vp, _d, _l],
    "demsph_sph_write_vtu": [_vp, C.c_char_p, _long, _int],
    "demsph_sph_num_list_shapes": [],
    "demsph_sph_set_list_shape": [_vp, _int],
    "demsph_sph_copy_members": [_vp, _vp, _int, _i, _i, _i, _d],
    "demsph_sph_num": [_vp, _int, _l],
    "demsph_sph_member_create": [_pvp, _vp],
    "demsph_sph_member_destroy": [_vp],
    "demsph_sph_member_add": [_vp, _int, _long, _d, _d, _d, _d, _d, _d],
    "demsph_sph_member_seal": [_vp],
    "demsph_sph_member_count": [_vp, _int, _l],
    "demsph_sph_assemble": [_vp, _int, _pvp, _d, _d, _d, _d, _dbl, _int],
    "demsph_sph_num_pairs": [_vp, _int, _l],
    "demsph_sph_step_index": [_vp, _l, _d],
    "demsph_sph_get": [_vp, _int, _d, _d, _d, _d, _d, _d, _d],
    "demsph_sph_set": [_vp, _d, _d, _d, _d, _d],
    "demsph_sph_get_pairs": [_vp, _int, _i, _i],
    "demsph_sph_couple_balls": [_vp, _vp, _long, _i, _dbl, _dbl, _dbl, _dbl, _dbl],
    "demsph_sph_couple_step": [_vp, _vp, _long, _int],
    "demsph_sph_num_markers": [_vp, _l, _l],
    "demsph_sph_get_markers": [_vp, _d, _d, _d, _d, _i],
    "demsph_sph_get_coupling": [_vp, _i, _d, _d],
    "buildHashStartEnd": [_vp, _vp, _vp, _vp, C.c_size_t, C.c_size_t, C.c_size_t, C.c_size_t, _vp],
    "buildPrefixSum": [_vp, _vp, C.c_size_t, _vp],
    "demsph_build_hash_start_end_noalloc": [_vp, _vp, _vp, _vp, C.c_size_t, C.c_size_t, _vp],
}
_RESTYPE = {
    "demsph_last_error": C.c_char_p,
    "demsph_version": C.c_char_p,
    "demsph_kernel_launches": C.c_longlong,
    "buildHashStartEnd": None,
    "buildPrefixSum": None,
    "launchAddConstantForce": None,
    "launchAddGlobalDampingForceTorque": None,
    "launchAddBuoyancyDrag": None,
}

_lib = None


class DemsphError(RuntimeError):
    def __init__(self, code, func, msg):
        super().__init__(f"{func} failed with status {code}: {msg}")
        self.code = code


def lib():
    """Loads the native library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} not found: the CUDA library is not built "
                "(run `python -m this_studio_b200.build`)")
        L = C.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = _RESTYPE.get(name, C.c_int)
        _lib = L
    return _lib


def call(name, *args):
    rc = getattr(lib(), name)(*args)
    if rc != OK:
        msg = lib().demsph_last_error().decode(errors="replace")
        raise DemsphError(rc, name, msg)
    return rc


def kernel_launches() -> int:
    return int(lib().demsph_kernel_launches())


def retain_device_memory(nbytes: int) -> None:
    """Keeps up to nbytes of freed scene memory in this process's pool."""
    call("demsph_retain_device_memory", int(nbytes))
