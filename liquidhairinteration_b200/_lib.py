"""Loads liblhi.so (built in-tree by ``make -C liquidhairinteration_b200``)
and declares the ctypes signatures of every entry point of include/lhi.h.

There is no fallback: if the library is missing, importing the model raises.
"""
import ctypes as C
import os

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblhi.so")

_vp = C.c_void_p
_h = C.c_void_p  # lhi_liquid*

# name -> (argtypes); every function returns int unless listed in _RESTYPE
SIGNATURES = {
    "lhi_liquid_create": [C.POINTER(abi.GridDesc), C.POINTER(abi.SolverParams), C.POINTER(abi.LiquidParams),
                          C.c_int32, C.POINTER(_h)],
    "lhi_liquid_destroy": [_h],
    "lhi_last_error": [],
    "lhi_liquid_precision": [_h, C.POINTER(C.c_int32)],
    "lhi_liquid_sync": [_h],
    "lhi_liquid_get_dx": [_h, C.POINTER(C.c_double)],
    "lhi_liquid_set_boundary": [_h, C.POINTER(abi.BoundaryNode), C.c_int32, C.c_int32],
    "lhi_liquid_set_solid_phi": [_h, _vp],
    "lhi_liquid_set_particles": [_h, C.c_int64, _vp, _vp, _vp],
    "lhi_liquid_get_particles": [_h, _vp, _vp, _vp],
    "lhi_liquid_num_particles": [_h, C.POINTER(C.c_int64)],
    "lhi_liquid_pre_step": [_h, C.c_double],
    "lhi_liquid_step": [_h, C.c_double],
    "lhi_liquid_post_step": [_h, C.c_double],
    "lhi_liquid_clear": [_h],
    "lhi_liquid_sort_particles": [_h],
    "lhi_liquid_compute_liquid_phi": [_h],
    "lhi_liquid_particle_to_grid": [_h],
    "lhi_liquid_apply_gravity": [_h, C.c_double],
    "lhi_liquid_projection": [_h, C.c_double],
    "lhi_liquid_velocity_update": [_h, C.c_double],
    "lhi_liquid_extrapolate": [_h],
    "lhi_liquid_grid_to_particle": [_h],
    "lhi_liquid_advect_particles": [_h, C.c_double],
    "lhi_liquid_compute_divergence": [_h, C.POINTER(C.c_double), C.POINTER(C.c_double)],
    "lhi_solver_spmv": [_h, C.POINTER(C.c_double), C.POINTER(C.c_int32)],
    "lhi_liquid_render": [_h, C.POINTER(abi.RenderParams), _vp, _vp],
    "lhi_liquid_correct_volume": [_h, C.c_double],
    "lhi_debug_set_stage_wait_limit": [C.c_double],
    "lhi_liquid_get_cfl": [_h, C.POINTER(C.c_double)],
    "lhi_net_create": [C.c_uint64, C.POINTER(C.c_void_p)],
    "lhi_net_destroy": [C.c_void_p],
    "lhi_net_num_params": [C.POINTER(C.c_int64)],
    "lhi_net_get_params": [C.c_void_p, _vp],
    "lhi_net_set_params": [C.c_void_p, _vp],
    "lhi_net_save": [C.c_void_p, C.c_char_p],
    "lhi_net_set_relu": [C.c_void_p, C.c_int32],
    "lhi_net_set_sparse": [C.c_void_p, C.c_int32],
    "lhi_net_load": [C.c_void_p, C.c_char_p],
    "lhi_solver_set_network": [_h, C.c_void_p, C.c_int32],
    "lhi_solver_learned_stats": [_h, C.POINTER(C.c_int32), C.POINTER(C.c_int32)],
    "lhi_solver_record_residuals": [_h, C.c_int32],
    "lhi_solver_num_snapshots": [_h, C.POINTER(C.c_int32)],
    "lhi_solver_get_snapshot": [_h, C.c_int32, _vp],
    "lhi_net_train": [C.c_void_p, _h, C.c_int32, C.c_int32, C.c_double, C.c_uint64, C.POINTER(C.c_double),
                      C.POINTER(C.c_double)],
    "lhi_net_tensor_core_selftest": [C.c_int32, C.c_int32, _vp, _vp, _vp, C.POINTER(C.c_int32)],
    "lhi_net_forward_host": [C.c_void_p, C.POINTER(C.c_int32), _vp, _vp, _vp, C.c_double, _vp],
    "lhi_net_backward_host": [C.c_void_p, C.POINTER(C.c_int32), _vp, _vp, _vp, C.c_double, _vp, _vp],
    "lhi_divergence_noalloc": [C.POINTER(C.c_int32), C.c_double, C.c_int32, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                               C.POINTER(C.c_double), C.POINTER(C.c_double)],
    "lhi_solver_init": [_h],
    "lhi_solver_build_rhs": [_h],
    "lhi_solver_build_lhs": [_h, C.c_double, C.c_double],
    "lhi_solver_apply_preconditioner": [_h],
    "lhi_solver_solve": [_h, C.c_double, C.c_double, C.POINTER(abi.SolveStats)],
    "lhi_solver_get_stats": [_h, C.POINTER(abi.SolveStats)],
    "lhi_solver_get_ax": [_h, C.c_int32, _vp, _vp],
    "lhi_solver_active_tiles": [_h, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int32)],
    "lhi_liquid_field_size": [_h, C.c_int32, C.c_int32, C.POINTER(C.c_int64), C.POINTER(C.c_int32)],
    "lhi_liquid_get_field": [_h, C.c_int32, C.c_int32, _vp],
    "lhi_liquid_set_field": [_h, C.c_int32, C.c_int32, _vp],
    "lhi_liquid_stream": [_h, C.POINTER(C.c_void_p)],
    "lhi_liquid_set_async": [_h, C.c_int32],
    "lhi_solver_graph_error": [_h],
    "lhi_kernel_launch_count": [C.POINTER(C.c_int64)],
    "lhi_liquid_profile": [_h, C.c_int32],
    "lhi_liquid_profile_read": [_h, C.c_int32, C.POINTER(C.c_int64), C.POINTER(C.c_double)],
    "lhi_boundary_eval": [C.POINTER(abi.BoundaryNode), C.c_int32, C.c_int32, C.c_int32, _vp, C.c_int64, _vp],
    "lhi_scene_seed_particles": [C.POINTER(abi.GridDesc), C.POINTER(abi.BoundaryNode), C.c_int32, C.c_int32,
                                 C.POINTER(abi.FluidPrim), C.c_int32, C.c_uint64, C.c_int32,
                                 C.POINTER(C.c_int64), _vp, _vp],
    "lhi_scene_spawn_lattice": [C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_double, C.c_int64, C.c_int32,
                                C.POINTER(C.c_int64), _vp],
}
_RESTYPE = {"lhi_last_error": C.c_char_p, "lhi_solver_graph_error": C.c_char_p}

_LIB = None


def lib():
    """The loaded liblhi.so (raises OSError if it has not been built)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} not found: build it with `make -C {HERE}` "
                          "(there is no CPU fallback for the liquid step)")
        L = C.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = _RESTYPE.get(name, C.c_int)
        _LIB = L
    return _LIB


class LhiError(RuntimeError):
    """A non-zero status from the C-ABI; ``code`` is the LHI_E_* value."""

    def __init__(self, code, func, msg):
        self.code = code
        super().__init__(f"{func} failed with {abi.STATUS_NAMES.get(code, code)}: {msg}")


def check(rc, func="lhi call"):
    if rc != abi.LHI_OK:
        msg = lib().lhi_last_error()
        raise LhiError(rc, func, msg.decode() if msg else "")
    return rc


def call(name, *args):
    return check(getattr(lib(), name)(*args), name)
