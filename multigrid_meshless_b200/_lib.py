"""ctypes binding of libmgm.so (the C ABI declared in include/mgm.h).

The library is loaded from this package directory.  There is no CPU
fallback: if the shared library is missing or no CUDA device is present,
calls fail loudly.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmgm.so")

dp = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
ip = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
vp = C.c_void_p

# status codes (include/mgm.h)
MGM_OK, MGM_ERR_CUDA, MGM_ERR_ARG, MGM_ERR_DIVERGED, MGM_ERR_TIMEOUT, MGM_ERR_NOMEM, MGM_ERR_STATE = range(7)
MODE_REFERENCE, MODE_FP64, MODE_FP32_IR = 0, 1, 2
GUESS_EXTRAPOLATE, GUESS_LEARNED = 1, 2
NOALLOC_MAX_NODES = 2097152  # MGM_NOALLOC_MAX_NODES
BC_LID, BC_TAYLOR_COUETTE = 0, 1
SETUP_REFERENCE_TRANSFER = 1
BATCH_AUTOTUNE = 1
FIELD = {"u": 0, "v": 1, "w": 2, "p": 3, "u_new": 4, "v_new": 5, "w_new": 6, "u_old": 7, "v_old": 8, "w_old": 9,
         "res": 10, "source": 11, "dpdn": 12, "dpdx": 13, "dpdy": 14, "dpdz": 15, "p_old": 16, "pprime": 3}
TIMPLE_PARTS = {"momentum": 0, "mass": 1, "pressure": 2, "update": 3, "boundary_pressure": 4}

# every exported entry point and its argument types (restype int unless noted)
SIGNATURES = {
    "mgm_last_error": ([], C.c_char_p),
    "mgm_set_device": ([C.c_int], C.c_int),
    "mgm_kernel_launches": ([], C.c_longlong),
    "mgm_version": ([], C.c_int),
    "mgm_knn_cloud": ([C.c_int, C.c_int, C.c_int, dp, dp, dp, u8p, C.c_int, ip], C.c_int),
    "mgm_nearest_points": ([C.c_int, dp, dp, dp, C.c_int, dp, dp, dp, C.c_int, ip], C.c_int),
    "mgm_bfs_order": ([C.c_int, C.c_int, ip, ip], C.c_int),
    "mgm_apply_order": ([C.c_int, C.c_int, ip, dp, dp, dp, dp, dp, dp, u8p, ip], C.c_int),
    "mgm_correct_normals": ([C.c_int, C.c_int, dp, dp, dp, u8p, ip, dp, dp, dp], C.c_int),
    "mgm_avg_dx": ([C.c_int, C.c_int, C.c_int, dp, dp, dp, u8p, ip, C.POINTER(C.c_double)], C.c_int),
    "mgm_avg_dx_noalloc": ([C.c_int, C.c_int, C.c_int, vp, vp, vp, vp, vp, vp, vp], C.c_int),
    "mgm_derivative_weights": ([C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, dp, dp, dp, dp, dp, dp, u8p, ip,
                                dp, dp, vp, dp, dp], C.c_int),
    "mgm_transfer_weights": ([C.c_int, dp, dp, dp, u8p, ip, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                              C.c_int, dp, dp, dp, ip, dp], C.c_int),
    "mgm_spmv": ([C.c_int, C.c_int, dp, ip, dp, dp], C.c_int),
    "mgm_write_solution": ([vp, C.c_char_p, C.c_int], C.c_int),
    "mgm_checkpoint_save": ([vp, C.c_char_p], C.c_int),
    "mgm_checkpoint_load": ([vp, C.c_char_p], C.c_int),
    "mgm_timple_run": ([vp, C.c_int, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_longlong),
                        C.POINTER(C.c_double)], C.c_int),
    "mgm_gauss_jordan": ([C.c_int, dp, dp], C.c_int),
    "mgm_laplacian_for_poisson": ([C.c_int, C.c_int, C.c_int, dp, dp, vp, dp, dp, dp, vp, u8p, dp], C.c_int),
    "mgm_ref_routine": ([vp, C.c_int, C.c_int], C.c_int),
    "mgm_heat_init": ([vp, C.c_int], C.c_int),
    "mgm_heat_step": ([vp, C.POINTER(C.c_double)], C.c_int),
    "mgm_mesh_read": ([C.c_char_p, C.c_int, C.POINTER(vp)], C.c_int),
    "mgm_mesh_info": ([vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_double)],
                      C.c_int),
    "mgm_mesh_get": ([vp, dp, dp, dp, dp, dp, dp, u8p, u8p], C.c_int),
    "mgm_mesh_free": ([vp], None),
    "mgm_create": ([C.c_int, C.c_int, C.c_int], vp),
    "mgm_destroy": ([vp], None),
    "mgm_set_level": ([vp, C.c_int, C.c_int, C.c_int, dp, dp, dp, dp, dp, dp, u8p, C.c_int, C.c_int], C.c_int),
    "mgm_setup": ([vp, C.c_int], C.c_int),
    "mgm_load_level": ([vp, C.c_int, C.c_int, C.c_int, dp, dp, dp, dp, dp, dp, u8p, C.c_int, C.c_int, ip, dp, dp, vp,
                        dp, dp, ip, ip, C.c_double], C.c_int),
    "mgm_load_transfer": ([vp, C.c_int, vp, vp], C.c_int),
    "mgm_prepare": ([vp], C.c_int),
    "mgm_level_size": ([vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                        C.POINTER(C.c_int)], C.c_int),
    "mgm_level_d_avg": ([vp, C.c_int, C.POINTER(C.c_double)], C.c_int),
    "mgm_get_geometry": ([vp, C.c_int, vp, vp, vp, vp, vp, vp, vp, vp], C.c_int),
    "mgm_get_operators": ([vp, C.c_int, vp, vp, vp, vp, vp], C.c_int),
    "mgm_get_transfer": ([vp, C.c_int, vp, vp, vp, vp], C.c_int),
    "mgm_get_solver_transfer": ([vp, C.c_int, vp, vp], C.c_int),
    "mgm_get_compact": ([vp, C.c_int, C.c_int, vp, vp, vp], C.c_int),
    "mgm_set_flow": ([vp, C.c_double, C.c_double, C.c_float, C.c_int, C.c_int, C.c_double], C.c_int),
    "mgm_get_dt": ([vp, C.POINTER(C.c_double)], C.c_int),
    "mgm_set_field": ([vp, C.c_int, C.c_int, dp], C.c_int),
    "mgm_get_field": ([vp, C.c_int, C.c_int, dp], C.c_int),
    "mgm_apply_bc": ([vp, C.c_int], C.c_int),
    "mgm_step": ([vp, C.c_int, C.POINTER(C.c_double)], C.c_int),
    "mgm_set_solver": ([vp, C.c_double, C.c_int, C.c_int, C.c_double], C.c_int),
    "mgm_use_graphs": ([vp, C.c_int], C.c_int),
    "mgm_use_launch_chaining": ([vp, C.c_int], C.c_int),
    "mgm_use_fused_coarse": ([vp, C.c_int], C.c_int),
    "mgm_fused_coarse_available": ([vp, C.POINTER(C.c_int)], C.c_int),
    "mgm_selftest_barrier_timeout": ([vp, C.POINTER(C.c_int)], C.c_int),
    "mgm_use_step_graph": ([vp, C.c_int], C.c_int),
    "mgm_solve_counters": ([vp, vp, vp, vp], C.c_int),
    "mgm_solve_start_residual": ([vp, C.POINTER(C.c_double)], C.c_int),
    "mgm_set_initial_guess": ([vp, C.c_int], C.c_int),
    "mgm_use_compact": ([vp, C.c_int], C.c_int),
    "mgm_use_tiled": ([vp, C.c_int], C.c_int),
    "mgm_use_half_operator": ([vp, C.c_int], C.c_int),
    "mgm_set_compatible_rhs": ([vp, C.c_int], C.c_int),
    "mgm_set_timple": ([vp, C.c_int, C.c_int, C.c_double, C.c_double], C.c_int),
    "mgm_timple_step": ([vp, C.c_int, C.POINTER(C.c_double)], C.c_int),
    "mgm_timple_part": ([vp, C.c_int, C.c_int], C.c_int),
    "mgm_last_solve": ([vp, C.POINTER(C.c_int), C.POINTER(C.c_double)], C.c_int),
    "mgm_intermediate_velocity": ([vp], C.c_int),
    "mgm_mass_residual": ([vp], C.c_int),
    "mgm_poisson": ([vp, C.c_int], C.c_int),
    "mgm_update_velocity": ([vp, C.POINTER(C.c_double)], C.c_int),
    "mgm_last_steady_error": ([vp, C.POINTER(C.c_double)], C.c_int),
    "mgm_solve_poisson": ([vp, C.c_int, dp, dp, C.POINTER(C.c_int), C.POINTER(C.c_double)], C.c_int),
    "mgm_sync": ([vp], C.c_int),
    "mgm_reference_set_poisson_mode": ([C.c_int], None),
    "mgm_reference_set_compatible_rhs": ([C.c_int], None),
    "mgm_mpnn_init": ([vp, C.c_ulonglong, C.c_int], C.c_int),
    "mgm_mpnn_num_params": ([], C.c_int),
    "mgm_mpnn_params": ([vp, vp, vp], C.c_int),
    "mgm_mpnn_loss_grad": ([vp, vp, vp, vp, vp, C.POINTER(C.c_double), vp, vp], C.c_int),
    "mgm_mpnn_predict": ([vp, vp, vp, vp, vp], C.c_int),
    "mgm_mpnn_collect": ([vp, C.c_int, C.c_int], C.c_int),
    "mgm_mpnn_dataset_size": ([vp, C.POINTER(C.c_int)], C.c_int),
    "mgm_mpnn_train": ([vp, C.c_int, C.c_int, C.c_int, C.c_float, C.c_ulonglong, vp], C.c_int),
    "mgm_mpnn_eval": ([vp, C.c_int, C.c_int, C.POINTER(C.c_double)], C.c_int),
    "mgm_set_warm_start": ([vp, C.c_int], C.c_int),
    "mgm_mpnn_set_loss": ([vp, C.c_float, C.c_float], C.c_int),
    "mgm_set_warm_smoothing": ([vp, C.c_int], C.c_int),
    "mgm_last_learned_alpha": ([vp, C.POINTER(C.c_double)], C.c_int),
    "mgm_run_steps": ([vp, C.c_int, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_longlong),
                       C.POINTER(C.c_double)], C.c_int),
    "mgm_step_host": ([vp, C.c_int, vp, vp, vp, vp, vp, vp, vp, C.POINTER(C.c_double)], C.c_int),
    "mgm_host_alloc": ([C.c_size_t], vp),
    "mgm_host_free": ([vp], None),
    "mgm_profile_smoother": ([vp, C.c_int], C.c_int),
    "mgm_profile_read": ([vp, C.POINTER(C.c_double), C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)], C.c_int),
    "mgm_batch_create": ([C.c_int, C.c_int, C.c_int], vp),
    "mgm_batch_destroy": ([vp], None),
    "mgm_batch_set_level": ([vp, C.c_int, C.c_int, C.c_int, dp, dp, dp, dp, dp, dp, u8p, C.c_int, ip], C.c_int),
    "mgm_batch_setup": ([vp, C.c_int], C.c_int),
    "mgm_batch_weights_report": ([vp, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_longlong),
                                  C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)], C.c_int),
    "mgm_batch_num_classes": ([vp, C.POINTER(C.c_int)], C.c_int),
    "mgm_batch_class": ([vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_longlong), C.POINTER(C.c_int),
                         C.POINTER(C.c_double)], C.c_int),
    "mgm_batch_level_size": ([vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_longlong),
                              C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)], C.c_int),
    "mgm_batch_get_level": ([vp, C.c_int] + [vp] * 15, C.c_int),
    "mgm_batch_get_transfer": ([vp, C.c_int] + [vp] * 8, C.c_int),
    "mgm_batch_set_solver": ([vp, C.c_double, C.c_int, C.c_int, C.c_double], C.c_int),
    "mgm_batch_solve": ([vp, C.c_int, C.c_int, dp, dp, C.POINTER(C.c_int), dp, C.POINTER(C.c_double)], C.c_int),
}

_LIB = None


class MgmError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[mgm status {code}] {msg}")
        self.code = code


def load(path: str = LIB_PATH):
    """Loads libmgm.so (once).  Raises if it is missing: there is no fallback."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing: build it with `python -m multigrid_meshless_b200.build`")
        lib = C.CDLL(path)
        for name, (args, res) in SIGNATURES.items():
            f = getattr(lib, name)
            f.argtypes = args
            f.restype = res
        _LIB = lib
    return _LIB


def check(status: int):
    if status != MGM_OK:
        raise MgmError(status, load().mgm_last_error().decode(errors="replace"))


def ptr(a):
    return None if a is None else a.ctypes.data
