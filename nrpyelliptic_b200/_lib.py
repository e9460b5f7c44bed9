"""Loader for the in-tree CUDA library libnrpyell_gpu.so (ctypes).

There is no CPU fallback: if the library is missing, loading raises, and on
a machine without a GPU the compute entry points report a CUDA error.
"""
import ctypes as C
import os

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libnrpyell_gpu.so")

_lib = None

P = C.POINTER
PREAL = abi.PREAL
XX = abi.PREAL * 3

EXPORTS = {
    # reference prototypes
    "MoL_malloc_y_n_gfs": (None, [P(abi.paramstruct), P(abi.MoL_gridfunctions_struct)]),
    "MoL_free_memory_y_n_gfs": (None, [P(abi.paramstruct), P(abi.MoL_gridfunctions_struct)]),
    "MoL_malloc_non_y_n_gfs": (None, [P(abi.paramstruct), P(abi.MoL_gridfunctions_struct)]),
    "MoL_free_memory_non_y_n_gfs": (None, [P(abi.paramstruct), P(abi.MoL_gridfunctions_struct)]),
    "MoL_step_forward_in_time": (None, [P(abi.griddata_struct), C.c_double]),
    "rhs_eval": (None, [P(abi.paramstruct), P(abi.rfm_struct), PREAL, PREAL, PREAL]),
    "apply_bcs_outerradiation_and_inner": (None, [P(abi.paramstruct), P(abi.bc_struct), XX, PREAL, PREAL, PREAL,
                                                  PREAL]),
    "apply_bcs_inner_only": (None, [P(abi.paramstruct), P(abi.bc_struct), PREAL]),
    "apply_bcs_outerextrap_and_inner": (None, [P(abi.paramstruct), P(abi.bc_struct), PREAL]),
    "residual_all_points": (None, [P(abi.paramstruct), P(abi.rfm_struct), PREAL, PREAL, PREAL]),
    "L2_norm_of_gf": (C.c_double, [P(abi.paramstruct), C.c_int, C.c_double, XX, PREAL]),
    "L2_norm_of_gf_noalloc": (C.c_double, [P(abi.paramstruct), C.c_int, C.c_double, XX, PREAL]),
    # extensions
    "nrpyell_last_status": (C.c_int, []),
    "nrpyell_gpu_last_status": (C.c_int, []),
    "nrpyell_last_error": (C.c_char_p, []),
    "nrpyell_clear_status": (None, []),
    "nrpyell_set_exit_on_error": (None, [C.c_int]),
    "nrpyell_abi_layout": (C.c_int, [P(C.c_int), C.c_int]),
    "nrpyell_launch_count": (C.c_longlong, []),
    "nrpyell_device_alloc_count": (C.c_longlong, []),
    "nrpyell_copy_bandwidth": (C.c_double, [C.c_size_t, C.c_int]),
    "nrpyell_set_step_mode": (None, [C.c_int]),
    "nrpyell_get_step_mode": (C.c_int, []),
    "nrpyell_set_device": (C.c_int, [C.c_int]),
    "nrpyell_set_async": (None, [C.c_int]),
    "nrpyell_set_tile": (None, [C.c_int]),
    "nrpyell_set_programmatic_launch": (None, [C.c_int]),
    "nrpyell_get_programmatic_launch": (C.c_int, []),
    "nrpyell_get_tile": (C.c_int, [P(abi.paramstruct), C.c_int, P(C.c_int), P(C.c_int), P(C.c_int)]),
    "nrpyell_num_tiles": (C.c_int, []),
    "nrpyell_tile_info": (C.c_int, [C.c_int, P(C.c_int), P(C.c_int), P(C.c_int)]),
    "nrpyell_synchronize": (None, []),
    "nrpyell_event_record": (C.c_int, [C.c_int]),
    "nrpyell_event_elapsed_ms": (C.c_float, [C.c_int, C.c_int]),
    "nrpyell_flush_l2": (None, []),
    "nrpyell_time_fused": (C.c_int, [P(abi.griddata_struct), C.c_double, C.c_int, C.c_int, P(C.c_double),
                                     P(C.c_double)]),
    "nrpyell_release_tables": (None, []),
    "nrpyell_device_malloc": (C.c_void_p, [C.c_size_t]),
    "nrpyell_device_free": (None, [C.c_void_p]),
    "nrpyell_host_pinned_malloc": (C.c_void_p, [C.c_size_t]),
    "nrpyell_host_pinned_free": (None, [C.c_void_p]),
    "nrpyell_memcpy": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int]),
    "nrpyell_memset": (C.c_int, [C.c_void_p, C.c_int, C.c_size_t]),
    "nrpyell_set_Cparameters_to_default": (None, [P(abi.paramstruct)]),
    "nrpyell_set_Nxx_dxx_invdx_params__and__xx": (None, [C.c_int, P(C.c_int), P(abi.paramstruct), XX]),
    "nrpyell_free_xx": (None, [XX]),
    "nrpyell_bcstruct_set_up": (None, [P(abi.paramstruct), P(abi.bc_struct)]),
    "nrpyell_bcstruct_free": (None, [P(abi.bc_struct)]),
    "nrpyell_rfm_precompute_rfmstruct_malloc": (None, [P(abi.paramstruct), P(abi.rfm_struct)]),
    "nrpyell_rfm_precompute_rfmstruct_define": (None, [P(abi.paramstruct), XX, P(abi.rfm_struct)]),
    "nrpyell_rfm_precompute_rfmstruct_freemem": (None, [P(abi.paramstruct), P(abi.rfm_struct)]),
    "nrpyell_find_timestep": (C.c_double, [P(abi.paramstruct), XX, C.c_double]),
    "nrpyell_auxevol_gfs_all_points": (None, [P(abi.paramstruct), XX, PREAL]),
    "nrpyell_wavespeed_gf_all_points": (None, [P(abi.paramstruct), C.c_double, C.c_double, XX, PREAL]),
    "nrpyell_compute_wavespeed_at_OB": (C.c_double, [P(abi.paramstruct), PREAL]),
    "nrpyell_auxevol_device": (C.c_int, [P(abi.paramstruct), XX, C.c_double, C.c_double, PREAL]),
    "nrpyell_relax": (C.c_int, [P(abi.griddata_struct), C.c_double, C.c_double, C.c_int, C.c_double, P(C.c_int),
                                P(C.c_double), PREAL]),
    "nrpyell_relax_mixed": (C.c_int, [P(abi.griddata_struct), C.c_double, C.c_double, C.c_double, C.c_int,
                                      C.c_int, C.c_double, P(C.c_int), P(C.c_int), P(C.c_double), PREAL]),
    "nrpyell_relax_et": (C.c_int, [P(abi.griddata_struct), C.c_double, C.c_double, C.c_int, C.c_int, C.c_double,
                                   P(C.c_int), P(C.c_double)]),
    "nrpyell_compute_TRC": (C.c_double, [C.c_double] * 6),
    "nrpyell_set_optimum_eta_damping": (None, [C.c_double, C.c_double, P(abi.paramstruct)]),
    "nrpyell_setup_tables_device": (C.c_int, [P(abi.paramstruct), XX, P(abi.rfm_struct), P(abi.bc_struct)]),
    "nrpyell_device_tables_read": (C.c_longlong, [P(abi.paramstruct), XX, P(abi.rfm_struct), P(abi.bc_struct), C.c_int,
                                                  C.c_void_p, C.c_longlong]),
    "nrpyell_initial_lapse": (C.c_int, [P(abi.paramstruct), C.c_int, PREAL, PREAL, C.c_int, C.c_double, PREAL]),
    "nrpyell_interpolate_solution": (C.c_int, [P(abi.paramstruct), XX, PREAL, C.c_int, PREAL, C.c_int, PREAL, PREAL,
                                               PREAL, PREAL]),
    "nrpyell_relax_batch": (C.c_int, [C.c_int, P(abi.griddata_struct), PREAL, C.c_double, C.c_int, C.c_double,
                                      P(C.c_int), PREAL]),
    "nrpyell_relax_batch_mixed": (C.c_int, [C.c_int, P(abi.griddata_struct), PREAL, C.c_double, C.c_double, C.c_int,
                                            C.c_int, C.c_double, P(C.c_int), P(C.c_int), PREAL]),
    "nrpyell_mlp_create": (C.c_void_p, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint]),
    "nrpyell_mlp_destroy": (None, [C.c_void_p]),
    "nrpyell_mlp_num_params": (C.c_longlong, [C.c_void_p]),
    "nrpyell_mlp_get_params": (C.c_int, [C.c_void_p, C.c_void_p]),
    "nrpyell_mlp_set_params": (C.c_int, [C.c_void_p, C.c_void_p]),
    "nrpyell_mlp_predict": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    "nrpyell_mlp_loss_grad": (C.c_double, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    "nrpyell_mlp_train": (C.c_double, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_float,
                                       C.c_uint, C.c_void_p]),
    "nrpyell_pod_guess": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_longlong, C.c_void_p, C.c_double,
                                    C.c_void_p]),
    "nrpyell_relax_host": (C.c_int, [P(abi.paramstruct), XX, P(abi.bc_struct), P(abi.rfm_struct), PREAL, PREAL,
                                     C.c_double, C.c_double, C.c_int, C.c_double, P(C.c_int), P(C.c_double)]),
}


def lib_path():
    return LIB_PATH


def load(exit_on_error=False):
    """Load libnrpyell_gpu.so once and return it (raises if it is missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libnrpyell_gpu.so is not built; run nrpyelliptic_b200.build.build() "
                               "(or __graft_entry__.build())")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in EXPORTS.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
    _lib.nrpyell_set_exit_on_error(1 if exit_on_error else 0)
    return _lib


def check(lib):
    """Raise RuntimeError with the library's message if a call failed."""
    if lib.nrpyell_last_status() != 0:
        msg = lib.nrpyell_last_error().decode()
        lib.nrpyell_clear_status()
        raise RuntimeError("libnrpyell_gpu: " + msg)
