"""ctypes mirrors of the C structs in include/nrpyell_abi.h.

The layout is the reference's NRPy_basic_defines.h:40-269 (paramstruct,
rfm_struct, bc_struct, MoL_gridfunctions_struct, griddata_struct); the test
suite compares sizes and offsets with the compiled library.
"""
import ctypes as C

NGHOSTS = 5
NUM_EVOL_GFS = 2
NUM_AUXEVOL_GFS = 3
UUGF, VVGF = 0, 1
ADD_TIMES_AUUGF, PSI_BACKGROUNDGF, WAVESPEEDGF = 0, 1, 2
EXTRAPOLATION_OUTER_BCS, RADIATION_OUTER_BCS = 0, 1

REAL = C.c_double
PREAL = C.POINTER(C.c_double)

PARAM_REALS = [
    "AMAX",
    "Cart_CoM_offsetx", "Cart_CoM_offsety", "Cart_CoM_offsetz",
    "Cart_originx", "Cart_originy", "Cart_originz",
    "P0_x", "P0_y", "P0_z", "P1_x", "P1_y", "P1_z",
    "S0_x", "S0_y", "S0_z", "S1_x", "S1_y", "S1_z",
    "SINHWAA", "bScale", "bare_mass_0", "bare_mass_1",
    "dxx0", "dxx1", "dxx2", "eta_damping",
    "f0_of_xx0", "f0_of_xx0__D0", "f0_of_xx0__DD00", "f0_of_xx0__DDD000",
    "f1_of_xx1", "f1_of_xx1__D1", "f1_of_xx1__DD11", "f1_of_xx1__DDD111",
    "f2_of_xx0_xx1", "f2_of_xx0_xx1__D0", "f2_of_xx0_xx1__D1", "f2_of_xx0_xx1__DD00", "f2_of_xx0_xx1__DD11",
    "f2_of_xx1", "f2_of_xx1__D1", "f2_of_xx1__DD11", "f2_of_xx1__DDD111",
    "f3_of_xx0", "f3_of_xx0__D0", "f3_of_xx0__DD00",
    "f4_of_xx2", "f4_of_xx2__D2", "f4_of_xx2__DD22",
    "invdx0", "invdx1", "invdx2",
    "puncture_0_x", "puncture_0_y", "puncture_0_z",
    "puncture_1_x", "puncture_1_y", "puncture_1_z",
    "time", "uu_wavespeed_at_OB", "vv_wavespeed_at_OB",
    "xx0", "xx1", "xx2", "xxmax0", "xxmax1", "xxmax2", "xxmin0", "xxmin1", "xxmin2",
]
PARAM_INTS = ["Nxx0", "Nxx1", "Nxx2", "Nxx_plus_2NGHOSTS0", "Nxx_plus_2NGHOSTS1", "Nxx_plus_2NGHOSTS2",
              "has_outer_boundary", "outer_bc_type"]


class paramstruct(C.Structure):
    _fields_ = [(n, C.c_double) for n in PARAM_REALS] + [(n, C.c_int) for n in PARAM_INTS]


RFM_FIELDS = ["f0_of_xx0", "f0_of_xx0__D0", "f0_of_xx0__DD00", "f0_of_xx0__DDD000",
              "f1_of_xx1", "f1_of_xx1__D1", "f1_of_xx1__DD11",
              "f2_of_xx0_xx1", "f2_of_xx0_xx1__D0", "f2_of_xx0_xx1__D1", "f2_of_xx0_xx1__DD00", "f2_of_xx0_xx1__DD11",
              "f3_of_xx0", "f3_of_xx0__D0", "f3_of_xx0__DD00"]


class rfm_struct(C.Structure):
    _fields_ = [(n, PREAL) for n in RFM_FIELDS]


class innerpt_bc_struct(C.Structure):
    _fields_ = [("dstpt", C.c_int), ("srcpt", C.c_int), ("parity", C.c_int8 * 10)]


class outerpt_bc_struct(C.Structure):
    _fields_ = [("i0", C.c_short), ("i1", C.c_short), ("i2", C.c_short),
                ("FACEX0", C.c_int8), ("FACEX1", C.c_int8), ("FACEX2", C.c_int8)]


class bc_info_struct(C.Structure):
    _fields_ = [("num_inner_boundary_points", C.c_int),
                ("num_pure_outer_boundary_points", (C.c_int * 3) * NGHOSTS),
                ("bc_loop_bounds", ((C.c_int * 6) * 6) * NGHOSTS)]


class bc_struct(C.Structure):
    _fields_ = [("inner_bc_array", C.POINTER(innerpt_bc_struct)),
                ("pure_outer_bc_array", C.POINTER(outerpt_bc_struct) * (NGHOSTS * 3)),
                ("bc_info", bc_info_struct)]


class MoL_gridfunctions_struct(C.Structure):
    _fields_ = [("y_n_gfs", PREAL), ("y_nplus1_running_total_gfs", PREAL), ("k_odd_gfs", PREAL),
                ("k_even_gfs", PREAL), ("auxevol_gfs", PREAL), ("diagnostic_output_gfs", PREAL)]


class griddata_struct(C.Structure):
    _fields_ = [("params", paramstruct), ("xx", PREAL * 3), ("bcstruct", bc_struct),
                ("rfmstruct", rfm_struct), ("gridfuncs", MoL_gridfunctions_struct)]


def layout():
    """Same order as nrpyell_abi_layout() in the C library."""
    return [C.sizeof(paramstruct), C.sizeof(rfm_struct), C.sizeof(innerpt_bc_struct),
            C.sizeof(outerpt_bc_struct), C.sizeof(bc_info_struct), C.sizeof(bc_struct),
            C.sizeof(MoL_gridfunctions_struct), C.sizeof(griddata_struct),
            paramstruct.Nxx0.offset, paramstruct.outer_bc_type.offset,
            griddata_struct.xx.offset, griddata_struct.bcstruct.offset,
            griddata_struct.rfmstruct.offset, griddata_struct.gridfuncs.offset, NGHOSTS]


def declare_reference_api(lib):
    """Attach argtypes/restype for the reference prototypes
    (NRPy_function_prototypes.h) to a loaded library, GPU or CPU build."""
    P = C.POINTER
    sig = {
        "rhs_eval": (None, [P(paramstruct), P(rfm_struct), PREAL, PREAL, PREAL]),
        "residual_all_points": (None, [P(paramstruct), P(rfm_struct), PREAL, PREAL, PREAL]),
        "apply_bcs_outerradiation_and_inner": (None, [P(paramstruct), P(bc_struct), PREAL * 3, PREAL, PREAL,
                                                      PREAL, PREAL]),
        "apply_bcs_inner_only": (None, [P(paramstruct), P(bc_struct), PREAL]),
        "apply_bcs_outerextrap_and_inner": (None, [P(paramstruct), P(bc_struct), PREAL]),
        "MoL_step_forward_in_time": (None, [P(griddata_struct), C.c_double]),
        "L2_norm_of_gf": (C.c_double, [P(paramstruct), C.c_int, C.c_double, PREAL * 3, PREAL]),
        "MoL_malloc_y_n_gfs": (None, [P(paramstruct), P(MoL_gridfunctions_struct)]),
        "MoL_malloc_non_y_n_gfs": (None, [P(paramstruct), P(MoL_gridfunctions_struct)]),
        "MoL_free_memory_y_n_gfs": (None, [P(paramstruct), P(MoL_gridfunctions_struct)]),
        "MoL_free_memory_non_y_n_gfs": (None, [P(paramstruct), P(MoL_gridfunctions_struct)]),
    }
    for name, (res, args) in sig.items():
        if hasattr(lib, name):
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
    return lib
