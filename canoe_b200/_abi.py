"""ctypes mirror of include/canoe_b200.h and the loader of the CUDA library.

The library is built in-tree (``python -m canoe_b200.build``) and there is
no fallback: importing :data:`lib` when the shared object is missing raises.
"""
import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_int, c_int32, c_int64, c_uint32, c_void_p

MAX_NY = 8
MAX_VAPOR = 4
NGHOST = 3

BC_REFLECT, BC_PERIODIC, BC_OUTFLOW, BC_EXO3, BC_BLOCK = 0, 1, 2, 3, 4
RECON_PLM, RECON_PPM = 2, 3
RS_LMARS, RS_HLLC = 0, 1
FP64, FP32_PERTURBATION = 0, 1


class Thermo(ctypes.Structure):
    _fields_ = [
        ("ny", c_int32), ("nvapor", c_int32),
        ("rd", c_double), ("gammad", c_double), ("grav", c_double),
        ("cv_ratio_m1", c_double * MAX_NY),
        ("inv_mu_ratio_m1", c_double * MAX_NY),
        ("u0", c_double * MAX_NY),
        ("liq_slot", c_int32 * MAX_VAPOR), ("ice_slot", c_int32 * MAX_VAPOR),
        ("t3", c_double * MAX_VAPOR), ("p3", c_double * MAX_VAPOR),
        ("beta_l", c_double * MAX_VAPOR), ("delta_l", c_double * MAX_VAPOR),
        ("beta_s", c_double * MAX_VAPOR), ("delta_s", c_double * MAX_VAPOR),
    ]


class SatOpts(ctypes.Structure):
    _fields_ = [("tol", c_double), ("max_iter", c_int32), ("warm", c_int32)]


class BlockConfig(ctypes.Structure):
    _fields_ = [
        ("nx1", c_int32), ("nx2", c_int32), ("nx3", c_int32),
        ("bc", c_int32 * 6),
        ("x2min", c_double), ("x3min", c_double),
        ("dx2", c_double), ("dx3", c_double),
        ("h_x1f", POINTER(c_double)),
        ("recon", c_int32), ("rsolver", c_int32), ("implicit_flag", c_int32),
        ("precision", c_int32), ("satadj", c_int32),
        ("cfl", c_double),
        ("thermo", Thermo),
    ]


class ShellConfig(ctypes.Structure):
    _fields_ = [
        ("nx1", c_int32), ("nside", c_int32), ("bc_x1", c_int32 * 2),
        ("h_x1f", POINTER(c_double)),
        ("recon", c_int32), ("rsolver", c_int32), ("implicit_flag", c_int32),
        ("precision", c_int32),
        ("cfl", c_double),
        ("thermo", Thermo),
    ]


HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libcanoe_b200.so")

# (name, restype, argtypes) of every entry point declared in the header
SIGNATURES = [
    ("canoe_version", c_char_p, []),
    ("canoe_last_error", c_char_p, []),
    ("canoe_device_sm_count", c_int, [POINTER(c_int)]),
    ("canoe_riemann_lmars", c_int, [POINTER(Thermo), c_int, c_void_p, c_void_p, c_void_p, c_int64, c_void_p]),
    ("canoe_riemann_hllc", c_int, [POINTER(Thermo), c_int, c_void_p, c_void_p, c_void_p, c_int64, c_void_p]),
    ("canoe_saturation_adjust", c_int, [POINTER(Thermo), POINTER(SatOpts), c_void_p, c_int64,
                                        c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    ("canoe_block_create", c_int, [POINTER(BlockConfig), POINTER(c_void_p)]),
    ("canoe_block_destroy", c_int, [c_void_p]),
    ("canoe_block_dims", c_int, [c_void_p, POINTER(c_int32), POINTER(c_int32), POINTER(c_int32), POINTER(c_int32)]),
    ("canoe_block_set_conserved", c_int, [c_void_p, c_void_p]),
    ("canoe_block_get_conserved", c_int, [c_void_p, c_void_p]),
    ("canoe_block_get_primitive", c_int, [c_void_p, c_void_p]),
    ("canoe_block_device_ptrs", c_int, [c_void_p, POINTER(c_void_p), POINTER(c_void_p)]),
    ("canoe_block_set_stream", c_int, [c_void_p, c_void_p]),
    ("canoe_block_calculate_fluxes", c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    ("canoe_block_solve_implicit", c_int, [c_void_p, c_void_p, c_double]),
    ("canoe_block_use_graph", c_int, [c_void_p, c_int]),
    ("canoe_block_synchronize", c_int, [c_void_p]),
    ("canoe_block_set_fixed_dt", c_int, [c_void_p, c_double]),
    ("canoe_block_set_diffusion", c_int, [c_void_p, c_double, c_double]),
    ("canoe_block_step_profile", c_int, [c_void_p, c_double, POINTER(ctypes.c_float), c_int]),
    ("canoe_block_step", c_int, [c_void_p, c_double]),
    ("canoe_block_step_noalloc", c_int, [POINTER(BlockConfig), c_void_p, c_void_p, c_void_p,
                                         c_double, c_void_p]),
    ("canoe_block_new_dt", c_int, [c_void_p, POINTER(c_double)]),
    ("canoe_block_error_word", c_int, [c_void_p, POINTER(c_uint32)]),
    ("canoe_block_set_mlp", c_int, [c_void_p, c_void_p]),
    ("canoe_block_satadj_stats", c_int, [c_void_p, c_void_p]),
    ("canoe_mlp_create", c_int, [ctypes.c_uint64, POINTER(c_void_p)]),
    ("canoe_mlp_destroy", c_int, [c_void_p]),
    ("canoe_mlp_nparams", c_int, []),
    ("canoe_mlp_set_params", c_int, [c_void_p, c_void_p]),
    ("canoe_mlp_get_params", c_int, [c_void_p, c_void_p]),
    ("canoe_mlp_set_normalization", c_int, [c_void_p, c_void_p, c_void_p, ctypes.c_float,
                                            ctypes.c_float]),
    ("canoe_mlp_get_normalization", c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    ("canoe_mlp_loss_grad", c_int, [c_void_p, c_void_p, c_void_p, c_int64, c_void_p, c_void_p,
                                    c_void_p]),
    ("canoe_mlp_adam_step", c_int, [c_void_p, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                    ctypes.c_float, c_void_p]),
    ("canoe_mlp_forward", c_int, [c_void_p, c_void_p, c_void_p, c_int64, c_int, c_void_p]),
    ("canoe_block_set_column_threads", c_int, [c_void_p, c_int]),
    ("canoe_block_set_flux_run", c_int, [c_void_p, c_int]),
    ("canoe_block_get_shapes", c_int, [c_void_p, c_void_p, c_void_p]),
    ("canoe_selftest_bounded_wait", c_int, [c_int, c_int, c_void_p]),
    ("canoe_selftest_umma_wait", c_int, [c_int, c_int, c_void_p]),
    ("canoe_measure_fma_peak", c_int, [c_int, POINTER(c_double)]),
    ("canoe_block_set_neighbor", c_int, [c_void_p, c_int, c_void_p]),
    ("canoe_block_stage", c_int, [c_void_p, c_int, c_double]),
    ("canoe_block_exchange_ghosts", c_int, [c_void_p]),
    ("canoe_block_side_doubles", c_int, [c_void_p, c_int, POINTER(c_int64)]),
    ("canoe_block_pack_side", c_int, [c_void_p, c_int, c_void_p]),
    ("canoe_block_unpack_side", c_int, [c_void_p, c_int, c_void_p]),
    ("canoe_mesh_create", c_int, [c_void_p, c_int, POINTER(c_void_p)]),
    ("canoe_mesh_destroy", c_int, [c_void_p]),
    ("canoe_mesh_use_graph", c_int, [c_void_p, c_int]),
    ("canoe_mesh_step", c_int, [c_void_p, c_double]),
    ("canoe_mesh_new_dt", c_int, [c_void_p, POINTER(c_double)]),
    ("canoe_mesh_synchronize", c_int, [c_void_p]),
    ("canoe_batch_create", c_int, [c_void_p, c_int, POINTER(c_void_p)]),
    ("canoe_batch_destroy", c_int, [c_void_p]),
    ("canoe_batch_use_graph", c_int, [c_void_p, c_int]),
    ("canoe_batch_step", c_int, [c_void_p]),
    ("canoe_batch_synchronize", c_int, [c_void_p]),
    ("canoe_batch_autotune", c_int, [c_void_p, c_void_p]),
    ("canoe_shell_create", c_int, [POINTER(ShellConfig), POINTER(c_void_p)]),
    ("canoe_shell_destroy", c_int, [c_void_p]),
    ("canoe_shell_dims", c_int, [c_void_p, POINTER(c_int32), POINTER(c_int32), POINTER(c_int32),
                                 POINTER(c_int32)]),
    ("canoe_shell_set_stream", c_int, [c_void_p, c_void_p]),
    ("canoe_shell_set_conserved", c_int, [c_void_p, c_void_p, c_int]),
    ("canoe_shell_get_conserved", c_int, [c_void_p, c_void_p]),
    ("canoe_shell_get_primitive", c_int, [c_void_p, c_void_p]),
    ("canoe_shell_fill_ghosts", c_int, [c_void_p]),
    ("canoe_shell_calculate_fluxes", c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    ("canoe_shell_step", c_int, [c_void_p, c_double]),
    ("canoe_shell_synchronize", c_int, [c_void_p]),
    ("canoe_shell_error_word", c_int, [c_void_p, POINTER(c_uint32)]),
    ("canoe_saturation_adjust_learned", c_int, [POINTER(Thermo), POINTER(SatOpts), c_void_p,
                                                c_void_p, c_int64, c_void_p, c_void_p, c_void_p,
                                                c_void_p, c_void_p]),
]


class CanoeError(RuntimeError):
    pass


_lib = None


def load():
    """Load the CUDA library (raises CanoeError if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise CanoeError(
            f"CUDA library {LIB_PATH} is missing: build it with `python -m canoe_b200.build`")
    lib = ctypes.CDLL(LIB_PATH)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc, what=""):
    if rc != 0:
        msg = load().canoe_last_error().decode()
        raise CanoeError(f"{what} failed with status {rc}: {msg}")
