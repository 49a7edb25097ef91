"""ctypes binding of libufem_gpu.so (the C ABI in include/ufem_gpu.h).

The library is built in-tree (``python -m ufem_b200.build``) and loaded from
``ufem_b200/lib/libufem_gpu.so``.  There is no CPU fallback: loading fails
loudly when the library is missing, and every call returns the reference's
AF_* codes, which the Python layer turns into exceptions.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libufem_gpu.so")

_lib = None

_l = C.POINTER(C.c_long)
_d = C.POINTER(C.c_double)
_i = C.POINTER(C.c_int)


class Tables(C.Structure):
    """ufem_tables: the reference's flat model tables (fem/fem_data.c)."""
    _fields_ = [
        ("nLen", C.c_long), ("n_x", _d), ("n_y", _d), ("n_z", _d),
        ("eLen", C.c_long), ("eType", _l), ("eRS", _l), ("eMP", _l), ("eFrom", _l), ("eNodesL", _l),
        ("rsLen", C.c_long), ("rsType", _l), ("rsFrom", _l), ("rsLenL", C.c_long), ("rsValL", _d),
        ("mpLen", C.c_long), ("mpType", _l), ("mpFrom", _l), ("mpLenL", C.c_long), ("mpValL", _d),
        ("nlLen", C.c_long), ("nlNode", _l), ("nlType", _l), ("nlDir", _l), ("nlVal", _d),
    ]


class McOptions(C.Structure):
    _fields_ = [("precision", C.c_int), ("tol", C.c_double), ("max_iters", C.c_long),
                ("replace_every", C.c_long), ("replace_near", C.c_double), ("use_graphs", C.c_int),
                ("tiles_per_block", C.c_int), ("unroll", C.c_int), ("lane_samples", C.c_int),
                ("coarse", C.c_int)]


class WarmOptions(C.Structure):
    _fields_ = [("n_modes", C.c_int), ("n_hidden", C.c_int), ("n_feat", C.c_int), ("feat_cols", C.c_long * 32),
                ("feat_log", C.c_int * 32), ("scale_col", C.c_long), ("n_snapshots", C.c_long),
                ("power_iters", C.c_int), ("epochs", C.c_int), ("batch", C.c_int), ("lr", C.c_float),
                ("seed", C.c_ulonglong), ("guess_mode", C.c_int), ("n_coarse", C.c_int), ("snap_tol", C.c_double),
                ("order_samples", C.c_int)]


class WarmTrainStats(C.Structure):
    _fields_ = [("cold_iters_max", C.c_long), ("cold_iters_mean", C.c_double), ("ms_solve", C.c_double),
                ("ms_basis", C.c_double), ("ms_train", C.c_double), ("sigma2", C.c_double * 80),
                ("loss_first", C.c_float), ("loss_last", C.c_float), ("epochs", C.c_int), ("steps", C.c_long),
                ("coarse_modes", C.c_int)]


class WarmStats(C.Structure):
    _fields_ = [("nsamp", C.c_long), ("fallbacks", C.c_long), ("guess_err_mean", C.c_double),
                ("guess_err_max", C.c_double), ("iters_mean", C.c_double), ("iters_max", C.c_long),
                ("cold_cap", C.c_long), ("ms_guess", C.c_double), ("ms_solve", C.c_double),
                ("ms_fallback", C.c_double), ("ms_total", C.c_double), ("kernel_launches", C.c_long),
                ("pcg_ms", C.c_double), ("pcg_bytes", C.c_double), ("pcg_launches", C.c_long)]


class McStats(C.Structure):
    _fields_ = [("ms_assemble", C.c_double), ("ms_pcg", C.c_double), ("ms_refine", C.c_double),
                ("ms_outputs", C.c_double), ("ms_total", C.c_double), ("pcg_iterations", C.c_long),
                ("pcg_bytes", C.c_double), ("spmv_bytes", C.c_double), ("kernel_launches", C.c_long),
                ("pcg_launches", C.c_long), ("pcg_launch_ms", C.c_double * 16), ("tiles_per_block", C.c_int),
                ("unroll", C.c_int), ("lane_samples", C.c_int), ("coarse_modes", C.c_int),
                ("phase_wall_ms", C.c_double * 6), ("phase_busy_ms", C.c_double * 6),
                ("true_residual_passes", C.c_long)]


_SIGS = {
    "ufem_last_error": (C.c_char_p, []),
    "ufem_device_info": (C.c_int, [_i, _i, _i, _l]),
    "ufem_selftest_barrier_timeout": (C.c_int, [C.c_int, C.c_int, _i, _d]),
    "ufem_selftest_mma_wait_timeout": (C.c_int, [C.c_long, _i]),
    "ufem_model_create": (C.c_int, [C.POINTER(Tables), C.POINTER(C.c_void_p)]),
    "ufem_read_input": (C.c_int, [C.c_char_p, C.POINTER(C.c_void_p)]),
    "ufem_convert_input": (C.c_int, [C.c_char_p, C.c_char_p]),
    "ufem_model_free": (None, [C.c_void_p]),
    "ufem_model_set_mc_vars": (C.c_int, [C.c_void_p, C.c_long, C.c_long, _l]),
    "ufem_ndof": (C.c_long, [C.c_void_p]),
    "ufem_get_ndoffld": (C.c_int, [C.c_void_p, _l]),
    "ufem_export_rowslot": (C.c_int, [C.c_void_p, _l, _l, _l, _l]),
    "ufem_bsr_shape": (C.c_int, [C.c_void_p, _l, _l, _l]),
    "ufem_get_bsr_pattern": (C.c_int, [C.c_void_p, _i, _i]),
    "ufem_num_colours": (C.c_long, [C.c_void_p]),
    "ufem_get_element_colours": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "ufem_fill_K": (C.c_int, [C.c_void_p, C.c_long]),
    "ufem_add_loads": (C.c_int, [C.c_void_p]),
    "ufem_add_disps": (C.c_int, [C.c_void_p]),
    "ufem_solve": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_long, _l]),
    "ufem_fem_solve": (C.c_int, [C.c_void_p, C.c_int, _l]),
    "ufem_get_u": (C.c_int, [C.c_void_p, _d]),
    "ufem_set_u": (C.c_int, [C.c_void_p, _d]),
    "ufem_get_F": (C.c_int, [C.c_void_p, _d]),
    "ufem_get_K_values": (C.c_int, [C.c_void_p, _d]),
    "ufem_get_element_matrices": (C.c_int, [C.c_void_p, _d]),
    "ufem_get_stresses": (C.c_int, [C.c_void_p, _d, _d]),
    "ufem_num_reactions": (C.c_long, [C.c_void_p]),
    "ufem_get_reactions": (C.c_int, [C.c_void_p, _l, _l, _d]),
    "ufem_get_phase_ms": (C.c_int, [C.c_void_p, _d, _d, _d, _d]),
    "ufem_get_ingest_ms": (C.c_int, [C.c_void_p, _d]),
    "ufem_eqs_cgwj": (C.c_int, [C.c_long, _l, _l, _l, _d, _d, _d, C.c_double, C.c_long]),
    "ufem_eqs_bicgs": (C.c_int, [C.c_long, _l, _l, _l, _d, _d, _d, C.c_double, C.c_long]),
    "ufem_eqs_cgwssor": (C.c_int, [C.c_long, _l, _l, _l, _d, _d, _d, C.c_double, C.c_long]),
    "ufem_eqs_cgwj_noalloc": (C.c_int, [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_void_p, C.c_double, C.c_long, _l]),
    "monte_dlib_interface_type": (C.c_long, []),
    "monte_nums_of_vars": (None, [C.c_char_p, _l, _l, _l]),
    "monte_ivar_name": (C.c_char_p, [C.c_char_p, C.c_long]),
    "monte_ovar_name": (C.c_char_p, [C.c_char_p, C.c_long]),
    "monte_init_lib_stuff": (C.c_int, [C.c_char_p]),
    "monte_clean_lib_stuff": (C.c_int, [C.c_char_p]),
    "monte_solution": (C.c_int, [C.c_char_p, _d, _d, C.c_long]),
    "monte_solution_batch": (C.c_int, [C.c_char_p, C.c_long, _d, _d, C.c_long, _i]),
    "ufem_mc_default_options": (None, [C.POINTER(McOptions)]),
    "ufem_mc_solve": (C.c_int, [C.c_int, C.POINTER(C.c_void_p), _l, C.POINTER(_d), C.POINTER(_d),
                                C.POINTER(_i), C.POINTER(_l), C.POINTER(_d), C.POINTER(McOptions)]),
    "ufem_mc_solve_device": (C.c_int, [C.c_int, C.POINTER(C.c_void_p), _l, C.POINTER(C.c_void_p),
                                       C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                       C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.POINTER(McOptions)]),
    "ufem_mc_get_stats": (C.c_int, [C.POINTER(McStats)]),
    "ufem_mc_autotune": (C.c_int, [C.c_int, C.POINTER(C.c_void_p), _l, C.POINTER(C.c_void_p), C.POINTER(McOptions),
                                   C.c_char_p, C.POINTER(McOptions)]),
    "ufem_mc_solve_serial": (C.c_int, [C.c_void_p, C.c_long, _d, _d, _i, _l, C.c_double]),
    "ufem_mc_set_coarse": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "ufem_mlp_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_ulonglong, C.POINTER(C.c_void_p)]),
    "ufem_mlp_free": (None, [C.c_void_p]),
    "ufem_mlp_num_params": (C.c_long, [C.c_void_p]),
    "ufem_mlp_get_params": (C.c_int, [C.c_void_p, C.POINTER(C.c_float)]),
    "ufem_mlp_set_params": (C.c_int, [C.c_void_p, C.POINTER(C.c_float)]),
    "ufem_mlp_forward": (C.c_int, [C.c_void_p, C.c_long, C.c_void_p, C.c_void_p]),
    "ufem_mlp_gradients": (C.c_int, [C.c_void_p, C.c_long, C.c_void_p, C.c_void_p, C.POINTER(C.c_float),
                                     C.POINTER(C.c_float)]),
    "ufem_mlp_train_step": (C.c_int, [C.c_void_p, C.c_long, C.c_void_p, C.c_void_p, C.c_float,
                                      C.POINTER(C.c_float)]),
    "ufem_tc_gemm_bf16": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
    "ufem_warm_default_options": (None, [C.POINTER(WarmOptions)]),
    "ufem_warm_create": (C.c_int, [C.c_void_p, C.POINTER(WarmOptions), C.POINTER(C.c_void_p)]),
    "ufem_warm_free": (None, [C.c_void_p]),
    "ufem_warm_train": (C.c_int, [C.c_void_p, C.c_long, C.c_void_p, C.POINTER(McOptions),
                                  C.POINTER(WarmTrainStats)]),
    "ufem_warm_guess": (C.c_int, [C.c_void_p, C.c_long, C.c_void_p, C.c_void_p]),
    "ufem_warm_solve": (C.c_int, [C.c_void_p, C.c_long, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                  C.POINTER(McOptions), C.POINTER(WarmStats)]),
    "ufem_warm_set_guess_mode": (C.c_int, [C.c_void_p, C.c_int]),
    "ufem_warm_set_guess_scale": (C.c_int, [C.c_void_p, C.c_double]),
    "ufem_warm_get_basis": (C.c_int, [C.c_void_p, _d, _d]),
    "ufem_dgemm_f64": (C.c_int, [C.c_int, C.c_int, C.c_long, C.c_void_p, C.c_void_p, C.c_void_p]),
    "ufem_sym_eig": (C.c_int, [C.c_int, _d, _d, _d, _i]),
}

# every symbol include/ufem_gpu.h declares (checked by the CPU test suite)
EXPORTED = sorted(_SIGS)


def load():
    """Load libufem_gpu.so or raise: the product has no CPU fallback."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"libufem_gpu.so is not built ({LIB_PATH}); run python -m ufem_b200.build")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class UfemError(RuntimeError):
    def __init__(self, fn: str, rv: int):
        msg = load().ufem_last_error()
        super().__init__(f"{fn} returned {rv}: {msg.decode() if msg else ''}")
        self.rv = rv


def check(fn: str, rv: int) -> int:
    if rv != 0:
        raise UfemError(fn, rv)
    return rv
