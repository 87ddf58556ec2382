"""ctypes binding of the in-tree C ABI (include/hsc_c_api.h, libhsc_b200.so).

Loading fails loudly: there is no CPU fallback for the solver.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import os

HERE = Path(__file__).resolve().parent
# HSC_LIB selects another in-tree build of the same ABI (the self-checking one)
LIB_PATH = HERE / os.environ.get("HSC_LIB", "libhsc_b200.so")

HSC_OK = 0
HSC_ERR_INVALID = 1
HSC_ERR_NONSPD = 2
HSC_ERR_BREAKDOWN = 3
HSC_ERR_NOCONV = 4
HSC_ERR_NONDESCENT = 5
HSC_ERR_RESIDUAL = 6
HSC_ERR_CUDA = 7
HSC_ERR_TIMEOUT = 8
HSC_ERR_ALLOC = 9
HSC_ERR_NOTREADY = 10
STATUS_NAMES = {0: "ok", 1: "invalid", 2: "nonspd", 3: "breakdown", 4: "noconv", 5: "nondescent",
                6: "residual", 7: "cuda", 8: "timeout", 9: "alloc", 10: "notready"}

HSC_FP64, HSC_FP32, HSC_BF16 = 0, 1, 2
HSC_ABD_NEUMANN, HSC_ABD_ADAPTIVE, HSC_ABD_EXACT = 0, 1, 2
HSC_PRECOND_NEUMANN, HSC_PRECOND_POLY, HSC_PRECOND_SCHUR_POLY, HSC_PRECOND_LEARNED = 0, 1, 2, 3
HSC_PRECOND_BLOCK, HSC_PRECOND_BLOCK_LEARNED = 4, 5
HSC_MAX_POLY = 16
HSC_FEATURES, HSC_MLP_HIDDEN, HSC_MLP_OUT, HSC_MLP_PARAMS = 16, 64, 8, 5768


class Options(C.Structure):
    _fields_ = [
        ("max_rank", C.c_int32),
        ("aca_rtol", C.c_double),
        ("neumann_order", C.c_int32),
        ("omega", C.c_double),
        ("max_iter", C.c_int32),
        ("tol", C.c_double),
        ("abd_inverse", C.c_int32),
        ("abd_inverse_tol", C.c_double),
        ("full_residual_limit", C.c_double),
        ("precision", C.c_int32),
        ("preconditioner", C.c_int32),
        ("poly_degree", C.c_int32),
        ("poly_weights", C.c_double * HSC_MAX_POLY),
        ("residual_replacement", C.c_int32),
        ("refine_target", C.c_double),
        ("max_refinements", C.c_int32),
        ("fallback_on_stall", C.c_int32),
        ("threads_per_row", C.c_int32),
        ("spin_limit", C.c_int64),
        ("check_residual", C.c_int32),
        ("trace_iterations", C.c_int32),
        ("resident", C.c_int32),
        ("fuse_update", C.c_int32),
        ("aca_cluster", C.c_int32),
        ("reorder", C.c_int32),
        ("aca_components", C.c_int32),
        ("lanczos_stats", C.c_int32),
        ("coupled_part_weight", C.c_double),
        ("graph_replay", C.c_int32),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("status", C.c_int32),
        ("fem_dofs", C.c_int32), ("abd_dofs", C.c_int32), ("active_fem_dofs", C.c_int32), ("rank", C.c_int32),
        ("pcg_iterations", C.c_int32), ("neumann_doublings", C.c_int32), ("refinement_steps", C.c_int32),
        ("precision", C.c_int32), ("preconditioner", C.c_int32), ("fallback", C.c_int32), ("accepted", C.c_int32),
        ("residual_replacements", C.c_int32),
        ("aca_relative_error", C.c_double),
        ("schur_relative_residual", C.c_double),
        ("full_relative_residual", C.c_double),
        ("abd_inverse_residual", C.c_double),
        ("full_residual_limit", C.c_double),
        ("descent", C.c_double),
        ("setup_ms", C.c_double), ("pcg_ms", C.c_double), ("total_ms", C.c_double),
        ("lanczos_min", C.c_double), ("lanczos_max", C.c_double),
        ("stage_ms", C.c_double * 8),
        ("nnzb", C.c_int64),
        ("analysis_ms", C.c_double),
    ]

    def as_dict(self):
        d = {name: getattr(self, name) for name, _ in self._fields_}
        d["stage_ms"] = list(self.stage_ms)
        return d


class BCOO3(C.Structure):
    _fields_ = [("d_rows", C.c_void_p), ("d_cols", C.c_void_p), ("d_values", C.c_void_p),
                ("nnzb", C.c_int64), ("nblock", C.c_int32)]


class Layout(C.Structure):
    _fields_ = [("qo", C.c_int32), ("qm", C.c_int32), ("fo", C.c_int32), ("fn", C.c_int32)]


# the exported symbols, as include/hsc_c_api.h declares them
EXPORTS = {
    "hsc_options_default": (C.c_int, [C.POINTER(Options)]),
    "hsc_options_reference": (C.c_int, [C.POINTER(Options)]),
    "hsc_create": (C.c_int, [C.POINTER(Options), C.POINTER(C.c_void_p)]),
    "hsc_destroy": (None, [C.c_void_p]),
    "hsc_set_options": (C.c_int, [C.c_void_p, C.POINTER(Options)]),
    "hsc_last_error": (C.c_char_p, [C.c_void_p]),
    "hsc_solve": (C.c_int, [C.c_void_p, C.POINTER(BCOO3), C.POINTER(Layout), C.c_void_p, C.c_void_p,
                            C.c_void_p, C.POINTER(Stats)]),
    "hsc_solve_batch": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(BCOO3), C.POINTER(Layout),
                                  C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.c_int32, C.c_void_p,
                                  C.POINTER(Stats)]),
    "hsc_spmv": (C.c_int, [C.c_void_p, C.POINTER(BCOO3), C.POINTER(Layout), C.c_void_p, C.c_void_p, C.c_void_p]),
    "hsc_spmv_noalloc": (C.c_int, [C.POINTER(BCOO3), C.c_void_p, C.c_void_p, C.c_void_p]),
    "hsc_get_factors": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                  C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.c_void_p]),
    "hsc_get_abd_inverse": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p]),
    "hsc_debug_block_plan": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32]),
    "hsc_get_partition": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.c_void_p,
                                    C.c_void_p]),
    "hsc_partition_nodes": (C.c_int, [C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]),
    "hsc_get_trace": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "hsc_version": (C.c_int, []),
    "hsc_kernel_launches": (C.c_longlong, []),
    "hsc_debug_checks": (C.c_int, [C.POINTER(C.c_longlong)]),
    "hsc_debug_barrier_selftest": (C.c_int, [C.c_int32, C.c_int32, C.c_int64, C.c_int64, C.POINTER(C.c_int32),
                                             C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "hsc_debug_dmv_accumulate": (C.c_int, [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double,
                                           C.c_void_p]),
    "hsc_set_learned_model": (C.c_int, [C.c_void_p, C.c_void_p]),
    "hsc_get_features": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p]),
    "hsc_get_poly_weights": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.POINTER(C.c_int32)]),
    "hsc_get_lanczos": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.POINTER(C.c_int32)]),
    "hsc_mlp_forward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                  C.c_void_p, C.c_void_p]),
    "hsc_mlp_backward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "hsc_poly_ls_loss": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_float,
                                   C.c_void_p, C.c_void_p, C.c_void_p]),
    "hsc_adam_step": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_float,
                                C.c_float, C.c_float, C.c_float, C.c_float, C.c_int32, C.c_void_p]),
    "hsc_fem_assembler_create": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_double, C.c_double,
                                           C.c_double, C.c_int32, C.POINTER(C.c_void_p)]),
    "hsc_fem_assembler_destroy": (None, [C.c_void_p]),
    "hsc_fem_pattern": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_int64)]),
    "hsc_fem_assemble": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_int32),
                                   C.c_void_p]),
    "hsc_fem_feasible_step": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_int32,
                                        C.POINTER(C.c_double), C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                        C.c_void_p]),
    "hsc_coupling_assembler_create": (C.c_int, [C.c_int32, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_int32,
                                                C.c_void_p, C.c_int32, C.c_int32, C.c_int32,
                                                C.POINTER(C.c_void_p)]),
    "hsc_coupling_assembler_destroy": (C.c_int, [C.c_void_p]),
    "hsc_coupling_assemble": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32,
                                        C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.c_void_p]),
    "hsc_coupling_read": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.c_void_p]),
}

_LIB = None


def load():
    """Load libhsc_b200.so and declare every exported signature."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m hsc_reimpl_b200.build` "
                           "(the solver has no CPU fallback)")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in EXPORTS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


class HSCError(RuntimeError):
    def __init__(self, code, message):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {message}")
        self.code = code
