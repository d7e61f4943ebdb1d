"""ctypes binding of the C ABI (include/mspai_b200.h, include/mspai_b200_io.h).

The shared library is built in-tree (mspai_b200/libmspai_b200.so, sm_100a).
There is no fallback: if the library is missing, importing the compute entry
points raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmspai_b200.so")

MSPAI_OK = 0
ERRORS = {
    1: "MSPAI_ERR_PARAM", 2: "MSPAI_ERR_INPUT", 3: "MSPAI_ERR_SINGULAR",
    4: "MSPAI_ERR_CAPACITY", 5: "MSPAI_ERR_CUDA", 6: "MSPAI_ERR_NO_DEVICE",
    7: "MSPAI_ERR_STATE", 8: "MSPAI_ERR_IO", 9: "MSPAI_ERR_ALLOC",
}
MEM_HOST, MEM_DEVICE = 0, 1
PREC_FP64, PREC_MIXED = 0, 1


class mspai_csc(ctypes.Structure):
    _fields_ = [("nrows", ctypes.c_int32), ("ncols", ctypes.c_int32), ("nnz", ctypes.c_int64),
                ("colptr", ctypes.c_void_p), ("rowidx", ctypes.c_void_p),
                ("values", ctypes.c_void_p), ("mem", ctypes.c_int32)]


class mspai_params(ctypes.Structure):
    _fields_ = [("ep", ctypes.c_double), ("mn", ctypes.c_int32), ("ns", ctypes.c_int32),
                ("um", ctypes.c_int32), ("hs", ctypes.c_int32), ("cs", ctypes.c_int32),
                ("qr", ctypes.c_int32), ("ch", ctypes.c_int32), ("fg", ctypes.c_double),
                ("pk", ctypes.c_int32), ("pm", ctypes.c_int32), ("schur", ctypes.c_int32),
                ("rho", ctypes.c_double), ("bs", ctypes.c_int32), ("target", ctypes.c_int32),
                ("probing", ctypes.c_int32), ("prec", ctypes.c_int32), ("refine", ctypes.c_int32),
                ("batched", ctypes.c_int32), ("verbose", ctypes.c_int32),
                ("col_begin", ctypes.c_int32), ("col_end", ctypes.c_int32),
                ("keep_factors", ctypes.c_int32), ("reuse_factors", ctypes.c_int32)]


class mspai_stats(ctypes.Structure):
    _fields_ = [("columns", ctypes.c_int64), ("ls_solves", ctypes.c_int64),
                ("nnz_m", ctypes.c_int64), ("singular_columns", ctypes.c_int64),
                ("capacity_columns", ctypes.c_int64), ("bucket_columns", ctypes.c_int64 * 4),
                ("flops", ctypes.c_double), ("flops_dense", ctypes.c_double),
                ("gather_bytes", ctypes.c_double), ("setup_ms", ctypes.c_double),
                ("kernel_ms", ctypes.c_double * 4), ("kernel_launches", ctypes.c_int64),
                ("bucket_flops", ctypes.c_double * 4),
                ("reused_columns", ctypes.c_int64), ("factor_reuse_columns", ctypes.c_int64)]


class mspai_tuning(ctypes.Structure):
    _fields_ = [("smem_kb", ctypes.c_int32), ("fixed_arena_kb", ctypes.c_int32),
                ("fixed_arena_large_kb", ctypes.c_int32), ("warp_emax", ctypes.c_int32),
                ("warp_nmax", ctypes.c_int32), ("w_smem_kb", ctypes.c_int32),
                ("warp_emax_adaptive", ctypes.c_int32), ("warp_nmax_adaptive", ctypes.c_int32)]


class mspai_matrix(ctypes.Structure):
    _fields_ = [("nrows", ctypes.c_int32), ("ncols", ctypes.c_int32), ("nnz", ctypes.c_int64),
                ("colptr", ctypes.POINTER(ctypes.c_int64)),
                ("rowidx", ctypes.POINTER(ctypes.c_int32)),
                ("values", ctypes.POINTER(ctypes.c_double)), ("symmetric", ctypes.c_int32)]


# Every symbol the headers declare (checked by the CPU test suite).
EXPORTED = [
    "mspai_default_params", "mspai_validate_params", "mspai_create", "mspai_setup",
    "mspai_apply", "mspai_tune",
    "mspai_result_nnz", "mspai_result_copy", "mspai_column_info", "mspai_get_stats",
    "mspai_adjoint", "mspai_adjoint_weighted", "mspai_last_error", "mspai_free", "mspai_version",
    "mspai_matrix_view", "mspai_matrix_free", "mspai_mm_read", "mspai_mm_write",
    "mspai_probing_assemble", "mspai_pattern_generate", "mspai_row_structure",
    "mspai_measure_fma_peak", "mspai_setup_fixed_noalloc", "mspai_block_pattern_generate",
    "mspai_pattern_power2", "mspai_get_tuning", "mspai_set_tuning", "mspai_pattern_powers",
]

_lib = None


def load() -> ctypes.CDLL:
    """Loads the in-tree library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with "
                          "`make -C mspai_b200/csrc` (or __graft_entry__.build())")
    lib = ctypes.CDLL(LIB_PATH)
    V, I, P = ctypes.c_void_p, ctypes.c_int, ctypes.POINTER
    lib.mspai_default_params.argtypes = [P(mspai_params)]
    lib.mspai_default_params.restype = None
    lib.mspai_validate_params.argtypes = [P(mspai_params), ctypes.c_char_p, ctypes.c_int32]
    lib.mspai_validate_params.restype = I
    lib.mspai_create.argtypes = [P(V), ctypes.c_int32, V]
    lib.mspai_create.restype = I
    lib.mspai_setup.argtypes = [V, P(mspai_csc), P(mspai_csc), P(mspai_csc), P(mspai_csc),
                                P(mspai_csc), P(mspai_params)]
    lib.mspai_setup.restype = I
    lib.mspai_result_nnz.argtypes = [V, P(ctypes.c_int64)]
    lib.mspai_result_nnz.restype = I
    lib.mspai_result_copy.argtypes = [V, V, V, V, ctypes.c_int32]
    lib.mspai_result_copy.restype = I
    lib.mspai_tune.argtypes = [V, P(mspai_csc), P(mspai_csc), P(mspai_csc), P(mspai_csc),
                               P(mspai_csc), P(mspai_params), ctypes.c_int32,
                               P(ctypes.c_int32)]
    lib.mspai_tune.restype = I
    lib.mspai_get_tuning.argtypes = [V, P(mspai_tuning)]
    lib.mspai_get_tuning.restype = I
    lib.mspai_set_tuning.argtypes = [V, P(mspai_tuning)]
    lib.mspai_set_tuning.restype = I
    lib.mspai_apply.argtypes = [V, V, V, ctypes.c_int32]
    lib.mspai_apply.restype = I
    lib.mspai_column_info.argtypes = [V, V, V, V]
    lib.mspai_column_info.restype = I
    lib.mspai_get_stats.argtypes = [V, P(mspai_stats)]
    lib.mspai_get_stats.restype = I
    lib.mspai_adjoint.argtypes = [V, P(mspai_csc), P(mspai_csc), V, V, V,
                                  P(ctypes.c_double), ctypes.c_int32]
    lib.mspai_adjoint.restype = I
    lib.mspai_adjoint_weighted.argtypes = [V, P(mspai_csc), P(mspai_csc), V, ctypes.c_double, V,
                                           V, P(ctypes.c_double), ctypes.c_int32]
    lib.mspai_adjoint_weighted.restype = I
    lib.mspai_last_error.argtypes = [V]
    lib.mspai_last_error.restype = ctypes.c_char_p
    lib.mspai_free.argtypes = [V]
    lib.mspai_free.restype = None
    lib.mspai_measure_fma_peak.argtypes = [ctypes.c_int32, ctypes.c_int32,
                                           ctypes.POINTER(ctypes.c_double)]
    lib.mspai_measure_fma_peak.restype = I
    lib.mspai_setup_fixed_noalloc.argtypes = [P(mspai_csc), P(mspai_csc), P(mspai_csc),
                                              P(mspai_params), V, V, V, V, ctypes.c_char_p,
                                              ctypes.c_int32]
    lib.mspai_setup_fixed_noalloc.restype = I
    lib.mspai_version.argtypes = []
    lib.mspai_version.restype = ctypes.c_char_p
    lib.mspai_mm_read.argtypes = [ctypes.c_char_p, P(mspai_matrix), ctypes.c_char_p,
                                  ctypes.c_int32]
    lib.mspai_mm_read.restype = I
    lib.mspai_mm_write.argtypes = [ctypes.c_char_p, P(mspai_csc), ctypes.c_char_p,
                                   ctypes.c_int32]
    lib.mspai_mm_write.restype = I
    lib.mspai_matrix_free.argtypes = [P(mspai_matrix)]
    lib.mspai_matrix_free.restype = None
    lib.mspai_probing_assemble.argtypes = [P(mspai_csc), P(mspai_csc), P(mspai_csc),
                                           ctypes.c_double, P(mspai_matrix), P(mspai_matrix),
                                           ctypes.c_char_p, ctypes.c_int32]
    lib.mspai_probing_assemble.restype = I
    lib.mspai_pattern_generate.argtypes = [P(mspai_csc), ctypes.c_int32, P(mspai_matrix)]
    lib.mspai_pattern_generate.restype = I
    lib.mspai_block_pattern_generate.argtypes = [P(mspai_csc), ctypes.c_int32, ctypes.c_int32,
                                                 P(mspai_matrix)]
    lib.mspai_block_pattern_generate.restype = I
    lib.mspai_pattern_power2.argtypes = [P(mspai_csc), ctypes.c_double, ctypes.c_int32,
                                         P(mspai_matrix), ctypes.c_char_p, ctypes.c_int32]
    lib.mspai_pattern_power2.restype = I
    lib.mspai_pattern_powers.argtypes = [P(mspai_csc), ctypes.c_int32, ctypes.c_int32,
                                         P(mspai_matrix), ctypes.c_char_p, ctypes.c_int32]
    lib.mspai_pattern_powers.restype = I
    lib.mspai_row_structure.argtypes = [P(mspai_csc), ctypes.c_int32, P(mspai_matrix)]
    lib.mspai_row_structure.restype = I
    _lib = lib
    return lib


class MspaiError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{ERRORS.get(code, code)}: {message}")
        self.code = code
