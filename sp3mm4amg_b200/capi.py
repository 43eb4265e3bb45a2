"""ctypes binding of ``lib/libsp3mm_b200.so`` (declared in include/sp3mm_b200.h).

Loading fails loudly when the library is missing: there is no CPU path.
"""
from __future__ import annotations

import ctypes
import os

from .spmat import CONFIG_P, SPMAT_P, idx_t, spmat

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libsp3mm_b200.so")

# Reference-named entry points (per OFF_F suffix).
SPMM_UB_NAMES = ("spmmSerial_", "spmmRowByRow_", "spmmRowByRow1DBlocks_", "spmmRowByRow2DBlocks_",
                 "spmmRowByRow2DBlocksAllocated_")
SPMM_SYMBNUM_NAMES = ("spmmRowByRow_SymbNum_", "spmmRowByRow1DBlocks_SymbNum_",
                      "spmmRowByRow2DBlocks_SymbNum_", "spmmRowByRow2DBlocksAllocated_SymbNum_")
SP3MM_NAMES = ("sp3mmRowByRowPair_", "sp3mmRowByRowMerged_", "sp3mmRowByRowPair_SymbNum_",
               "sp3mmRowByRowMerged_SymbNum_", "sp3mmRowByRowPairRight_")
SIZE_NAMES = ("SpMM_Symb___", "spMMSizeUpperbound_", "spMMSizeUpperboundColParts_")

# Layer-2 names with (restype, argtypes).
_c = ctypes
DEVICE_API = {
    "sp3mm_ctx_create": (_c.c_int, [_c.c_int, _c.POINTER(_c.c_void_p)]),
    "sp3mm_ctx_destroy": (_c.c_int, [_c.c_void_p]),
    "sp3mm_ctx_set_stream": (_c.c_int, [_c.c_void_p, _c.c_void_p]),
    "sp3mm_ctx_stream": (_c.c_void_p, [_c.c_void_p]),
    "sp3mm_ctx_set_workspace_limit": (_c.c_int, [_c.c_void_p, _c.c_size_t]),
    "sp3mm_ctx_trim": (_c.c_int, [_c.c_void_p]),
    "sp3mm_ctx_last_error": (_c.c_char_p, [_c.c_void_p]),
    "sp3mm_ctx_launches": (_c.c_uint64, [_c.c_void_p]),
    "sp3mm_ctx_sync": (_c.c_int, [_c.c_void_p]),
    "sp3mm_ctx_set_tuning": (_c.c_int, [_c.c_void_p, _c.c_int, _c.c_int, _c.c_int]),
    "sp3mm_ctx_set_profiling": (_c.c_int, [_c.c_void_p, _c.c_int]),
    "sp3mm_ctx_profile_report": (_c.c_int, [_c.c_void_p, _c.c_char_p, _c.c_size_t]),
    "sp3mm_dcsr_upload": (_c.c_int, [_c.c_void_p, SPMAT_P, _c.c_int, _c.c_int, _c.c_void_p]),
    "sp3mm_dcsr_upload_arrays": (_c.c_int, [_c.c_void_p, _c.c_int64, _c.c_int64, _c.c_int64,
                                            _c.c_void_p, _c.c_void_p, _c.c_void_p, _c.c_int,
                                            _c.c_void_p]),
    "sp3mm_dcsr_download": (_c.c_int, [_c.c_void_p, _c.c_void_p, _c.c_int,
                                       _c.POINTER(_c.c_void_p)]),
    "sp3mm_dcsr_download_arrays": (_c.c_int, [_c.c_void_p, _c.c_void_p, _c.c_void_p,
                                              _c.c_void_p, _c.c_void_p]),
    "sp3mm_dcsr_free": (_c.c_int, [_c.c_void_p, _c.c_void_p]),
    "sp3mm_dcsr_set_values": (_c.c_int, [_c.c_void_p, _c.c_void_p, _c.c_void_p]),
    "sp3mm_spmm": (_c.c_int, [_c.c_void_p, _c.c_void_p, _c.c_void_p, _c.c_int, _c.c_int,
                              _c.c_void_p]),
    "sp3mm_rap": (_c.c_int, [_c.c_void_p, _c.c_void_p, _c.c_void_p, _c.c_void_p, _c.c_int,
                             _c.c_int, _c.c_int, _c.c_void_p]),
    "sp3mm_spmm_rowsizes": (_c.c_int, [_c.c_void_p, _c.c_void_p, _c.c_void_p, _c.c_int,
                                       _c.c_void_p, _c.POINTER(_c.c_int64)]),
    "sp3mm_transpose": (_c.c_int, [_c.c_void_p, _c.c_void_p, _c.c_void_p]),
    "sp3mm_rap_direct_noalloc": (_c.c_int, [_c.c_void_p, _c.c_void_p, _c.c_void_p, _c.c_void_p,
                                            _c.c_void_p, _c.c_void_p, _c.c_int64,
                                            _c.POINTER(_c.c_int64), _c.c_void_p]),
    "sp3mm_rap_memory_estimate": (_c.c_int, [_c.c_void_p, _c.c_void_p, _c.c_void_p, _c.c_int,
                                             _c.c_int, _c.POINTER(_c.c_size_t)]),
    "sp3mm_block_prolongator": (_c.c_int, [_c.c_void_p, _c.c_void_p, _c.c_void_p, _c.c_int,
                                           _c.c_int, _c.c_double, _c.c_int, _c.c_void_p]),
    "sp3mm_hierarchy_build": (_c.c_int, [_c.c_void_p, _c.c_void_p, _c.c_void_p, _c.c_int,
                                         _c.c_int, _c.c_double, _c.c_int64, _c.c_int, _c.c_int,
                                         _c.c_int, _c.c_int, _c.POINTER(_c.c_void_p)]),
    "sp3mm_hierarchy_levels": (_c.c_int, [_c.c_void_p]),
    "sp3mm_hierarchy_get": (_c.c_int, [_c.c_void_p, _c.c_int, _c.c_void_p, _c.c_void_p,
                                       _c.c_void_p]),
    "sp3mm_hierarchy_free": (_c.c_int, [_c.c_void_p, _c.c_void_p]),
    "sp3mm_hierarchy_build_batch": (_c.c_int, [_c.c_void_p, _c.c_int, _c.c_void_p, _c.c_void_p,
                                               _c.c_void_p, _c.c_int, _c.c_double, _c.c_int64,
                                               _c.c_int, _c.c_int, _c.c_void_p]),
    "sp3mm_batch_create": (_c.c_int, [_c.c_void_p, _c.c_int, _c.c_void_p, _c.c_void_p,
                                      _c.c_void_p, _c.c_void_p, _c.c_int,
                                      _c.POINTER(_c.c_void_p)]),
    "sp3mm_batch_set_tuning": (_c.c_int, [_c.c_void_p, _c.c_int, _c.c_int, _c.c_int, _c.c_int,
                                          _c.c_void_p]),
    "sp3mm_batch_set_flavour": (_c.c_int, [_c.c_void_p, _c.c_int]),
    "sp3mm_batch_plan": (_c.c_int, [_c.c_void_p]),
    "sp3mm_batch_execute": (_c.c_int, [_c.c_void_p]),
    "sp3mm_batch_run": (_c.c_int, [_c.c_void_p]),
    "sp3mm_batch_autotune": (_c.c_int, [_c.c_void_p, _c.c_int, _c.c_char_p, _c.c_size_t]),
    "sp3mm_batch_result": (_c.c_int, [_c.c_void_p, _c.c_int, _c.c_void_p]),
    "sp3mm_batch_info": (_c.c_int, [_c.c_void_p, _c.POINTER(_c.c_int64),
                                    _c.POINTER(_c.c_int64), _c.POINTER(_c.c_int),
                                    _c.POINTER(_c.c_int), _c.POINTER(_c.c_int64)]),
    "sp3mm_batch_free": (_c.c_int, [_c.c_void_p]),
    "sp3mm_server_create": (_c.c_int, [_c.c_void_p, _c.c_int, _c.c_double,
                                       _c.POINTER(_c.c_void_p)]),
    "sp3mm_server_now": (_c.c_double, [_c.c_void_p]),
    "sp3mm_server_submit": (_c.c_int, [_c.c_void_p, _c.c_int64, _c.c_int64, _c.c_void_p,
                                       _c.c_void_p, _c.c_void_p, _c.c_void_p, _c.c_int,
                                       _c.c_int, _c.c_double, _c.c_int64, _c.c_int, _c.c_int,
                                       _c.c_double, _c.POINTER(_c.c_int64)]),
    "sp3mm_server_submit_ops": (_c.c_int, [_c.c_void_p, _c.c_int64, _c.c_int64, _c.c_void_p,
                                           _c.c_void_p, _c.c_void_p, _c.c_int, _c.c_void_p,
                                           _c.c_void_p, _c.c_void_p, _c.c_void_p, _c.c_void_p,
                                           _c.c_void_p, _c.c_int, _c.c_double,
                                           _c.POINTER(_c.c_int64)]),
    "sp3mm_server_step": (_c.c_int, [_c.c_void_p, _c.POINTER(_c.c_int)]),
    "sp3mm_server_poll": (_c.c_int, [_c.c_void_p, _c.c_int64, _c.POINTER(_c.c_int),
                                     _c.POINTER(_c.c_double), _c.POINTER(_c.c_double)]),
    "sp3mm_server_take": (_c.c_int, [_c.c_void_p, _c.c_int64, _c.POINTER(_c.c_void_p)]),
    "sp3mm_server_stats": (_c.c_int, [_c.c_void_p, _c.POINTER(_c.c_int64),
                                      _c.POINTER(_c.c_int64), _c.POINTER(_c.c_double),
                                      _c.POINTER(_c.c_double), _c.POINTER(_c.c_double),
                                      _c.POINTER(_c.c_int64), _c.POINTER(_c.c_int),
                                      _c.POINTER(_c.c_int64)]),
    "sp3mm_server_free": (_c.c_int, [_c.c_void_p]),
}

# Host-side MatrixMarket entry points with (restype, argtypes).
HOST_API = {
    "MMtoCSR": (_c.c_void_p, [_c.c_char_p]),
    "colsOffsetsPartitioningUnifRanges_0": (_c.c_void_p, [SPMAT_P, _c.c_uint]),
    "colsOffsetsPartitioningUnifRanges_1": (_c.c_void_p, [SPMAT_P, _c.c_uint]),
    "colsPartitioningUnifRanges_0": (_c.c_void_p, [SPMAT_P, _c.c_uint]),
    "colsPartitioningUnifRanges_1": (_c.c_void_p, [SPMAT_P, _c.c_uint]),
    "colsPartitioningUnifRangesOffsetsAux_0": (_c.c_void_p, [SPMAT_P, _c.c_uint, _c.c_void_p]),
    "colsPartitioningUnifRangesOffsetsAux_1": (_c.c_void_p, [SPMAT_P, _c.c_uint, _c.c_void_p]),
    "sp3mm_write_mm": (_c.c_int, [SPMAT_P, _c.c_int, _c.c_char_p]),
    "sp3mm_spmat_sort_rows": (_c.c_int, [SPMAT_P, _c.c_int]),
}

# Error codes, flavours, variants, value types (include/sp3mm_b200.h).
SP3MM_OK, SP3MM_ECUDA, SP3MM_EINVAL, SP3MM_ENOMEM, SP3MM_ELIMIT, SP3MM_EDEVICE = range(6)
UB, SYMBNUM = 0, 1
BATCH_SPMM, BATCH_RAP = 0, 1
PAIR, DIRECT, PAIR_RIGHT = 0, 1, 2
F64, F32 = 0, 1


class sp3mm_dcsr(ctypes.Structure):
    _fields_ = [
        ("M", ctypes.c_int32),
        ("N", ctypes.c_int32),
        ("nnz", ctypes.c_int64),
        ("row_ptr", ctypes.c_void_p),
        ("col", ctypes.c_void_p),
        ("val", ctypes.c_void_p),
        ("val_type", ctypes.c_int32),
        ("max_row", ctypes.c_int32),
    ]


def all_symbols() -> list[str]:
    """Every symbol include/sp3mm_b200.h declares (functions and globals)."""
    names = []
    for off in (0, 1):
        for n in SPMM_UB_NAMES + SPMM_SYMBNUM_NAMES + SP3MM_NAMES + SIZE_NAMES:
            names.append(f"{n}{off}")
    names += list(DEVICE_API)
    names += list(HOST_API)
    names += ["Start", "End", "Elapsed", "ElapsedInternal"]
    return names


_LIB = None


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load the CUDA library (raises if it was not built)."""
    global _LIB
    if _LIB is not None and path == LIB_PATH:
        return _LIB
    if not os.path.exists(path):
        raise RuntimeError(
            f"{path} is missing: build it with `make -C sp3mm4amg_b200/csrc` "
            "(the library has no CPU fallback)")
    lib = ctypes.CDLL(path)
    for off in (0, 1):
        for n in SPMM_UB_NAMES + SPMM_SYMBNUM_NAMES:
            f = getattr(lib, f"{n}{off}")
            f.restype = ctypes.c_void_p
            f.argtypes = [SPMAT_P, SPMAT_P, CONFIG_P]
        for n in SP3MM_NAMES:
            f = getattr(lib, f"{n}{off}")
            f.restype = ctypes.c_void_p
            f.argtypes = [SPMAT_P, SPMAT_P, SPMAT_P, CONFIG_P, ctypes.c_void_p]
        f = getattr(lib, f"SpMM_Symb___{off}")
        f.restype = ctypes.c_void_p
        f.argtypes = [ctypes.c_int, SPMAT_P, SPMAT_P]
        f = getattr(lib, f"spMMSizeUpperbound_{off}")
        f.restype = ctypes.c_void_p
        f.argtypes = [SPMAT_P, SPMAT_P]
        f = getattr(lib, f"spMMSizeUpperboundColParts_{off}")
        f.restype = ctypes.c_void_p
        f.argtypes = [SPMAT_P, SPMAT_P, ctypes.c_ushort, ctypes.POINTER(idx_t)]
    for name, (res, args) in list(DEVICE_API.items()) + list(HOST_API.items()):
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    if path == LIB_PATH:
        _LIB = lib
    return lib


def global_double(lib: ctypes.CDLL, name: str) -> float:
    return ctypes.c_double.in_dll(lib, name).value
