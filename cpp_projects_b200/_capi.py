"""ctypes binding of the C ABI declared in include/bfs.h.

The shared library is built in-tree (``python -m cpp_projects_b200.build``)
and loaded from ``cpp_projects_b200/lib``.  There is no fallback: if the
library is missing, importing a compute entry point raises.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libbfs_b200.so"

BFS_OK, BFS_ERR_ARG, BFS_ERR_CUDA, BFS_ERR_OVERFLOW, BFS_ERR_TIMEOUT, BFS_ERR_ALLOC, \
    BFS_ERR_UNSUPPORTED = range(7)
STATUS_NAMES = {0: "BFS_OK", 1: "BFS_ERR_ARG", 2: "BFS_ERR_CUDA", 3: "BFS_ERR_OVERFLOW",
                4: "BFS_ERR_TIMEOUT", 5: "BFS_ERR_ALLOC", 6: "BFS_ERR_UNSUPPORTED"}
BFS_WIDTHS_POW2, BFS_WIDTHS_ALL = 0, 1
BFS_FDMT_EXTERNAL_WS = 1
BFS_FUSE_AUTOTUNE = -2
BFS_SEG_SINGLE_BUFFER = 1
BFS_PREC_F32, BFS_PREC_F16, BFS_PREC_BF16 = 0, 1, 2
BFS_PLAN_KEITH, BFS_PLAN_PRAVIR = 0, 1


class BfsError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class FdmtDesc(ctypes.Structure):
    _fields_ = [("fmin", ctypes.c_float), ("fmax", ctypes.c_float), ("nchan", ctypes.c_int),
                ("ncols", ctypes.c_int), ("max_dt", ctypes.c_int), ("plan_kind", ctypes.c_int),
                ("precision", ctypes.c_int), ("fuse_depth", ctypes.c_int),
                ("flags", ctypes.c_int), ("head_tile", ctypes.c_int), ("dt_min", ctypes.c_int),
                ("dt_step", ctypes.c_int), ("tsamp", ctypes.c_float), ("seg_levels", ctypes.c_int),
                ("seg_rows", ctypes.c_int), ("seg_threads", ctypes.c_int), ("seg_flags", ctypes.c_int)]


class FdmtInfo(ctypes.Structure):
    _fields_ = [("niter", ctypes.c_int), ("rows_level0", ctypes.c_int),
                ("fuse_depth", ctypes.c_int), ("rows_total", ctypes.c_int64),
                ("workspace_bytes", ctypes.c_size_t), ("alg_bytes", ctypes.c_double),
                ("out_rows", ctypes.c_int), ("hbm_passes", ctypes.c_int), ("seg_levels", ctypes.c_int),
                ("sched_bytes", ctypes.c_double)]


class ChunkDesc(ctypes.Structure):
    _fields_ = [("fmin", ctypes.c_float), ("fmax", ctypes.c_float), ("npol", ctypes.c_int),
                ("nchan", ctypes.c_int), ("len_sft", ctypes.c_int), ("nbin", ctypes.c_int),
                ("nfft", ctypes.c_int), ("noverlap", ctypes.c_int), ("tsamp", ctypes.c_float),
                ("max_dt", ctypes.c_int), ("reserved", ctypes.c_int * 6)]


class BatchDesc(ctypes.Structure):
    _fields_ = [("nbeams", ctypes.c_int), ("beams", ctypes.POINTER(FdmtDesc)),
                ("widths_mode", ctypes.c_int), ("param", ctypes.c_int), ("thr", ctypes.c_float),
                ("metrics", ctypes.c_int * 3), ("capacity", ctypes.c_uint32),
                ("use_graph", ctypes.c_int), ("reserved", ctypes.c_int * 8)]


class GuppiHeader(ctypes.Structure):
    _fields_ = [("nbits", ctypes.c_int), ("chan_bw", ctypes.c_float), ("npol", ctypes.c_int),
                ("directio", ctypes.c_int), ("obsfreq", ctypes.c_float), ("nchan", ctypes.c_int),
                ("obsbw", ctypes.c_float), ("blocsize", ctypes.c_int64), ("telescope", ctypes.c_int),
                ("tbin", ctypes.c_float), ("straight_order", ctypes.c_int), ("data_offset", ctypes.c_int64),
                ("nsamp", ctypes.c_int64), ("fmin", ctypes.c_float), ("fmax", ctypes.c_float),
                ("reserved", ctypes.c_int * 4)]


class GuppiSession(ctypes.Structure):
    _fields_ = [("len_sft", ctypes.c_int), ("noverlap", ctypes.c_int), ("len_chunk", ctypes.c_int64),
                ("ncoherent", ctypes.c_int), ("optimal_overlap", ctypes.c_int), ("fmin", ctypes.c_float),
                ("fmax", ctypes.c_float), ("tsamp", ctypes.c_float), ("d_min", ctypes.c_float),
                ("d_max", ctypes.c_float), ("reserved", ctypes.c_int * 4)]


class Cand(ctypes.Structure):
    _fields_ = [("mt", ctypes.c_int), ("mdt", ctypes.c_int), ("mwidth", ctypes.c_int),
                ("msnr", ctypes.c_float)]


_P = ctypes.c_void_p
_I = ctypes.c_int
_U32 = ctypes.c_uint32
_I64 = ctypes.c_int64
_F = ctypes.c_float

# name -> (restype, argtypes)
_SIGNATURES = {
    "bfs_last_error": (ctypes.c_char_p, []),
    "bfs_version": (ctypes.c_char_p, []),
    "bfs_trim_scratch": (_I, []),
    "bfs_fdmt_plan_create": (_I, [ctypes.POINTER(FdmtDesc), ctypes.POINTER(_P)]),
    "bfs_fdmt_plan_create_host": (_I, [ctypes.POINTER(FdmtDesc), ctypes.POINTER(_P)]),
    "bfs_fdmt_autotune": (_I, [ctypes.POINTER(FdmtDesc), ctypes.POINTER(_I), ctypes.POINTER(_I),
                               ctypes.POINTER(_F)]),
    "bfs_fdmt_autotune_desc": (_I, [ctypes.POINTER(FdmtDesc), ctypes.POINTER(FdmtDesc), ctypes.POINTER(_F)]),
    "bfs_fdmt_plan_passes": (_I, [_P, ctypes.POINTER(_I), _P, _I]),
    "bfs_fdmt_plan_segment": (_I, [_P, _I, _P, _I, _P, _I]),
    "bfs_fdmt_plan_destroy": (_I, [_P]),
    "bfs_fdmt_plan_info": (_I, [_P, ctypes.POINTER(FdmtInfo)]),
    "bfs_fdmt_plan_rows": (_I, [_P, _P, _I]),
    "bfs_fdmt_plan_tables": (_I, [_P, _I, _P, _P, _P, _I]),
    "bfs_fdmt_plan_head": (_I, [_P, _P, _P, _I, _P, _I]),
    "bfs_fdmt_execute": (_I, [_P, _P, _P, _I, _P]),
    "bfs_fdmt_workspace_size": (_I, [_P, ctypes.POINTER(ctypes.c_size_t)]),
    "bfs_fdmt_execute_ws": (_I, [_P, _P, _P, _I, _P, ctypes.c_size_t, _P]),
    "bfs_fdmt_execute_noalloc": (_I, [_P, _P, _P, _I, _P]),
    "bfs_selftest_divide": (_I, [_I, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint32), _P]),
    "bfs_fdmt_noalloc_scratch_bytes": (_I, [_P, ctypes.POINTER(ctypes.c_size_t),
                                            ctypes.POINTER(ctypes.c_size_t)]),
    "bfs_preproc_calc_fdmt_inputs": (_I, [_P, _I, _I, _P, _P, _P]),
    "bfs_fdmt_normalize": (_I, [_P, _P, _I64, _P, _P]),
    "bfs_norm_rows": (_I, [_P, _P, _I, _I, _P, _P]),
    "bfs_row_stats": (_I, [_P, _I, _I, _P, _P]),
    "bfs_boxcar_gather": (_I, [_P, _I, _I, _P, _F, _P, _I, _I, _I, _P, _U32,
                               ctypes.POINTER(_U32), _P]),
    "bfs_cluster": (_I, [_P, _U32, _P, _P, _P, _P, ctypes.POINTER(_U32), _P]),
    "bfs_select_delegates": (_I, [_P, _P, _U32, _P, _U32, _P, _P]),
    "bfs_cluster_grouped": (_I, [_P, _U32, _P, _U32, _P, _P, _P, _P, ctypes.POINTER(_U32), _P]),
    "bfs_fdmt_plan_delays": (_I, [_P, _P, _I, _P, _P, _I]),
    "bfs_fdmt_execute_row_mask": (_I, [_P, _P, _I, _P, _P]),
    "bfs_fdmt_adjoint": (_I, [_P, _P, _P, _P]),
    "bfs_fdmt_adjoint_workspace_size": (_I, [_P, ctypes.POINTER(ctypes.c_size_t)]),
    "bfs_fdmt_adjoint_ws": (_I, [_P, _P, _P, _P, ctypes.c_size_t, _P]),
    "bfs_boxcar_snr_cells": (_I, [_P, _I, _I, _P, _P, _I, _P, _P]),
    "bfs_boxcar_snr_cells_adjoint": (_I, [_P, _I, _I, _P, _P, _I, _P, _P, _P, _P]),
    "bfs_cut_fragment": (_I, [_P, _I, _I, _I, _I, _P, ctypes.POINTER(_I), ctypes.POINTER(_I),
                              ctypes.POINTER(_I), _P]),
    "bfs_guppi_parse_header": (_I, [_P, ctypes.c_size_t, _P]),
    "bfs_guppi_open": (_I, [ctypes.c_char_p, ctypes.POINTER(_P)]),
    "bfs_guppi_close": (_I, [_P]),
    "bfs_guppi_blocks": (_I, [_P, ctypes.POINTER(_I)]),
    "bfs_guppi_block_header": (_I, [_P, _I, _P]),
    "bfs_guppi_chunk_count": (_I, [_P, _I, ctypes.c_int64, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)]),
    "bfs_guppi_read_chunk": (_I, [_P, _I, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, _P, ctypes.c_size_t]),
    "bfs_guppi_reader_create": (_I, [_P, ctypes.c_int64, ctypes.c_int64, _I, _I, ctypes.POINTER(_P)]),
    "bfs_guppi_reader_next": (_I, [_P, _P, _P, ctypes.POINTER(_P), ctypes.POINTER(_I),
                                   ctypes.POINTER(ctypes.c_int64)]),
    "bfs_guppi_reader_destroy": (_I, [_P]),
    "bfs_guppi_session_plan": (_I, [_P, ctypes.c_float, ctypes.c_double, ctypes.c_double, _I, _I, _P]),
    "bfs_batch_create": (_I, [ctypes.POINTER(BatchDesc), ctypes.POINTER(_P)]),
    "bfs_batch_destroy": (_I, [_P]),
    "bfs_batch_run": (_I, [_P, _P, _P]),
    "bfs_batch_submit": (_I, [_P, _P, _P]),
    "bfs_batch_collect": (_I, [_P, _P]),
    "bfs_batch_run_host": (_I, [_P, _P, _P, _P]),
    "bfs_batch_counts": (_I, [_P, ctypes.POINTER(_U32), ctypes.POINTER(_U32)]),
    "bfs_batch_beam_results": (_I, [_P, _I, _P, _P, _I, ctypes.POINTER(_I), ctypes.POINTER(_U32)]),
    "bfs_chunk_create": (_I, [ctypes.POINTER(ChunkDesc), ctypes.POINTER(_P)]),
    "bfs_chunk_destroy": (_I, [_P]),
    "bfs_chunk_info": (_I, [_P, _P, _I]),
    "bfs_chunk_coherent_dms": (_I, [ctypes.c_double, ctypes.c_double, _I, _P, _I]),
    "bfs_chunk_unpack": (_I, [_P, _P, _P, _P]),
    "bfs_chunk_forward_fft": (_I, [_P, _P, _P]),
    "bfs_chunk_voltages": (_I, [_P, _P, ctypes.c_double, _P, _P]),
    "bfs_chunk_detect": (_I, [_P, _P, ctypes.c_double, _P, _P]),
    "bfs_chunk_detect_spectrum": (_I, [_P, _P, ctypes.c_double, _P, _P]),
    "bfs_chunk_process": (_I, [_P, _P, _P, _I, _P, _P]),
    "bfs_chunk_unpack_fft": (_I, [_P, _P, _P, _P]),
    "bfs_chunk_process_raw": (_I, [_P, _P, _P, _P, _I, _P, _P]),
    "bfs_chunk_process_spectrum": (_I, [_P, _P, _P, _I, _P, _P]),
}

_lib = None


def lib() -> ctypes.CDLL:
    """Load (once) and return the native library; raise if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"native library {LIB_PATH} is missing: run "
                          "`python -m cpp_projects_b200.build` (there is no CPU fallback)")
    l = ctypes.CDLL(str(LIB_PATH), mode=os.RTLD_NOW | os.RTLD_LOCAL)
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(l, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    _lib = l
    return l


def declared_symbols() -> list[str]:
    return [n for n in _SIGNATURES]


def check(status: int) -> None:
    if status != BFS_OK:
        msg = lib().bfs_last_error()
        raise BfsError(status, msg.decode() if msg else "")


def call(name: str, *args) -> None:
    check(getattr(lib(), name)(*args))
