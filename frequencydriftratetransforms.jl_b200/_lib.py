"""ctypes binding of libfdrb200.so (the C ABI declared in include/fdr_b200.h).

The library is the only compute path: if it is missing or fails to load, importing the
package raises.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# FDR_B200_DEBUG=1 loads the debug build (index checks recorded in device fault words)
LIB_PATH = os.path.join(HERE, "libfdrb200_debug.so" if os.environ.get("FDR_B200_DEBUG") == "1"
                        else "libfdrb200.so")

# status codes (fdr_status)
FDR_OK = 0
FDR_ERR_INVALID_ARGUMENT = 1
FDR_ERR_UNSUPPORTED_SIZE = 2
FDR_ERR_UNSUPPORTED_WINDOW = 3
FDR_ERR_OUT_OF_MEMORY = 4
FDR_ERR_CUDA = 5
FDR_ERR_CAPACITY = 6
FDR_ERR_NO_DEVICE = 7

FDR_WINDOW_RECT = 0
FDR_WINDOW_HAMMING = 1
FDR_WINDOW_CUSTOM = 2

FDR_ZDT_OUTPUT_ALIGNED = 0x1
FDR_ZDT_EXACT_PHASE = 0x2
FDR_ZDT_STAGED_ONLY = 0x4
FDR_ZDT_MIXED_PRECISION = 0x8
FDR_ZDT_FAST_STATS = 0x10

FDR_SNR_F64 = 1
FDR_SNR_F32 = 2

FDR_RATES_F64 = 0
FDR_RATES_F32 = 1


class FDRError(RuntimeError):
    """A nonzero fdr_status from the library (the reference throws the equivalent)."""

    def __init__(self, status, message):
        super().__init__(message)
        self.status = status


class CapacityError(FDRError):
    pass


class fdr_zdt_info(C.Structure):
    _fields_ = [
        ("Nf", C.c_int64), ("Nt", C.c_int64), ("Nr", C.c_int64), ("Nl", C.c_int64),
        ("K", C.c_int64), ("r0", C.c_float), ("dr", C.c_float), ("flags", C.c_uint32),
        ("fused", C.c_int32), ("bytes", C.c_int64), ("nfactors", C.c_int32),
        ("factors", C.c_int64 * 8),
    ]


class fdr_hit_cluster(C.Structure):
    _fields_ = [("peak_i", C.c_int64), ("peak_j", C.c_int64), ("peak_value", C.c_float),
                ("reserved", C.c_int32), ("count", C.c_int64), ("i_min", C.c_int64),
                ("i_max", C.c_int64), ("j_min", C.c_int64), ("j_max", C.c_int64),
                ("first", C.c_int64)]


class fdr_batch_channel(C.Structure):
    _fields_ = [("Nf", C.c_int64), ("Nt", C.c_int64), ("Nr", C.c_int64), ("r0", C.c_float),
                ("dr", C.c_float), ("spectrogram", C.c_void_p), ("fdr", C.c_void_p)]


P = C.c_void_p
I64 = C.c_int64
F32 = C.c_float
F64 = C.c_double
INT = C.c_int

# name -> (restype, argtypes)
SIGNATURES = {
    "fdr_version": (C.c_char_p, []),
    "fdr_last_error_string": (C.c_char_p, []),
    "fdr_status_string": (C.c_char_p, [INT]),
    "fdr_kernel_launches": (I64, []),
    "fdr_synchronize": (INT, [P]),
    "fdr_selftest_bounded_wait": (INT, [I64, P]),
    "fdr_debug_build": (INT, []),
    "fdr_debug_fault": (INT, [C.POINTER(C.c_uint64), P]),
    "fdr_calc_nl": (I64, [I64, I64, C.POINTER(I64), INT]),
    "fdr_grow_nr": (I64, [I64, I64, C.POINTER(I64), INT]),
    "fdr_estimate_memory": (I64, [I64, I64, I64, I64, I64, C.POINTER(I64), INT]),
    "fdr_zdt_create": (INT, [C.POINTER(P), P, I64, I64, F32, F32, I64, C.POINTER(I64), INT,
                             C.c_uint32, P]),
    "fdr_zdt_destroy": (INT, [P]),
    "fdr_zdt_get_info": (INT, [P, C.POINTER(fdr_zdt_info)]),
    "fdr_zdt_fused_split": (INT, [I64, I64, I64, C.c_uint32, C.POINTER(I64), C.POINTER(I64)]),
    "fdr_zdt_buffers": (INT, [P, C.POINTER(P), C.POINTER(P), C.POINTER(P)]),
    "fdr_zdt_input": (INT, [P, P, P]),
    "fdr_zdt_preprocess": (INT, [P, F32, P]),
    "fdr_zdt_convolve": (INT, [P, P]),
    "fdr_zdt_postprocess": (INT, [P, INT, P, P]),
    "fdr_zdt_output": (INT, [P, P, P]),
    "fdr_zdt_execute": (INT, [P, P, C.POINTER(F32), I64, C.POINTER(P), INT, P, P]),
    "fdr_zdtfdr_protohits": (INT, [P, P, C.POINTER(F32), I64, C.POINTER(P), INT, P, F64, INT, P,
                                   I64, C.POINTER(I64), C.POINTER(F64), P]),
    "fdr_zdt_execute_blocks": (INT, [P, P, C.POINTER(C.c_int32), I64, P, INT, P, P]),
    "fdr_zdtfdr_blocks_protohits": (INT, [P, P, C.POINTER(C.c_int32), I64, P, INT, P, F64, INT, P,
                                          I64, C.POINTER(I64), C.POINTER(F64), P]),
    "fdr_zdt_set_timing": (INT, [P, INT]),
    "fdr_zdt_stage_times": (INT, [P, C.POINTER(F32), INT, C.POINTER(INT),
                                  C.POINTER(C.c_char_p)]),
    "fdr_batch_create": (INT, [C.POINTER(P), C.POINTER(fdr_batch_channel), I64, INT, P]),
    "fdr_batch_autotune": (INT, [P, P]),
    "fdr_batch_capture": (INT, [P, P]),
    "fdr_batch_launch": (INT, [P, P]),
    "fdr_batch_get_tuning": (INT, [P, C.POINTER(INT), INT, C.POINTER(INT), C.POINTER(INT)]),
    "fdr_batch_info": (INT, [P, C.POINTER(I64), C.POINTER(I64), C.POINTER(I64), C.POINTER(INT)]),
    "fdr_batch_destroy": (INT, [P]),
    "fdr_propose_create": (INT, [C.POINTER(P), INT, INT, INT, INT, INT, INT, C.c_uint64]),
    "fdr_propose_destroy": (INT, [P]),
    "fdr_propose_num_params": (INT, [P, C.POINTER(I64)]),
    "fdr_propose_features": (INT, [P, I64, I64, INT, INT, P, P]),
    "fdr_propose_lag_features": (INT, [P, I64, I64, INT, INT, INT, P, P]),
    "fdr_propose_input": (INT, [P, I64, I64, INT, INT, INT, P, P]),
    "fdr_propose_forward": (INT, [P, P, INT, P, P]),
    "fdr_propose_gradients": (INT, [P, P, P, INT, P, P, P, P]),
    "fdr_propose_train_step": (INT, [P, P, P, INT, F32, P, P, P]),
    "fdr_propose_get_state": (INT, [P, P, P, P, C.POINTER(I64)]),
    "fdr_propose_set_state": (INT, [P, P, P, P, I64]),
    "fdr_intshift": (INT, [P, I64, I64, F64, INT, P, P]),
    "fdr_intfdr": (INT, [P, I64, I64, C.POINTER(F64), I64, INT, P, P]),
    "fdr_intfdr_shifts": (INT, [P, I64, I64, C.POINTER(I64), I64, P, P]),
    "fdr_taylor_tree": (INT, [P, I64, I64, INT, INT, P, P]),
    "fdr_fftfdr_workspace": (INT, [C.POINTER(P), P, I64, I64, P]),
    "fdr_fftfdr_workspace_update": (INT, [P, P, I64, I64, P]),
    "fdr_fftfdr_destroy": (INT, [P]),
    "fdr_fftfdr_rfft_buffer": (INT, [P, C.POINTER(P)]),
    "fdr_fdshiftsum": (INT, [P, F32, P, P]),
    "fdr_fdshift": (INT, [P, F32, P, P]),
    "fdr_fftfdr": (INT, [P, C.POINTER(F32), I64, P, P]),
    "fdr_stats": (INT, [C.POINTER(P), I64, I64, I64, C.POINTER(F64), C.POINTER(F64), P]),
    "fdr_stats_noalloc": (INT, [P, I64, I64, C.POINTER(F64), C.POINTER(F64), P]),
    "fdr_normalize": (INT, [C.POINTER(P), I64, I64, I64, F32, F32, P]),
    "fdr_findprotohits": (INT, [C.POINTER(P), I64, I64, I64, F64, INT, P, I64,
                                C.POINTER(I64), C.POINTER(F64), P]),
    "fdr_cluster_protohits": (INT, [P, I64, I64, I64, INT, INT, C.POINTER(P), I64, I64, P, P,
                                    I64, C.POINTER(I64), P]),
    "fdr_lz4_decompress": (INT, [P, I64, P, I64, C.POINTER(I64)]),
    "fdr_lz4_compress": (INT, [P, I64, P, I64, C.POINTER(I64)]),
    "fdr_bitshuffle_lz4_decode": (INT, [P, I64, INT, P, I64, C.POINTER(I64), C.POINTER(I64)]),
    "fdr_bitshuffle_lz4_encode": (INT, [P, I64, INT, I64, P, I64, C.POINTER(I64)]),
    "fdr_bitunshuffle": (INT, [P, I64, INT, I64, P, P]),
}

_lib = None


def load(path: str | None = None):
    """Load libfdrb200.so and declare every C-ABI signature (raises if it is missing)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise ImportError(
            f"libfdrb200.so not found at {p}; build it with "
            "`python frequencydriftratetransforms.jl_b200/build.py` (nvcc, sm_100a)")
    lib = C.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def lib():
    return load()


def check(status: int):
    if status != FDR_OK:
        msg = lib().fdr_last_error_string().decode(errors="replace")
        if status == FDR_ERR_CAPACITY:
            raise CapacityError(status, msg)
        raise FDRError(status, msg)


def snr_mode(threshold, snr):
    """The `snr` argument of the proto-hit searches for a Python threshold: 0 without snr;
    with snr, the type Julia's promotion gives fdrdenormalize(threshold, m, s) =
    threshold*s + m for Float32 m and s: Float32 for an integer or numpy float32 threshold
    (FDR_SNR_F32), Float64 for a Python or numpy float64 (FDR_SNR_F64)."""
    import numpy as np
    if not snr:
        return 0
    if isinstance(threshold, (bool, int, np.integer, np.float32)):
        return FDR_SNR_F32
    return FDR_SNR_F64


def i64_array(values):
    vals = list(values)
    return (I64 * max(1, len(vals)))(*vals), len(vals)
