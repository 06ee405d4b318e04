"""ctypes binding of libj2kb200.so (the C ABI declared in include/j2k_b200.h).

The library is the product: there is no CPU fallback.  Importing this module on a machine
where the shared library is missing raises immediately with the build command to run.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libj2kb200.so")

J2K_OK = 0
STATUS = {0: "ok", -1: "invalid argument", -2: "CUDA error", -3: "out of memory",
          -4: "device-reported error", -5: "output capacity exceeded", -6: "unsupported",
          -7: "device wait timed out", -8: "host error"}
U8, I16, I32, F32 = 0, 1, 2, 3
MCT_NONE, MCT_RCT, MCT_ICT = 0, 1, 2
ORDER_T800, ORDER_REF = 0, 1
W53, W97 = 53, 97
BAND_LL, BAND_HL, BAND_LH, BAND_HH = 0, 1, 2, 3

CB_DESC = np.dtype([("offset", "<u4"), ("length", "<i4"), ("numbps", "u1"), ("npasses", "u1"),
                    ("orient", "u1"), ("band", "u1"), ("x0", "<u2"), ("y0", "<u2"),
                    ("cw", "<u2"), ("ch", "<u2"), ("comp", "<u2"), ("reserved", "<u2")])
assert CB_DESC.itemsize == 24


class EncParams(C.Structure):
    _fields_ = [("levels", C.c_int), ("cbw", C.c_int), ("cbh", C.c_int), ("order", C.c_int),
                ("steps", C.c_void_p), ("target_bytes", C.c_size_t), ("layers", C.c_int),
                ("layer_bytes", C.c_void_p), ("cblk_style", C.c_int), ("pass_ends", C.c_void_p)]


# code-block styles (T.800 Table A.19) and the pass-end stride per code-block
CBLK_BYPASS, CBLK_RESET, CBLK_TERMALL = 1, 2, 4
PASS_STRIDE = 92


J2K_MAX_BANDS = 97


class StreamInfo(C.Structure):
    _fields_ = [("w", C.c_uint32), ("h", C.c_uint32), ("ncomp", C.c_int), ("levels", C.c_int), ("cbw", C.c_int),
                ("cbh", C.c_int), ("lossless", C.c_int), ("mct", C.c_int), ("guard", C.c_int),
                ("precision", C.c_int), ("layers", C.c_int), ("progression", C.c_int),
                ("steps", C.c_float * J2K_MAX_BANDS), ("cblk_style", C.c_int)]


class J2KError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS.get(status, status)} ({status}): {msg}")
        self.status = status


_lib = None

# name -> (restype, argtypes)
P, S, I = C.c_void_p, C.c_size_t, C.c_int
SIGS = {
    "j2k_ctx_create": (I, [I, C.POINTER(P)]),
    "j2k_ctx_destroy": (I, [P]),
    "j2k_ctx_set_stream": (I, [P, P]),
    "j2k_ctx_use_own_stream": (I, [P]),
    "j2k_ctx_stream": (P, [P]),
    "j2k_stream_sync": (I, [P]),
    "j2k_last_error": (C.c_char_p, [P]),
    "j2k_ctx_set_tuning": (I, [P, I, I]),
    "j2k_status_string": (C.c_char_p, [I]),
    "j2k_version": (I, []),
    "j2k_rgb_to_planar": (I, [P, P, S, I, I, I, P, S, S, S, S]),
    "j2k_planar_to_rgb": (I, [P, P, I, S, S, I, I, P, S, S, S]),
    "j2k_dwt_forward": (I, [P, I, I, P, S, P, S, S, S, I, P]),
    "j2k_dwt_inverse": (I, [P, I, I, P, S, P, S, S, S, I, P]),
    "j2k_dwt_forward_noalloc": (I, [P, I, I, P, S, P, S, S, S, I, P]),
    "j2k_dwt_forward_batch": (I, [P, I, I, P, S, S, P, S, S, I, S, S, I, P]),
    "j2k_dwt_inverse_batch": (I, [P, I, I, P, S, S, P, S, S, I, S, S, I, P]),
    "j2k_codeblock_count": (S, [S, S, I, I, I]),
    "j2k_codestream_read": (I, [P, S, P, P, P, P, S, P, P, S]),
    "j2k_codestream_read_layers": (I, [P, S, I, P, P, P, P, S, P, P, S]),
    "j2k_codestream_write": (I, [C.c_uint32, C.c_uint32, I, I, I, I, I, P, P, S, P, S, I, P, P, P, S, P]),
    "j2k_bpc_encode": (I, [P, P, S, S, S, I, I, I, P, P, S]),
    "j2k_bpc_decode": (I, [P, P, P, S, P, S, S, S, I, I, I]),
    "j2k_encoder_create": (I, [P, I, I, C.POINTER(P)]),
    "j2k_encoder_destroy": (I, [P]),
    "j2k_encoder_run": (I, [P, P, I, I, S, S, S, S, P]),
    "j2k_encoder_run_interleaved": (I, [P, P, I, S, I, S, S, P]),
    "j2k_encoder_map_dwt_out": (I, [P, C.POINTER(P), C.POINTER(S)]),
    "j2k_encoder_unmap_dwt_out": (I, [P, P]),
    "j2k_encoder_get_codeblocks": (I, [P, P, C.POINTER(S), P, S, C.POINTER(S)]),
    "j2k_encoder_get_codestream": (I, [P, P, S, C.POINTER(S)]),
    "j2k_encoder_get_pass_ends": (I, [P, P, S, C.POINTER(S)]),
    "j2k_codestream_pass_ends": (I, [P, S, I, P, S, C.POINTER(S), P, S]),
    "j2k_encoder_device_results": (I, [P, C.POINTER(P), C.POINTER(P), C.POINTER(S), C.POINTER(S)]),
    "j2k_decoder_create": (I, [P, I, C.POINTER(P)]),
    "j2k_decoder_destroy": (I, [P]),
    "j2k_decoder_run_codeblocks": (I, [P, P, P, S, I, I, S, S, P, P, I, S]),
    "j2k_decoder_run_batch": (I, [P, P, I]),
    "j2k_decoder_run_codestreams": (I, [P, P, P, I, I, P]),
    "j2k_codestream_info": (I, [P, S, P, P, S]),
    "j2k_encoder_autotune": (I, [P, I, P]),
    "j2k_dwt97_forward_adjoint": (I, [P, P, P, I, S, S, I]),
    "j2k_dwt97_inverse_adjoint": (I, [P, P, P, I, S, S, I]),
    "j2k_relaxed_quant_forward": (I, [P, P, P, I, S, S, I, P, C.c_uint64, P, I]),
    "j2k_relaxed_quant_backward": (I, [P, P, P, P, I, S, S, I, P, C.c_uint64, C.c_float, P, I]),
    "j2k_relaxed_quant_forward_noise": (I, [P, P, P, P, I, S, S, I, P, C.c_uint64, P, I]),
    "j2k_relaxed_quant_backward_scaled": (I, [P, P, P, P, I, S, S, I, P, C.c_uint64, P, C.c_float, P, C.c_float,
                                              P, I]),
    "j2k_dwt97_residual_partials": (S, [S, S, I]),
    "j2k_dwt97_rd_finalize": (I, [P, P, S, P, S, C.c_double, C.c_float, P]),
    "j2k_dwt97_band_sum": (I, [P, P, I, I, I, P]),
    "j2k_dwt97_inverse_residual": (I, [P, P, P, P, I, S, S, I, P]),
    "j2k_dwt97_forward_adjoint_residual": (I, [P, P, P, P, C.c_float, P, I, S, S, I]),
    "j2k_dwt97_rd_parts": (S, [P, S, S, I]),
    "j2k_dwt97_rd_forward": (I, [P, P, P, P, P, I, S, S, I, P, C.c_uint64, P, P]),
    "j2k_dwt97_rd_backward": (I, [P, P, P, P, P, C.c_float, P, C.c_float, P, P, I, S, S, I, P]),
    "j2k_batch_create": (I, [P, P, I, C.POINTER(P)]),
    "j2k_batch_destroy": (I, [P]),
    "j2k_batch_pack": (I, [P, C.POINTER(S)]),
    "j2k_batch_read_packed": (I, [P, P, P, S]),
    "j2k_batch_image_jobs": (I, [P, C.POINTER(S)]),
    "j2k_batch_input": (I, [P, C.POINTER(P), P]),
    "j2k_batch_encode": (I, [P, P, I]),
    "j2k_batch_encode_async": (I, [P, P, I]),
    "j2k_batch_upload": (I, [P, P, I]),
    "j2k_batch_set_option": (I, [P, I, I]),
    "j2k_batch_get_option": (I, [P, I, C.POINTER(I)]),
    "j2k_batch_autotune": (I, [P, I, P]),
    "j2k_batch_get_codeblocks": (I, [P, I, P, C.POINTER(S), P, S, C.POINTER(S)]),
    "j2k_batch_get_codestream": (I, [P, I, P, S, C.POINTER(S)]),
}


class BatchImage(C.Structure):
    _fields_ = [("w", C.c_uint32), ("h", C.c_uint32), ("ncomp", C.c_int), ("kernel", C.c_int),
                ("levels", C.c_int), ("cb", C.c_int), ("steps", C.c_void_p)]


class DecodeItem(C.Structure):
    _fields_ = [("w", C.c_uint32), ("h", C.c_uint32), ("ncomp", C.c_int), ("lossless", C.c_int),
                ("levels", C.c_int), ("cbw", C.c_int), ("cbh", C.c_int), ("steps", C.c_void_p),
                ("descs", C.c_void_p), ("count", C.c_size_t), ("bytes", C.c_void_p), ("nbytes", C.c_size_t),
                ("out", C.c_void_p), ("cblk_style", C.c_int), ("pass_ends", C.c_void_p)]


def exported_symbols():
    return sorted(SIGS)


def lib():
    """Loads libj2kb200.so; raises if it has not been built (no fallback path exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -c 'import __graft_entry__ as g; "
                              f"g.build()'` (or python roger_b200/build.py) first")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(status, ctx=None):
    if status != J2K_OK:
        msg = lib().j2k_last_error(ctx).decode() if ctx else ""
        raise J2KError(status, msg)
    return status
