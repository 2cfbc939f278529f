"""ctypes binding of the native library libldpc_b200.so (C ABI: include/ldpc_b200.h).

The library is built in-tree by ``python -m fast_ldpc_decoder_for_gpu_fixed_b200.build``.
There is no fallback: when the library is missing, every decode raises.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libldpc_b200.so")

LDPC_OK = 0
ERRORS = {-1: "LDPC_ERR_ARG", -2: "LDPC_ERR_CUDA", -3: "LDPC_ERR_UNSUPPORTED", -4: "LDPC_ERR_NOMEM",
          -5: "LDPC_ERR_SHAPE"}
KINDS = {"MS": 0, "FMS": 0, "OMS": 1, "NMS": 2, "2NMS": 3, "XMS": 4, "LEARNED": 5}
PACKS = {"AUTO": -1, "SIMD4": 0, "F16X2": 1, "I8": 2, "FRAME": 3, "F16X2_SPLIT": 4}
OUT_BYTES, OUT_PACKED = 0, 1
FLAG_EARLY_STOP = 1
FLAG_EARLY_STOP_FRAMES = 4
FLAG_FLOODING = 8
FLAG_EARLY_STOP_PAIRS = 16
BATCH_GRAPH = 2
EARLY_STOP_DEFAULT_SLACK = 128
EARLY_SLACK_ANY = 1 << 30
TRAIN_QUANTIZED, TRAIN_FRAME_LOSS = 1, 2

# every entry point declared in include/ldpc_b200.h: name -> (restype, argtypes)
_P = ctypes.c_void_p
_I = ctypes.c_int
_SZ = ctypes.c_size_t
SIGNATURES = {
    "ldpc_code_create_from_table": (_I, [ctypes.POINTER(_P), _I, _I, _I, _I, _I, _I, _I, _I, _P]),
    "ldpc_code_create": (_I, [ctypes.POINTER(_P), _I, _I, _P, _P, _P]),
    "ldpc_code_load": (_I, [ctypes.POINTER(_P), ctypes.c_char_p]),
    "ldpc_code_create_qc": (_I, [ctypes.POINTER(_P), _I, _I, _I, _P]),
    "ldpc_code_info": (_I, [_P, _P]),
    "ldpc_code_destroy": (None, [_P]),
    "ldpc_decoder_create": (_I, [ctypes.POINTER(_P), _P, _I, _SZ, _I, _I]),
    "ldpc_decode_host": (_I, [_P, _P, _P, _I]),
    "ldpc_decode_host_ex": (_I, [_P, _P, _P, _I, _I, _P, _P]),
    "ldpc_decode_device": (_I, [_P, _P, _P, _SZ, _I, _I, _P, _P, _P]),
    "ldpc_decode_device_state": (_I, [_P, _P, _P, _SZ, _I, _P, _P, _P, _P]),
    "ldpc_decoder_info": (_I, [_P, _P]),
    "ldpc_decoder_set_learned": (_I, [_P, _I, _P, _P]),
    "ldpc_decoder_set_early_stop": (_I, [_P, _I, _I]),
    "ldpc_decoder_status": (_I, [_P, _P]),
    "ldpc_decoder_destroy": (_I, [_P]),
    "ldpc_batch_create": (_I, [ctypes.POINTER(_P), _P, _I, _I, _I, _I]),
    "ldpc_batch_decode": (_I, [_P, _P, _P, _P, _I, _I, _P, _P, _P]),
    "ldpc_batch_autotune": (_I, [_P, _P, _P, _P, _I, _P, ctypes.POINTER(ctypes.c_double), _P]),
    "ldpc_batch_set_learned": (_I, [_P, _I, _P, _P]),
    "ldpc_batch_configure": (_I, [_P, _I, _I, _I, _I]),
    "ldpc_batch_set_early_stop": (_I, [_P, _I, _I]),
    "ldpc_batch_info": (_I, [_P, _P]),
    "ldpc_batch_code_info": (_I, [_P, _I, _P]),
    "ldpc_batch_set_code_kernel": (_I, [_P, _I, _I]),
    "ldpc_batch_destroy": (_I, [_P]),
    "ldpc_train_step": (_I, [_P, _P, _P, _P, _SZ, _I, _I, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "ldpc_train_stash_bytes": (_SZ, [_P, _SZ, _I]),
    "ldpc_last_error_string": (ctypes.c_char_p, []),
    "ldpc_version": (_I, []),
    "ldpc_simd_selftest": (_I, [_I, _P, _P, _P, _SZ, _P]),
    "ldpc_probe_int_peak": (_I, [ctypes.POINTER(ctypes.c_double), _P]),
    "ldpc_sigma": (ctypes.c_double, [ctypes.c_double, ctypes.c_double, _I]),
    "ldpc_channel_awgn": (_I, [_P, _SZ, _I, ctypes.c_float, ctypes.c_uint64, ctypes.c_uint64, _P, _SZ, _P]),
    "ldpc_philox": (_I, [_P, _SZ, ctypes.c_uint64, ctypes.c_uint64, _P]),
    "ldpc_count_errors": (_I, [_P, _SZ, _I, _I, _P, _SZ, _P, _P]),
    "ldpc_decode_noalloc": (_I, [_P, _I, _I, _P, _P, _SZ, _I, _P]),
    "ldpc_simulate": (_I, [_P, _SZ, _I, ctypes.c_float, ctypes.c_uint64, ctypes.c_uint64, _P, _SZ, _I, _P, _P, _P]),
}


class LdpcError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (%d): %s" % (ERRORS.get(code, "LDPC_ERR"), code, msg))
        self.code = code


_lib = None


def lib():
    """Loads the native library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("native library %s is missing; build it with "
                              "`python -m fast_ldpc_decoder_for_gpu_fixed_b200.build`" % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def last_error():
    return lib().ldpc_last_error_string().decode(errors="replace")


def check(rc):
    if rc != LDPC_OK:
        raise LdpcError(rc, last_error())
    return rc
