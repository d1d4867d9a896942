"""ctypes binding of libspektri_b200.so (the C ABI in include/spektri_b200.h).

The shared library is built in place by ``spektri_b200.build.build()``.  There
is no fallback: if the library cannot be loaded, importing the binding raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libspektri_b200.so")

SK_OK = 0
SK_WARN_FILTER = 1
SK_ERR_ARG = -1
SK_ERR_FILTER = -2
SK_ERR_CUDA = -3
SK_ERR_NOMEM = -4
SK_ERR_TIMEOUT = -5
SK_ERR_UNSUPPORTED = -6
SK_ERR_STATE = -7

SPEC_U8, SPEC_U16, SPEC_F32 = 0, 1, 2
MODE_PLAIN, MODE_BATCHED = 0, 1
AGC_SSB, AGC_AM, AGC_AM_ENVELOPE, ENVELOPE = 1, 2, 3, 4


class SpektriError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"spektri_b200 error {code}: {msg}")
        self.code = code


class Params(C.Structure):
    _fields_ = [("fs_in", C.c_double), ("fc_in", C.c_double), ("fft_size", C.c_uint32),
                ("ffts_per_buf", C.c_uint32), ("averages", C.c_uint32), ("input_format", C.c_int32),
                ("spectrum_format", C.c_int32), ("mode", C.c_int32), ("device", C.c_int32),
                ("flags", C.c_uint32)]


class Filter(C.Structure):
    _fields_ = [("fs_out", C.c_double), ("fc_out", C.c_double), ("weights", C.c_void_p),
                ("transition", C.c_uint32), ("reserved", C.c_uint32)]


class PlanInfo(C.Structure):
    _fields_ = [("new_samples", C.c_uint64), ("overlap", C.c_uint64), ("total", C.c_uint64),
                ("raw_bytes", C.c_uint64), ("result_bins", C.c_uint32), ("n_channels", C.c_uint32),
                ("max_spectra", C.c_uint32), ("spectrum_bytes", C.c_uint32)]


class ChannelInfo(C.Structure):
    _fields_ = [("bins", C.c_uint32), ("filter_index", C.c_int32), ("first", C.c_int64),
                ("fs_out", C.c_double), ("fc_out", C.c_double), ("out_samples", C.c_uint64)]


class Result(C.Structure):
    _fields_ = [("n_spectra", C.c_uint32), ("reserved", C.c_uint32), ("spectrum_seq0", C.c_uint64)]


# (name, restype, argtypes) of every exported symbol; the CPU test checks
# that each one declared in the header is exported.
PROTOTYPES = [
    ("sk_freq_to_bins", C.c_int, [C.c_double, C.c_double, C.c_uint64, C.c_double, C.c_double,
                                  C.POINTER(C.c_uint32), C.POINTER(C.c_int64)]),
    ("sk_freq_to_bins_exact", C.c_int, [C.c_double, C.c_double, C.c_uint64, C.c_double, C.c_double,
                                        C.POINTER(C.c_uint32), C.POINTER(C.c_int64)]),
    ("sk_bins_to_freq", C.c_int, [C.c_double, C.c_double, C.c_uint64, C.c_uint32, C.c_int64,
                                  C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    ("sk_raised_cosine_weights", C.c_int, [C.c_uint32, C.c_void_p]),
    ("sk_tukey_weights", C.c_int, [C.c_uint32, C.c_uint32, C.c_void_p]),
    ("sk_serialize_metadata", C.c_int, [C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint32]),
    ("sk_signal_topic", C.c_int, [C.c_void_p, C.c_double, C.c_double]),
    ("sk_spectrum_topic", C.c_int, [C.c_void_p, C.c_int32, C.c_double, C.c_double]),
    ("sk_format_bytes", C.c_int, [C.c_int32]),
    ("sk_format_is_complex", C.c_int, [C.c_int32]),
    ("sk_last_error", C.c_char_p, []),
    ("sk_version", C.c_char_p, []),
    ("sk_plan_create", C.c_int, [C.POINTER(Params), C.c_void_p, C.c_int32, C.c_void_p, C.POINTER(C.c_void_p)]),
    ("sk_plan_info_get", C.c_int, [C.c_void_p, C.POINTER(PlanInfo)]),
    ("sk_plan_channel", C.c_int, [C.c_void_p, C.c_int32, C.POINTER(ChannelInfo)]),
    ("sk_plan_destroy", None, [C.c_void_p]),
    ("sk_set_weights", C.c_int, [C.c_void_p, C.c_int32, C.c_void_p]),
    ("sk_get_weights", C.c_int, [C.c_void_p, C.c_int32, C.c_void_p]),
    ("sk_process", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(Result)]),
    ("sk_process_device", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(Result), C.c_void_p]),
    ("sk_synchronize", C.c_int, [C.c_void_p]),
    ("sk_plan_set_carry", C.c_int, [C.c_void_p, C.c_void_p]),
    ("sk_launches_per_call", C.c_int, [C.c_void_p]),
    ("sk_spectra_device", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("sk_spectra_window_device", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("sk_fcfb_forward_device", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("sk_fcfb_backward_device", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.c_void_p]),
    ("sk_plan_autotune", C.c_int, [C.c_void_p, C.c_char_p, C.POINTER(C.c_double)]),
    ("sk_plan_set_tuning", C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32]),
    ("sk_plan_get_tuning", C.c_int, [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    ("sk_plan_set_timing", C.c_int, [C.c_void_p, C.c_int]),
    ("sk_plan_timing", C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_uint64)]),
    ("sk_plan_set_trace", C.c_int, [C.c_void_p, C.c_int]),
    ("sk_plan_trace", C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_uint64)]),
    ("sk_spectra_noalloc", C.c_int, [C.c_void_p, C.c_int32, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p]),
    ("sk_ddc_create", C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int64, C.c_int64, C.c_int32,
                                C.POINTER(C.c_void_p)]),
    ("sk_ddc_outputs", C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(C.c_uint64)]),
    ("sk_ddc_process_device", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.POINTER(C.c_uint64),
                                        C.c_void_p]),
    ("sk_ddc_destroy", None, [C.c_void_p]),
    ("sk_agc_create", C.c_int, [C.c_int32, C.c_int32, C.POINTER(C.c_void_p)]),
    ("sk_agc_process_device", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p]),
    ("sk_agc_destroy", None, [C.c_void_p]),
    ("sk_host_alloc", C.c_void_p, [C.c_size_t]),
    ("sk_host_free", None, [C.c_void_p]),
]

_lib = None


def lib() -> C.CDLL:
    """Load the library (once).  Raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'` "
                              "or `make -C spektri_b200`")
        L = C.CDLL(LIB_PATH)
        for name, res, args in PROTOTYPES:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def last_error() -> str:
    return lib().sk_last_error().decode(errors="replace")


def check(rc: int, what: str = "") -> int:
    if rc < 0:
        raise SpektriError(rc, f"{what}: {last_error()}" if what else last_error())
    return rc
