"""ctypes wrapper around the FP32 C++ restatement (``oracle/spektri_oracle.cpp``).

TEST INFRASTRUCTURE ONLY: used by tests, the smoke check and the benchmark's
CPU-baseline leg as the checker.  The product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import threading

import numpy as np

from .oracle64 import fmt_code, is_complex, bytes_per_sample

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(BUILD, "liboracle.so")
CLI = os.path.join(BUILD, "spektri_oracle")
_lock = threading.Lock()
_lib = None


def build(force: bool = False) -> None:
    """Compile the restatement with its Makefile (gcc only, seconds)."""
    src = os.path.join(HERE, "spektri_oracle.cpp")
    fresh = all(os.path.exists(p) and os.path.getmtime(p) >= os.path.getmtime(src) for p in (LIB, CLI))
    if fresh and not force:
        return
    subprocess.run(["make", "-s", "-C", HERE], check=True)


class _Params(C.Structure):
    _fields_ = [("fs_in", C.c_double), ("fc_in", C.c_double), ("fft_size", C.c_int32),
                ("ffts_per_buf", C.c_int32), ("averages", C.c_int32), ("input_format", C.c_int32),
                ("spectrum_format", C.c_int32), ("n_threads", C.c_int32)]


class _Filter(C.Structure):
    _fields_ = [("fs_out", C.c_double), ("fc_out", C.c_double),
                ("weights", C.c_void_p), ("transition", C.c_int32)]


def lib() -> C.CDLL:
    global _lib
    with _lock:
        if _lib is None:
            build()
            L = C.CDLL(LIB)
            L.orc_create.restype = C.c_void_p
            L.orc_create.argtypes = [C.POINTER(_Params), C.POINTER(_Filter), C.c_int32, C.POINTER(C.c_int32)]
            L.orc_destroy.argtypes = [C.c_void_p]
            L.orc_info.argtypes = [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                   C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
            L.orc_channel.argtypes = [C.c_void_p, C.c_int32, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
            L.orc_max_spectra.argtypes = [C.c_void_p]
            L.orc_process.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.POINTER(C.c_int32), C.POINTER(C.c_uint64)]
            L.orc_two_real_ffts.argtypes = [C.c_int32] + [C.c_void_p] * 5
            L.orc_fft.argtypes = [C.c_int32, C.c_int32, C.c_void_p]
            L.orc_freq_to_bins.argtypes = [C.c_double, C.c_double, C.c_int64, C.c_double, C.c_double,
                                           C.c_int32, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
            L.orc_bins_to_freq.argtypes = [C.c_double, C.c_double, C.c_int64, C.c_int64, C.c_int64,
                                           C.POINTER(C.c_double), C.POINTER(C.c_double)]
            L.orc_tukey.argtypes = [C.c_int32, C.c_int32, C.c_void_p]
            L.orc_raised_cosine.argtypes = [C.c_int32, C.c_void_p]
            _lib = L
    return _lib


SPEC_FORMATS = {"u8": 0, "u16": 1, "f32": 2}


class Oracle32:
    """Streaming FP32 restatement: same constructor shape as the product's
    ``spektri_b200.Plan``; ``process(raw)`` returns (spectra, outputs)."""

    def __init__(self, fs_in, fc_in, fft_size, ffts_per_buf, averages, input_format, filters,
                 spectrum_format="f32", n_threads=None):
        L = lib()
        self.fmt = fmt_code(input_format)
        self.spec_fmt = SPEC_FORMATS[spectrum_format]
        p = _Params(float(fs_in), float(fc_in), int(fft_size), int(ffts_per_buf), int(averages),
                    self.fmt, self.spec_fmt, int(n_threads or os.cpu_count() or 1))
        self._keep = []
        fl = (_Filter * max(1, len(filters)))()
        for i, f in enumerate(filters):
            w = f.get("weights")
            ptr = None
            if w is not None:
                w = np.ascontiguousarray(w, dtype=np.complex64)
                self._keep.append(w)
                ptr = w.ctypes.data
            fl[i] = _Filter(float(f["fs_out"]), float(f["fc_out"]), ptr, int(f.get("transition", 0)))
        st = (C.c_int32 * max(1, len(filters)))()
        self.h = L.orc_create(C.byref(p), fl, len(filters), st)
        if not self.h:
            raise ValueError("oracle rejected the parameters")
        self.filter_status = list(st)[: len(filters)]
        nn, ov, K, nch = C.c_int64(), C.c_int64(), C.c_int32(), C.c_int32()
        L.orc_info(self.h, C.byref(nn), C.byref(ov), C.byref(K), C.byref(nch))
        self.new, self.overlap, self.K, self.n_channels = nn.value, ov.value, K.value, nch.value
        self.ffts_per_buf = int(ffts_per_buf)
        self.channels = []
        for c in range(self.n_channels):
            b, f0 = C.c_int64(), C.c_int64()
            L.orc_channel(self.h, c, C.byref(b), C.byref(f0))
            self.channels.append((b.value, f0.value))
        self.max_spectra = L.orc_max_spectra(self.h)
        self.raw_bytes = self.new * bytes_per_sample(self.fmt)

    def out_samples(self, c):
        return self.ffts_per_buf * (self.channels[c][0] // 8 * 6)

    def process(self, raw):
        L = lib()
        raw = np.ascontiguousarray(np.frombuffer(raw, np.uint8) if isinstance(raw, (bytes, bytearray)) else raw.view(np.uint8))
        assert raw.nbytes == self.raw_bytes, (raw.nbytes, self.raw_bytes)
        outs = [np.empty(self.out_samples(c), np.complex64) for c in range(self.n_channels)]
        ptrs = (C.c_void_p * max(1, self.n_channels))(*[o.ctypes.data for o in outs])
        sb = {0: 1, 1: 2, 2: 4}[self.spec_fmt]
        spec = np.empty(self.max_spectra * self.K * sb, np.uint8)
        ns, seq0 = C.c_int32(), C.c_uint64()
        L.orc_process(self.h, raw.ctypes.data, ptrs, spec.ctypes.data, C.byref(ns), C.byref(seq0))
        dt = {0: np.uint8, 1: ">u2", 2: np.float32}[self.spec_fmt]
        spectra = [(seq0.value + r, spec[r * self.K * sb:(r + 1) * self.K * sb].view(dt).copy())
                   for r in range(ns.value)]
        return spectra, outs

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            lib().orc_destroy(h)
            self.h = None


def two_real_ffts(window, in0, in1):
    L = lib()
    n = len(window)
    a = [np.ascontiguousarray(x, np.float32) for x in (window, in0, in1)]
    o0 = np.empty(n // 2 + 1, np.complex64)
    o1 = np.empty(n // 2 + 1, np.complex64)
    L.orc_two_real_ffts(n, a[0].ctypes.data, a[1].ctypes.data, a[2].ctypes.data, o0.ctypes.data, o1.ctypes.data)
    return o0, o1


def fft(x, sign=-1):
    x = np.ascontiguousarray(x, np.complex64).copy()
    lib().orc_fft(len(x), sign, x.ctypes.data)
    return x


def freq_to_bins(fs, fc, N, fs_out, fc_out, exact=False):
    b, f = C.c_int64(), C.c_int64()
    r = lib().orc_freq_to_bins(fs, fc, N, fs_out, fc_out, int(exact), C.byref(b), C.byref(f))
    return (b.value, f.value) if r == 0 else None


def bins_to_freq(fs, fc, N, bins, first):
    a, b = C.c_double(), C.c_double()
    lib().orc_bins_to_freq(fs, fc, N, bins, first, C.byref(a), C.byref(b))
    return a.value, b.value


def tukey(n, tw):
    o = np.empty(n, np.complex64)
    lib().orc_tukey(n, tw, o.ctypes.data)
    return o.real.copy()


def raised_cosine(n):
    o = np.empty(n, np.complex64)
    lib().orc_raised_cosine(n, o.ctypes.data)
    return o.real.copy()
