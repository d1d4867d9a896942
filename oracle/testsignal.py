"""Test infrastructure, not product code: a restatement of the reference's
sweep generator (testsignal/src/main.rs:27-77), the checker for
spektri_b200/bin/testsignal.  Only tests/ imports it.

float32 arithmetic step by step as in main.rs:40-76 (numpy float32 scalars,
no fused operations), with the C library's cosf, sinf and fmodf, which Rust's
f32::cos / f32::sin / `%` call on Linux.  The reference cannot be built here
(no Rust toolchain), so this restatement is pinned by the source alone.
"""
from __future__ import annotations

import ctypes
import ctypes.util

import numpy as np

_m = ctypes.CDLL(ctypes.util.find_library("m"))
for _f in ("cosf", "sinf"):
    getattr(_m, _f).restype = ctypes.c_float
    getattr(_m, _f).argtypes = [ctypes.c_float]
_m.fmodf.restype = ctypes.c_float
_m.fmodf.argtypes = [ctypes.c_float, ctypes.c_float]

FORMATS = {"s16le": 0x08, "f32le": 0x1C, "cs16le": 0x48, "cf32le": 0x5C}


def testsignal(fmt: str, nsamples: int) -> bytes:
    code = FORMATS[fmt.lower()]
    is_iq = (code & 0xC0) == 0x40
    is_s16 = (code & 0x1F) == 0x08
    buflen = 1024
    nbufs = nsamples // buflen
    PI = np.float32(np.pi)
    init_freq = -PI
    two_pi = np.float32(2.0) * PI
    freq_step = two_pi / (np.float32(buflen) * np.float32(nbufs)) if nbufs else np.float32(0)
    phase = np.float32(0.0)
    n = buflen * nbufs
    i_part = np.empty(n, np.float32)
    q_part = np.empty(n, np.float32)
    for c in range(n):
        i_part[c] = _m.cosf(phase)
        if is_iq:
            q_part[c] = _m.sinf(phase)
        freq = np.float32(init_freq + np.float32(freq_step * np.float32(c)))
        phase = np.float32(_m.fmodf(np.float32(phase + freq), two_pi))
    conv = (lambda v: np.trunc(v * np.float32(32767.0)).astype("<i2")) if is_s16 else (lambda v: v.astype("<f4"))
    i_part = conv(i_part)
    if is_iq:
        q_part = conv(q_part)
        return np.stack([i_part, q_part], axis=1).reshape(-1).tobytes()
    return i_part.tobytes()
