"""Host-side mirror of the reference's DSP interface, over the C ABI.

Names, argument meaning and error behaviour follow tejeez/spektri:

* ``DspParams`` / ``FilterParams``      spektri/src/dsp.rs:22-33, dsp/fcfb.rs:206-210
* ``DspState.init`` -> (state, InputBufferSize)   dsp.rs:76-111
* ``DspState.process`` (process_real / process_complex)   dsp.rs:114-160
* ``freq_to_bins`` / ``bins_to_freq`` / ``freq_to_bins_exact``   dsp/fcfb.rs:225-285
* ``serialize_metadata`` / ``serialize_signal_topic`` / ``serialize_spectrum_topic``   dsp/data.rs:110-171
* ``parse_filter_params``   main.rs:70-91 (``fs=..:fc=..[:file=..]``, plus ``tw=`` and ``w=``)
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from ._lib import check, lib, SK_ERR_FILTER
from .plan import Plan, format_code


def freq_to_bins(fs_in, fc_in, fft_size, fs_out, fc_out):
    """(bins, first) or None (fcfb.rs:225-252)."""
    b, f = C.c_uint32(), C.c_int64()
    rc = lib().sk_freq_to_bins(fs_in, fc_in, fft_size, fs_out, fc_out, C.byref(b), C.byref(f))
    if rc == SK_ERR_FILTER:
        return None
    check(rc)
    return b.value, f.value


def freq_to_bins_exact(fs_in, fc_in, fft_size, fs_out, fc_out):
    """(bins, first) when the parameters are exactly representable, else None (fcfb.rs:274-285)."""
    b, f = C.c_uint32(), C.c_int64()
    rc = lib().sk_freq_to_bins_exact(fs_in, fc_in, fft_size, fs_out, fc_out, C.byref(b), C.byref(f))
    if rc == SK_ERR_FILTER:
        return None
    check(rc)
    return b.value, f.value


def bins_to_freq(fs_in, fc_in, fft_size, bins, first):
    """(fs_out, fc_out) (fcfb.rs:257-268)."""
    a, c = C.c_double(), C.c_double()
    check(lib().sk_bins_to_freq(fs_in, fc_in, fft_size, bins, first, C.byref(a), C.byref(c)))
    return a.value, c.value


def raised_cosine_weights(n: int) -> np.ndarray:
    """fcfb.rs:197-203 as complex64."""
    w = np.empty(n, np.complex64)
    check(lib().sk_raised_cosine_weights(n, w.ctypes.data))
    return w


def tukey_weights(n: int, tw: int) -> np.ndarray:
    """Periodic Tukey weights with ``tw`` taper bins per side, complex64."""
    w = np.empty(n, np.complex64)
    check(lib().sk_tukey_weights(n, tw, w.ctypes.data))
    return w


def serialize_metadata(seq: int, secs: int, nanos: int) -> bytes:
    b = (C.c_uint8 * 24)()
    check(lib().sk_serialize_metadata(b, seq, secs, nanos))
    return bytes(b)


def serialize_signal_topic(fs: float, fc: float) -> bytes:
    b = (C.c_uint8 * 24)()
    check(lib().sk_signal_topic(b, fs, fc))
    return bytes(b)


def serialize_spectrum_topic(fd: float, f0: float, spectrum_format: str = "u8") -> bytes:
    b = (C.c_uint8 * 24)()
    check(lib().sk_spectrum_topic(b, {"u8": 0, "u16": 1, "f32": 2}[spectrum_format], fd, f0))
    return bytes(b)


@dataclass
class OutputParams:
    filename: Optional[str] = None


@dataclass
class FilterParams:
    fs_out: float
    fc_out: float
    output: OutputParams = field(default_factory=OutputParams)
    transition: int = 0                 # tw=: Tukey taper bins (0 = reference raised cosine)
    weights: Optional[np.ndarray] = None  # w=: complex64 weights, natural order


def parse_filter_params(s: str) -> FilterParams:
    """main.rs:70-91: ``key=value`` pairs separated by ':'.  Missing fs/fc or
    malformed numbers raise ValueError (the reference panics)."""
    m = {}
    for part in s.split(":"):
        if "=" not in part:
            raise ValueError(f"malformed filter parameter {part!r}")
        k, v = part.split("=", 1)
        m[k] = v
    fp = FilterParams(fs_out=float(m["fs"]), fc_out=float(m["fc"]), output=OutputParams(m.get("file")))
    if "tw" in m:
        fp.transition = int(m["tw"])
    if "w" in m:
        fp.weights = np.fromfile(m["w"], dtype="<c8")
    return fp


@dataclass
class DspParams:
    complex: bool
    fs_in: float
    fc_in: float
    fft_size: int
    scaling: float
    ffts_per_buf: int
    spectrum_format: str
    spectrum_averages: int
    filters: list
    input_format: str = "s16le"
    mode: str = "batched"
    device: int = 0


@dataclass
class InputBufferSize:
    new: int
    overlap: int
    total: int


class DspState:
    """DspState on the GPU.  ``process(raw)`` takes the new raw bytes of one
    buffer (the overlap is carried inside) and returns (spectra, outputs)."""

    def __init__(self, plan: Plan, params: DspParams):
        self.plan = plan
        self.params = params

    @classmethod
    def init(cls, params: DspParams):
        filters = []
        for f in params.filters:
            d = dict(fs_out=f.fs_out, fc_out=f.fc_out, transition=f.transition)
            if f.weights is not None:
                d["weights"] = f.weights
            filters.append(d)
        plan = Plan(params.fs_in, params.fft_size, format_code(params.input_format), filters, fc_in=params.fc_in,
                    ffts_per_buf=params.ffts_per_buf, averages=params.spectrum_averages,
                    spectrum_format=params.spectrum_format, mode=params.mode, device=params.device)
        return cls(plan, params), InputBufferSize(plan.new_samples, plan.overlap, plan.total)

    def process(self, raw):
        return self.plan.process(raw)
