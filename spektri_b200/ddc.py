"""GPU rational downconverter: the reference's RationalDdc and DesignDdc
(tools/ddc.py:51-177) on a channel's complex64 output stream.

``RationalDdc(taps, interpolation, decimation, freq_num, freq_den)`` mirrors
the reference class: ``execute(x)`` consumes a chunk of samples and returns
the outputs it completes, with the FIR history and the oscillator and
polyphase phases carried to the next call.  ``design_ddc(fs_in, fs_out, fc)``
is DesignDdc: a Blackman-windowed FIR of (11 decimation) // interpolation *
interpolation taps at cutoff 1/decimation, times interpolation, and the
oscillator frequency -fc/fs_in as an exact fraction.  The arithmetic runs in
libspektri_b200.so (sk_ddc_*); there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
from fractions import Fraction

import numpy as np

from ._lib import check, lib


class RationalDdc:
    def __init__(self, taps, interpolation=1, decimation=1, freq_num=0, freq_den=1, device=0):
        taps = np.ascontiguousarray(np.asarray(taps, dtype=np.float32))
        self.interpolation, self.decimation = int(interpolation), int(decimation)
        self.freq_num, self.freq_den = int(freq_num), int(freq_den)
        self.device = int(device)
        self.taps = taps
        h = C.c_void_p()
        check(lib().sk_ddc_create(taps.ctypes.data, taps.size, self.interpolation, self.decimation, self.freq_num,
                                  self.freq_den, self.device, C.byref(h)), "sk_ddc_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().sk_ddc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def outputs_for(self, n_in: int) -> int:
        """How many outputs the next call of n_in samples completes."""
        n = C.c_uint64()
        check(lib().sk_ddc_outputs(self._h, int(n_in), C.byref(n)), "sk_ddc_outputs")
        return n.value

    def execute_device(self, x, out, stream=None) -> int:
        """x, out: torch complex64 CUDA tensors (out holds outputs_for(len(x))).
        Enqueues on ``stream`` (default: torch's current stream); returns the
        number of outputs written."""
        import torch
        if stream is None:
            stream = torch.cuda.current_stream(self.device)
        s = stream.cuda_stream if hasattr(stream, "cuda_stream") else stream
        n = C.c_uint64()
        check(lib().sk_ddc_process_device(self._h, x.data_ptr(), x.numel(), out.data_ptr(), C.byref(n), s),
              "sk_ddc_process_device")
        return n.value

    def execute(self, x):
        """RationalDdc.execute (ddc.py:93-145): numpy or torch complex64 in,
        the completed outputs out (same kind as the input)."""
        import torch
        is_np = isinstance(x, np.ndarray)
        xt = torch.from_numpy(np.ascontiguousarray(x, dtype=np.complex64)) if is_np else x
        xt = xt.to(device=f"cuda:{self.device}", dtype=torch.complex64).contiguous()
        out = torch.empty(max(1, self.outputs_for(xt.numel())), dtype=torch.complex64, device=xt.device)
        n = self.execute_device(xt, out)
        out = out[:n]
        if is_np:
            torch.cuda.synchronize(self.device)
            return out.cpu().numpy()
        return out


def design_taps(fs_in, fs_out, fc=0):
    """DesignDdc's parameters (ddc.py:148-177): (taps, interpolation,
    decimation, freq_num, freq_den)."""
    from scipy import signal
    fs_in, fs_out, fc = Fraction(fs_in), Fraction(fs_out), Fraction(fc)
    freq = -fc / fs_in
    r = fs_out / fs_in
    interp, decim = r.numerator, r.denominator
    taps = signal.firwin((11 * decim) // interp * interp, 1.0 / decim, window="blackman") * interp
    return taps.astype(np.float32), interp, decim, freq.numerator, freq.denominator


def design_ddc(fs_in, fs_out, fc=0, device=0) -> RationalDdc:
    """DesignDdc (ddc.py:148-177) on the GPU."""
    taps, i, d, num, den = design_taps(fs_in, fs_out, fc)
    return RationalDdc(taps, i, d, num, den, device=device)
