"""GPU demodulators for a channel's complex64 output stream: the reference's
tools/demodulator.py on the device.

``SsbDemodulator``, ``AmDemodulator`` and ``IqDemodulator`` take the
reference's constructor arguments (fs_in, fc_in, fc_demod, mode, enable_agc)
and build the same chains (demodulator.py:106-197):

  SSB: DesignDdc to 16 kHz centred 1.5 kHz beside fc_demod, a 64-tap
       Hann low-pass at 1400 Hz decimating by 2, a mixer by 3/16 of the
       rate towards the audio band, SsbAgc, real part (8 kHz audio)
  AM : DesignDdc to 16 kHz at fc_demod, a 64-tap Hann low-pass at 3000 Hz,
       |s|, AmAgc (16 kHz audio)
  IQ : DesignDdc to 20 kHz, DesignDdc to 200 Hz, a 32-tap Hann low-pass at
       40 Hz decimating by 2 (complex 100 Hz)

Every stage runs in libspektri_b200.so: the downconverters on sk_ddc_*, the
envelope and the gain controls (``SsbAgc``, ``AmAgc``) on sk_agc_*.  State
carries across ``execute`` calls as in the reference's objects.  There is no
CPU path.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, lib
from .ddc import RationalDdc, design_ddc


def _to_device(x, device, dtype):
    import torch
    is_np = isinstance(x, np.ndarray)
    if is_np:
        x = torch.from_numpy(np.ascontiguousarray(x))
    return x.to(device=f"cuda:{device}", dtype=dtype).contiguous(), is_np


class Agc:
    """One post-detection stage on the device (sk_agc_*): kind is
    AGC_SSB (complex in and out), AGC_AM (real), AGC_AM_ENVELOPE (|s| of
    complex input, then AmAgc) or ENVELOPE (|s| alone)."""

    def __init__(self, kind: int, device: int = 0):
        self.kind, self.device = int(kind), int(device)
        h = C.c_void_p()
        check(lib().sk_agc_create(self.kind, self.device, C.byref(h)), "sk_agc_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().sk_agc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def execute_device(self, x, out, stream=None):
        """x, out: contiguous CUDA tensors of the stage's input and output
        types, out as long as x; enqueued on ``stream`` (default: torch's
        current stream)."""
        import torch
        if stream is None:
            stream = torch.cuda.current_stream(self.device)
        s = stream.cuda_stream if hasattr(stream, "cuda_stream") else stream
        check(lib().sk_agc_process_device(self._h, x.data_ptr(), x.numel(), out.data_ptr(), s),
              "sk_agc_process_device")
        return out

    def execute(self, x):
        import torch
        cin = self.kind != _lib.AGC_AM
        xt, is_np = _to_device(x, self.device, torch.complex64 if cin else torch.float32)
        out = torch.empty(xt.numel(), device=xt.device,
                          dtype=torch.complex64 if self.kind == _lib.AGC_SSB else torch.float32)
        if xt.numel():
            self.execute_device(xt, out)
        if is_np:
            torch.cuda.synchronize(self.device)
            return out.cpu().numpy()
        return out


class SsbAgc(Agc):
    """SsbAgc (demodulator.py:16-65): complex64 in, complex64 out."""

    def __init__(self, device: int = 0):
        super().__init__(_lib.AGC_SSB, device)


class AmAgc(Agc):
    """AmAgc (demodulator.py:68-103): float32 in, float32 out."""

    def __init__(self, device: int = 0):
        super().__init__(_lib.AGC_AM, device)


def _hann_lowpass(ntaps, cutoff, fs):
    from scipy import signal
    return signal.firwin(ntaps, cutoff, window="hann", fs=fs)


def _run_ddc(stage: RationalDdc, x):
    import torch
    out = torch.empty(max(1, stage.outputs_for(x.numel())), dtype=torch.complex64, device=x.device)
    n = stage.execute_device(x, out)
    return out[:n]


class _Chain:
    """A device chain of downconverters followed by an optional detector /
    gain stage; execute(x) takes numpy or torch input and returns the same
    kind."""

    device = 0
    stages: list
    post: Agc | None = None
    real_out = False

    def execute_device(self, x):
        s = x
        for st in self.stages:
            s = _run_ddc(st, s)
        if self.post is not None:
            import torch
            out = torch.empty(s.numel(), device=s.device,
                              dtype=torch.complex64 if self.post.kind == _lib.AGC_SSB else torch.float32)
            if s.numel():
                self.post.execute_device(s, out)
            s = out
        if self.real_out and s.is_complex():
            s = s.real
        return s

    def execute(self, x):
        import torch
        xt, is_np = _to_device(x, self.device, torch.complex64)
        y = self.execute_device(xt)
        if is_np:
            torch.cuda.synchronize(self.device)
            return y.cpu().numpy()
        return y


class SsbDemodulator(_Chain):
    """SsbDemodulator (demodulator.py:106-137): Weaver-method SSB, 8 kHz
    audio.  mode 'usb' or anything else for LSB, as in the reference."""

    def __init__(self, fs_in, fc_in, fc_demod, mode="lsb", enable_agc=True, device=0):
        self.device = int(device)
        sideband = 1 if mode == "usb" else -1
        self.stages = [
            design_ddc(fs_in, 16000, fc_demod + 1500 * sideband - fc_in, device=self.device),
            RationalDdc(_hann_lowpass(64, 1400, 16000), decimation=2, device=self.device),
            RationalDdc(np.ones(1, np.float32), freq_num=3 * sideband, freq_den=16, device=self.device),
        ]
        self.post = Agc(_lib.AGC_SSB, self.device) if enable_agc else None
        self.real_out = True


class AmDemodulator(_Chain):
    """AmDemodulator (demodulator.py:139-162): envelope detection, 16 kHz
    audio."""

    def __init__(self, fs_in, fc_in, fc_demod, mode="am", enable_agc=True, device=0):
        self.device = int(device)
        self.stages = [
            design_ddc(fs_in, 16000, fc_demod - fc_in, device=self.device),
            RationalDdc(_hann_lowpass(64, 3000, 16000), decimation=1, device=self.device),
        ]
        self.post = Agc(_lib.AGC_AM_ENVELOPE if enable_agc else _lib.ENVELOPE, self.device)
        self.real_out = True


class IqDemodulator(_Chain):
    """IqDemodulator (demodulator.py:165-197): complex I/Q at 100 Hz."""

    def __init__(self, fs_in, fc_in, fc_demod, mode="", enable_agc=True, device=0):
        self.device = int(device)
        self.stages = [
            design_ddc(fs_in, 20000, fc_demod - fc_in, device=self.device),
            design_ddc(20000, 200, 0, device=self.device),
            RationalDdc(_hann_lowpass(32, 40, 200), decimation=2, device=self.device),
        ]
        self.post = None
        self.real_out = False
