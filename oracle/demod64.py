"""Test infrastructure, not product code: an FP64 restatement of the
reference's demodulators (tools/demodulator.py), the checker for the GPU
chains in spektri_b200/demod.py.  Only tests/ and tests/golden/make_golden.py
import it.

SsbAgc (demodulator.py:16-65) and AmAgc (:68-103) follow one average
amplitude pa (0 at the start) through the stream:
  SsbAgc: p = |s|, pd = p - pa, pa += pd * (pd >= 0 ? attack : release),
          s *= amplitude / pa (0 when pa <= 0), then if |s|^2 > clip,
          s *= sqrt(clip / |s|^2)         attack 0.002, release 0.0002,
                                          clip 0.9, amplitude 0.25
  AmAgc : pd = s - pa, pa += pd * speed, s = s * (amplitude / pa) - amplitude
          (0 when pa <= 0)                speed 0.0002, amplitude 0.25
with the constants as the float32 values the reference uses.  The chains
(SsbDemodulator :106-137, AmDemodulator :139-162, IqDemodulator :165-197)
are restated on ddc64.RationalDdc64 with the taps rounded to float32 as
RationalDdc stores them (ddc.py:73).
"""
from __future__ import annotations

import numpy as np

from .ddc64 import RationalDdc64, design_taps

F32 = lambda v: float(np.float32(v))
ATTACK, RELEASE, CLIP, AMPLITUDE, AM_SPEED = F32(0.002), F32(0.0002), F32(0.9), F32(0.25), F32(0.0002)


class SsbAgc64:
    def __init__(self):
        self.pa = 0.0

    def execute(self, x):
        x = np.asarray(x, np.complex128)
        y = np.zeros_like(x)
        pa = self.pa
        for i, s in enumerate(x):
            pd = abs(s) - pa
            pa += pd * (ATTACK if pd >= 0 else RELEASE)
            s = s * (AMPLITUDE / pa) if pa > 0 else 0j
            p = s.real ** 2 + s.imag ** 2
            if p > CLIP:
                s *= np.sqrt(CLIP / p)
            y[i] = s
        self.pa = pa
        return y


class AmAgc64:
    def __init__(self):
        self.pa = 0.0

    def execute(self, x):
        x = np.asarray(x, np.float64)
        y = np.zeros_like(x)
        pa = self.pa
        for i, s in enumerate(x):
            pa += (s - pa) * AM_SPEED
            y[i] = s * (AMPLITUDE / pa) - AMPLITUDE if pa > 0 else 0.0
        self.pa = pa
        return y


def _ddc(fs_in, fs_out, fc):
    taps, i, d, num, den = design_taps(fs_in, fs_out, fc)
    return RationalDdc64(taps, i, d, num, den)


def _lowpass(ntaps, cutoff, fs, decimation, **kw):
    from scipy import signal
    taps = signal.firwin(ntaps, cutoff, window="hann", fs=fs).astype(np.float32)
    return RationalDdc64(taps, 1, decimation, **kw)


class _Chain64:
    stages: list
    post = None
    envelope = False
    real_out = False

    def execute(self, x):
        s = np.asarray(x, np.complex128)
        for st in self.stages:
            s = st.execute(s)
        if self.envelope:
            s = np.abs(s)
        if self.post is not None:
            s = self.post.execute(s)
        return s.real if self.real_out else s


class SsbDemodulator64(_Chain64):
    def __init__(self, fs_in, fc_in, fc_demod, mode="lsb", enable_agc=True):
        sideband = 1 if mode == "usb" else -1
        self.stages = [_ddc(fs_in, 16000, fc_demod + 1500 * sideband - fc_in),
                       _lowpass(64, 1400, 16000, 2),
                       RationalDdc64(np.ones(1, np.float32), 1, 1, 3 * sideband, 16)]
        self.post = SsbAgc64() if enable_agc else None
        self.real_out = True


class AmDemodulator64(_Chain64):
    def __init__(self, fs_in, fc_in, fc_demod, mode="am", enable_agc=True):
        self.stages = [_ddc(fs_in, 16000, fc_demod - fc_in), _lowpass(64, 3000, 16000, 1)]
        self.envelope = True
        self.post = AmAgc64() if enable_agc else None
        self.real_out = True


class IqDemodulator64(_Chain64):
    def __init__(self, fs_in, fc_in, fc_demod, mode="", enable_agc=True):
        self.stages = [_ddc(fs_in, 20000, fc_demod - fc_in), _ddc(20000, 200, 0), _lowpass(32, 40, 200, 2)]


# The seeded test streams, complex baseband around fc_in: noise plus carriers
# (offset from fc_in in Hz, amplitude, modulation frequency Hz, AM depth),
# with the amplitude stepped down by 5x for the second half so that the gain
# controls attack and release.
CASES = [
    dict(kind="ssb", mode="usb", agc=True, fs_in=64000, fc_in=0, fc_demod=10000, n=64000, seed=11,
         tones=[(10700.0, 0.3, 0.0, 0.0), (8800.0, 0.2, 0.0, 0.0)]),
    dict(kind="ssb", mode="lsb", agc=True, fs_in=48000, fc_in=1000000, fc_demod=1005000, n=48000, seed=12,
         tones=[(4100.0, 0.3, 0.0, 0.0), (6300.0, 0.1, 0.0, 0.0)]),
    dict(kind="ssb", mode="usb", agc=False, fs_in=64000, fc_in=0, fc_demod=10000, n=32000, seed=13,
         tones=[(11000.0, 0.3, 0.0, 0.0)]),
    dict(kind="am", mode="am", agc=True, fs_in=64000, fc_in=0, fc_demod=-8000, n=64000, seed=14,
         tones=[(-8000.0, 0.4, 400.0, 0.5)]),
    dict(kind="am", mode="am", agc=False, fs_in=64000, fc_in=0, fc_demod=-8000, n=32000, seed=15,
         tones=[(-8000.0, 0.4, 700.0, 0.3)]),
    dict(kind="iq", mode="", agc=True, fs_in=40000, fc_in=0, fc_demod=3000, n=40000, seed=16,
         tones=[(3020.0, 0.3, 0.0, 0.0)]),
]


def stimulus(case):
    n, fs = case["n"], case["fs_in"]
    rng = np.random.default_rng(case["seed"])
    t = np.arange(n) / fs
    x = 0.02 * (rng.standard_normal(n) + 1j * rng.standard_normal(n))
    for f, a, fm, m in case["tones"]:
        x = x + a * (1 + m * np.cos(2 * np.pi * fm * t)) * np.exp(2j * np.pi * f * t)
    x[n // 2:] *= 0.2
    return x.astype(np.complex64)


def agc_edges():
    """Edge streams for the gain controls alone: silence (the average
    amplitude stays 0, outputs 0), an impulse into silence (the SSB clip and
    the release), and a step from silence (the attack)."""
    z = np.zeros(64, np.complex64)
    imp = np.zeros(96, np.complex64)
    imp[0] = 1 + 1j
    step = np.concatenate([np.zeros(16), 0.5 * np.exp(2j * np.pi * 0.01 * np.arange(5000))]).astype(np.complex64)
    return {"silence": z, "impulse": imp, "step": step}


def make(case, cls_map):
    """The case's demodulator from cls_map = {"ssb": ..., "am": ..., "iq": ...}."""
    return cls_map[case["kind"]](case["fs_in"], case["fc_in"], case["fc_demod"], case["mode"], case["agc"])


ORACLE = {"ssb": SsbDemodulator64, "am": AmDemodulator64, "iq": IqDemodulator64}
