"""Test infrastructure, not product code: an FP64 restatement of the
reference's rational downconverter (tools/ddc.py), the checker for the GPU
DDC stage (spektri_b200/ddc.py).  Only tests/ imports it.

RationalDdc (tools/ddc.py:51-145): each input sample x[s] is mixed with a
repeating local-oscillator table lo[k] = exp(2 pi i (k num mod den) / den)
(ddc.py:20-34, k = s mod den), pushed into a FIR history, and the polyphase
phase advances by `interpolation`; every time it reaches `decimation` it
drops by `decimation` and one output is formed from the `firlen` newest
mixed samples with the taps of that phase (ddc.py:113-141):

    y[o] = sum_j taps[p_o + j * interpolation] * mixed[s_o - firlen + 1 + j]

Closed form used here (the phase starts at 0): after S input samples
T(S) = floor(S * interpolation / decimation) outputs exist; output o comes
from sample s_o = ceil((o + 1) * decimation / interpolation) - 1 with phase
p_o = (s_o + 1) * interpolation - (o + 1) * decimation.  Mixed samples
before the stream start are zero (the FIR buffer starts zeroed, ddc.py:84).
DesignDdc (ddc.py:148-177) is restated in design_taps.
"""
from __future__ import annotations

from fractions import Fraction

import numpy as np


def lo_table(num: int, den: int) -> np.ndarray:
    """ddc.py:20-34: phases (k num mod den) * (2 pi / den) in float32, cos + i sin."""
    if num == 0:
        return np.ones(1, np.complex128)
    k = (np.arange(den, dtype=np.int64) * num) % den
    ph = k.astype(np.float32) * np.float32(2.0 * np.pi / den)
    return np.cos(ph.astype(np.float64)) + 1j * np.sin(ph.astype(np.float64))


def design_taps(fs_in, fs_out, fc):
    """DesignDdc (ddc.py:148-177): (taps, interpolation, decimation, num, den)."""
    from scipy import signal
    fs_in, fs_out, fc = Fraction(fs_in), Fraction(fs_out), Fraction(fc)
    freq = -fc / fs_in
    r = fs_out / fs_in
    interp, decim = r.numerator, r.denominator
    taps = signal.firwin((11 * decim) // interp * interp, 1.0 / decim, window="blackman") * interp
    return taps.astype(np.float32), interp, decim, freq.numerator, freq.denominator


class RationalDdc64:
    """Streaming FP64 RationalDdc: execute(x) consumes a chunk and returns
    the outputs it completes, like ddc.py:93-145."""

    def __init__(self, taps, interpolation=1, decimation=1, freq_num=0, freq_den=1):
        self.taps = np.asarray(taps, np.float64)
        self.interp, self.decim = int(interpolation), int(decimation)
        self.firlen = len(self.taps) // self.interp
        self.lo = lo_table(int(freq_num), int(freq_den))
        self.mixed = np.zeros(0, np.complex128)      # every mixed sample so far
        self.n_in = 0
        self.n_out = 0

    def execute(self, x):
        x = np.asarray(x, np.complex128)
        s = np.arange(self.n_in, self.n_in + len(x))
        self.mixed = np.concatenate([self.mixed, x * self.lo[s % len(self.lo)]])
        self.n_in += len(x)
        total = self.n_in * self.interp // self.decim
        o = np.arange(self.n_out, total, dtype=np.int64)
        self.n_out = total
        s_o = -((-(o + 1) * self.decim) // self.interp) - 1            # ceil((o+1) d / i) - 1
        p_o = (s_o + 1) * self.interp - (o + 1) * self.decim
        j = np.arange(self.firlen)
        idx = s_o[:, None] - self.firlen + 1 + j[None, :]
        hist = np.where(idx >= 0, self.mixed[np.maximum(idx, 0)], 0)
        taps = self.taps[p_o[:, None] + j[None, :] * self.interp]
        return (taps * hist).sum(axis=1)
