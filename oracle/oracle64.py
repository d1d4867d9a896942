"""FP64 numpy oracle for the spektri filter-bank + Welch spectrum path.

TEST INFRASTRUCTURE ONLY.  Nothing in the product (``spektri_b200``) imports
this module; tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg use it as a checker.

It restates, in float64, the math of the reference (tejeez/spektri, Rust):

* input conversion ......... spektri/src/inputformats.rs:12-155
* buffer assembly .......... spektri/src/main.rs:154-193 (real), :113-152 (complex)
* window / block slicing ... spektri/src/dsp.rs:70-79, 114-160
* forward FFT .............. spektri/src/dsp/multifft.rs:34-95 (rustfft 6.0.1:
  unnormalised DFT, exponent sign -1)
* Welch accumulation ....... spektri/src/dsp/spectrum.rs:82-163
* modulo/mirror bin access . spektri/src/dsp/fftutil.rs:8-22
* filter bank .............. spektri/src/dsp/fcfb.rs:154-203 (inverse DFT sign +1,
  unnormalised; keep samples [n/8, 7n/8))
* bin arithmetic ........... spektri/src/dsp/fcfb.rs:225-285

The constants that the reference holds in f32 (the window value
``scaling/N`` and the filter weights) are taken as their f32 values and then
used exactly in f64, so the f64 result is the exact-arithmetic answer for the
same inputs: the error floor against which FP32 results are measured.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

# DataFormat codes, spektri/src/dsp/data.rs:79-96
FORMATS = {
    "s8": 0x04, "s16le": 0x08, "s16be": 0x09, "f32le": 0x1C, "f32be": 0x1D, "u8": 0x24,
    "cs8": 0x44, "cs16le": 0x48, "cs16be": 0x49, "cf32le": 0x5C, "cf32be": 0x5D, "cu8": 0x64,
}
CODE_TO_NAME = {v: k for k, v in FORMATS.items()}


def fmt_code(fmt) -> int:
    return FORMATS[fmt.lower()] if isinstance(fmt, str) else int(fmt)


def is_complex(fmt) -> bool:
    """inputformats.rs:29-44: the top two bits of the format code say complex."""
    return (fmt_code(fmt) & 0xC0) == 0x40


def bytes_per_sample(fmt) -> int:
    """inputformats.rs:12-27."""
    c = fmt_code(fmt)
    bits = {2: 8, 4: 16, 6: 32}[(c >> 1) & 7]
    return bits // 8 * (2 if is_complex(c) else 1)


def input_scaling(fmt) -> np.float32:
    """inputformats.rs:47-62: 1/i8::MAX, 1/i16::MAX or 1, computed in f32."""
    c = fmt_code(fmt)
    bits = {2: 8, 4: 16, 6: 32}[(c >> 1) & 7]
    if bits == 8:
        return np.float32(1.0) / np.float32(127.0)
    if bits == 16:
        return np.float32(1.0) / np.float32(32767.0)
    return np.float32(1.0)


def convert(raw: bytes | np.ndarray, fmt) -> np.ndarray:
    """inputformats.rs:65-155 -> float32 (real) or complex64 samples.

    U8 subtracts 127.4 in f32 (:68-71); every other format converts exactly.
    """
    c = fmt_code(fmt)
    raw = np.frombuffer(raw, dtype=np.uint8) if not isinstance(raw, np.ndarray) else raw.view(np.uint8)
    name = CODE_TO_NAME[c].lstrip("c")
    dt = {"u8": np.uint8, "s8": np.int8, "s16le": "<i2", "s16be": ">i2",
          "f32le": "<f4", "f32be": ">f4"}[name]
    v = raw.view(dt)
    if name == "u8":
        f = v.astype(np.float32) - np.float32(127.4)
    else:
        f = v.astype(np.float32)
    if is_complex(c):
        return (f[0::2] + 1j * f[1::2].astype(np.float64)).astype(np.complex64)
    return f


# ---------------------------------------------------------------- bin arithmetic

def _round_half_away(v: float) -> float:
    """Rust f64::round: half-way cases away from zero."""
    return math.copysign(math.floor(abs(v) + 0.5), v) if abs(v) < 2**52 else v


def freq_to_bins(fs_in, fc_in, fft_size, fs_out, fc_out):
    """fcfb.rs:225-252.  Returns (bins, first) or None."""
    def nearest_multiple(value, multiple):
        r = _round_half_away(value / float(multiple)) * float(multiple)
        if math.isnan(r):
            return 0
        return int(max(min(r, 2**63 - 1), -2**63))
    spacing = fs_in / float(fft_size)
    bins = nearest_multiple(fs_out / spacing, 4)
    center = nearest_multiple((fc_out - fc_in) / spacing, 4)
    if bins > 0:
        return bins, center - bins // 2
    return None


def bins_to_freq(fs_in, fc_in, fft_size, bins, first):
    """fcfb.rs:257-268."""
    spacing = fs_in / float(fft_size)
    return spacing * float(bins), fc_in + spacing * float(first + bins // 2)


def freq_to_bins_exact(fs_in, fc_in, fft_size, fs_out, fc_out):
    """fcfb.rs:274-285: accept only an exact f64 round trip."""
    bn = freq_to_bins(fs_in, fc_in, fft_size, fs_out, fc_out)
    if bn is None:
        return None
    if bins_to_freq(fs_in, fc_in, fft_size, *bn) == (fs_out, fc_out):
        return bn
    return None


# ---------------------------------------------------------------- weights

_libm = None


def _cosf(x: np.ndarray) -> np.ndarray:
    """The platform libm ``cosf`` (what Rust's f32::cos calls on Linux); numpy's
    own float32 cos rounds differently in the last place."""
    global _libm
    if _libm is None:
        import ctypes
        _libm = ctypes.CDLL("libm.so.6")
        _libm.cosf.restype = ctypes.c_float
        _libm.cosf.argtypes = [ctypes.c_float]
    return np.array([_libm.cosf(float(v)) for v in x], dtype=np.float32)


_rc_cache: dict = {}


def raised_cosine_weights(n: int) -> np.ndarray:
    """fcfb.rs:197-203, evaluated in f32 exactly as the reference does."""
    if n not in _rc_cache:
        f = np.float32(2.0 * np.float32(math.pi)) / np.float32(n)
        i = np.arange(n, dtype=np.float32)
        _rc_cache[n] = (np.float32(0.5) - np.float32(0.5) * _cosf((i * f).astype(np.float32))).astype(np.float32)
    return _rc_cache[n].copy()


def tukey_weights(n: int, tw: int) -> np.ndarray:
    """Periodic Tukey window with ``tw`` taper bins per side, as
    prototyping/fcfb.py:122 designs it (``tukey(n, 2*tw/n, sym=False)``).

    Evaluated in f64 and rounded to f32.  tw >= n/2 gives the full Hann window.
    """
    if tw <= 0:
        return np.ones(n, dtype=np.float32)
    m = n + 1                       # periodic = symmetric of length n+1, last dropped
    alpha = 2.0 * tw / n
    if alpha >= 1.0:
        k = np.arange(n)
        return (0.5 - 0.5 * np.cos(2 * np.pi * k / n)).astype(np.float32)
    width = int(np.floor(alpha * (m - 1) / 2.0))
    k = np.arange(m, dtype=np.float64)
    w = np.ones(m)
    a = k[: width + 1]
    w[: width + 1] = 0.5 * (1 + np.cos(np.pi * (-1 + 2.0 * a / alpha / (m - 1))))
    c = k[m - width - 1:]
    w[m - width - 1:] = 0.5 * (1 + np.cos(np.pi * (-2.0 / alpha + 1 + 2.0 * c / alpha / (m - 1))))
    return w[:n].astype(np.float32)


# ---------------------------------------------------------------- spectra

def get_bins(X: np.ndarray, fft_size: int, idx: np.ndarray) -> np.ndarray:
    """fftutil.rs:8-22, vectorised over indices; X has shape [..., K]."""
    m = np.mod(idx, fft_size)
    K = X.shape[-1]
    direct = m < K
    out = np.empty(X.shape[:-1] + idx.shape, dtype=X.dtype)
    out[..., direct] = X[..., m[direct]]
    out[..., ~direct] = np.conj(X[..., fft_size - m[~direct]])
    return out


def welch_terms(X: np.ndarray, fft_size: int) -> np.ndarray:
    """spectrum.rs:90-111: c_k = X[k] - (X[k-1] + X[k+1])/2, |c_k|^2, per block."""
    K = X.shape[-1]
    k = np.arange(K)
    left = get_bins(X, fft_size, k - 1)
    right = get_bins(X, fft_size, k + 1)
    c = X - (left + right) * 0.5
    return c.real ** 2 + c.imag ** 2


def quantize(acc_mean_db: np.ndarray, spec_fmt: str) -> np.ndarray:
    """spectrum.rs:133-151 on a dB array.  Rust's float->int casts saturate and
    send NaN to 0."""
    if spec_fmt == "u8":
        v = np.clip(np.nan_to_num(acc_mean_db * 2.0 + 250.0, nan=0.0, neginf=0.0), 0, 255)
        return np.trunc(v).astype(np.uint8)
    if spec_fmt == "u16":
        v = np.clip(np.nan_to_num(acc_mean_db * 20.0 + 4000.0, nan=0.0, neginf=0.0), 0, 4095)
        return np.trunc(v).astype(">u2")
    raise ValueError(spec_fmt)


# ---------------------------------------------------------------- pipeline

@dataclass
class Channel:
    bins: int
    first: int
    weights: np.ndarray          # complex128 [bins], natural order: W[j] scales bin first+j


@dataclass
class Oracle64:
    """Streaming FP64 restatement of DspState + main loop.

    ``process(raw)`` consumes one buffer of ``new`` raw samples (main.rs:176)
    and returns (spectra, channel_outputs): spectra is a list of
    (spectrum_seq, power) with power = acc/accn (float64), channel_outputs a
    list of complex128 arrays of B*3n/4 samples, in filter order.
    """
    fmt: str | int
    fft_size: int
    ffts_per_buf: int
    averages: int
    channels: list[Channel]
    acc: np.ndarray = field(init=False)
    accn: int = field(init=False, default=0)
    spec_seq: int = field(init=False, default=0)

    def __post_init__(self):
        self.cplx = is_complex(self.fmt)
        N = self.fft_size
        self.overlap = N // 4                       # dsp.rs:77
        self.hop = N - self.overlap                 # dsp.rs:78
        self.new = self.hop * self.ffts_per_buf     # dsp.rs:107-110
        self.total = self.new + self.overlap
        self.K = N if self.cplx else N // 2 + 1     # dsp.rs:79
        # dsp.rs:70-73: rectangular window scaling/N in f32
        self.w = float(np.float32(input_scaling(self.fmt) / np.float32(N)))
        self.buf = np.zeros(self.total, dtype=np.complex128 if self.cplx else np.float64)
        self.acc = np.zeros(self.K)

    def spectra_of(self, raw: bytes | np.ndarray) -> np.ndarray:
        """Advance the overlap buffer by one raw buffer and return X [B, K]."""
        self.buf[: self.overlap] = self.buf[self.new: self.total]          # main.rs:173
        self.buf[self.overlap:] = convert(raw, self.fmt)                  # main.rs:181
        N, I = self.fft_size, self.hop
        idx = np.arange(self.ffts_per_buf)[:, None] * I + np.arange(N)[None, :]
        blocks = self.buf[idx] * self.w
        if self.cplx:
            return np.fft.fft(blocks, axis=1)
        return np.fft.rfft(blocks, axis=1)

    def process(self, raw):
        X = self.spectra_of(raw)
        spectra = []
        P = welch_terms(X, self.fft_size)
        for b in range(self.ffts_per_buf):
            self.acc += P[b]
            self.accn += 1
            if self.accn >= self.averages:                                # spectrum.rs:116
                spectra.append((self.spec_seq, self.acc / self.accn))
                self.acc = np.zeros(self.K)
                self.accn = 0
                self.spec_seq += 1
        outs = [self.channel_output(X, ch) for ch in self.channels]
        return spectra, outs

    def channel_output(self, X: np.ndarray, ch: Channel) -> np.ndarray:
        """fcfb.rs:154-188 for every block of X; returns B*3n/4 samples."""
        n = ch.bins
        j = (np.arange(n) + n // 2) % n                                   # fcfb.rs:166-169
        g = get_bins(X, self.fft_size, ch.first + j) * ch.weights[j]
        y = np.fft.ifft(g, axis=1) * n                                    # unnormalised
        return y[:, n // 8: n // 8 * 7].reshape(-1)                       # fcfb.rs:177


def rel_rms(a: np.ndarray, ref: np.ndarray) -> float:
    """||a - ref|| / ||ref|| (0 when both are zero)."""
    a = np.asarray(a, dtype=np.complex128 if np.iscomplexobj(a) or np.iscomplexobj(ref) else np.float64)
    ref = np.asarray(ref, dtype=a.dtype)
    den = np.sqrt(np.sum(np.abs(ref) ** 2))
    num = np.sqrt(np.sum(np.abs(a - ref) ** 2))
    if den == 0:
        return 0.0 if num == 0 else float("inf")
    return float(num / den)
