"""Seeded synthetic workloads standing in for the five benchmark configurations.

Every stream is int16 (real ``s16le`` or interleaved ``cs16le``) built from
Gaussian noise, tones and band-limited noise carriers, clipped to int16.
Channel layouts (IFFT sizes, centre bins as multiples of 4 — fcfb.rs:232-242
needs that for an exact filter — and taper widths) come from a separate RNG
stream (seed + 1000).  ``stream_numpy`` makes any window of a stream on the
CPU; ``stream_torch`` makes a whole stream on the GPU for benchmarking (the
same recipe, different random numbers).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Workload:
    name: str
    fmt: str                  # "s16le" or "cs16le"
    fs: float                 # input sample rate (Hz)
    fc: float                 # input centre frequency (Hz)
    fft_size: int
    ffts_per_buf: int
    averages: int
    n_samples: int            # stream length (samples; IQ pairs for complex)
    seed: int
    noise_sigma: float
    n_tones: int
    tone_amp: tuple           # (lo, hi) LSB; log-uniform when hi/lo > 10
    n_carriers: int = 0
    carrier_bw: tuple = (3e3, 20e3)
    channels: list = field(default_factory=list)   # dicts: n, centre, transition, trainable

    @property
    def complex(self) -> bool:
        return self.fmt.startswith("c")

    @property
    def spacing(self) -> float:
        return self.fs / self.fft_size

    @property
    def hop(self) -> int:
        return self.fft_size - self.fft_size // 4

    @property
    def samples_per_buffer(self) -> int:
        return self.hop * self.ffts_per_buf

    @property
    def bytes_per_sample(self) -> int:
        return 4 if self.complex else 2

    def filters(self):
        """Plan filter dicts (fs_out, fc_out exact by construction)."""
        out = []
        for c in self.channels:
            d = dict(fs_out=self.spacing * c["n"], fc_out=self.fc + self.spacing * c["centre"])
            if c.get("transition"):
                d["transition"] = int(c["transition"])
            out.append(d)
        return out

    def alg_bytes_per_sample(self) -> float:
        """Input bytes + channel output bytes (8 B per complex64 output) per
        input sample; each block emits sum(3n/4) outputs per 3N/4 inputs."""
        sum_n = sum(c["n"] for c in self.channels)
        return self.bytes_per_sample + 8.0 * sum_n / self.fft_size

    def scaled(self, n_samples: int):
        """The same configuration on a shorter stream."""
        w = Workload(**{k: getattr(self, k) for k in self.__dataclass_fields__})
        w.n_samples = int(n_samples)
        return w


def _draw_channels(rng, count, log2_lo, log2_hi, N, complex_input, tw=None, tw_range=None):
    ch = []
    for _ in range(count):
        n = 1 << int(rng.integers(log2_lo, log2_hi + 1))
        if complex_input:
            centre = 4 * int(rng.integers(-N // 8, N // 8))
        else:
            centre = 4 * int(rng.integers(0, N // 8 + 1))          # 0 .. N/2
        if tw_range is not None:
            t = min(int(rng.integers(tw_range[0], tw_range[1] + 1)), n // 2)
        else:
            t = tw or 0
        ch.append(dict(n=n, centre=centre, transition=t))
    return ch


def c1() -> Workload:
    """Plain small CPU-runnable case: 2^22 real samples, N=4096, 4 x n=256."""
    w = Workload("c1_plain_small", "s16le", 4.096e6, 0.0, 4096, 8, 64, 1 << 22, 1, 1000.0, 5, (100.0, 5000.0))
    rng = np.random.default_rng(w.seed + 1000)
    w.channels = [dict(n=256, centre=4 * int(rng.integers(32, 480)), transition=28) for _ in range(4)]
    return w


def c2() -> Workload:
    """RX888-like: 2^30 real samples at 64.8 MS/s, N=65536, 32 channels n=256..4096."""
    w = Workload("c2_rx888", "s16le", 64.8e6, 0.0, 65536, 64, 256, 1 << 30, 2, 500.0, 200,
                 (8.0, 8000.0), n_carriers=50)
    rng = np.random.default_rng(w.seed + 1000)
    w.channels = _draw_channels(rng, 32, 8, 12, w.fft_size, False)
    return w


def c3() -> Workload:
    """Batching: the C2 stream, 256 channels n=64..8192, taper 8..64 bins, B=64."""
    w = c2()
    w.name = "c3_batched_256ch"
    rng = np.random.default_rng(3 + 1000)
    w.channels = _draw_channels(rng, 256, 6, 13, w.fft_size, False, tw_range=(8, 64))
    return w


def c4() -> Workload:
    """Differentiation: 2^24 real samples, N=32768, 64 channels of n=1024."""
    w = Workload("c4_differentiable", "s16le", 32.768e6, 0.0, 32768, 16, 10**9, 1 << 24, 4, 500.0, 64,
                 (8.0, 8000.0), n_carriers=16)
    rng = np.random.default_rng(w.seed + 1000)
    w.channels = _draw_channels(rng, 64, 10, 10, w.fft_size, False, tw=64)
    return w


def c5() -> Workload:
    """Large complex channelizer: cs16, N=2^20, 2048 channels n=64..8192."""
    w = Workload("c5_cs16_2048ch", "cs16le", 122.88e6, 0.0, 1 << 20, 8, 64, 1 << 31, 5, 300.0, 2000,
                 (3.0, 3000.0), n_carriers=500, carrier_bw=(5e3, 50e3))
    rng = np.random.default_rng(w.seed + 1000)
    w.channels = _draw_channels(rng, 2048, 6, 13, w.fft_size, True, tw_range=(8, 64))
    return w


WORKLOADS = {"c1": c1, "c2": c2, "c3": c3, "c4": c4, "c5": c5}


def _signal_params(w: Workload):
    rng = np.random.default_rng(w.seed)
    lo, hi = w.tone_amp
    half = 0.5 if w.complex else 0.5
    f_tone = rng.uniform(-half if w.complex else 0.0, half, w.n_tones)        # cycles / sample
    if hi / lo > 10:
        a_tone = np.exp(rng.uniform(math.log(lo), math.log(hi), w.n_tones))
    else:
        a_tone = rng.uniform(lo, hi, w.n_tones)
    p_tone = rng.uniform(0, 2 * math.pi, w.n_tones)
    bw = rng.uniform(w.carrier_bw[0], w.carrier_bw[1], w.n_carriers) / w.fs
    f_car = rng.uniform(-half if w.complex else 0.0, half, w.n_carriers)
    a_car = np.exp(rng.uniform(math.log(lo), math.log(hi), w.n_carriers)) if w.n_carriers else np.zeros(0)
    return f_tone, a_tone, p_tone, f_car, bw, a_car


CHUNK = 1 << 20


def stream_numpy(w: Workload, start: int, count: int) -> np.ndarray:
    """Samples [start, start+count) of the stream as raw int16 (interleaved
    I/Q for complex).  Chunks of 2^20 samples are seeded by (seed, chunk)."""
    f_tone, a_tone, p_tone, f_car, bw, a_car = _signal_params(w)
    out = np.empty(count * (2 if w.complex else 1), np.int16)
    pos = start
    while pos < start + count:
        ch = pos // CHUNK
        lo = pos - ch * CHUNK
        hi = min(CHUNK, start + count - ch * CHUNK)
        x = _chunk_numpy(w, ch, f_tone, a_tone, p_tone, f_car, bw, a_car)[lo:hi]
        o = pos - start
        if w.complex:
            out[2 * o: 2 * (o + hi - lo)] = x
        else:
            out[o: o + hi - lo] = x
        pos += hi - lo
    return out


def _chunk_numpy(w, ch, f_tone, a_tone, p_tone, f_car, bw, a_car):
    rng = np.random.default_rng([w.seed, ch])
    t = np.arange(ch * CHUNK, (ch + 1) * CHUNK, dtype=np.float64)
    if w.complex:
        z = (rng.standard_normal(CHUNK) + 1j * rng.standard_normal(CHUNK)) * (w.noise_sigma / math.sqrt(2))
        for f, a, p in zip(f_tone, a_tone, p_tone):
            z += a * np.exp(1j * (2 * math.pi * ((f * t) % 1.0) + p))
    else:
        z = rng.standard_normal(CHUNK) * w.noise_sigma
        for f, a, p in zip(f_tone, a_tone, p_tone):
            z += a * np.cos(2 * math.pi * ((f * t) % 1.0) + p)
    if len(f_car):
        spec = np.zeros(CHUNK, np.complex128)
        k = np.fft.fftfreq(CHUNK)
        for f, b, a in zip(f_car, bw, a_car):
            m = np.abs(k - f) < b / 2
            nb = int(m.sum())
            if nb:
                spec[m] += (rng.standard_normal(nb) + 1j * rng.standard_normal(nb)) * a * math.sqrt(CHUNK / nb / 2)
        c = np.fft.ifft(spec)
        z = z + (c if w.complex else c.real * math.sqrt(2))
    if w.complex:
        iq = np.stack([z.real, z.imag], axis=1).reshape(-1)
        return np.clip(np.round(iq), -32768, 32767).astype(np.int16)
    return np.clip(np.round(z), -32768, 32767).astype(np.int16)


def stream_torch(w: Workload, count: int, device="cuda", chunk: int = 1 << 24):
    """``count`` samples of the workload generated on the GPU (uint8 view of
    int16 data), for benchmarking at full size."""
    import torch
    f_tone, a_tone, p_tone, f_car, bw, a_car = _signal_params(w)
    g = torch.Generator(device=device)
    g.manual_seed(w.seed)
    comp = 2 if w.complex else 1
    out = torch.empty(count * comp, dtype=torch.int16, device=device)
    ft = torch.tensor(f_tone, dtype=torch.float64, device=device)
    at = torch.tensor(a_tone, dtype=torch.float32, device=device)
    pt = torch.tensor(p_tone, dtype=torch.float32, device=device)
    for s in range(0, count, chunk):
        n = min(chunk, count - s)
        t = torch.arange(s, s + n, dtype=torch.float64, device=device)
        if w.complex:
            z = torch.randn(n, dtype=torch.complex64, device=device, generator=g) * w.noise_sigma
        else:
            z = torch.randn(n, dtype=torch.float32, device=device, generator=g) * w.noise_sigma
        for i in range(0, len(f_tone), 16):
            ph = (torch.outer(t, ft[i:i + 16]) % 1.0).float() * (2 * math.pi) + pt[i:i + 16]
            if w.complex:
                z += (torch.polar(at[i:i + 16].expand_as(ph), ph)).sum(dim=1)
            else:
                z += (torch.cos(ph) * at[i:i + 16]).sum(dim=1)
        if len(f_car):
            L = n
            k = torch.fft.fftfreq(L, device=device, dtype=torch.float64)
            spec = torch.zeros(L, dtype=torch.complex64, device=device)
            for f, b, a in zip(f_car, bw, a_car):
                m = (k - f).abs() < b / 2
                nb = int(m.sum())
                if nb:
                    spec[m] += torch.randn(nb, dtype=torch.complex64, device=device, generator=g) * float(a * math.sqrt(L / nb / 2))
            c = torch.fft.ifft(spec)
            z = z + (c if w.complex else c.real * math.sqrt(2))
        if w.complex:
            v = torch.stack([z.real, z.imag], dim=1).reshape(-1)
            out[2 * s: 2 * (s + n)] = torch.clamp(torch.round(v), -32768, 32767).to(torch.int16)
        else:
            out[s: s + n] = torch.clamp(torch.round(z), -32768, 32767).to(torch.int16)
    return out.view(torch.uint8)
