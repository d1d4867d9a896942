"""Gradient-based design of the channels' complex frequency-domain weights.

The filter bank's channel outputs are differentiable in the weights through
the adjoint kernel (``spektri_b200.autograd``).  A design batch holds one
probe per block: block b's spectrum is that of a single tone at a chosen
frequency, windowed and scaled exactly like an input block (rectangular
window scaling/N, dsp.rs:70-73), so one filter-bank call measures every
channel's response to every probe tone.  The loss per channel is

    1e3 * mean stop-band output power / P_ref  +  mean (pass-band power / P_ref - 1)^2

with P_ref the output power of a pass-band tone through all-ones weights:
stop-band energy weighted 1e3 plus pass-band ripple against an ideal flat
response.  Pass tones lie inside [first + tw, first + n - tw) (tw = taper
bins); stop tones lie outside the channel's n bins, up to n/2 beyond.  Adam
updates the real and imaginary parts.  The designed weights are written as
complex64 files that the plain path loads (filter key ``w=`` of the host
binary, or ``weights`` of ``Plan``).
"""
from __future__ import annotations

import math
import os

import numpy as np
import torch

from .autograd import fcfb
from .plan import Plan


def tone_spectra(freqs_bins, N: int, real_input: bool, scale: float, seed: int = 0, device="cuda"):
    """[len(freqs), K] complex64 spectra of unit tones at the given (fractional)
    bin frequencies, random phases, each windowed by `scale` (= scaling/N)."""
    g = torch.Generator(device="cpu").manual_seed(seed)
    f = torch.as_tensor(np.asarray(freqs_bins, dtype=np.float64)).to(device)
    ph = (torch.rand(len(f), generator=g, dtype=torch.float64) * 2 * math.pi).to(device)
    t = torch.arange(N, dtype=torch.float64, device=device)
    arg = 2 * math.pi * f[:, None] * t[None, :] / N + ph[:, None]
    amp = 16384.0 * scale
    if real_input:
        x = amp * torch.cos(arg)
        X = torch.fft.rfft(x, dim=1)
    else:
        x = amp * torch.exp(1j * arg)
        X = torch.fft.fft(x, dim=1)
    return X.to(torch.complex64)


class WeightDesign:
    """Holds a plan whose B = number of probe tones, the probe spectra and the
    per-channel bookkeeping; ``loss(W)`` is differentiable in W."""

    def __init__(self, fs_in, fft_size, channels, real_input=True, n_pass=12, n_stop=12, transition=None,
                 seed=0, device=0):
        # channels: list of (fs_out, fc_out); all IFFT sizes from the bin arithmetic
        self.N = fft_size
        self.real = real_input
        fmt = "s16le" if real_input else "cs16le"
        self.nc = len(channels)
        rng = np.random.default_rng(seed)
        probes, owner, kind = [], [], []
        spacing = fs_in / fft_size
        info = []
        for c, (fs_out, fc_out) in enumerate(channels):
            n = int(round(fs_out / spacing))
            centre = int(round(fc_out / spacing))
            first = centre - n // 2
            tw = transition if transition is not None else n // 8
            info.append((n, first, tw))
            lo_b = 1 if real_input else -fft_size // 2
            hi_b = fft_size // 2 - 1 if real_input else fft_size // 2 - 1
            pf = rng.uniform(first + tw, first + n - tw, n_pass)
            side = rng.random(n_stop) < 0.5
            sf = np.where(side, rng.uniform(first - n / 2, first - 1, n_stop), rng.uniform(first + n + 1, first + 3 * n / 2, n_stop))
            for f, k in [(x, 0) for x in pf] + [(x, 1) for x in sf]:
                if lo_b <= f <= hi_b:
                    probes.append(f)
                    owner.append(c)
                    kind.append(k)
        B = len(probes)
        if real_input and B % 2:
            probes.append(probes[-1]); owner.append(owner[-1]); kind.append(kind[-1]); B += 1
        self.B = B
        self.info = info
        filters = [dict(fs_out=fs, fc_out=fc) for fs, fc in channels]
        self.plan = Plan(fs_in, fft_size, fmt, filters, ffts_per_buf=B, averages=10**9, spectrum_format="f32",
                         mode="batched", device=device)
        assert self.plan.n_channels == self.nc, "every design channel must be exact"
        scale = (1.0 / 32767.0) / fft_size
        self.X = tone_spectra(probes, fft_size, real_input, scale, seed=seed + 1, device=f"cuda:{device}")
        self.owner = torch.tensor(owner, device=self.X.device)
        self.kind = torch.tensor(kind, device=self.X.device)
        ones = [torch.ones(n, dtype=torch.complex64, device=self.X.device) for n, _, _ in info]
        with torch.no_grad():
            y1 = fcfb(self.plan, self.X, ones)
            self.p_ref = []
            for c in range(self.nc):
                p = self._block_power(y1[c], c)
                m = (self.owner == c) & (self.kind == 0)
                self.p_ref.append(p[m].mean().clamp_min(1e-30))

    def _block_power(self, y, c):
        n = self.info[c][0]
        return (y.view(self.B, n // 8 * 6).abs() ** 2).mean(dim=1)

    def loss(self, W, per_channel=False):
        ys = fcfb(self.plan, self.X, W)
        losses = []
        for c in range(self.nc):
            p = self._block_power(ys[c], c) / self.p_ref[c]
            mp = (self.owner == c) & (self.kind == 0)
            ms = (self.owner == c) & (self.kind == 1)
            stop = p[ms].mean() if ms.any() else p.new_zeros(())
            ripple = ((p[mp] - 1.0) ** 2).mean() if mp.any() else p.new_zeros(())
            losses.append(1e3 * stop + ripple)
        total = torch.stack(losses).sum()
        return (total, losses) if per_channel else total

    def initial_weights(self, kind="tukey"):
        from .dsp import tukey_weights, raised_cosine_weights
        out = []
        for n, _, tw in self.info:
            w = tukey_weights(n, tw) if kind == "tukey" else raised_cosine_weights(n)
            out.append(torch.from_numpy(w).to(self.X.device))
        return out


def adam_design(wd: WeightDesign, steps=500, lr=2e-3, init="tukey", log_every=0):
    """Optimise real and imaginary parts with Adam; returns (weights, history)."""
    W = [torch.view_as_real(w.clone()).requires_grad_(True) for w in wd.initial_weights(init)]
    opt = torch.optim.Adam(W, lr=lr)
    hist = []
    for it in range(steps):
        opt.zero_grad(set_to_none=True)
        loss = wd.loss([torch.view_as_complex(w) for w in W])
        loss.backward()
        opt.step()
        hist.append(float(loss.detach()))
        if log_every and it % log_every == 0:
            print(f"step {it:4d} loss {hist[-1]:.6g}")
    return [torch.view_as_complex(w.detach()).clone() for w in W], hist


def save_weights(directory, weights):
    """One complex64 little-endian file per channel (filter key w=<path>)."""
    os.makedirs(directory, exist_ok=True)
    paths = []
    for i, w in enumerate(weights):
        p = os.path.join(directory, f"channel{i:04d}.c64")
        np.ascontiguousarray(w.detach().cpu().numpy().astype("<c8")).tofile(p)
        paths.append(p)
    return paths


def main(argv=None):
    import argparse
    ap = argparse.ArgumentParser(description="Adam design of filter-bank weights (complex64 files for w=)")
    ap.add_argument("--samplerate", type=float, required=True)
    ap.add_argument("--fftsize", type=int, required=True)
    ap.add_argument("--inputformat", default="s16le")
    ap.add_argument("--filters", nargs="+", required=True, help="fs=..:fc=.. per channel")
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--out", required=True)
    a = ap.parse_args(argv)
    from .dsp import parse_filter_params
    fl = [parse_filter_params(s) for s in a.filters]
    wd = WeightDesign(a.samplerate, a.fftsize, [(f.fs_out, f.fc_out) for f in fl],
                      real_input=not a.inputformat.lower().startswith("c"))
    w0 = wd.initial_weights()
    l0 = float(wd.loss(w0))
    W, hist = adam_design(wd, a.steps, a.lr, log_every=max(1, a.steps // 10))
    paths = save_weights(a.out, W)
    print(f"loss {l0:.6g} -> {hist[-1]:.6g}; weights: {paths[0]} .. ({len(paths)} files)")


if __name__ == "__main__":
    main()
