"""The downstream rational downconverter (tools/ddc.py:51-177).

CPU: the FP64 restatement (oracle/ddc64.py) and the tap design against the
reference's own outputs (tests/golden/ddc_ref.npz, made by importing
tools/ddc.py and running it on seeded input in uneven chunks).
GPU: the CUDA stage (sk_ddc_*) against the same fixtures (relative RMS
<= 1e-5), invariance to how the stream is cut into calls (bit-exact), and
chained after the filter bank on a channel's output stream.
"""
import os

import numpy as np
import pytest

from oracle import ddc64
from oracle.oracle64 import rel_rms

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ddc_ref.npz")
TOL = 1e-5
CHUNKS = [517, 1999, 64, 3001, 1, 1000, 4096]


def cases():
    d = np.load(GOLDEN)
    n = len([k for k in d.files if k.startswith("cfg")])
    for i in range(n):
        cfg = [int(v) for v in d[f"cfg{i}"]]
        yield dict(interp=cfg[0], decim=cfg[1], num=cfg[2], den=cfg[3], fs_in=cfg[4], fs_out=cfg[5], fc=cfg[6],
                   taps=d[f"taps{i}"], x=d[f"in{i}"], y=d[f"out{i}"])


def chunked(fn, x, sizes=CHUNKS):
    out, pos, k = [], 0, 0
    while pos < len(x):
        c = sizes[k % len(sizes)]
        out.append(fn(x[pos:pos + c]))
        pos += c
        k += 1
    return np.concatenate(out)


def test_restatement_and_design_match_reference_outputs():
    from spektri_b200 import ddc
    for c in cases():
        taps, i, d, num, den = ddc.design_taps(c["fs_in"], c["fs_out"], c["fc"])
        assert (i, d, num, den) == (c["interp"], c["decim"], c["num"], c["den"])
        assert np.array_equal(taps, c["taps"])
        o = ddc64.RationalDdc64(c["taps"], i, d, num, den)
        y = chunked(o.execute, c["x"])
        assert y.shape == c["y"].shape
        assert rel_rms(y, c["y"]) < 1e-6


@pytest.mark.gpu
def test_gpu_ddc_matches_reference_outputs():
    from spektri_b200 import ddc
    for c in cases():
        g = ddc.RationalDdc(c["taps"], c["interp"], c["decim"], c["num"], c["den"])
        y = chunked(g.execute, c["x"])
        assert y.shape == c["y"].shape
        e = rel_rms(y, c["y"])
        assert e < TOL, e
        # the designed object is the same stage
        g2 = ddc.design_ddc(c["fs_in"], c["fs_out"], c["fc"])
        y2 = chunked(g2.execute, c["x"], [c["x"].size])
        assert np.array_equal(y, y2)             # how the stream is cut into calls does not matter


@pytest.mark.gpu
def test_gpu_ddc_after_the_filter_bank():
    """A channel of the plain small configuration (n = 256 bins at 1 kHz
    spacing: 256 kHz complex output) mixed down by 12 kHz and resampled to
    48 kHz, over 6 buffers, against the FP64 restatement fed with the
    channel's own output."""
    import torch
    from spektri_b200 import Plan, ddc, workloads
    w = workloads.c1()
    nb = 6
    raw = workloads.stream_numpy(w, 0, nb * w.samples_per_buffer).view(np.uint8)
    plan = Plan(w.fs, w.fft_size, w.fmt, w.filters()[:1], ffts_per_buf=w.ffts_per_buf, averages=8,
                spectrum_format="f32")
    fs_ch = plan.channels[0]["fs_out"]
    g = ddc.design_ddc(fs_ch, 48000, 12000)
    taps, i, d, num, den = ddc.design_taps(fs_ch, 48000, 12000)
    ref = ddc64.RationalDdc64(taps, i, d, num, den)
    ys, rs = [], []
    for r in np.split(raw, nb):
        _, outs = plan.process(r)
        x = torch.from_numpy(outs[0]).cuda()
        ys.append(g.execute(x).cpu().numpy())
        rs.append(ref.execute(outs[0]))
    y, r = np.concatenate(ys), np.concatenate(rs)
    assert y.shape == r.shape and y.size == nb * plan.channels[0]["out_samples"] * 3 // 16
    assert rel_rms(y, r) < TOL
