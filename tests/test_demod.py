"""The downstream demodulators (tools/demodulator.py:16-197).

CPU: the FP64 restatement (oracle/demod64.py) against the reference's own
outputs (tests/golden/demod_ref.npz, made by importing tools/demodulator.py
and running it on the seeded streams of demod64.CASES in uneven chunks).
GPU: the device chains (spektri_b200/demod.py) against the same fixtures and
the restatement (relative RMS <= 1e-5 over the whole output and over its
last three quarters, after the gain controls settle), invariance to how the
stream is cut into calls (bit-exact), and the gain-control stages alone
across their 4096-sample segments and on the reference's outputs for
silence, an impulse and a step (demod64.agc_edges).
"""
import os

import numpy as np
import pytest

from oracle import demod64
from oracle.oracle64 import rel_rms

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "demod_ref.npz")
TOL = 1e-5


def chunked(fn, x, sizes):
    out, pos, k = [], 0, 0
    while pos < len(x):
        c = sizes[k % len(sizes)]
        out.append(np.asarray(fn(x[pos:pos + c])))
        pos += c
        k += 1
    return np.concatenate(out)


def errors(y, r):
    q = len(r) // 4
    return rel_rms(y, r), rel_rms(y[q:], r[q:])


def test_restatement_matches_reference_outputs():
    d = np.load(GOLDEN)
    assert len([k for k in d.files if k.startswith("out")]) == len(demod64.CASES)
    for i, case in enumerate(demod64.CASES):
        o = demod64.make(case, demod64.ORACLE)
        y = chunked(o.execute, demod64.stimulus(case), [4096, 333, 1000, 7, 2500])
        r = d[f"out{i}"]
        assert y.shape == r.shape, (i, y.shape, r.shape)
        assert max(errors(y, r)) < 5e-6, (i, errors(y, r))


def _edge_check(y, r):
    if not np.any(r):
        assert not np.any(y)                                   # silence stays exactly 0
    else:
        assert rel_rms(y, r) < TOL, rel_rms(y, r)


def test_restatement_gain_controls_on_edge_streams():
    """SsbAgc / AmAgc alone on silence (the average amplitude stays 0: the
    reference's pa <= 0 branch gives 0), an impulse into silence (the SSB clip,
    then release) and a step from silence (attack), each in two calls."""
    d = np.load(GOLDEN)
    for name, x in demod64.agc_edges().items():
        h = len(x) // 3
        ssb, am = demod64.SsbAgc64(), demod64.AmAgc64()
        env = np.abs(x.astype(np.complex128))
        _edge_check(np.concatenate([ssb.execute(x[:h]), ssb.execute(x[h:])]), d[f"agc_ssb_{name}"])
        _edge_check(np.concatenate([am.execute(env[:h]), am.execute(env[h:])]), d[f"agc_am_{name}"])


@pytest.mark.gpu
def test_gpu_gain_controls_on_edge_streams():
    """The device gain controls on the same edge streams and calls."""
    from spektri_b200 import _lib, demod
    d = np.load(GOLDEN)
    for name, x in demod64.agc_edges().items():
        h = len(x) // 3
        env = np.abs(x).astype(np.float32)
        ssb, am = demod.Agc(_lib.AGC_SSB), demod.Agc(_lib.AGC_AM)
        y = np.concatenate([ssb.execute(x[:h]), ssb.execute(x[h:])])
        assert y.dtype == np.complex64 and y.shape == x.shape
        _edge_check(y, d[f"agc_ssb_{name}"])
        ya = np.concatenate([am.execute(env[:h]), am.execute(env[h:])])
        assert ya.dtype == np.float32 and ya.shape == x.shape
        _edge_check(ya, d[f"agc_am_{name}"])
        if name == "impulse":
            assert abs(np.abs(y[0]) ** 2 - 0.9) < 1e-5          # clipped to |s|^2 = 0.9 (demodulator.py:58-60)


@pytest.mark.gpu
def test_gpu_demodulators_match_reference_outputs():
    from spektri_b200 import demod
    d = np.load(GOLDEN)
    cls = {"ssb": demod.SsbDemodulator, "am": demod.AmDemodulator, "iq": demod.IqDemodulator}
    for i, case in enumerate(demod64.CASES):
        x = demod64.stimulus(case)
        g = demod64.make(case, cls)
        y = chunked(g.execute, x, [517, 1999, 64, 3001, 1, 8192])
        r = d[f"out{i}"]
        assert y.shape == r.shape and y.dtype == r.dtype, (i, y.shape, y.dtype, r.shape, r.dtype)
        assert max(errors(y, r)) < TOL, (i, errors(y, r))
        o = demod64.make(case, demod64.ORACLE)
        assert max(errors(y, o.execute(x))) < TOL
        g2 = demod64.make(case, cls)
        assert np.array_equal(y, chunked(g2.execute, x, [len(x)]))   # the cut into calls does not matter


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["ssb", "am", "am_envelope", "envelope"])
def test_gpu_gain_control_stages(kind):
    """Each post-detection stage alone on 3 calls totalling 21 000 samples
    (segments of 4096 inside a call, carried state between calls), with the
    amplitude stepped up and down so that both the attack and the release
    branches of SsbAgc run."""
    import torch
    from spektri_b200 import _lib, demod
    rng = np.random.default_rng(7)
    n = 21000
    env = np.where((np.arange(n) // 3000) % 2 == 0, 1.0, 0.1) * (1 + 0.5 * np.sin(np.arange(n) / 300))
    z = (env * (rng.standard_normal(n) + 1j * rng.standard_normal(n)) * 0.3).astype(np.complex64)
    code = {"ssb": _lib.AGC_SSB, "am": _lib.AGC_AM, "am_envelope": _lib.AGC_AM_ENVELOPE,
            "envelope": _lib.ENVELOPE}[kind]
    x = np.abs(z).astype(np.float32) if kind == "am" else z
    g = demod.Agc(code)
    y = chunked(g.execute, x, [5000, 9001, 6999])
    if kind == "ssb":
        r = demod64.SsbAgc64().execute(z)
    elif kind in ("am", "am_envelope"):
        r = demod64.AmAgc64().execute(np.abs(z.astype(np.complex128)))
    else:
        r = np.abs(z.astype(np.complex128))
    assert y.shape == (n,) and y.dtype == (np.complex64 if kind == "ssb" else np.float32)
    assert max(errors(y, r)) < TOL, errors(y, r)
    y2 = demod.Agc(code).execute(torch.from_numpy(x).cuda()).cpu().numpy()
    assert np.array_equal(y, y2)
    if kind == "ssb":
        assert np.max(np.abs(y) ** 2) <= 0.9 * (1 + 1e-6)                # the clip (demodulator.py:58-60)


@pytest.mark.gpu
def test_gpu_am_demodulator_after_the_filter_bank():
    """An AM carrier at 5 kHz from the centre of a 256-bin channel of the
    plain small configuration: the filter bank's channel output fed to the
    device AM demodulator over 6 buffers equals the FP64 restatement fed with
    the same channel output."""
    import torch
    from spektri_b200 import Plan, demod, workloads
    w = workloads.c1()
    nb = 6
    raw = workloads.stream_numpy(w, 0, nb * w.samples_per_buffer).view(np.uint8)
    plan = Plan(w.fs, w.fft_size, w.fmt, w.filters()[:1], ffts_per_buf=w.ffts_per_buf, averages=8,
                spectrum_format="f32")
    ch = plan.channels[0]
    fs_ch = int(round(ch["fs_out"]))
    g = demod.AmDemodulator(fs_ch, 0, 5000)
    o = demod64.AmDemodulator64(fs_ch, 0, 5000)
    ys, rs = [], []
    for r in np.split(raw, nb):
        _, outs = plan.process(r)
        ys.append(g.execute(torch.from_numpy(outs[0]).cuda()).cpu().numpy())
        rs.append(o.execute(outs[0]))
    y, r = np.concatenate(ys), np.concatenate(rs)
    assert y.shape == r.shape and y.size > 0
    assert max(errors(y, r)) < TOL, errors(y, r)
