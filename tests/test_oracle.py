"""Pins the checker before anything is compared with it (CPU only).

* the FP32 restatement and the FP64 oracle against the reference's own
  known-answer tests (multifft.rs:98-132, fcfb.rs:288-312);
* both against the reference's Python model of the filter bank
  (prototyping/fcfb.py, fixtures made by tests/golden/make_golden.py);
* FP32 restatement against FP64 oracle on streaming cases (all 12 formats,
  real and complex), within the 1e-5 relative-RMS bar.
"""
import json
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle32, oracle64
from oracle.oracle64 import rel_rms

TOL = 1e-5


def test_kat_two_real_ffts(golden_dir):
    kat = json.load(open(os.path.join(golden_dir, "kat_two_real_fft.json")))
    o0, o1 = oracle32.two_real_ffts(kat["window"], kat["input0"], kat["input1"])
    e0 = np.array([complex(*v) for v in kat["expected0"]])
    e1 = np.array([complex(*v) for v in kat["expected1"]])
    tol = kat["tolerance"]
    assert np.all(np.abs(o0.real - e0.real) < tol) and np.all(np.abs(o0.imag - e0.imag) < tol)
    assert np.all(np.abs(o1.real - e1.real) < tol) and np.all(np.abs(o1.imag - e1.imag) < tol)
    # the FP64 oracle reads the same numbers
    w = np.array(kat["window"])
    r0 = np.fft.rfft(np.array(kat["input0"]) * w)
    r1 = np.fft.rfft(np.array(kat["input1"]) * w)
    assert np.max(np.abs(r0 - e0)) < tol and np.max(np.abs(r1 - e1)) < tol


def test_kat_freq_to_bins(golden_dir):
    kat = json.load(open(os.path.join(golden_dir, "kat_freq_to_bins.json")))
    for c in kat["cases"]:
        args = (c["fs_in"], c["fc_in"], c["fft_size"], c["fs_out"], c["fc_out"])
        assert oracle64.freq_to_bins(*args) == (c["bins"], c["first"])
        assert oracle32.freq_to_bins(*args) == (c["bins"], c["first"])
        if c["exact"]:
            assert oracle64.freq_to_bins_exact(*args) == (c["bins"], c["first"])
            assert oracle32.freq_to_bins(*args, exact=True) == (c["bins"], c["first"])
            assert oracle64.bins_to_freq(c["fs_in"], c["fc_in"], c["fft_size"], c["bins"], c["first"]) == (c["fs_out"], c["fc_out"])


def test_freq_to_bins_agree_randomised():
    rng = np.random.default_rng(7)
    for _ in range(2000):
        N = int(2 ** rng.integers(8, 21))
        fs = float(rng.choice([64.8e6, 131.072e6, 128e6, 1.024e6, 163.84e6, 48000.0 * rng.integers(1, 100)]))
        fc = float(rng.choice([0.0, 1e6, -2.5e6, rng.normal(0, 1e7)]))
        sp = fs / N
        if rng.random() < 0.5:
            fs_out = sp * 4 * int(rng.integers(-2, 3000))
            fc_out = fc + sp * 4 * int(rng.integers(-N // 8, N // 8))
        else:
            fs_out, fc_out = float(rng.uniform(-1e5, 3e6)), float(rng.normal(0, fs / 4))
        for exact in (False, True):
            a = (oracle64.freq_to_bins_exact if exact else oracle64.freq_to_bins)(fs, fc, N, fs_out, fc_out)
            b = oracle32.freq_to_bins(fs, fc, N, fs_out, fc_out, exact=exact)
            assert a == b, (fs, fc, N, fs_out, fc_out, exact)


@pytest.mark.parametrize("n", [1, 2, 4, 8, 12, 16, 20, 28, 60, 64, 96, 256, 1000, 4096, 65536])
def test_restated_fft_matches_dft(n):
    rng = np.random.default_rng(n)
    x = (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex64)
    for sign in (-1, 1):
        y = oracle32.fft(x, sign)
        ref = np.fft.fft(x.astype(np.complex128)) if sign < 0 else np.fft.ifft(x.astype(np.complex128)) * n
        assert rel_rms(y, ref) < 1e-6


def test_weights_match_design_formulae():
    from scipy.signal import windows
    for n in (16, 64, 256, 1024, 8192):
        assert np.array_equal(oracle32.raised_cosine(n), oracle64.raised_cosine_weights(n))
        for tw in (1, 8, 28, 64, n // 2):
            if tw > n // 2:
                continue
            ref = windows.tukey(n, 2.0 * tw / n, sym=False)
            assert np.max(np.abs(oracle64.tukey_weights(n, tw) - ref)) < 1e-6
            assert np.max(np.abs(oracle32.tukey(n, tw) - oracle64.tukey_weights(n, tw))) <= 1.2e-7
    # the 256-bin / 28-bin design: W[0]=0, flat top of ones
    w = oracle64.tukey_weights(256, 28)
    assert w[0] == 0 and np.all(w[28:229] == 1.0)


def _proto_cases(golden_dir):
    z = np.load(os.path.join(golden_dir, "proto_fcfb.npz"))
    for kind in ("real", "complex"):
        N, B, nbuf, nch = (int(v) for v in z[f"{kind}_params"])
        raw = z[f"{kind}_raw"]
        chans = [(int(z[f"{kind}_{c}_meta"][0]), int(z[f"{kind}_{c}_meta"][1]), z[f"{kind}_{c}_weights"], z[f"{kind}_{c}_out"])
                 for c in range(nch)]
        yield kind, N, B, nbuf, raw, chans


def test_oracles_match_reference_python_model(golden_dir):
    """prototyping/fcfb.py run as an overlap-save bank: its stream is the Rust
    stream delayed by n/8 samples."""
    for kind, N, B, nbuf, raw, chans in _proto_cases(golden_dir):
        fmt = "s16le" if kind == "real" else "cs16le"
        fs = float(N * 1000)
        filters = [dict(fs_out=1000.0 * n, fc_out=1000.0 * (first + n // 2), weights=w.astype(np.complex64))
                   for n, first, w, _ in chans]
        o64 = oracle64.Oracle64(fmt, N, B, 10**9, [oracle64.Channel(n, first, w.astype(np.complex128)) for n, first, w, _ in chans])
        o32 = oracle32.Oracle32(fs, 0.0, N, B, 10**9, fmt, filters)
        assert [tuple(c) for c in o32.channels] == [(n, first) for n, first, _, _ in chans]
        per = len(raw) // nbuf
        s64 = [[] for _ in chans]
        s32 = [[] for _ in chans]
        for b in range(nbuf):
            chunk = raw[b * per:(b + 1) * per]
            _, a = o64.process(chunk.tobytes())
            _, c = o32.process(chunk.tobytes())
            for i in range(len(chans)):
                s64[i].append(a[i]); s32[i].append(c[i])
        for i, (n, first, w, proto) in enumerate(chans):
            y64 = np.concatenate(s64[i]); y32 = np.concatenate(s32[i])
            p = proto[n // 8: n // 8 + len(y64)]
            # the prototype holds back the last n/8 samples of its final step
            assert len(p) >= len(y64) - n // 8
            m = len(p)
            assert rel_rms(y64[:m], p) < 1e-12, (kind, n)
            assert rel_rms(y32[:m], p) < TOL, (kind, n, rel_rms(y32[:m], p))


def _stream(fmt, nsamp, rng):
    cplx = oracle64.is_complex(fmt)
    name = oracle64.CODE_TO_NAME[oracle64.fmt_code(fmt)].lstrip("c")
    count = nsamp * (2 if cplx else 1)
    if name in ("s16le", "s16be"):
        v = np.clip(np.round(rng.normal(0, 3000, count)), -32768, 32767).astype("<i2" if name == "s16le" else ">i2")
    elif name == "s8":
        v = np.clip(np.round(rng.normal(0, 30, count)), -128, 127).astype(np.int8)
    elif name == "u8":
        v = np.clip(np.round(rng.normal(127, 30, count)), 0, 255).astype(np.uint8)
    else:
        v = rng.normal(0, 0.2, count).astype("<f4" if name == "f32le" else ">f4")
    return v.tobytes()


@pytest.mark.parametrize("fmt", sorted(oracle64.FORMATS))
def test_fp32_restatement_vs_fp64(fmt):
    rng = np.random.default_rng(oracle64.fmt_code(fmt))
    N, B, avg = 1024, 6, 5
    fs = 1024e3
    cplx = oracle64.is_complex(fmt)
    chans = [(64, 100), (128, -300 if cplx else 260), (32, 480), (256, 8)]
    filters = [dict(fs_out=1000.0 * n, fc_out=1000.0 * (first + n // 2)) for n, first in chans]
    filters.append(dict(fs_out=1000.0 * 64, fc_out=1000.0 * 33 + 0.5))          # invalid: dropped
    o32 = oracle32.Oracle32(fs, 0.0, N, B, avg, fmt, filters, spectrum_format="f32")
    o32u = oracle32.Oracle32(fs, 0.0, N, B, avg, fmt, filters, spectrum_format="u8")
    assert o32.filter_status[-1] != 0 and o32.n_channels == len(chans)
    o64 = oracle64.Oracle64(fmt, N, B, avg, [oracle64.Channel(n, f, oracle64.raised_cosine_weights(n).astype(np.complex128)) for n, f in chans])
    nbuf = 4
    for b in range(nbuf):
        raw = _stream(fmt, o32.new, rng)
        sp32, out32 = o32.process(raw)
        spu, _ = o32u.process(raw)
        sp64, out64 = o64.process(raw)
        assert [s for s, _ in sp32] == [s for s, _ in sp64]
        for (_, a), (_, r), (_, q) in zip(sp32, sp64, spu):
            assert rel_rms(a, r) < TOL
            db = 10 * np.log10(r)
            qref = oracle64.quantize(db, "u8")
            assert np.max(np.abs(q.astype(int) - qref.astype(int))) <= 1
        for a, r in zip(out32, out64):
            assert rel_rms(a, r) < TOL


def test_oracle_cli_framing(tmp_path):
    """The restated main loop: headers (seq, fake clock), record sizes, tail drop."""
    oracle32.build()
    N, B = 256, 4
    I = N * 3 // 4
    nbuf = 3
    rng = np.random.default_rng(5)
    raw = np.clip(np.round(rng.normal(0, 2000, nbuf * B * I + 77)), -32768, 32767).astype("<i2")
    f0 = tmp_path / "c0.bin"
    args = [oracle32.CLI, "--samplerate=256000", "--centerfreq=1000", "-n", str(N), "--fftbuf", str(B),
            "--averages=6", "-I", "S16LE", "--spectrumformat=u8", "--fake-clock=1700000000,250000000",
            "--filters", f"fs=32000:fc=9000:file={f0}", "fs=3000:fc=0"]
    res = subprocess.run(args, input=raw.tobytes(), capture_output=True, check=True)
    assert b"Invalid filter parameters" in res.stderr
    data = f0.read_bytes()
    n = 32
    rec = 24 + B * (3 * n // 4) * 8
    assert len(data) == nbuf * rec                         # short tail dropped (main.rs:176-178)
    for s in range(nbuf):
        seq, secs, nanos, zero = np.frombuffer(data[s * rec: s * rec + 24], dtype=np.dtype([("a", "<u8"), ("b", "<u8"), ("c", "<u4"), ("d", "<u4")]))[0]
        t = 1700000000 * 10**9 + s * 250000000
        assert (seq, secs, nanos, zero) == (s, t // 10**9, t % 10**9, 0)
    # spectrum: 12 blocks, averages 6 -> 2 records of K=129 u8 on stdout
    K = N // 2 + 1
    out = res.stdout
    assert len(out) == 2 * (24 + K)
    assert np.frombuffer(out[0:8], "<u8")[0] == 0 and np.frombuffer(out[24 + K: 32 + K], "<u8")[0] == 1
