#!/usr/bin/env python3
"""Generate the golden fixtures under tests/golden/ from the reference tree.

Run in a container that has the reference checked out, naming its root:
``python tests/golden/make_golden.py <reference root>`` or with the
SPEKTRI_REFERENCE environment variable.  The GPU box does not have the
reference, so the outputs are committed and the tests only read them.

Fixtures:
  kat_two_real_fft.json  the known-answer vectors of spektri/src/dsp/multifft.rs:98-132
                         (read from the Rust source text, tolerance 1e-4 as there)
  kat_freq_to_bins.json  the case of spektri/src/dsp/fcfb.rs:288-312
  proto_fcfb.npz         outputs of prototyping/fcfb.py:17-87 (the reference's own
                         Python model of the filter bank, imported and run here) on
                         seeded int16 streams, real and complex, for several channels
  wire_topics.json       topic / metadata bytes from tools/spektri.py:15-42
  ddc_ref.npz            outputs of tools/ddc.py:51-177 (RationalDdc designed by
                         DesignDdc, imported and run here; needs numba and scipy)
                         on seeded complex streams fed in uneven chunks
  demod_ref.npz          outputs of tools/demodulator.py:106-197 (SsbDemodulator,
                         AmDemodulator, IqDemodulator with their gain controls,
                         imported and run here; needs numba and scipy) on the
                         seeded streams of oracle/demod64.py's CASES, fed in
                         uneven chunks, and of SsbAgc / AmAgc alone on the edge
                         streams of demod64.agc_edges (silence, impulse, step)
"""
import importlib.util
import json
import os
import re
import struct
import sys

import numpy as np

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SPEKTRI_REFERENCE", "")
OUT = os.path.dirname(os.path.abspath(__file__))


def load_module(path, name):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def kat_two_real_fft():
    src = open(os.path.join(REF, "spektri/src/dsp/multifft.rs")).read()
    body = src[src.index("fn test_two_real_ffts"):]
    cplx = re.findall(r"vec!\[\s*(Complex\{.*?\})\s*\]", body, re.S)
    def parse_c(s):
        return [[float(a), float(b)] for a, b in re.findall(r"re:\s*([-\d.]+)\s*,\s*im:\s*([-\d.]+)", s)]
    exp0, exp1 = parse_c(cplx[0]), parse_c(cplx[1])
    reals = re.findall(r"&vec!\[([-\d.,\s]+)\]", body)
    win, in0, in1 = [[float(v) for v in r.split(",") if v.strip()] for r in reals[:3]]
    tol = float(re.findall(r"check_difference\(&out0, &expected_out0, ([\d.]+)\)", body)[0])
    return {"source": "spektri/src/dsp/multifft.rs:98-132", "n": len(win), "window": win,
            "input0": in0, "input1": in1, "expected0": exp0, "expected1": exp1, "tolerance": tol}


def kat_freq_to_bins():
    src = open(os.path.join(REF, "spektri/src/dsp/fcfb.rs")).read()
    m = re.search(r"test\((\d+),\s*([\d.e]+),\s*([\d.e]+),\s*([\d.e]+),\s*([\d.e]+),\s*(\d+),\s*(\d+),\s*(true|false)\)", src)
    n, fs, fc, fso, fco, bins, first, exact = m.groups()
    return {"source": "spektri/src/dsp/fcfb.rs:288-312",
            "cases": [{"fft_size": int(n), "fs_in": float(fs), "fc_in": float(fc), "fs_out": float(fso),
                       "fc_out": float(fco), "bins": int(bins), "first": int(first), "exact": exact == "true"}]}


def raised_cosine_f32(n):
    import ctypes
    libm = ctypes.CDLL("libm.so.6"); libm.cosf.restype = ctypes.c_float; libm.cosf.argtypes = [ctypes.c_float]
    # fcfb.rs:197-203 in f32 (the same values the filter bank uses)
    f = np.float32(2.0 * np.float32(np.pi)) / np.float32(n)
    i = np.arange(n, dtype=np.float32)
    c = np.array([libm.cosf(float(v)) for v in (i * f).astype(np.float32)], np.float32)
    return (np.float32(0.5) - np.float32(0.5) * c).astype(np.float32)


def proto_fcfb():
    """Run prototyping/fcfb.py:fcfb() as an overlap-save bank equivalent to the
    Rust filter: prewindow = scaling/N (dsp.rs:70-73), postwindow keeps
    [n/8, 7n/8) (fcfb.rs:177), overlap 0.25.  Its output stream equals the Rust
    stream delayed by n/8 samples (the prototype emits the tail of the previous
    step first)."""
    fcfb = load_module(os.path.join(REF, "prototyping/fcfb.py"), "proto_fcfb").fcfb
    rng = np.random.default_rng(1234)
    cases = {}
    N, B, nbuf = 512, 4, 4
    I = N - N // 4
    for kind in ("real", "complex"):
        nnew = B * I * nbuf
        if kind == "real":
            t = np.arange(nnew)
            x = 3000 * np.cos(2 * np.pi * 0.0731 * t + 0.3) + 800 * np.cos(2 * np.pi * 0.3117 * t) + rng.normal(0, 300, nnew)
            raw = np.clip(np.round(x), -32768, 32767).astype("<i2")
            xf = raw.astype(np.float64)
        else:
            t = np.arange(nnew)
            z = 2500 * np.exp(2j * np.pi * (-0.2113 * t)) + 900 * np.exp(2j * np.pi * 0.0517 * t) \
                + rng.normal(0, 250, nnew) + 1j * rng.normal(0, 250, nnew)
            iq = np.stack([np.round(z.real), np.round(z.imag)], axis=1)
            raw = np.clip(iq, -32768, 32767).astype("<i2").reshape(-1)
            xf = raw[0::2].astype(np.float64) + 1j * raw[1::2].astype(np.float64)
        w = np.float32(np.float32(1.0) / np.float32(32767.0) / np.float32(N))
        # main.rs:165: the stream starts with N/4 zeros; one extra hop of zeros
        # lets the prototype's loop (fcfb.py:60, t < len - N) reach the last block.
        stream = np.concatenate([np.zeros(N // 4, xf.dtype), xf, np.zeros(I, xf.dtype)])
        # centre bins (first + n/2) are multiples of 4, as fcfb.rs:232-242 requires
        chans = [(64, 40), (32, -20), (128, 100), (16, 252)] if kind == "real" else [(64, -152), (32, 28), (128, 300)]
        for ci, (n, first) in enumerate(chans):
            weights = raised_cosine_f32(n)
            post = np.zeros(n, np.float32)
            post[n // 8: 7 * n // 8] = 1
            pre = np.full(N, w, np.float32)
            y = fcfb(stream, first + n // 2, pre, weights, post, 0.25)
            cases[f"{kind}_{ci}_out"] = y
            cases[f"{kind}_{ci}_meta"] = np.array([n, first], np.int64)
            cases[f"{kind}_{ci}_weights"] = weights
        cases[f"{kind}_raw"] = raw
        cases[f"{kind}_params"] = np.array([N, B, nbuf, len(chans)], np.int64)
    np.savez_compressed(os.path.join(OUT, "proto_fcfb.npz"), **cases)


def wire_topics():
    sys.modules.setdefault("zmq", __import__("zmq"))
    sp = load_module(os.path.join(REF, "tools/spektri.py"), "spektri_tools")
    cases = []
    for fs, fc in [(64000.0, 80000.0), (500000.0, 50.25e6), (80000.0, 0.0), (988.76953125 * 256, -1234.5)]:
        cases.append({"fs": fs, "fc": fc, "topic_hex": sp.signal_topic(fs, fc).hex()})
    msg = struct.pack("<QQII", 123456789, 1700000000, 987654321, 0) + b"\x00" * 8
    md = sp.unpack_metadata(msg)
    return {"source": "tools/spektri.py:15-42", "signal_topics": cases,
            "spectrum_topic_prefix_hex": sp.spectrum_topic().hex(),
            "metadata_hex": msg[:24].hex(), "metadata": [md.seq, md.time_s, md.time_ns]}


DDC_CASES = [                      # (fs_in, fs_out, fc, samples)
    (256000, 48000, 12000, 6000),
    (64000, 16000, -3000, 4000),
    (500000, 16000, 500, 12000),
]


def ddc_ref():
    """RationalDdc outputs of the reference (tools/ddc.py) on seeded input,
    fed in chunks of uneven size (the state carries across calls); the
    reference's output buffer holds 1000 samples per call (ddc.py:105), so
    chunks stay below 1000 * decimation / interpolation input samples."""
    ddc = load_module(os.path.join(REF, "tools/ddc.py"), "ref_ddc")
    out = {}
    rng = np.random.default_rng(2024)
    for i, (fs_in, fs_out, fc, n) in enumerate(DDC_CASES):
        d = ddc.DesignDdc(fs_in, fs_out, fc)
        x = ((rng.standard_normal(n) + 1j * rng.standard_normal(n)) * 0.3).astype(np.complex64)
        t = np.arange(n)
        x += (0.5 * np.exp(2j * np.pi * (fc + 0.1 * fs_out) / fs_in * t)).astype(np.complex64)
        limit = max(1, 1000 * d.decimation // d.interpolation - 1)
        ys, pos, k = [], 0, 0
        while pos < n:
            c = min(n - pos, min(limit, [517, 1999, 64, 3001, 1][k % 5]))
            ys.append(d.execute(x[pos:pos + c]))
            pos += c
            k += 1
        y = np.concatenate(ys)
        from fractions import Fraction
        f = -Fraction(fc) / Fraction(fs_in)
        out[f"in{i}"] = x
        out[f"taps{i}"] = np.asarray(d.taps, np.float32)
        out[f"cfg{i}"] = np.array([d.interpolation, d.decimation, f.numerator, f.denominator, fs_in, fs_out, fc],
                                  np.int64)
        out[f"out{i}"] = y
    np.savez_compressed(os.path.join(OUT, "ddc_ref.npz"), **out)


def demod_ref():
    """Demodulator outputs of the reference (tools/demodulator.py) on the
    seeded streams of oracle/demod64.py's CASES, fed in uneven chunks; each
    RationalDdc stage's output buffer holds 1000 samples per call
    (ddc.py:105), so chunks stay below 1000 * decimation / interpolation of
    the first stage."""
    sys.path.insert(0, os.path.join(REF, "tools"))
    sys.path.insert(0, os.path.dirname(os.path.dirname(OUT)))
    import demodulator
    from oracle import demod64
    out = {}
    for i, case in enumerate(demod64.CASES):
        d = demod64.make(case, {"ssb": demodulator.SsbDemodulator, "am": demodulator.AmDemodulator,
                                "iq": demodulator.IqDemodulator})
        x = demod64.stimulus(case)
        first = d.ddc
        limit = max(1, 1000 * first.decimation // first.interpolation - 1)
        ys, pos, k = [], 0, 0
        while pos < len(x):
            c = min(len(x) - pos, limit, [517, 1999, 64, 3001, 1][k % 5])
            ys.append(np.array(d.execute(x[pos:pos + c])))
            pos += c
            k += 1
        out[f"out{i}"] = np.concatenate(ys)
    # the gain controls alone on their edge streams, in two calls each
    for name, x in demod64.agc_edges().items():
        h = len(x) // 3
        ssb, am = demodulator.SsbAgc(), demodulator.AmAgc()
        env = np.abs(x).astype(np.float32)
        out[f"agc_ssb_{name}"] = np.concatenate([ssb.execute(x[:h].copy()), ssb.execute(x[h:].copy())])
        out[f"agc_am_{name}"] = np.concatenate([am.execute(env[:h].copy()), am.execute(env[h:].copy())])
    np.savez_compressed(os.path.join(OUT, "demod_ref.npz"), **out)


if __name__ == "__main__":
    if not REF or not os.path.isdir(os.path.join(REF, "spektri")):
        sys.exit("usage: make_golden.py <reference root>  (or set SPEKTRI_REFERENCE): the tejeez/spektri tree")
    with open(os.path.join(OUT, "kat_two_real_fft.json"), "w") as f:
        json.dump(kat_two_real_fft(), f, indent=1)
    with open(os.path.join(OUT, "kat_freq_to_bins.json"), "w") as f:
        json.dump(kat_freq_to_bins(), f, indent=1)
    with open(os.path.join(OUT, "wire_topics.json"), "w") as f:
        json.dump(wire_topics(), f, indent=1)
    proto_fcfb()
    ddc_ref()
    demod_ref()
    print("golden fixtures written to", OUT)
