"""C ABI checks that need no GPU: the library loads, exports every symbol the
header declares, and its host-only functions agree bit for bit with the
oracle (bin arithmetic, weights) and the reference's wire format."""
import json
import os
import re

import numpy as np
import pytest

from oracle import oracle32, oracle64
from spektri_b200 import _lib, dsp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "spektri_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(sk_[a-z0-9_]+)\s*\(", src)))


def test_every_declared_symbol_is_exported_and_bound():
    L = _lib.lib()
    names = header_functions()
    assert len(names) >= 29
    bound = {n for n, _, _ in _lib.PROTOTYPES}
    for n in names:
        assert hasattr(L, n), n
        assert n in bound, f"{n} has no ctypes prototype"


def test_header_constants_match_the_binding():
    """Every status and kind code the header defines has the same value in
    the ctypes binding (a drifted constant would select the wrong stage)."""
    src = open(os.path.join(ROOT, "include", "spektri_b200.h")).read()
    defs = {k: int(v) for k, v in re.findall(r"#define\s+(SK_[A-Z0-9_]+)\s+(-?\d+)\b", src)}
    names = {"SK_OK": "SK_OK", "SK_WARN_FILTER": "SK_WARN_FILTER", "SK_ERR_ARG": "SK_ERR_ARG",
             "SK_ERR_FILTER": "SK_ERR_FILTER", "SK_ERR_CUDA": "SK_ERR_CUDA", "SK_ERR_NOMEM": "SK_ERR_NOMEM",
             "SK_ERR_TIMEOUT": "SK_ERR_TIMEOUT", "SK_ERR_UNSUPPORTED": "SK_ERR_UNSUPPORTED",
             "SK_ERR_STATE": "SK_ERR_STATE", "SK_AGC_SSB": "AGC_SSB", "SK_AGC_AM": "AGC_AM",
             "SK_AGC_AM_ENVELOPE": "AGC_AM_ENVELOPE", "SK_ENVELOPE": "ENVELOPE"}
    for h, py in names.items():
        assert defs[h] == getattr(_lib, py), h


def test_no_gpu_fails_loudly_without_fallback():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from spektri_b200 import Plan, SpektriError
    with pytest.raises(SpektriError) as e:
        Plan(1e6, 1024, "s16le", [])
    assert e.value.code == _lib.SK_ERR_CUDA


def test_bins_bit_exact_against_oracle():
    rng = np.random.default_rng(3)
    for _ in range(3000):
        N = int(2 ** rng.integers(6, 21))
        fs = float(rng.choice([64.8e6, 131.072e6, 128e6, 1.024e6, 163.84e6, 48000.0 * int(rng.integers(1, 100))]))
        fc = float(rng.choice([0.0, 1e6, -2.5e6, rng.normal(0, 1e7)]))
        sp = fs / N
        if rng.random() < 0.6:
            fs_out = sp * 4 * int(rng.integers(-2, 3000))
            fc_out = fc + sp * 4 * int(rng.integers(-N // 8, N // 8))
        else:
            fs_out, fc_out = float(rng.uniform(-1e5, 3e6)), float(rng.normal(0, fs / 4))
        a = dsp.freq_to_bins(fs, fc, N, fs_out, fc_out)
        b = oracle64.freq_to_bins(fs, fc, N, fs_out, fc_out)
        assert a == b
        assert dsp.freq_to_bins_exact(fs, fc, N, fs_out, fc_out) == oracle64.freq_to_bins_exact(fs, fc, N, fs_out, fc_out)
        if a:
            assert dsp.bins_to_freq(fs, fc, N, *a) == oracle64.bins_to_freq(fs, fc, N, *a)


def test_kat_freq_to_bins(golden_dir):
    kat = json.load(open(os.path.join(golden_dir, "kat_freq_to_bins.json")))
    for c in kat["cases"]:
        args = (c["fs_in"], c["fc_in"], c["fft_size"], c["fs_out"], c["fc_out"])
        assert dsp.freq_to_bins(*args) == (c["bins"], c["first"])
        assert dsp.freq_to_bins_exact(*args) == (c["bins"], c["first"])


def test_weights_match_oracle():
    for n in (4, 16, 64, 256, 1024, 8192):
        assert np.array_equal(dsp.raised_cosine_weights(n).real, oracle32.raised_cosine(n))
        assert np.all(dsp.raised_cosine_weights(n).imag == 0)
        for tw in (0, 1, 8, 28, 64, n // 2):
            if tw > n // 2:
                continue
            a = dsp.tukey_weights(n, tw).real
            assert np.array_equal(a, oracle32.tukey(n, tw)), (n, tw)
            if tw:
                assert np.max(np.abs(a - oracle64.tukey_weights(n, tw))) <= 1.2e-7


def test_wire_format_matches_reference_tools(golden_dir):
    g = json.load(open(os.path.join(golden_dir, "wire_topics.json")))
    for c in g["signal_topics"]:
        assert dsp.serialize_signal_topic(c["fs"], c["fc"]).hex() == c["topic_hex"]
    assert dsp.serialize_spectrum_topic(1000.0, 0.0)[:8].hex() == g["spectrum_topic_prefix_hex"]
    assert dsp.serialize_spectrum_topic(1000.0, 5.0, "u16")[:8].hex() == g["spectrum_topic_prefix_hex"]
    assert dsp.serialize_spectrum_topic(1000.0, 5.0, "f32")[2] == 0x1C
    seq, s, ns = g["metadata"]
    assert dsp.serialize_metadata(seq, s, ns).hex() == g["metadata_hex"]


def test_format_tables():
    L = _lib.lib()
    for name, code in oracle64.FORMATS.items():
        assert L.sk_format_bytes(code) == oracle64.bytes_per_sample(code)
        assert L.sk_format_is_complex(code) == int(oracle64.is_complex(code))
    assert L.sk_format_bytes(0x33) < 0


def test_filter_grammar():
    f = dsp.parse_filter_params("fs=64000:fc=80000:file=/tmp/x.bin")
    assert (f.fs_out, f.fc_out, f.output.filename, f.transition) == (64000.0, 80000.0, "/tmp/x.bin", 0)
    f = dsp.parse_filter_params("fc=1e6:fs=2.5e5:tw=28")
    assert (f.fs_out, f.fc_out, f.transition) == (250000.0, 1e6, 28)
    with pytest.raises((ValueError, KeyError)):
        dsp.parse_filter_params("fs=64000")
    with pytest.raises(ValueError):
        dsp.parse_filter_params("fs=64000:fc")
    with pytest.raises(ValueError):
        dsp.parse_filter_params("fs=abc:fc=0")
