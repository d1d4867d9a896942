"""Parity at the benchmark configurations, with the reference's exact counts.

- The plain small configuration (N = 4096, B = 8, 4 channels of n = 256,
  64 averages) over its whole 2^22-sample stream, through the drop-in host
  binary: main.rs:162-181 turns it into 170 full buffers (24 576 new samples
  each, 1360 blocks) and drops the last 16 384 samples at the short read;
  spectrum.rs:112-161 emits 21 records from the first 1344 blocks.  Record
  headers (sequence numbers, injected-clock timestamps) equal the oracle CLI's
  byte for byte; payloads are within relative RMS 1e-5 of the FP64 oracle.
- The RX888-like configuration (N = 65536, B = 64, 32 channels of n =
  256..4096, 256 averages) over 4 buffers: the first f32 record completes on
  the 4th buffer; plain and batched execution agree bit for bit.
- The batching configuration (256 channels of n = 64..8192) over 4 buffers,
  one f32 plan and one u8 plan: the averages = 256 record in both formats
  (f32 within 1e-5, u8 within 1 LSB of the FP64 power in dB).
"""
import glob
import os
import subprocess

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from oracle import oracle32, oracle64
from oracle.oracle64 import rel_rms
from spektri_b200 import Plan, workloads

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HOST = os.path.join(ROOT, "spektri_b200", "bin", "spektri")
TOL = 1e-5


def _o64(plan, fmt):
    chans = [oracle64.Channel(c["bins"], c["first"], plan.get_weights(i).astype(np.complex128))
             for i, c in enumerate(plan.channels)]
    return oracle64.Oracle64(fmt, plan.fft_size, plan.ffts_per_buf, plan.averages, chans)


def _libzmq_env():
    """The host binary dlopens libzmq: point it at pyzmq's bundled copy."""
    import zmq
    base = os.path.dirname(os.path.dirname(zmq.__file__))
    cands = glob.glob(os.path.join(base, "pyzmq.libs", "libzmq*.so*")) + \
        glob.glob(os.path.join(os.path.dirname(zmq.__file__), "*libzmq*.so*"))
    return dict(os.environ, SPEKTRI_LIBZMQ=cands[0] if cands else "")


def _records(data, rec_bytes):
    assert len(data) % rec_bytes == 0, (len(data), rec_bytes)
    return [data[i:i + rec_bytes] for i in range(0, len(data), rec_bytes)]


def test_c1_whole_stream_counts_and_parity(tmp_path):
    assert os.path.exists(HOST), "build spektri_b200/bin/spektri first"
    oracle32.build()
    w = workloads.c1()
    assert w.n_samples == 1 << 22
    raw = workloads.stream_numpy(w, 0, w.n_samples)
    infile = tmp_path / "c1.s16"
    raw.tofile(infile)
    per_buf = w.samples_per_buffer
    n_buf, tail = divmod(w.n_samples, per_buf)
    assert (per_buf, n_buf, tail) == (24576, 170, 16384)
    n_blocks = n_buf * w.ffts_per_buf
    n_rec = n_blocks // w.averages
    assert (n_blocks, n_rec, n_rec * w.averages) == (1360, 21, 1344)

    filt = [f"fs={f['fs_out']:.17g}:fc={f['fc_out']:.17g}:tw={f['transition']}" for f in w.filters()]
    common = [f"--samplerate={w.fs:.17g}", "-n", str(w.fft_size), "--fftbuf", str(w.ffts_per_buf),
              f"--averages={w.averages}", "-I", "s16le", "--spectrumformat=f32", "--fake-clock=1700000000,7500000"]

    def run(binary, name):
        d = tmp_path / name
        d.mkdir()
        files = [d / f"c{i}.bin" for i in range(len(filt))]
        args = [binary] + common + ["--zmqbind", f"ipc://{d}/sk.zmq", "--filters"] + \
            [f"{s}:file={p}" for s, p in zip(filt, files)]
        r = subprocess.run(args, stdin=open(infile, "rb"), capture_output=True, timeout=600, env=_libzmq_env())
        assert r.returncode == 0, r.stderr.decode()[-2000:]
        return r.stdout, [p.read_bytes() for p in files]

    out_o, files_o = run(oracle32.CLI, "oracle")
    out_h, files_h = run(HOST, "host")

    # channel records: 170 per filter, seq 0..169, headers equal to the oracle CLI's
    keep = w.ffts_per_buf * (256 // 8 * 6)
    rec = 24 + 8 * keep
    o64 = oracle64.Oracle64(w.fmt, w.fft_size, w.ffts_per_buf, w.averages,
                            [oracle64.Channel(256, oracle32.freq_to_bins(w.fs, w.fc, w.fft_size, f["fs_out"],
                                                                         f["fc_out"], exact=True)[1],
                                              oracle32.tukey(256, f["transition"]).astype(np.complex128))
                             for f in w.filters()])
    recs_h = [_records(f, rec) for f in files_h]
    recs_o = [_records(f, rec) for f in files_o]
    for rh, ro in zip(recs_h, recs_o):
        assert len(rh) == len(ro) == n_buf
        assert [r[:24] for r in rh] == [r[:24] for r in ro]
        assert [int.from_bytes(r[:8], "little") for r in rh] == list(range(n_buf))
    # spectrum records on stdout: 21, f32 K = 2049 bins each
    K = w.fft_size // 2 + 1
    sh = _records(out_h, 24 + 4 * K)
    so = _records(out_o, 24 + 4 * K)
    assert len(sh) == len(so) == n_rec
    assert [r[:24] for r in sh] == [r[:24] for r in so]
    # payloads against FP64, buffer by buffer over the whole stream
    raws = np.split(raw[: n_buf * per_buf].view(np.uint8), n_buf)
    worst = 0.0
    got_spec = []
    for b, r in enumerate(raws):
        sp64, outs64 = o64.process(r)
        got_spec += [p for _, p in sp64]
        for c in range(len(filt)):
            y = np.frombuffer(recs_h[c][b][24:], np.complex64)
            e = rel_rms(y, outs64[c])
            worst = max(worst, e)
            assert e < TOL, (b, c, e)
    assert len(got_spec) == n_rec
    for r, p in zip(sh, got_spec):
        e = rel_rms(np.frombuffer(r[24:], np.float32), p)
        worst = max(worst, e)
        assert e < TOL, e
    print(f"c1 whole stream: {n_buf} buffers, {n_blocks} blocks, {n_rec} records, tail {tail} dropped; "
          f"worst rel rms {worst:.2e}")


def test_c2_rx888_config_against_oracle():
    w = workloads.c2()
    nbuf = w.averages // w.ffts_per_buf                        # 256 / 64 = 4: one record, on the last buffer
    x = workloads.stream_torch(w, nbuf * w.samples_per_buffer, "cuda").cpu().numpy()
    raws = np.split(x, nbuf)
    pb = Plan(w.fs, w.fft_size, w.fmt, w.filters(), fc_in=w.fc, ffts_per_buf=w.ffts_per_buf, averages=w.averages,
              spectrum_format="f32", mode="batched")
    pp = Plan(w.fs, w.fft_size, w.fmt, w.filters(), fc_in=w.fc, ffts_per_buf=w.ffts_per_buf, averages=w.averages,
              spectrum_format="f32", mode="plain")
    assert pb.n_channels == 32
    assert {c["bins"] for c in pb.channels} <= {256, 512, 1024, 2048, 4096}
    o64 = _o64(pb, w.fmt)
    worst = 0.0
    for i, r in enumerate(raws):
        sb, ob = pb.process(r)
        sp, op = pp.process(r)
        s64, o = o64.process(r)
        assert [s for s, _ in sb] == [s for s, _ in sp] == [s for s, _ in s64] == ([0] if i == nbuf - 1 else [])
        for a, b in zip(ob, op):
            assert np.array_equal(a, b)
        for (_, a), (_, ref) in zip(sb, s64):
            e = rel_rms(a, ref)
            worst = max(worst, e)
            assert e < TOL, e
        for c, (a, ref) in enumerate(zip(ob, o)):
            e = rel_rms(a, ref)
            worst = max(worst, e)
            assert e < TOL, (i, c, e)
    print(f"c2: worst rel rms {worst:.2e}")


def test_c3_batching_config_records_f32_and_u8():
    w = workloads.c3()
    nbuf = w.averages // w.ffts_per_buf
    x = workloads.stream_torch(w, nbuf * w.samples_per_buffer, "cuda").cpu().numpy()
    raws = np.split(x, nbuf)
    pf = Plan(w.fs, w.fft_size, w.fmt, w.filters(), fc_in=w.fc, ffts_per_buf=w.ffts_per_buf, averages=w.averages,
              spectrum_format="f32", mode="batched")
    pu = Plan(w.fs, w.fft_size, w.fmt, w.filters(), fc_in=w.fc, ffts_per_buf=w.ffts_per_buf, averages=w.averages,
              spectrum_format="u8", mode="batched")
    assert pf.n_channels == 256
    o64 = _o64(pf, w.fmt)
    worst = 0.0
    for i, r in enumerate(raws):
        sf, of = pf.process(r)
        su, ou = pu.process(r)
        s64, o = o64.process(r)
        want = [0] if i == nbuf - 1 else []
        assert [s for s, _ in sf] == [s for s, _ in su] == [s for s, _ in s64] == want
        for a, b in zip(of, ou):
            assert np.array_equal(a, b)
        for (_, a), (_, q), (_, ref) in zip(sf, su, s64):
            e = rel_rms(a, ref)
            worst = max(worst, e)
            assert e < TOL, e
            codes = oracle64.quantize(10 * np.log10(ref), "u8")
            assert np.max(np.abs(q.astype(np.int64) - codes.astype(np.int64))) <= 1
        errs = [rel_rms(a, ref) for a, ref in zip(of, o)]
        worst = max(worst, max(errs))
        assert max(errs) < TOL, (i, int(np.argmax(errs)), max(errs))
    print(f"c3: worst rel rms {worst:.2e}")
