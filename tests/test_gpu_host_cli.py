"""The drop-in host binary (spektri_b200/bin/spektri) against the oracle's
restatement of the reference main loop (oracle/_build/spektri_oracle).

Same command line and stdin on both; with --fake-clock the record headers
(seq, seconds, nanoseconds) must match byte for byte, the per-filter files and
the spectrum records on stdout must have the same framing, sample payloads
within relative RMS 1e-5, u8 spectrum codes within 1 LSB.  The ZeroMQ PUB
socket must carry (topic, record) pairs whose topics are the reference's
serialize_signal_topic / serialize_spectrum_topic bytes (data.rs:137-171,
tools/spektri.py:15-36) and whose records equal the file records.
"""
import glob
import json
import os
import subprocess
import threading
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from oracle import oracle32
from oracle.oracle64 import rel_rms
from spektri_b200 import workloads

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HOST = os.path.join(ROOT, "spektri_b200", "bin", "spektri")


def libzmq_path():
    import zmq
    base = os.path.dirname(os.path.dirname(zmq.__file__))
    cands = glob.glob(os.path.join(base, "pyzmq.libs", "libzmq*.so*")) + glob.glob(os.path.join(os.path.dirname(zmq.__file__), "*libzmq*.so*"))
    return cands[0] if cands else None


def split_records(data, payload_bytes):
    rec = 24 + payload_bytes
    assert len(data) % rec == 0, (len(data), rec)
    return [(data[i:i + 24], data[i + 24:i + rec]) for i in range(0, len(data), rec)]


def test_host_binary_matches_oracle_cli_and_publishes_zmq(tmp_path):
    import zmq
    assert os.path.exists(HOST), "build spektri_b200/bin/spektri first"
    oracle32.build()
    w = workloads.c1()
    nbuf = 10
    raw = workloads.stream_numpy(w, 0, nbuf * w.samples_per_buffer + 1000)      # + a short tail that is dropped
    infile = tmp_path / "in.s16"
    raw.tofile(infile)
    filt = [f"fs={f['fs_out']:.17g}:fc={f['fc_out']:.17g}" for f in w.filters()]
    common = [f"--samplerate={w.fs:.17g}", "-n", str(w.fft_size), "--fftbuf", str(w.ffts_per_buf), "--averages=16",
              "-I", "s16le", "--spectrumformat=u8", "--fake-clock=1700000000,123456789"]
    addr = f"ipc://{tmp_path}/sk.zmq"

    def run(binary, outdir):
        outdir.mkdir()
        files = [outdir / f"c{i}.bin" for i in range(len(filt))]
        fl = [f"{s}:file={p}" for s, p in zip(filt, files)] + ["fs=64000:fc=1001"]   # last one is invalid
        args = [binary] + common + ["--filters"] + fl + ["--zmqbind", addr]
        return args, files

    # oracle CLI
    args_o, files_o = run(oracle32.CLI, tmp_path / "oracle")
    ro = subprocess.run(args_o, stdin=open(infile, "rb"), capture_output=True, timeout=300)
    assert ro.returncode == 0, ro.stderr

    # device host binary, with a ZeroMQ subscriber
    args_h, files_h = run(HOST, tmp_path / "host")
    env = dict(os.environ, SPEKTRI_LIBZMQ=libzmq_path() or "")
    ctx = zmq.Context()
    sub = ctx.socket(zmq.SUB)
    sub.setsockopt(zmq.SUBSCRIBE, b"")
    sub.setsockopt(zmq.RCVHWM, 100000)
    sub.connect(addr)
    msgs = []
    stop = threading.Event()

    def recv():
        while not stop.is_set():
            if sub.poll(100):
                msgs.append(sub.recv_multipart())

    th = threading.Thread(target=recv, daemon=True)
    th.start()
    p = subprocess.Popen(args_h, stdin=subprocess.PIPE, stdout=subprocess.PIPE, stderr=subprocess.PIPE, env=env)
    time.sleep(1.5)                                  # bind + subscription before the first record
    out, err = p.communicate(open(infile, "rb").read(), timeout=300)
    time.sleep(0.5)
    stop.set()
    th.join()
    sub.close()
    ctx.term()
    assert p.returncode == 0, err
    assert b"Invalid filter parameters" in err and b"Invalid filter parameters" in ro.stderr

    # per-filter files: framing exact, payload within tolerance
    for fo, fh, f in zip(files_o, files_h, w.filters()):
        n = int(round(f["fs_out"] / w.spacing))
        pb = w.ffts_per_buf * (n // 8 * 6) * 8
        ro_recs = split_records(fo.read_bytes(), pb)
        rh_recs = split_records(fh.read_bytes(), pb)
        assert len(ro_recs) == len(rh_recs) == nbuf
        for (ho, po), (hh, ph) in zip(ro_recs, rh_recs):
            assert ho == hh
            assert rel_rms(np.frombuffer(ph, np.complex64), np.frombuffer(po, np.complex64)) < 1e-5
    # spectrum records on stdout
    K = w.fft_size // 2 + 1
    so = split_records(ro.stdout, K)
    sh = split_records(out, K)
    assert len(so) == len(sh) == nbuf * w.ffts_per_buf // 16
    for (ho, po), (hh, ph) in zip(so, sh):
        assert ho == hh
        assert np.max(np.abs(np.frombuffer(po, np.uint8).astype(int) - np.frombuffer(ph, np.uint8).astype(int))) <= 1

    # ZeroMQ: topics from the reference's wire format, bodies equal to the records
    golden = json.load(open(os.path.join(ROOT, "tests", "golden", "wire_topics.json")))
    from spektri_b200 import dsp
    sig_topics = {dsp.serialize_signal_topic(f["fs_out"], f["fc_out"]): i for i, f in enumerate(w.filters())}
    spec_topic = dsp.serialize_spectrum_topic(w.spacing, w.fc, "u8")
    assert spec_topic[:8].hex() == golden["spectrum_topic_prefix_hex"]
    got_sig = {i: [] for i in range(len(filt))}
    got_spec = []
    for m in msgs:
        assert len(m) == 2 and len(m[0]) == 24
        if m[0] == spec_topic:
            got_spec.append(m[1])
        else:
            got_sig[sig_topics[m[0]]].append(m[1])
    assert got_spec == [h + p for h, p in sh]
    for i, fh in enumerate(files_h):
        pb = len(fh.read_bytes()) // nbuf
        recs = [fh.read_bytes()[k * pb:(k + 1) * pb] for k in range(nbuf)]
        assert got_sig[i] == recs
        seqs = [int.from_bytes(r[:8], "little") for r in got_sig[i]]
        assert seqs == list(range(nbuf))                      # contiguous, like test/zmq_rx.py checks


def test_host_binary_error_behaviour(tmp_path):
    env = dict(os.environ, SPEKTRI_LIBZMQ=libzmq_path() or "")
    addr = f"--zmqbind=ipc://{tmp_path}/e.zmq"
    r = subprocess.run([HOST, "-I", "s16le", addr], capture_output=True, env=env, timeout=60)
    assert r.returncode == 1 and b"samplerate" in r.stderr                  # clap: required argument
    r = subprocess.run([HOST, "-s", "1e6", "-I", "s17le", addr], capture_output=True, env=env, timeout=60)
    assert r.returncode == 1                                                 # clap: invalid value
    r = subprocess.run([HOST, "-s", "1e6", "-I", "s16le", "--filters", "fs=1000", addr], capture_output=True,
                       env=env, timeout=60)
    assert r.returncode == 101                                               # main.rs:85-86 unwrap panics
    r = subprocess.run([HOST, "-s", "1e6", "-I", "s16le", "--fftbuf", "3", addr], input=b"", capture_output=True,
                       env=env, timeout=60)
    assert r.returncode != 0                                                 # odd fftbuf (multifft.rs:57-61)
    # empty stdin: clean exit, no output
    r = subprocess.run([HOST, "-s", "1024000", "-n", "1024", "-I", "s16le", addr], input=b"", capture_output=True,
                       env=env, timeout=120)
    assert r.returncode == 0 and r.stdout == b""


def test_host_binary_streams_c3(tmp_path):
    """The pipelined binary on the batching configuration (N = 65536, 256
    channels, B = 64): stdin, GPU call and output overlap; every buffer's
    spectrum records arrive on stdout and the run's throughput is printed
    (two stream lengths, so start-up cancels)."""
    assert os.path.exists(HOST), "build spektri_b200/bin/spektri first"
    w = workloads.c3()
    filt = [f"fs={f['fs_out']:.17g}:fc={f['fc_out']:.17g}:tw={f.get('transition', 0)}" for f in w.filters()]
    args = [HOST, f"--samplerate={w.fs:.17g}", f"--centerfreq={w.fc:.17g}", "-n", str(w.fft_size), "--fftbuf",
            str(w.ffts_per_buf), f"--averages={w.averages}", "-I", "s16le", "--spectrumformat=u8",
            f"--zmqbind=ipc://{tmp_path}/sk.zmq", "--filters"] + filt
    env = dict(os.environ, SPEKTRI_LIBZMQ=libzmq_path())         # a PUB socket with no subscriber
    times = {}
    rng = np.random.default_rng(3)
    for nbuf in (4, 20):
        raw = rng.integers(-3000, 3000, nbuf * w.samples_per_buffer, dtype=np.int16)
        infile = tmp_path / f"in{nbuf}.s16"
        raw.tofile(infile)
        t0 = time.perf_counter()
        with open(infile, "rb") as fin:
            r = subprocess.run(args, stdin=fin, stdout=subprocess.PIPE, stderr=subprocess.PIPE, env=env, timeout=600)
        times[nbuf] = time.perf_counter() - t0
        assert r.returncode == 0, r.stderr.decode()[-2000:]
        n_spec = nbuf * w.ffts_per_buf // w.averages
        assert len(r.stdout) == n_spec * (24 + w.fft_size // 2 + 1)
    per_buf = (times[20] - times[4]) / 16
    print(f"host binary, C3: {w.samples_per_buffer / per_buf / 1e6:.1f} Msamples/s "
          f"({per_buf * 1e3:.2f} ms per buffer of {w.samples_per_buffer} samples)")


def test_sweep_through_host_binary(tmp_path):
    """The reference's integration stimulus (test/test_spectrum.sh:7-16): the
    testsignal sweep piped into the drop-in binary and into the oracle CLI.
    Same record headers, u8 spectra within 1 LSB, channel records within
    relative RMS 1e-5, and the spectral peak walks up the band record by
    record as the sweep does (-pi to pi rad/sample over the run)."""
    oracle32.build()
    tsig = os.path.join(ROOT, "spektri_b200", "bin", "testsignal")
    N, B, avg, n = 4096, 8, 8, 1 << 20
    sig = subprocess.run([tsig, "-f", "cf32le", "-n", str(n)], capture_output=True, timeout=120, check=True).stdout
    infile = tmp_path / "sweep.cf32"
    infile.write_bytes(sig)
    fs = 4.096e6
    common = [f"--samplerate={fs:.17g}", "-n", str(N), "--fftbuf", str(B), f"--averages={avg}", "-I", "cf32le",
              "--spectrumformat=u8", "--fake-clock=1700000000,1000000"]
    env = dict(os.environ, SPEKTRI_LIBZMQ=libzmq_path() or "")

    def run(binary, name):
        d = tmp_path / name
        d.mkdir()
        f = d / "ch.bin"
        args = [binary] + common + ["--zmqbind", f"ipc://{d}/sk.zmq", "--filters", f"fs=256000:fc=-1024000:file={f}"]
        r = subprocess.run(args, stdin=open(infile, "rb"), capture_output=True, timeout=300, env=env)
        assert r.returncode == 0, r.stderr.decode()[-2000:]
        return r.stdout, f.read_bytes()

    out_o, ch_o = run(oracle32.CLI, "oracle")
    out_h, ch_h = run(HOST, "host")
    so, sh = split_records(out_o, N), split_records(out_h, N)
    assert len(so) == len(sh) == (n // (3 * N // 4 * B)) * B // avg
    peaks = []
    for (ho, po), (hh, ph) in zip(so, sh):
        assert ho == hh
        a, b = np.frombuffer(po, np.uint8).astype(int), np.frombuffer(ph, np.uint8).astype(int)
        assert np.max(np.abs(a - b)) <= 1
        k = int(np.argmax(b))
        peaks.append(k if k < N // 2 else k - N)               # signed bin: -N/2 .. N/2
    steps = np.diff(np.array(peaks))
    assert np.mean(steps > 0) > 0.9, peaks                     # the sweep rises through the band
    keep = B * 256 // 8 * 6 * 8
    ro, rh = split_records(ch_o, keep), split_records(ch_h, keep)
    assert len(ro) == len(rh) and [h for h, _ in ro] == [h for h, _ in rh]
    # over the whole run (the sweep crosses the channel once; elsewhere the
    # channel holds only leakage, where both FP32 paths differ by rounding)
    yo = np.concatenate([np.frombuffer(p, np.complex64) for _, p in ro])
    yh = np.concatenate([np.frombuffer(p, np.complex64) for _, p in rh])
    assert rel_rms(yh, yo) < 1e-5
