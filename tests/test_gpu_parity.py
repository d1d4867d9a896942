"""GPU parity: the CUDA path (through the C ABI) against the oracle.

Bars: relative RMS <= 1e-5 against the FP64 oracle for channel outputs and
f32 spectra; u8/u16 spectrum codes within 1 LSB; bin indices, record counts,
sequence numbers and sample counts exact.  Plain and batched execution must
agree bit for bit (same kernels, different scheduling).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from oracle import oracle32, oracle64
from oracle.oracle64 import rel_rms
from spektri_b200 import Plan, workloads
from spektri_b200._lib import SK_ERR_FILTER, SK_ERR_UNSUPPORTED, SpektriError

TOL = 1e-5


def _o64(plan, fmt, chans_w=None):
    chans = []
    for i, c in enumerate(plan.channels):
        w = plan.get_weights(i).astype(np.complex128) if chans_w is None else chans_w[i]
        chans.append(oracle64.Channel(c["bins"], c["first"], w))
    return oracle64.Oracle64(fmt, plan.fft_size, plan.ffts_per_buf, plan.averages, chans)


def make_plan(fs, N, fmt, filters, B, averages, spec="f32", mode="batched", fc=0.0):
    return Plan(fs, N, fmt, filters, fc_in=fc, ffts_per_buf=B, averages=averages, spectrum_format=spec, mode=mode)


def run_compare(plan, fmt, raws, o64=None, tol=TOL, check_o32=None):
    o64 = o64 or _o64(plan, fmt)
    worst = 0.0
    for raw in raws:
        sp, outs = plan.process(raw)
        sp64, outs64 = o64.process(raw)
        assert [s for s, _ in sp] == [s for s, _ in sp64]
        for (_, a), (_, r) in zip(sp, sp64):
            if plan.spectrum_format == 2:
                e = rel_rms(a, r)
                worst = max(worst, e)
                assert e < tol, e
            else:
                q = oracle64.quantize(10 * np.log10(r), "u8" if plan.spectrum_format == 0 else "u16")
                assert np.max(np.abs(a.astype(np.int64) - q.astype(np.int64))) <= 1
        for c, (a, r) in enumerate(zip(outs, outs64)):
            assert a.shape == r.shape
            e = rel_rms(a, r)
            worst = max(worst, e)
            assert e < tol, (c, plan.channels[c], e)
        if check_o32 is not None:
            sp32, outs32 = check_o32.process(raw)
            for a, r in zip(outs, outs32):
                assert rel_rms(a, r) < 2 * tol
    return worst


def test_c1_plain_small_vs_oracles():
    w = workloads.c1()
    nbuf = 12
    raw = workloads.stream_numpy(w, 0, nbuf * w.samples_per_buffer)
    raws = np.split(raw.view(np.uint8), nbuf)
    for mode in ("plain", "batched"):
        plan = make_plan(w.fs, w.fft_size, w.fmt, w.filters(), w.ffts_per_buf, w.averages, mode=mode)
        assert [c["bins"] for c in plan.channels] == [256] * 4
        o32 = oracle32.Oracle32(w.fs, w.fc, w.fft_size, w.ffts_per_buf, w.averages, w.fmt, w.filters())
        assert [(c["bins"], c["first"]) for c in plan.channels] == o32.channels
        worst = run_compare(plan, w.fmt, raws, check_o32=o32)
        print(f"c1 {mode}: worst rel rms {worst:.2e}")


@pytest.mark.parametrize("fmt", sorted(oracle64.FORMATS))
def test_all_formats_small(fmt):
    rng = np.random.default_rng(oracle64.fmt_code(fmt))
    N, B, avg = 1024, 6, 4
    cplx = oracle64.is_complex(fmt)
    chans = [(64, 100), (128, -300 if cplx else 260), (32, 480), (256, 8), (4, 14), (1024, 512), (16, -8)]
    filters = [dict(fs_out=1000.0 * n, fc_out=1000.0 * (first + n // 2)) for n, first in chans]
    plan = make_plan(1024e3, N, fmt, filters, B, avg)
    assert plan.n_channels == len(chans)
    from tests.test_oracle import _stream
    raws = [_stream(fmt, plan.new_samples, rng) for _ in range(5)]
    run_compare(plan, fmt, raws)


@pytest.mark.parametrize("fmt,N", [("s16le", 32768), ("s16le", 65536), ("cs16le", 4096),
                                   ("cs16le", 16384), ("cs16le", 65536), ("s16le", 8192), ("s16le", 16),
                                   ("cs16le", 1 << 17), ("s16le", 1 << 18), ("cs16le", 1 << 20), ("s16le", 1 << 22),
                                   ("s16le", 12288), ("s16le", 49152), ("s16le", 98304), ("cs16le", 12288),
                                   ("cs16le", 49152), ("cs16le", 98304), ("s16le", 20480), ("cs16le", 81920),
                                   ("cs16le", 48), ("s16le", 6144)])
def test_fft_sizes_and_split_paths(fmt, N):
    """Single-tile FFTs, the fused residue split (Nc = R1 * 8192, R1 = 2..8),
    the two-pass column/row FFT (R1 = 16..256, up to 2^20 complex and 2^22
    real points), the smallest size, and forward sizes 3 * 2^k and 5 * 2^k
    (the reference takes any --fftsize, main.rs:43-44, multifft.rs:25-30):
    a mixed-radix column pass (R1 = 3, 5, 6, 10, 12) and rows of M <= 8192."""
    rng = np.random.default_rng(N)
    B = 4 if N <= 1 << 17 else 2
    fs = float(N) * 1000.0
    cplx = fmt.startswith("c")
    ns = [n for n in (4, 64, 512, 2048, 8192) if n <= max(4, N // 2)]
    filters = []
    for n in ns:
        centre = 4 * int(rng.integers(-N // 8, N // 8)) if cplx else 4 * int(rng.integers(0, N // 8 + 1))
        filters.append(dict(fs_out=1000.0 * n, fc_out=1000.0 * centre))
    plan = make_plan(fs, N, fmt, filters, B, 3)
    from tests.test_oracle import _stream
    raws = [_stream(fmt, plan.new_samples, rng) for _ in range(3)]
    run_compare(plan, fmt, raws)


@pytest.mark.parametrize("spec", ["u8", "u16"])
def test_quantised_spectra(spec):
    w = workloads.c1()
    raw = workloads.stream_numpy(w, 0, 8 * w.samples_per_buffer).view(np.uint8)
    plan = make_plan(w.fs, w.fft_size, w.fmt, w.filters(), w.ffts_per_buf, 16, spec=spec)
    run_compare(plan, w.fmt, np.split(raw, 8))


def test_edge_channels_wrap_mirror_and_drops():
    """Channels across bin 0 and across Nyquist (conjugate mirror), wider than
    half the spectrum, smallest and largest sizes; inexact and unsupported
    filters are dropped with their status (fcfb.rs:58-61)."""
    N, B = 4096, 4
    fs = 4.096e6
    filters = [
        dict(fs_out=256e3, fc_out=0.0),                 # centred on bin 0: wraps to negative bins
        dict(fs_out=512e3, fc_out=2048e3),              # centred on Nyquist: mirrored bins
        dict(fs_out=8192e3, fc_out=1000e3),             # n = 8192 > N: wraps more than once
        dict(fs_out=4e3, fc_out=100e3),                 # n = 4
        dict(fs_out=64e3, fc_out=1001e3),               # centre not a multiple of 4: dropped
        dict(fs_out=48e3, fc_out=0.0),                  # n = 48: not a power of two (chirp-z)
        dict(fs_out=-4e3, fc_out=0.0),                  # bins <= 0: dropped
        dict(fs_out=9368e3, fc_out=0.0),                # n = 9368: beyond the device's chirp-z sizes
    ]
    plan = make_plan(fs, N, "s16le", filters, B, 5)
    assert plan.filter_status[:4] == [0, 0, 0, 0] and plan.filter_status[5] == 0
    assert plan.filter_status[4] == SK_ERR_FILTER and plan.filter_status[6] == SK_ERR_FILTER
    assert plan.filter_status[7] == SK_ERR_UNSUPPORTED
    o32 = oracle32.Oracle32(fs, 0.0, N, B, 5, "s16le", filters[:7])
    assert o32.filter_status[4] != 0 and o32.filter_status[6] != 0 and o32.filter_status[5] == 0
    assert [(c["bins"], c["first"]) for c in plan.channels] == [o32.channels[i] for i in (0, 1, 2, 3, 4)]
    rng = np.random.default_rng(11)
    from tests.test_oracle import _stream
    run_compare(plan, "s16le", [_stream("s16le", plan.new_samples, rng) for _ in range(4)])


def test_invalid_parameters_rejected():
    with pytest.raises(SpektriError):
        Plan(1e6, 1024, "s16le", [], ffts_per_buf=3)          # odd fftbuf with real input
    for N in (7 * 1024, 3 * 65536 * 2, 1000):                 # factor 7; complex length beyond 12 * 8192; 5^3
        with pytest.raises(SpektriError) as e:
            Plan(1e6, N, "cs16le", [], ffts_per_buf=2)
        assert e.value.code == SK_ERR_UNSUPPORTED
    with pytest.raises(SpektriError):
        Plan(1e6, 1000, "s16le", [], ffts_per_buf=2)          # 8 * 5^3: not a supported size
    with pytest.raises(SpektriError):
        Plan(1e6, 1 << 23, "s16le", [], ffts_per_buf=2)       # beyond 2^21 complex points
    p = Plan(1e6, 1024, "cs16le", [], ffts_per_buf=3)        # odd is fine for complex input
    assert p.n_channels == 0
    p.process(np.zeros(p.raw_bytes, np.uint8))


def test_c3_shape_plain_equals_batched_and_oracle():
    """The batching configuration (N=65536, 256 channels of 64..8192, B=64):
    two buffers against the FP64 oracle; plain and batched bit-identical."""
    w = workloads.c3()
    x = workloads.stream_torch(w, 2 * w.samples_per_buffer, "cuda").cpu().numpy()
    raws = np.split(x, 2)
    pb = make_plan(w.fs, w.fft_size, w.fmt, w.filters(), w.ffts_per_buf, w.averages, mode="batched")
    pp = make_plan(w.fs, w.fft_size, w.fmt, w.filters(), w.ffts_per_buf, w.averages, mode="plain")
    assert pb.n_channels == 256
    o64 = _o64(pb, w.fmt)
    for r in raws:
        sb, ob = pb.process(r)
        sp, op = pp.process(r)
        s64, o = o64.process(r)
        for a, b in zip(ob, op):
            assert np.array_equal(a, b)
        errs = [rel_rms(a, ref) for a, ref in zip(ob, o)]
        assert max(errs) < TOL, max(errs)


@pytest.mark.parametrize("spec", ["f32", "u8", "u16"])
def test_two_pass_complex_welch_records(spec):
    """Complex input through the two-pass FFT with 16 residue rows (N = 2^17,
    the transposing Welch kernel): 6 blocks per buffer and 4 averages, so
    records complete mid-buffer and the accumulator carries across buffers;
    f32 records within 1e-5 of FP64, u8/u16 codes within 1 LSB, channel
    outputs within 1e-5 (edge channels wrap past bin 0 and N - 1)."""
    N, B = 1 << 17, 6
    fs = N * 1000.0
    filters = [dict(fs_out=1000.0 * n, fc_out=1000.0 * f) for n, f in
               ((256, 0.0), (1024, -65536 + 8), (4096, 12340), (64, 65532))]
    plan = make_plan(fs, N, "cs16le", filters, B, 4, spec=spec)
    assert plan.n_channels == 4
    rng = np.random.default_rng(7)
    from tests.test_oracle import _stream
    run_compare(plan, "cs16le", [_stream("cs16le", plan.new_samples, rng) for _ in range(3)])


def test_c5_shape_complex_channelizer():
    """The large complex channelizer: cs16 input, forward FFT 2^20 (two-pass),
    2048 channels of 64..8192, B = 8 — one buffer against the FP64 oracle,
    spectrum included (64 averages span 8 buffers, so f32 records appear
    from the 8th call; the first call checks the outputs)."""
    w = workloads.c5()
    x = workloads.stream_torch(w, w.samples_per_buffer, "cuda").cpu().numpy()
    plan = make_plan(w.fs, w.fft_size, w.fmt, w.filters(), w.ffts_per_buf, 8)
    assert plan.n_channels == 2048
    o64 = _o64(plan, w.fmt)
    sp, outs = plan.process(x)
    sp64, o = o64.process(x)
    assert [s for s, _ in sp] == [s for s, _ in sp64] == [0]
    assert rel_rms(sp[0][1], sp64[0][1]) < TOL
    errs = [rel_rms(a, ref) for a, ref in zip(outs, o)]
    assert max(errs) < TOL, max(errs)


def test_device_path_matches_host_path():
    w = workloads.c1()
    raw = workloads.stream_numpy(w, 0, 3 * w.samples_per_buffer).view(np.uint8)
    ph = make_plan(w.fs, w.fft_size, w.fmt, w.filters(), w.ffts_per_buf, 8)
    pd = make_plan(w.fs, w.fft_size, w.fmt, w.filters(), w.ffts_per_buf, 8)
    for r in np.split(raw, 3):
        sh, oh = ph.process(r)
        rd = torch.from_numpy(r.copy()).cuda()
        outs = [torch.empty(c["out_samples"], dtype=torch.complex64, device="cuda") for c in pd.channels]
        spec = torch.empty(pd.max_spectra * pd.spectrum_bytes, dtype=torch.uint8, device="cuda")
        res = pd.process_device(rd, outs, spec)
        torch.cuda.synchronize()
        assert res.n_spectra == len(sh)
        for a, b in zip(oh, outs):
            assert np.array_equal(a, b.cpu().numpy())
        if sh:
            s = pd.split_spectra(spec.cpu().numpy(), res)
            for (q1, a), (q2, b) in zip(sh, s):
                assert q1 == q2 and np.array_equal(a, b)


@pytest.mark.parametrize("shape", [(8192, 256, 1), (8192, 512, 1), (8192, 512, 2), (4096, 256, 1), (4096, 256, 3)])
@pytest.mark.parametrize("mode", ["batched", "plain"])
def test_tile_shapes_against_oracle(shape, mode):
    """Every filter-bank tile shape the autotuner may pick meets the bar, for
    every IFFT size 4..8192 (radix plans differ between the shapes; 4096-point
    tiles run n = 8192 as two halves)."""
    N, B = 4096, 4
    sizes = [4, 8, 16, 32, 64, 128, 256, 512, 1024, 2048, 4096, 8192]
    filters = [dict(fs_out=1000.0 * n, fc_out=1000.0 * 4 * (37 * i + 5)) for i, n in enumerate(sizes)]
    plan = make_plan(N * 1000.0, N, "s16le", filters, B, 3, mode=mode)
    plan.set_tuning(*shape)
    assert plan.tuning() == shape
    rng = np.random.default_rng(21)
    from tests.test_oracle import _stream
    run_compare(plan, "s16le", [_stream("s16le", plan.new_samples, rng) for _ in range(3)])


def test_autotune_picks_and_caches(tmp_path):
    w = workloads.c1()
    plan = make_plan(w.fs, w.fft_size, w.fmt, w.filters(), w.ffts_per_buf, w.averages)
    cache = tmp_path / "tune.jsonl"
    t1 = plan.autotune(str(cache))
    assert t1[:2] in ((8192, 256), (8192, 512), (4096, 256)) and t1[2] >= 1 and t1[3] > 0
    lines = cache.read_text().splitlines()
    assert len(lines) == 1 and '"tile_size"' in lines[0]
    plan2 = make_plan(w.fs, w.fft_size, w.fmt, w.filters(), w.ffts_per_buf, w.averages)
    assert plan2.autotune(str(cache))[:3] == t1[:3]              # read back, not re-measured
    assert len(cache.read_text().splitlines()) == 1
    raw = workloads.stream_numpy(w, 0, 2 * w.samples_per_buffer).view(np.uint8)
    run_compare(plan2, w.fmt, np.split(raw, 2))


def test_graph_replay_matches_direct_launches():
    """Batched calls replay a captured CUDA graph (per-call kernel arguments
    patched in); with stage timing on the same plan launches directly.
    Switching back and forth mid-stream must give bit-identical outputs,
    spectra and carry state, across different output buffers."""
    w = workloads.c1()
    nb = 6
    raw = workloads.stream_numpy(w, 0, nb * w.samples_per_buffer).view(np.uint8)
    raws = np.split(raw, nb)
    ref = make_plan(w.fs, w.fft_size, w.fmt, w.filters(), w.ffts_per_buf, 16)
    mix = make_plan(w.fs, w.fft_size, w.fmt, w.filters(), w.ffts_per_buf, 16)
    for i, r in enumerate(raws):
        mix.set_timing(i % 3 == 1)
        sr, orf = ref.process(r)
        sm, om = mix.process(r)
        assert [s for s, _ in sr] == [s for s, _ in sm]
        for (_, a), (_, b) in zip(sr, sm):
            assert np.array_equal(a, b)
        for a, b in zip(orf, om):
            assert np.array_equal(a, b)
        # device path with fresh output tensors each call (the graph reads the table)
        outs = [torch.empty(c["out_samples"], dtype=torch.complex64, device="cuda") for c in mix.channels]
        spec = torch.empty(mix.max_spectra * mix.spectrum_bytes, dtype=torch.uint8, device="cuda")
        rd = torch.from_numpy(r.copy()).cuda()
        r1 = ref.process_device(rd, outs, spec)
        outs2 = [torch.empty_like(o) for o in outs]
        spec2 = torch.empty_like(spec)
        r2 = mix.process_device(rd, outs2, spec2)
        torch.cuda.synchronize()
        assert r1.n_spectra == r2.n_spectra
        for a, b in zip(outs, outs2):
            assert torch.equal(a, b)
    mix.set_timing(False)


@pytest.mark.parametrize("wl", ["c3", "c4", "c5"])
def test_dependent_launches_repeatable(wl):
    """In the batched graph every kernel after the first is a programmatic
    dependent launch: its CTAs start as the previous kernel's CTAs exit, claim
    tiles and stage metadata, and wait on the device for that kernel's writes;
    the forward kernel zeroes the tile cursors.  Over a dozen calls (two-pass
    forward FFTs, real and complex input) the graph's channel outputs and
    spectra must equal bit for bit those of the same plan launching stage by
    stage with stage timing on."""
    w = workloads.WORKLOADS[wl]()
    nb = 12
    stream = workloads.stream_torch(w, nb * w.samples_per_buffer, "cuda:0")
    rb = w.samples_per_buffer * w.bytes_per_sample
    plans = [Plan(w.fs, w.fft_size, w.fmt, w.filters(), fc_in=w.fc, ffts_per_buf=w.ffts_per_buf,
                  averages=w.averages, spectrum_format="f32", mode="batched") for _ in range(2)]
    plans[1].set_timing(True)
    bufs = [([torch.empty(c["out_samples"], dtype=torch.complex64, device="cuda") for c in p.channels],
             torch.empty(p.max_spectra * p.spectrum_bytes, dtype=torch.uint8, device="cuda")) for p in plans]
    for i in range(nb):
        raw = stream[i * rb:(i + 1) * rb]
        r = [p.process_device(raw, o, sp) for p, (o, sp) in zip(plans, bufs)]
        torch.cuda.synchronize()
        assert r[0].n_spectra == r[1].n_spectra
        n = r[0].n_spectra * plans[0].spectrum_bytes
        assert torch.equal(bufs[0][1][:n], bufs[1][1][:n])
        for a, b in zip(bufs[0][0], bufs[1][0]):
            assert torch.equal(a, b), i
    plans[1].set_timing(False)


def test_outputs_stay_inside_their_buffers():
    """Channel outputs are packed into one tensor with sentinel gaps between
    them; after processing every gap still holds its sentinel (n = 4 keeps
    no samples at all, fcfb.rs:177)."""
    N, B = 1024, 4
    sizes = [4, 8, 16, 64, 1024, 4, 8192]
    filters = [dict(fs_out=1000.0 * n, fc_out=1000.0 * 4 * (i + 3)) for i, n in enumerate(sizes)]
    for mode in ("batched", "plain"):
        plan = make_plan(1024e3, N, "s16le", filters, B, 3, mode=mode)
        assert plan.n_channels == len(sizes)
        assert [c["out_samples"] for c in plan.channels] == [B * (n // 8 * 6) for n in sizes]
        gap = 256
        total = sum(c["out_samples"] for c in plan.channels) + gap * (len(sizes) + 1)
        big = torch.full((total,), complex(12345.0, -6789.0), dtype=torch.complex64, device="cuda")
        outs, gaps, o = [], [], gap
        gaps.append((0, gap))
        for c in plan.channels:
            outs.append(big[o:o + c["out_samples"]])
            o += c["out_samples"]
            gaps.append((o, o + gap))
            o += gap
        spec = torch.empty(plan.max_spectra * plan.spectrum_bytes + 4096, dtype=torch.uint8, device="cuda")
        spec[plan.max_spectra * plan.spectrum_bytes:] = 77
        rng = np.random.default_rng(1)
        for _ in range(3):
            raw = torch.from_numpy(np.clip(rng.normal(0, 3000, plan.new_samples), -32768, 32767).astype("<i2").view(np.uint8)).cuda()
            plan.process_device(raw, outs, spec)
        torch.cuda.synchronize()
        for a, b in gaps:
            assert torch.all(big[a:b] == complex(12345.0, -6789.0)), (mode, a, b)
        assert torch.all(spec[plan.max_spectra * plan.spectrum_bytes:] == 77)


def test_weights_update_and_custom_complex_weights():
    w = workloads.c1()
    raw = workloads.stream_numpy(w, 0, 2 * w.samples_per_buffer).view(np.uint8)
    rng = np.random.default_rng(9)
    cw = [(rng.standard_normal(256) + 1j * rng.standard_normal(256)).astype(np.complex64) for _ in w.channels]
    filt = [dict(f, weights=cw[i]) for i, f in enumerate(w.filters())]
    plan = make_plan(w.fs, w.fft_size, w.fmt, filt, w.ffts_per_buf, 64)
    for i in range(plan.n_channels):
        assert np.array_equal(plan.get_weights(i), cw[i])
    o64 = _o64(plan, w.fmt, [c.astype(np.complex128) for c in cw])
    r0, r1 = np.split(raw, 2)
    run_compare(plan, w.fmt, [r0], o64=o64)
    new = (rng.standard_normal(256) + 1j * rng.standard_normal(256)).astype(np.complex64)
    plan.set_weights(2, new)
    o64.channels[2].weights = new.astype(np.complex128)
    run_compare(plan, w.fmt, [r1], o64=o64)


def test_time_shards_on_plans_reproduce_one_plan():
    """The multi-GPU split (spektri_b200.shard) run with one Plan per shard on
    this GPU, one after another: three shards of an 11-buffer stream, each
    primed with the raw samples before it, give, concatenated in shard order,
    the channel records and spectrum records (sequence numbers offset per
    shard) of one plan over the whole stream, bit for bit."""
    from spektri_b200 import shard
    N, B, avg, nbuf, world = 2048, 4, 8, 11, 3
    filters = [dict(fs_out=1000.0 * n, fc_out=1000.0 * f) for n, f in ((64, 300), (512, 640), (2048, 100))]
    rng = np.random.default_rng(23)
    from tests.test_oracle import _stream
    one = make_plan(N * 1000.0, N, "s16le", filters, B, avg)
    raws = [_stream("s16le", one.new_samples, rng) for _ in range(nbuf)]
    stream = np.concatenate([np.frombuffer(r, np.uint8) for r in raws])
    full = [one.process(r) for r in raws]
    shards = shard.plan_shards(nbuf, world, B, avg)
    offs = shard.spectrum_seq_offsets(shards, B, avg)
    assert [c for _, c in shards] == [4, 4, 3] and offs == [0, 2, 4]
    bps = one.raw_bytes // one.new_samples
    spectra, outs = [], []
    for (first, count), off in zip(shards, offs):
        p = make_plan(N * 1000.0, N, "s16le", filters, B, avg)
        carry = shard.carry_bytes(stream, first, one.new_samples, one.overlap, bps)
        if carry is not None:
            p.set_carry(carry)
        for b in range(first, first + count):
            sp, oc = p.process(raws[b])
            spectra += [(s + off, v) for s, v in sp]
            outs.append(oc)
        p.close()
    assert [s for s, _ in spectra] == [s for f in full for s, _ in f[0]]
    for (_, a), (_, r) in zip(spectra, [x for f in full for x in f[0]]):
        assert np.array_equal(a, r)
    for oc, f in zip(outs, full):
        for a, r in zip(oc, f[1]):
            assert np.array_equal(a, r)


@pytest.mark.parametrize("fmt,mode", [("s16le", "batched"), ("cf32le", "plain"), ("u8", "batched")])
def test_carry_starts_mid_stream(fmt, mode):
    """A plan primed with the N/4 samples before buffer k reproduces, bit for
    bit, what a plan that processed the whole stream emits from buffer k on
    (the time-shard contract): channel records and, at a Welch-window
    boundary, spectrum records (sequence numbers offset by the records before)."""
    from spektri_b200 import shard
    N, B, avg, nbuf = 2048, 4, 8, 8
    cplx = oracle64.is_complex(fmt)
    filters = [dict(fs_out=1000.0 * n, fc_out=1000.0 * f) for n, f in
               ((64, -300 if cplx else 300), (256, 512), (16, 100))]
    plans = [make_plan(N * 1000.0, N, fmt, filters, B, avg, mode=mode) for _ in range(2)]
    p0 = plans[0]
    rng = np.random.default_rng(5)
    from tests.test_oracle import _stream
    raws = [_stream(fmt, p0.new_samples, rng) for _ in range(nbuf)]
    stream = np.concatenate([np.frombuffer(r, np.uint8) for r in raws])
    full = [p0.process(r) for r in raws]
    bps = p0.raw_bytes // p0.new_samples
    for k in (shard.window_buffers(B, avg), 3):
        p1 = make_plan(N * 1000.0, N, fmt, filters, B, avg, mode=mode)
        p1.set_carry(shard.carry_bytes(stream, k, p0.new_samples, p0.overlap, bps))
        seq_off = k * B // avg
        for b in range(k, nbuf):
            sp, outs = p1.process(raws[b])
            for a, r in zip(outs, full[b][1]):
                assert np.array_equal(a, r), (fmt, k, b)
            if k * B % avg == 0:
                assert [s + seq_off for s, _ in sp] == [s for s, _ in full[b][0]]
                for (_, a), (_, r) in zip(sp, full[b][0]):
                    assert np.array_equal(a, r)
    with pytest.raises(ValueError):
        p0.set_carry(np.zeros(3, np.uint8))


CHIRP_SIZES = [12, 20, 28, 36, 100, 300, 1000, 1012, 2340]
CHIRP_SIZES_BIG = [3000, 4036, 4680]                    # chirp-z transforms of 8192 points
CHIRP_SIZES_16K = [4684, 6000, 8188, 9000, 9364]        # 16384 points: their own kernel, any tile shape


@pytest.mark.parametrize("fmt", ["s16le", "cf32le"])
@pytest.mark.parametrize("mode", ["batched", "plain"])
@pytest.mark.parametrize("shape", [(8192, 256, 2), (4096, 256, 4)])
def test_chirp_sizes_against_oracle(fmt, mode, shape):
    """IFFT sizes that are multiples of 4 but not powers of two (the reference
    plans any size, fcfb.rs:150) run as chirp-z transforms; mixed with
    power-of-two channels in one plan, they meet the same bar."""
    N, B = 4096, 4
    cplx = oracle64.is_complex(fmt)
    sizes = CHIRP_SIZES + (CHIRP_SIZES_BIG if shape[0] == 8192 else []) + CHIRP_SIZES_16K + [64, 8192]
    filters = [dict(fs_out=1000.0 * n, fc_out=1000.0 * 4 * ((-1) ** i * (53 * i + 3) if cplx else 53 * i + 3))
               for i, n in enumerate(sizes)]
    plan = make_plan(N * 1000.0, N, fmt, filters, B, 3, mode=mode)
    assert [c["bins"] for c in plan.channels] == sizes
    plan.set_tuning(*shape)
    rng = np.random.default_rng(31)
    from tests.test_oracle import _stream
    worst = run_compare(plan, fmt, [_stream(fmt, plan.new_samples, rng) for _ in range(3)])
    print(f"chirp {fmt} {mode} {shape}: worst rel rms {worst:.2e}")


@pytest.mark.parametrize("fmt", ["s16le", "cs16le"])
@pytest.mark.parametrize("mode", ["batched", "plain"])
@pytest.mark.parametrize("shape", [(8192, 256, 2), (8192, 512, 2), (4096, 256, 4)])
def test_ifft_sizes_beyond_a_tile(fmt, mode, shape):
    """Power-of-two IFFT sizes above the tile size (the reference plans any
    size, fcfb.rs:150): n = P S runs as P independent S-point parts, one per
    output residue mod P, up to P = 8 (n = 2^16 on 8192-point tiles, 2^15 on
    4096-point ones), mixed with small sizes in one plan."""
    N, B = 65536, 4
    cplx = oracle64.is_complex(fmt)
    sizes = [64, 4096, 8192, 16384, 32768] + ([65536] if shape[0] == 8192 else [])
    filters = [dict(fs_out=1000.0 * n, fc_out=1000.0 * 4 * ((-1) ** i * (1789 * i + 5) if cplx else 1789 * i + 5))
               for i, n in enumerate(sizes)]
    plan = make_plan(N * 1000.0, N, fmt, filters, B, 3, mode=mode)
    assert [c["bins"] for c in plan.channels] == sizes
    plan.set_tuning(*shape)
    rng = np.random.default_rng(41)
    from tests.test_oracle import _stream
    worst = run_compare(plan, fmt, [_stream(fmt, plan.new_samples, rng) for _ in range(2)])
    print(f"split sizes {fmt} {mode} {shape}: worst rel rms {worst:.2e}")


def test_split_limits():
    """2^16-point IFFTs need 8 parts of an 8192-point tile: the 4096-point
    shape is refused for such a plan, and sizes above 2^16 are dropped."""
    N = 65536
    filters = [dict(fs_out=1000.0 * n, fc_out=0.0) for n in (65536, 131072, 64)]
    plan = make_plan(N * 1000.0, N, "s16le", filters, 2, 3)
    assert plan.filter_status == [0, SK_ERR_UNSUPPORTED, 0]
    with pytest.raises(SpektriError):
        plan.set_tuning(4096, 256, 1)
    plan.set_tuning(8192, 256, 1)


def test_chirp_limits():
    """Sizes whose chirp-z transform exceeds 16384 points (n > 9364) are
    dropped with a status; a 4096-point tile shape is refused while a plan
    holds a chirp-z size that needs 8192 points, and allowed with the 16384-point
    ones, which run in a kernel of their own."""
    N = 4096
    filters = [dict(fs_out=1000.0 * n, fc_out=0.0) for n in (4680, 9364, 9368, 12)]
    plan = make_plan(N * 1000.0, N, "s16le", filters, 4, 3)
    assert plan.filter_status == [0, 0, SK_ERR_UNSUPPORTED, 0]
    assert [c["bins"] for c in plan.channels] == [4680, 9364, 12]
    with pytest.raises(SpektriError):
        plan.set_tuning(4096, 256, 1)
    plan.set_tuning(8192, 256, 1)
    assert plan.autotune("")[0] == 8192                          # no cache file
    p16 = make_plan(N * 1000.0, N, "s16le", [filters[1], filters[3]], 4, 3)
    p16.set_tuning(4096, 256, 4)


def test_host_outputs_contiguous_and_separate():
    """The host path fills outputs laid out as one block with a single copy and
    separately allocated outputs with one copy each; both give the same bytes."""
    w = workloads.c1()
    raw = workloads.stream_numpy(w, 0, 2 * w.samples_per_buffer).view(np.uint8)
    r0, r1 = np.split(raw, 2)
    pa = make_plan(w.fs, w.fft_size, w.fmt, w.filters(), w.ffts_per_buf, 8)
    pb = make_plan(w.fs, w.fft_size, w.fmt, w.filters(), w.ffts_per_buf, 8)
    for r in (r0, r1):
        _, oa = pa.process(r)                                          # one block
        ob = [np.ascontiguousarray(np.full(c["out_samples"], np.nan, np.complex64)) for c in pb.channels]
        spec = np.empty(pb.max_spectra * pb.spectrum_bytes, np.uint8)
        pb.process_into(r, ob, spec)
        for a, b in zip(oa, ob):
            assert np.array_equal(a, b)
