"""The allocation-free spectra entry point (sk_spectra_noalloc) against the
FP64 oracle and the plan-based one (sk_spectra_device).

sk_spectra_noalloc exists for callers that may not allocate device memory:
real-time receive callbacks that cannot afford a cudaMalloc stall, and hosts
whose own memory pool owns the device.  It keeps its scratch in a static
device array, so these checks cover: the same spectra as the FP64 oracle and
the plan path (relative RMS <= 1e-5) on two calls in a row, whose second call
finds the first call's data still in the shared array; no change in free device
memory across calls; and a clear refusal of sizes beyond the array.

This file is collected last so that a failure here leaves every other test
already run.
"""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from oracle import oracle64
from spektri_b200 import Plan
from spektri_b200._lib import SK_ERR_ARG, SK_OK, last_error, lib

TOL = 1e-5
FMT = {"s16le": 0x08, "cs16le": 0x48, "f32le": 0x1C, "u8": 0x24}


def _rel(a, b):
    return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))


def _raw(rng, fmt, count):
    """count samples (components) of raw input in the format's own dtype."""
    if fmt == "f32le":
        return rng.normal(0, 3000, count).astype("<f4")
    if fmt == "u8":
        return rng.integers(0, 256, count).astype(np.uint8)
    return np.clip(np.round(rng.normal(0, 4000, count)), -32768, 32767).astype("<i2")


# Small N (Nc = 4 and 8, the smallest whole-block tile instances), odd block
# counts (real input: the plan path needs an even count, so those compare with
# the FP64 oracle alone), 32-bit and 8-bit formats, and the large sizes.
@pytest.mark.parametrize("fmt,N,B", [("s16le", 4096, 8), ("s16le", 65536, 8), ("cs16le", 16384, 4),
                                     ("cs16le", 65536, 2), ("s16le", 8, 3), ("cs16le", 16, 5), ("f32le", 1024, 6),
                                     ("u8", 256, 4)])
def test_noalloc_matches_oracle_and_plan_on_two_calls_in_a_row(fmt, N, B):
    """Two calls in a row, each window = [N/4 samples carried | 3N/4 * B new]:
    the spectra equal the FP64 oracle's (relative RMS <= 1e-5) and, where a
    plan can be made, the plan path's.  A priming buffer comes first so that
    every window's carried samples are real input (for u8 the reference's
    initial zeros are not a raw byte value)."""
    L = lib()
    cplx = fmt.startswith("c")
    comp = 2 if cplx else 1
    K = N if cplx else N // 2 + 1
    overlap, new = N // 4, (N - N // 4) * B
    rng = np.random.default_rng(N + B)
    bufs = [_raw(rng, fmt, new * comp) for _ in range(3)]
    o64 = oracle64.Oracle64(fmt, N, B, 10**9, [])
    o64.spectra_of(bufs[0].view(np.uint8))
    plan = None
    if cplx or B % 2 == 0:
        plan = Plan(N * 1000.0, N, fmt, [], ffts_per_buf=B, averages=10**6, spectrum_format="f32")
        assert plan.result_bins == K
    stream = torch.cuda.current_stream()
    x_ref = torch.empty(B, K, dtype=torch.complex64, device="cuda")
    x_new = torch.empty(B, K, dtype=torch.complex64, device="cuda")
    dev_new = [torch.from_numpy(b.view(np.uint8).copy()).cuda() for b in bufs]
    windows = [torch.from_numpy(np.concatenate([bufs[c - 1][-overlap * comp:], bufs[c]]).view(np.uint8).copy()).cuda()
               for c in (1, 2)]
    if plan is not None:
        plan.spectra_device(dev_new[0], x_ref, stream=stream)
    torch.cuda.synchronize()
    for call in range(2):
        x64 = torch.from_numpy(o64.spectra_of(bufs[call + 1].view(np.uint8))).cuda()
        rc = L.sk_spectra_noalloc(windows[call].data_ptr(), FMT[fmt], N, B, x_new.data_ptr(), stream.cuda_stream)
        assert rc == SK_OK, last_error()
        if plan is not None:
            plan.spectra_device(dev_new[call + 1], x_ref, stream=stream)
        torch.cuda.synchronize()
        e = _rel(x_new.to(torch.complex128), x64)
        assert e <= TOL, (call, e)
        if plan is not None:
            e = _rel(x_new, x_ref)
            assert e <= TOL, (call, e)


def test_noalloc_allocates_nothing_and_rejects_oversize():
    L = lib()
    N, B = 65536, 16
    new = (N - N // 4) * B + N // 4
    raw = torch.zeros(new, dtype=torch.int16, device="cuda").view(torch.uint8)
    X = torch.empty(B, N // 2 + 1, dtype=torch.complex64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    assert L.sk_spectra_noalloc(raw.data_ptr(), 0x08, N, B, X.data_ptr(), stream) == SK_OK
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        assert L.sk_spectra_noalloc(raw.data_ptr(), 0x08, N, B, X.data_ptr(), stream) == SK_OK
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    # 32765 twiddles + 65536 + 40 * 32768 complex elements exceed the 8 MiB array
    rc = L.sk_spectra_noalloc(raw.data_ptr(), 0x08, N, 40, X.data_ptr(), stream)
    assert rc == SK_ERR_ARG
    msg = last_error()
    assert "static" in msg and "at most 29 blocks" in msg, msg
