"""The allocation-free spectra entry point (sk_spectra_noalloc) against the
plan-based one (sk_spectra_device).

sk_spectra_noalloc exists for callers that may not allocate device memory:
real-time receive callbacks that cannot afford a cudaMalloc stall, and hosts
whose own memory pool owns the device.  It keeps its scratch in a static
device array, so these checks cover: the same spectra as the plan path
(relative RMS <= 1e-5) on two calls in a row, whose second call finds the
first call's data still in the shared array; no change in free device
memory across calls; and a clear refusal of sizes beyond the array.

This file is collected last so that a failure here leaves every other test
already run.
"""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from spektri_b200 import Plan
from spektri_b200._lib import SK_ERR_ARG, SK_OK, last_error, lib

TOL = 1e-5
FMT = {"s16le": 0x08, "cs16le": 0x48}


def _rel(a, b):
    return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))


@pytest.mark.parametrize("fmt,N,B", [("s16le", 4096, 8), ("s16le", 65536, 8), ("cs16le", 16384, 4), ("cs16le", 65536, 2)])
def test_noalloc_matches_plan_on_two_calls_in_a_row(fmt, N, B):
    L = lib()
    plan = Plan(N * 1000.0, N, fmt, [], ffts_per_buf=B, averages=10**6, spectrum_format="f32")
    K, overlap, new = plan.result_bins, N // 4, plan.new_samples
    comp = 2 if fmt.startswith("c") else 1
    rng = np.random.default_rng(N + B)
    bufs = [np.clip(np.round(rng.normal(0, 4000, new * comp)), -32768, 32767).astype("<i2") for _ in range(2)]
    stream = torch.cuda.current_stream()
    x_ref = torch.empty(B, K, dtype=torch.complex64, device="cuda")
    x_new = torch.empty(B, K, dtype=torch.complex64, device="cuda")
    carried = np.zeros(overlap * comp, np.int16)            # the reference's buffer starts with zeros
    dev_new = [torch.from_numpy(b.view(np.uint8).copy()).cuda() for b in bufs]
    windows = []
    for b in bufs:
        windows.append(torch.from_numpy(np.concatenate([carried, b]).view(np.uint8).copy()).cuda())
        carried = b[-overlap * comp:]
    torch.cuda.synchronize()
    for call in range(2):
        plan.spectra_device(dev_new[call], x_ref, stream=stream)
        rc = L.sk_spectra_noalloc(windows[call].data_ptr(), FMT[fmt], N, B, x_new.data_ptr(), stream.cuda_stream)
        assert rc == SK_OK, last_error()
        torch.cuda.synchronize()
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
