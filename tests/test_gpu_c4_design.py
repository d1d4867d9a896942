"""The differentiation configuration at its own size: a real int16 stream,
forward FFT 32768, 64 channels of n = 1024 with complex weights, 16 blocks per
buffer.  Gradients of the adjoint kernel against FP64 autograd on every
channel and against central finite differences (step 1e-3) on 8 random
channels; then 500 Adam steps of weight design over the same 64 channels,
whose weights are fed back into the plain path."""
import time

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from spektri_b200 import Plan, design, workloads
from spektri_b200 import autograd as AG
from tests.test_gpu_autograd import fcfb_ref, loss_of, rel


def c4_setup(seed=0):
    w = workloads.c4()
    plan = Plan(w.fs, w.fft_size, w.fmt, w.filters(), ffts_per_buf=w.ffts_per_buf, averages=10**6,
                spectrum_format="f32")
    assert plan.n_channels == 64 and all(c["bins"] == 1024 for c in plan.channels)
    raw = workloads.stream_numpy(w, 0, plan.total)
    win = torch.from_numpy(raw.view(np.uint8).copy()).cuda()
    X = AG.spectra_window(plan, win)
    rng = np.random.default_rng(seed)
    W = [torch.from_numpy((rng.standard_normal(1024) + 1j * rng.standard_normal(1024)).astype(np.complex64)).cuda()
         for _ in plan.channels]
    return w, plan, win, X, W, [(c["bins"], c["first"]) for c in plan.channels]


def test_c4_gradients_vs_fp64_and_finite_differences():
    w, plan, win, X, W, chans = c4_setup()
    N = plan.fft_size
    X64 = X.to(torch.complex128)
    g = torch.Generator(device="cpu").manual_seed(11)
    ref0 = fcfb_ref(X64, [v.to(torch.complex128) for v in W], chans, N, True)
    R = [torch.randn(r.numel(), dtype=torch.complex128, generator=g).cuda() * r.abs().mean() for r in ref0]
    Xg = X.clone().requires_grad_(True)
    Wg = [v.clone().requires_grad_(True) for v in W]
    ys = AG.fcfb(plan, Xg, Wg)
    for a, r in zip(ys, ref0):
        assert rel(a.to(torch.complex128), r) < 1e-5
    loss_of(ys, [r.to(torch.complex64) for r in R]).backward()
    Xr = X64.clone().requires_grad_(True)
    Wr = [v.to(torch.complex128).requires_grad_(True) for v in W]
    loss_of(fcfb_ref(Xr, Wr, chans, N, True), R).backward()
    worst = max(rel(a.grad.to(torch.complex128), b.grad) for a, b in zip(Wg, Wr))
    assert worst < 1e-4, worst
    assert rel(Xg.grad.to(torch.complex128), Xr.grad) < 1e-4
    rng = np.random.default_rng(12)
    h = 1e-3
    for c in rng.choice(len(W), 8, replace=False):
        v = torch.randn(1024, dtype=torch.complex128, generator=g).cuda()
        Wp = [x.to(torch.complex128) for x in W]
        Wm = [x.to(torch.complex128) for x in W]
        Wp[c] = Wp[c] + h * v
        Wm[c] = Wm[c] - h * v
        fd = (loss_of(fcfb_ref(X64, Wp, chans, N, True), R) - loss_of(fcfb_ref(X64, Wm, chans, N, True), R)) / (2 * h)
        ad = (Wg[c].grad.to(torch.complex128).conj() * v).real.sum()
        assert abs(float(ad - fd)) <= 1e-4 * abs(float(fd)) + 1e-12, (int(c), float(ad), float(fd))


def test_c4_adam_500_steps_and_plain_path(tmp_path):
    w = workloads.c4()
    chans = [(f["fs_out"], f["fc_out"]) for f in w.filters()]
    wd = design.WeightDesign(w.fs, w.fft_size, chans, real_input=True, n_pass=8, n_stop=8, seed=4)
    W0 = wd.initial_weights()
    with torch.no_grad():
        l0, per0 = wd.loss(W0, per_channel=True)
    t0 = time.perf_counter()
    W, hist = design.adam_design(wd, steps=500, lr=2e-3)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    with torch.no_grad():
        l1, per1 = wd.loss(W, per_channel=True)
    print(f"C4 design: {wd.B} probe blocks, 64 channels of 1024; loss {float(l0):.4g} -> {float(l1):.4g} "
          f"in 500 Adam steps ({dt:.1f} s); channels improved: "
          f"{sum(float(b) < float(a) for a, b in zip(per0, per1))}/64")
    assert float(l1) < 0.5 * float(l0)
    paths = design.save_weights(tmp_path, W)
    filt = [dict(f, weights=np.fromfile(p, "<c8")) for f, p in zip(w.filters(), paths)]
    plan = Plan(w.fs, w.fft_size, w.fmt, filt, ffts_per_buf=w.ffts_per_buf, averages=10**6, spectrum_format="f32",
                mode="plain")
    raw = workloads.stream_numpy(w, 0, plan.new_samples)
    _, outs = plan.process(raw.view(np.uint8))
    win = torch.from_numpy(np.concatenate([np.zeros(plan.overlap, "<i2"), raw]).view(np.uint8).copy()).cuda()
    ys = AG.fcfb(plan, AG.spectra_window(plan, win), [x.cuda() for x in W])
    for a, b in zip(outs, ys):
        assert np.array_equal(a, b.detach().cpu().numpy())
