"""Differentiable filter bank: the hand-written adjoint kernel through
torch.autograd against an FP64 torch-autograd restatement of fcfb.rs:154-188
(gather with modulo and conjugate mirror, weights, unnormalised inverse DFT,
keep [n/8, 7(n/8))), and against central finite differences (step 1e-3) on
8 random channels.  Bar: relative error <= 1e-4 for gradients, 1e-5 for the
forward outputs."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from spektri_b200 import Plan, workloads
from spektri_b200 import autograd as AG
from spektri_b200 import design


def fcfb_ref(X, W, chans, N, real):
    """FP64 restatement (torch ops, differentiable in X and W)."""
    K = X.shape[1]
    outs = []
    for (n, first), w in zip(chans, W):
        i = torch.arange(n, device=X.device)
        j = (i + n // 2) % n
        m = (first + j) % N
        if real:
            direct = m < K
            idx = torch.where(direct, m, N - m)
            G = X[:, idx]
            G = torch.where(direct, G, G.conj())
        else:
            G = X[:, m]
        y = torch.fft.ifft(w[j] * G, dim=1) * n
        outs.append(y[:, n // 8: n // 8 * 7].reshape(-1))
    return outs


def rel(a, b):
    a, b = a.detach(), b.detach()
    return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))


def setup(real=True, nch=16, B=6, N=4096, seed=0):
    rng = np.random.default_rng(seed)
    fs = float(N) * 1000.0
    chans = []
    for c in range(nch):
        n = int(2 ** rng.integers(4, 11))
        centre = 4 * int(rng.integers(0, N // 8)) if real else 4 * int(rng.integers(-N // 8, N // 8))
        chans.append(dict(fs_out=1000.0 * n, fc_out=1000.0 * centre))
    plan = Plan(fs, N, "s16le" if real else "cs16le", chans, ffts_per_buf=B, averages=10**6, spectrum_format="f32")
    comp = 1 if real else 2
    raw = np.clip(np.round(rng.normal(0, 3000, plan.total * comp)), -32768, 32767).astype("<i2")
    win = torch.from_numpy(raw.view(np.uint8).copy()).cuda()
    X = AG.spectra_window(plan, win)
    W = [torch.from_numpy((rng.standard_normal(c["bins"]) + 1j * rng.standard_normal(c["bins"])).astype(np.complex64)).cuda()
         for c in plan.channels]
    return plan, win, X, W, [(c["bins"], c["first"]) for c in plan.channels]


def loss_of(ys, R):
    return sum(((y.abs() ** 2).sum() * 0.5 + (y.conj() * r).real.sum()) for y, r in zip(ys, R))


@pytest.mark.parametrize("real", [True, False])
def test_forward_and_gradients_vs_fp64_autograd(real):
    plan, win, X, W, chans = setup(real)
    N = plan.fft_size
    Xg = X.clone().requires_grad_(True)
    Wg = [w.clone().requires_grad_(True) for w in W]
    ys = AG.fcfb(plan, Xg, Wg)
    X64 = X.to(torch.complex128).requires_grad_(True)
    W64 = [w.to(torch.complex128).requires_grad_(True) for w in W]
    ref = fcfb_ref(X64, W64, chans, N, real)
    for a, r in zip(ys, ref):
        if r.numel():
            assert rel(a.to(torch.complex128), r.detach()) < 1e-5
    g = torch.Generator(device="cpu").manual_seed(1)
    R = [torch.randn(r.numel(), dtype=torch.complex128, generator=g).cuda() * r.detach().abs().mean() for r in ref]
    loss_of(ys, [r.to(torch.complex64) for r in R]).backward()
    loss_of(ref, R).backward()
    for a, b in zip(Wg, W64):
        assert rel(a.grad.to(torch.complex128), b.grad) < 1e-4
    assert rel(Xg.grad.to(torch.complex128), X64.grad) < 1e-4


@pytest.mark.parametrize("real", [True, False])
def test_adjoint_is_bit_repeatable(real):
    """The adjoint sums in a fixed order (dW over blocks, dX over the channels
    that gather a bin; no atomics), so two backward passes on the same inputs
    give the same bits; overlapping channels exercise the dX gather lists."""
    plan, win, X, W, chans = setup(real, nch=24, B=8, seed=7)
    g = torch.Generator(device="cpu").manual_seed(2)
    dys = [torch.randn(c["out_samples"], dtype=torch.complex64, generator=g).cuda() for c in plan.channels]
    runs = []
    for _ in range(2):
        dW = [torch.empty_like(w) for w in W]
        dX = torch.zeros_like(X)
        plan.fcfb_backward_device(X, W, dys, dW, dX)
        torch.cuda.synchronize()
        runs.append((dW, dX))
    for a, b in zip(runs[0][0], runs[1][0]):
        assert torch.equal(a, b)
    assert torch.equal(runs[0][1], runs[1][1])
    assert float(runs[0][1].abs().sum()) > 0


def test_default_stream_outputs_are_ordered():
    """On torch's default stream (handle 0, passed to the C ABI as the legacy
    default stream rather than as NULL, which would select the plan's own
    non-blocking stream) every call's outputs are complete before torch reads
    them: 40 calls at a size where an unordered launch would still be
    running give the same bits, equal to FP64 within 1e-5."""
    rng = np.random.default_rng(21)
    N, B, n = 32768, 512, 1024
    chans = [dict(fs_out=1000.0 * n, fc_out=1000.0 * 4 * int(rng.integers(n // 8, N // 8 - n // 8))) for _ in range(64)]
    plan = Plan(N * 1000.0, N, "s16le", chans, ffts_per_buf=B, averages=10**9, spectrum_format="f32")
    K = plan.result_bins
    X = torch.from_numpy((rng.standard_normal((B, K)) + 1j * rng.standard_normal((B, K))).astype(np.complex64)).cuda()
    W = [torch.from_numpy((rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex64)).cuda()
         for _ in plan.channels]
    assert torch.cuda.current_stream().cuda_stream == 0
    with torch.no_grad():
        first = [y.clone() for y in AG.fcfb(plan, X, W)]
        for _ in range(40):
            ys = AG.fcfb(plan, X, W)
            assert all(torch.equal(a, b) for a, b in zip(ys, first))
    ref = fcfb_ref(X.to(torch.complex128), [w.to(torch.complex128) for w in W],
                   [(c["bins"], c["first"]) for c in plan.channels], N, True)
    assert max(rel(a.to(torch.complex128), r) for a, r in zip(first, ref)) < 1e-5


def test_conjugate_views_in_and_out():
    """Lazily conjugated tensors carry their values unconjugated plus a flag:
    weights passed as w.conj() and the gradients that flow back through
    y.conj() must reach the kernels resolved.  Loss sum Re(conj(y) r), whose
    output gradient is such a view, and weights given as a conj view."""
    plan, win, X, W, chans = setup(True, nch=8, seed=13)
    N = plan.fft_size
    g = torch.Generator(device="cpu").manual_seed(3)
    R = [torch.randn(c["out_samples"], dtype=torch.complex128, generator=g).cuda() for c in plan.channels]
    Wg = [w.clone().requires_grad_(True) for w in W]
    ys = AG.fcfb(plan, X, [w.conj() for w in Wg])
    sum((y.conj() * r.to(torch.complex64)).real.sum() for y, r in zip(ys, R)).backward()
    W64 = [w.to(torch.complex128).requires_grad_(True) for w in W]
    ref = fcfb_ref(X.to(torch.complex128), [w.conj() for w in W64], chans, N, True)
    for a, r in zip(ys, ref):
        assert rel(a.to(torch.complex128), r) < 1e-5
    sum((y.conj() * r).real.sum() for y, r in zip(ref, R)).backward()
    for a, b in zip(Wg, W64):
        assert rel(a.grad.to(torch.complex128), b.grad) < 1e-4


def test_gradients_vs_central_finite_differences():
    """Directional derivatives along random complex directions on 8 random
    channels: adjoint kernel vs (L(W + h v) - L(W - h v)) / 2h, h = 1e-3,
    with the loss evaluated in FP64."""
    plan, win, X, W, chans = setup(True, nch=16, seed=3)
    N = plan.fft_size
    X64 = X.to(torch.complex128)
    g = torch.Generator(device="cpu").manual_seed(5)
    ref0 = fcfb_ref(X64, [w.to(torch.complex128) for w in W], chans, N, True)
    R = [torch.randn(r.numel(), dtype=torch.complex128, generator=g).cuda() * (r.abs().mean() + 1e-30) for r in ref0]
    Wg = [w.clone().requires_grad_(True) for w in W]
    loss_of(AG.fcfb(plan, X, Wg), [r.to(torch.complex64) for r in R]).backward()
    rng = np.random.default_rng(9)
    pick = rng.choice(len(W), 8, replace=False)
    h = 1e-3
    for c in pick:
        v = torch.randn(W[c].numel(), dtype=torch.complex128, generator=g).cuda()
        Wp = [w.to(torch.complex128) for w in W]
        Wm = [w.to(torch.complex128) for w in W]
        Wp[c] = Wp[c] + h * v
        Wm[c] = Wm[c] - h * v
        fd = (loss_of(fcfb_ref(X64, Wp, chans, N, True), R) - loss_of(fcfb_ref(X64, Wm, chans, N, True), R)) / (2 * h)
        ad = (Wg[c].grad.to(torch.complex128).conj() * v).real.sum()
        assert abs(float(ad - fd)) <= 1e-4 * abs(float(fd)) + 1e-12, (c, float(ad), float(fd))


def test_recompute_path_matches_stored_spectra():
    plan, win, X, W, chans = setup(True, seed=7)
    g = torch.Generator(device="cpu").manual_seed(2)
    R = [torch.randn(c["out_samples"], dtype=torch.complex64, generator=g).cuda() for c in plan.channels]
    Wa = [w.clone().requires_grad_(True) for w in W]
    Wb = [w.clone().requires_grad_(True) for w in W]
    ya = AG.fcfb_windows(plan, [win], Wa, memory_budget=1 << 40)[0]        # spectra kept
    yb = AG.fcfb_windows(plan, [win], Wb, memory_budget=0)[0]              # recomputed in backward
    for a, b in zip(ya, yb):
        assert torch.equal(a, b)
    loss_of(ya, R).backward()
    loss_of(yb, R).backward()
    for a, b in zip(Wa, Wb):
        assert torch.equal(a.grad, b.grad)               # bit-identical spectra, fixed-order sums


def test_adam_design_lowers_loss_and_feeds_the_plain_path(tmp_path):
    N = 4096
    fs = N * 1000.0
    chans = [(256e3, 1000.0 * c) for c in (400, 812, 1200, 1604)]
    wd = design.WeightDesign(fs, N, chans, real_input=True, n_pass=8, n_stop=8, seed=1)
    w0 = wd.initial_weights()
    l0 = float(wd.loss(w0))
    W, hist = design.adam_design(wd, steps=80, lr=5e-3)
    assert hist[-1] < 0.7 * l0, (l0, hist[-1])
    paths = design.save_weights(tmp_path, W)
    # the plain path loads the files and reproduces the stage's outputs bit for bit
    filt = [dict(fs_out=fo, fc_out=fc, weights=np.fromfile(p, "<c8")) for (fo, fc), p in zip(chans, paths)]
    plan = Plan(fs, N, "s16le", filt, ffts_per_buf=4, averages=10**6, spectrum_format="f32", mode="plain")
    rng = np.random.default_rng(4)
    raw = np.clip(np.round(rng.normal(0, 3000, plan.new_samples)), -32768, 32767).astype("<i2")
    _, outs = plan.process(raw.view(np.uint8))
    win = torch.from_numpy(np.concatenate([np.zeros(N // 4, "<i2"), raw]).view(np.uint8).copy()).cuda()
    X = AG.spectra_window(plan, win)
    ys = AG.fcfb(plan, X, [w.cuda() for w in W])
    for a, b in zip(outs, ys):
        assert np.array_equal(a, b.detach().cpu().numpy())
