"""Differentiable filter-bank stage: ``torch.autograd.Function`` over the
hand-written forward and adjoint kernels (sk_fcfb_forward_device /
sk_fcfb_backward_device).

The stage is the channel computation of fcfb.rs:154-188 with complex weights:
    y_c[b] = keep_[n/8, 7(n/8))( IFFT_n( W_c[j] * get_bin(X[b], first_c + j) ) ),
    j = (i + n/2) mod n for IFFT input position i,
linear in both W and X.  Gradients follow torch's convention for complex
tensors (for a real loss, dL/dRe + i dL/dIm), so the adjoint is
dW = sum_b conj(G_b) FFT_n(pad(dy_b)) and dX = scatter(conj(W) FFT_n(pad(dy))).

Memory: a buffer's spectra take 8 K B bytes against 2 (N/4 + 3N/4 B) bytes of
int16 input.  ``fcfb_windows`` keeps the spectra for backward while they fit a
memory budget and otherwise keeps only the raw windows and recomputes each
window's forward FFT in backward (sk_spectra_window_device is stateless, so
the recomputed spectra are bit-identical to the forward ones).
"""
from __future__ import annotations

import torch

from .plan import Plan


def _plain(t: torch.Tensor) -> torch.Tensor:
    """The tensor's values in plain contiguous memory: a lazily conjugated or
    negated view (``y.conj()``, and the gradients that flow back through one)
    keeps its data unconjugated with a flag, which a raw pointer would lose."""
    return t.resolve_conj().resolve_neg().contiguous()


def _zeros_for(plan, X):
    return [torch.zeros(c["out_samples"], dtype=torch.complex64, device=X.device) for c in plan.channels]


class FcfbFunction(torch.autograd.Function):
    """y_0..y_{C-1} = fcfb(plan, X, W_0..W_{C-1}); X is [B, K] complex64."""

    @staticmethod
    def forward(ctx, plan: Plan, X: torch.Tensor, *W: torch.Tensor):
        ys = [torch.empty(c["out_samples"], dtype=torch.complex64, device=X.device) for c in plan.channels]
        Xc = _plain(X)
        Wc = [_plain(w) for w in W]
        plan.fcfb_forward_device(Xc, Wc, ys, stream=torch.cuda.current_stream(X.device))
        ctx.plan = plan
        ctx.save_for_backward(Xc, *Wc)
        return tuple(ys)

    @staticmethod
    def backward(ctx, *dys):
        X, *W = ctx.saved_tensors
        plan = ctx.plan
        zeros = _zeros_for(plan, X)
        dys = [z if d is None else _plain(d) for z, d in zip(zeros, dys)]
        dW = [torch.empty_like(w) for w in W]
        dX = torch.zeros_like(X) if ctx.needs_input_grad[1] else None
        plan.fcfb_backward_device(X, W, dys, dW, dX, stream=torch.cuda.current_stream(X.device))
        return (None, dX, *dW)


class FcfbRecompute(torch.autograd.Function):
    """fcfb over one raw window (N/4 + new samples), keeping only the window:
    backward recomputes its spectra instead of storing them."""

    @staticmethod
    def forward(ctx, plan: Plan, raw_window: torch.Tensor, *W: torch.Tensor):
        X = spectra_window(plan, raw_window)
        ys = [torch.empty(c["out_samples"], dtype=torch.complex64, device=raw_window.device) for c in plan.channels]
        Wc = [_plain(w) for w in W]
        plan.fcfb_forward_device(X, Wc, ys, stream=torch.cuda.current_stream(raw_window.device))
        ctx.plan = plan
        ctx.save_for_backward(raw_window, *Wc)
        return tuple(ys)

    @staticmethod
    def backward(ctx, *dys):
        raw_window, *W = ctx.saved_tensors
        plan = ctx.plan
        X = spectra_window(plan, raw_window)               # recomputed, bit-identical
        zeros = _zeros_for(plan, X)
        dys = [z if d is None else _plain(d) for z, d in zip(zeros, dys)]
        dW = [torch.empty_like(w) for w in W]
        plan.fcfb_backward_device(X, W, dys, dW, None, stream=torch.cuda.current_stream(X.device))
        return (None, None, *dW)


def fcfb(plan: Plan, X: torch.Tensor, weights):
    """Functional form: list of channel outputs (complex64, B*6(n/8) each)."""
    return list(FcfbFunction.apply(plan, X, *weights))


def spectra(plan: Plan, raw: torch.Tensor) -> torch.Tensor:
    """Forward FFTs of one buffer of new samples -> X [B, K] (advances the
    plan's overlap carry, like sk_process)."""
    X = torch.empty(plan.ffts_per_buf, plan.result_bins, dtype=torch.complex64, device=raw.device)
    plan.spectra_device(raw, X, stream=torch.cuda.current_stream(raw.device))
    return X


def spectra_window(plan: Plan, raw_window: torch.Tensor) -> torch.Tensor:
    """Forward FFTs of a whole window (N/4 + new samples) -> X [B, K];
    stateless."""
    X = torch.empty(plan.ffts_per_buf, plan.result_bins, dtype=torch.complex64, device=raw_window.device)
    plan.spectra_window_device(raw_window, X, stream=torch.cuda.current_stream(raw_window.device))
    return X


def spectra_bytes(plan: Plan) -> int:
    return plan.ffts_per_buf * plan.result_bins * 8


def fcfb_windows(plan: Plan, windows, weights, memory_budget: int = 1 << 30):
    """Channel outputs for a list of raw windows.  Spectra are kept for backward
    while they fit ``memory_budget`` bytes; beyond it each window is
    recomputed in backward.  Returns a list (per window) of output lists."""
    keep = len(windows) * spectra_bytes(plan) <= memory_budget
    outs = []
    for win in windows:
        if keep:
            outs.append(list(FcfbFunction.apply(plan, spectra_window(plan, win), *weights)))
        else:
            outs.append(list(FcfbRecompute.apply(plan, win, *weights)))
    return outs
