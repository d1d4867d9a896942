"""Differentiable filter-bank stage: ``torch.autograd.Function`` over the
hand-written forward and adjoint kernels (sk_fcfb_forward_device /
sk_fcfb_backward_device).

The stage is the channel computation of fcfb.rs:154-188 with complex weights:
    y_c[b] = keep_[n/8, 7n/8)( IFFT_n( W_c[j] * get_bin(X[b], first_c + j) ) ),
    j = (i + n/2) mod n for IFFT input position i,
linear in both W and X.  Gradients follow torch's convention for complex
tensors (for a real loss, dL/dRe + i dL/dIm), so the adjoint is
dW = sum_b conj(G_b) FFT_n(pad(dy_b)) and dX = scatter(conj(W) FFT_n(pad(dy))).

``SpectraSource`` feeds the stage with spectra from raw int16 buffers: when a
batch's spectra would not fit the memory budget, backward recomputes each
buffer's forward FFT instead of keeping it (the raw input is kept: 2 B per
sample instead of 8 B per bin).
"""
from __future__ import annotations

import torch

from .plan import Plan


class FcfbFunction(torch.autograd.Function):
    """y_0..y_{C-1} = fcfb(plan, X, W_0..W_{C-1})."""

    @staticmethod
    def forward(ctx, plan: Plan, X: torch.Tensor, *W: torch.Tensor):
        ys = [torch.empty(c["out_samples"], dtype=torch.complex64, device=X.device) for c in plan.channels]
        Xc = X.contiguous()
        Wc = [w.contiguous() for w in W]
        plan.fcfb_forward_device(Xc, Wc, ys, stream=torch.cuda.current_stream(X.device))
        ctx.plan = plan
        ctx.save_for_backward(Xc, *Wc)
        return tuple(ys)

    @staticmethod
    def backward(ctx, *dys):
        X, *W = ctx.saved_tensors
        plan = ctx.plan
        dys = [torch.zeros(c["out_samples"], dtype=torch.complex64, device=X.device) if d is None else d.contiguous()
               for c, d in zip(plan.channels, dys)]
        dW = [torch.empty_like(w) for w in W]
        dX = torch.zeros_like(X) if ctx.needs_input_grad[1] else None
        plan.fcfb_backward_device(X, W, dys, dW, dX, stream=torch.cuda.current_stream(X.device))
        return (None, dX, *dW)


def fcfb(plan: Plan, X: torch.Tensor, weights):
    """Functional form: list of channel outputs (complex64, B*3n/4 each)."""
    return list(FcfbFunction.apply(plan, X, *weights))


def spectra(plan: Plan, raw: torch.Tensor) -> torch.Tensor:
    """Forward FFTs of one buffer of raw samples -> X [B, K] complex64 (advances
    the plan's overlap carry)."""
    X = torch.empty(plan.ffts_per_buf, plan.result_bins, dtype=torch.complex64, device=raw.device)
    plan.spectra_device(raw, X, stream=torch.cuda.current_stream(raw.device))
    return X


class SpectraRecompute(torch.autograd.Function):
    """fcfb over one raw buffer, keeping only the raw samples: the spectra are
    recomputed in backward (with a copy of the carry the forward used)."""

    @staticmethod
    def forward(ctx, plan: Plan, spectra_plan: Plan, raw: torch.Tensor, *W: torch.Tensor):
        X = spectra(spectra_plan, raw)
        ys = [torch.empty(c["out_samples"], dtype=torch.complex64, device=raw.device) for c in plan.channels]
        plan.fcfb_forward_device(X, [w.contiguous() for w in W], ys, stream=torch.cuda.current_stream(raw.device))
        ctx.plan, ctx.spectra_plan = plan, spectra_plan
        ctx.save_for_backward(raw, *W)
        del X
        return tuple(ys)

    @staticmethod
    def backward(ctx, *dys):
        raw, *W = ctx.saved_tensors
        plan = ctx.plan
        X = spectra(ctx.spectra_plan, raw)          # recomputed, not stored
        dys = [torch.zeros(c["out_samples"], dtype=torch.complex64, device=raw.device) if d is None else d.contiguous()
               for c, d in zip(plan.channels, dys)]
        dW = [torch.empty_like(w) for w in W]
        plan.fcfb_backward_device(X, [w.contiguous() for w in W], dys, dW, None,
                                  stream=torch.cuda.current_stream(raw.device))
        return (None, None, None, *dW)
