"""torch.autograd.Function over the FP64 PT records and their adjoint.

`Spectrum(context, run, density)` is a differentiable map

    (T[levels], P[levels], S[lines], gamma_air[lines]) -> records[levels, n_sub, 20481]

whose forward pass is the library's FP64 computation (the `out64` records of
marfa_compute) and whose backward pass is `marfa_vjp`: the hand-written
adjoint kernels, which recompute the line shape instead of storing it.  The
derivative holds each line's multigrid placement, the Humlicek region choices
and the cascade clamp decisions fixed (the map is piecewise smooth).

PyTorch is only the autograd plumbing here: inputs may live on any device,
the computation runs in libmarfa_gpu.so and the records come back as a float64
tensor on the device of T.
"""
from __future__ import annotations

import dataclasses

import numpy as np
import torch

from .api import Context, Run


def _host(t: torch.Tensor) -> np.ndarray:
    return np.ascontiguousarray(t.detach().to("cpu", torch.float64).numpy())


class _SpectrumFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, T, P, S, gamma_air, model):
        model.context.set_line_params(_host(S), _host(gamma_air))
        _, out64 = model.context.compute(model.run, _host(P), _host(T), model.density, want64=True)
        ctx.model = model
        ctx.save_for_backward(T, P, S, gamma_air)
        return torch.from_numpy(out64).to(T.device)

    @staticmethod
    def backward(ctx, grad):
        T, P, S, gamma_air = ctx.saved_tensors
        model = ctx.model
        model.context.set_line_params(_host(S), _host(gamma_air))
        g = model.context.vjp(model.run, _host(P), _host(T), model.density, _host(grad))

        def back(a, like):
            return torch.from_numpy(a).to(device=like.device, dtype=like.dtype)

        return back(g["dT"], T), back(g["dP"], P), back(g["dS"], S), back(g["dgamma_air"], gamma_air), None


class Spectrum:
    """Differentiable PT records of one profile for a fixed line list."""

    def __init__(self, context: Context, run: Run, density):
        self.context = context
        self.run = dataclasses.replace(run, precision="fp64")
        self.density = np.ascontiguousarray(np.asarray(density, dtype=np.float64))

    def __call__(self, T: torch.Tensor, P: torch.Tensor, S: torch.Tensor,
                 gamma_air: torch.Tensor) -> torch.Tensor:
        return _SpectrumFn.apply(T, P, S, gamma_air, self)
