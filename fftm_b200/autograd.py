"""Differentiable spectral operators on the fftb kernels.

Each operator is a ``torch.autograd.Function`` whose backward runs the library's
hand-written adjoint kernels (no autograd through torch.fft):

* :func:`r2c`        forward R2C; backward = fftb_ffts_forward_adjoint (C2R of the
                     gradient with interior half-axis bins weighted 1/2)
* :func:`c2r`        unnormalised (or 1/N-normalised) C2R; backward =
                     fftb_ffts_backward_adjoint (R2C with interior bins doubled)
* :func:`poisson`    fused u = C2R(sign R2C(f) / |k|^2) / N; self-adjoint, so the
                     backward is the same fused solve
* :func:`filter_poisson`  fused Gaussian filter (optionally followed by the Poisson
                     multiply); self-adjoint

Gradients of complex tensors follow PyTorch's convention for real losses:
grad = dL/dRe + i dL/dIm, the G of the adjoint formulas.
"""
from __future__ import annotations

import torch


def _complex_dtype(obj):
    return torch.complex64 if obj.dtype == 0 else torch.complex128


def _real_dtype(obj):
    return torch.float32 if obj.dtype == 0 else torch.float64


class _R2C(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, obj):
        ctx.obj = obj
        spec = torch.empty(obj.spectrum_shape(), dtype=_complex_dtype(obj), device=x.device)
        obj.forward(x.contiguous(), spec)
        return spec

    @staticmethod
    def backward(ctx, g):
        obj = ctx.obj
        gs = g.contiguous().clone()          # the adjoint overwrites its input
        gx = torch.empty(obj.real_shape(), dtype=_real_dtype(obj), device=g.device)
        obj.forward_adjoint(gs, gx)
        return gx, None


class _C2R(torch.autograd.Function):
    @staticmethod
    def forward(ctx, spec, obj, normalized):
        ctx.obj = obj
        ctx.normalized = normalized
        out = torch.empty(obj.real_shape(), dtype=_real_dtype(obj), device=spec.device)
        obj.backward(spec.contiguous().clone(), out, normalized=normalized)
        return out

    @staticmethod
    def backward(ctx, g):
        obj = ctx.obj
        gs = torch.empty(obj.spectrum_shape(), dtype=_complex_dtype(obj), device=g.device)
        obj.backward_adjoint(g.contiguous(), gs)
        if ctx.normalized:
            n = 1
            for d in obj.dims:
                n *= d
            gs.mul_(1.0 / n)
        return gs, None, None


class _Poisson(torch.autograd.Function):
    @staticmethod
    def forward(ctx, f, obj, sign):
        ctx.obj = obj
        ctx.sign = sign
        out = torch.empty_like(f)
        obj.poisson(f.contiguous(), out, sign)
        return out

    @staticmethod
    def backward(ctx, g):
        out = torch.empty_like(g)
        ctx.obj.poisson(g.contiguous(), out, ctx.sign)
        return out, None, None


class _Filter(torch.autograd.Function):
    @staticmethod
    def forward(ctx, f, obj, sigma, poisson_sign):
        ctx.obj, ctx.sigma, ctx.ps = obj, sigma, poisson_sign
        out = torch.empty_like(f)
        obj.filter(f.contiguous(), out, sigma, poisson_sign)
        return out

    @staticmethod
    def backward(ctx, g):
        out = torch.empty_like(g)
        ctx.obj.filter(g.contiguous(), out, ctx.sigma, ctx.ps)
        return out, None, None, None


def r2c(x: torch.Tensor, obj) -> torch.Tensor:
    """R2C of x with obj (an initialised fftm_b200.ffts); differentiable."""
    return _R2C.apply(x, obj)


def c2r(spec: torch.Tensor, obj, normalized: bool = True) -> torch.Tensor:
    """C2R of spec (1/N-scaled if normalized); differentiable.  spec is not modified."""
    return _C2R.apply(spec, obj, normalized)


def poisson(f: torch.Tensor, obj, sign: float = -1.0) -> torch.Tensor:
    """Fused periodic Poisson solve; differentiable (self-adjoint)."""
    return _Poisson.apply(f, obj, sign)


def filter_poisson(f: torch.Tensor, obj, sigma: float, poisson_sign: float = 0.0) -> torch.Tensor:
    """Fused Gaussian filter (then Poisson multiply if poisson_sign != 0); differentiable."""
    return _Filter.apply(f, obj, sigma, poisson_sign)
