"""Parity with the reference's own cuFFT `ffts` path on the same GPU and the same seeded
inputs: tests/cufft_ref restates the exact cufftMakePlanMany64 plans of
source/ffts.hpp:677-776 and source/fftm.hpp:2941-2961 (auto-allocation off, one external
work area), the 4D stage order with its per-element transposes, and the Poisson example's
separate multiply and 1/N kernels.  fftb must give the same spectra, inverses and Poisson
solutions: relative L2 <= 2e-6 in float32 and <= 1e-12 in float64, and both are checked
against the FP64 oracle too."""
import os
import sys

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu
TOL32, TOL64 = 2e-6, 1e-12

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def env(torch_cuda):
    from fftm_b200 import build
    build.build()
    import cufft_ref
    cufft_ref.build()
    import fftm_b200
    return fftm_b200, cufft_ref


def _rel(a, b):
    import torch
    a = a.to(torch.complex128) if a.is_complex() else a.double()
    b = b.to(torch.complex128) if b.is_complex() else b.double()
    return float(torch.linalg.norm(a - b) / torch.linalg.norm(b))


def _np(t):
    import torch
    torch.cuda.synchronize()
    return t.cpu().numpy().astype(np.complex128 if t.is_complex() else np.float64)


@pytest.mark.parametrize("shape,dtype", [((64, 64, 64), "float32"), ((256, 256, 256), "float32"),
                                         ((96, 48, 80), "float32"), ((32, 24, 16), "float64")])
def test_3d_forward_backward_vs_reference_cufft(env, torch_cuda, shape, dtype):
    F, R = env
    torch = torch_cuda
    tdt = torch.float32 if dtype == "float32" else torch.float64
    cdt = torch.complex64 if dtype == "float32" else torch.complex128
    tol = TOL32 if dtype == "float32" else TOL64
    x_np = O.random_3d(*shape, 0x1234ABCDEF987654, single=dtype == "float32")
    x = torch.tensor(x_np, dtype=tdt, device="cuda")
    f = F.ffts(dtype).init(*shape)
    r = R.RefFfts(dtype, shape)
    X, Xr = (torch.empty(f.spectrum_shape(), dtype=cdt, device="cuda") for _ in range(2))
    f.forward(x, X)
    r.forward(x, Xr)
    assert _rel(X, Xr) <= tol
    if shape[0] <= 96:
        assert O.rel_l2(_np(Xr), O.ffts3d_forward(x_np)) <= tol    # the harness itself
    y, yr = torch.empty_like(x), torch.empty_like(x)
    f.backward(X.clone(), y)
    r.backward(Xr.clone(), yr)
    assert _rel(y, yr) <= tol


def test_3d_poisson_vs_reference_cufft(env, torch_cuda):
    F, R = env
    torch = torch_cuda
    n = 256
    g = 2 * np.pi * np.arange(n) / n
    rhs = (np.sin(g)[:, None, None] * np.sin(2 * g)[None, :, None] * np.cos(3 * g)[None, None, :]
           + 0.1 * np.random.default_rng(0).uniform(-1, 1, (n, n, n)))
    rhs -= rhs.mean()
    x = torch.from_numpy(rhs.astype(np.float32)).cuda()
    f = F.ffts("float32").init(n, n, n)
    r = R.RefFfts("float32", (n, n, n))
    u, ur = torch.empty_like(x), torch.empty_like(x)
    spec = torch.empty(f.spectrum_shape(), dtype=torch.complex64, device="cuda")
    f.poisson(x, u, -1.0)
    r.poisson(x.clone(), spec, ur, -1.0)
    assert _rel(u, ur) <= TOL32


@pytest.mark.parametrize("layout", ["pencil", "slab", "native_xzwy"])
@pytest.mark.parametrize("dims", [(16, 24, 32, 12), (64, 64, 64, 64)])
def test_4d_vs_reference_cufft(env, torch_cuda, layout, dims):
    F, R = env
    torch = torch_cuda
    f = F.ffts("float32", strategy_4d=layout).init(*dims)
    r = R.RefFfts("float32", dims, layout)
    gen = np.random.default_rng(1)
    x = torch.from_numpy(gen.standard_normal(f.real_shape()).astype(np.float32)).cuda()
    X, Xr = (torch.empty(f.spectrum_shape(), dtype=torch.complex64, device="cuda") for _ in range(2))
    f.forward(x, X)
    r.forward(x, Xr)
    assert _rel(X, Xr) <= TOL32
    if dims[0] <= 16:
        lay = {"pencil": O.PENCIL, "slab": O.SLAB, "native_xzwy": O.NATIVE_XZWY}[layout]
        ref = O.ffts4d_forward(lay, _np(x), dims)
        assert O.rel_l2(_np(Xr), ref) <= TOL32
    y, yr = torch.empty_like(x), torch.empty_like(x)
    f.backward(X.clone(), y)
    r.backward(Xr.clone(), yr)
    assert _rel(y, yr) <= TOL32
    assert _rel(yr / x.numel(), x) <= TOL32
