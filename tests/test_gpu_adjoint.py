"""GPU tests of the hand-written adjoint kernels and the autograd operators.

1. Dot-product identities <R2C x, G> = <x, R2C^T G> and <C2R Y, g> = <Y, C2R^T g>
   (real inner products, arbitrary complex G and Y) on every path: fused 3D, generic
   3D (odd sizes), 2D, and the three 4D layouts, f32 and f64.
2. The differentiable spectral pipeline at 128^3 f32: u = sin x cos y cos z
   + 0.05 N(0,1) (seed 4), w = Poisson(C2R(G(k) R2C(u)) / N) with the Gaussian
   G(k) = exp(-|k|^2 / (2 16^2)), loss = 0.5 ||w||^2.  Its gradient (adjoint kernels
   behind torch.autograd) is checked against torch autograd through torch.fft in
   float64, and against FP64 central finite differences on 64 random directions.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def F(torch_cuda):
    from fftm_b200 import build
    build.build()
    import fftm_b200
    return fftm_b200


def _rdot(a, b):
    import torch
    if a.is_complex():
        a = a.to(torch.complex128)
        b = b.to(torch.complex128)
        return float((a.real * b.real + a.imag * b.imag).sum())
    return float((a.double() * b.double()).sum())


CASES = [
    ("float32", (64, 64, 64), None), ("float32", (9, 10, 7), None), ("float64", (16, 12, 10), None),
    ("float32", (128, 64, 256), None),
    ("float32", (12, 20), None), ("float64", (7, 9), None),
    ("float32", (8, 6, 10, 12), "pencil"), ("float32", (8, 6, 10, 12), "slab"),
    ("float32", (8, 6, 10, 12), "native_xzwy"), ("float32", (32, 32, 64, 64), "native_xzwy"),
    ("float32", (32, 32, 64, 64), "slab"), ("float64", (6, 4, 8, 10), "native_xzwy"),
]


@pytest.mark.parametrize("dtype,dims,layout", CASES)
def test_adjoint_dot_products(F, torch_cuda, dtype, dims, layout):
    torch = torch_cuda
    f = F.ffts(dtype, strategy_4d=layout or "pencil").init(*dims)
    rt = torch.float32 if dtype == "float32" else torch.float64
    ct = torch.complex64 if dtype == "float32" else torch.complex128
    gen = torch.Generator(device="cuda").manual_seed(3)
    x = torch.randn(f.real_shape(), dtype=rt, device="cuda", generator=gen)
    Y = torch.randn(f.spectrum_shape(), dtype=ct, device="cuda", generator=gen)
    g = torch.randn(f.real_shape(), dtype=rt, device="cuda", generator=gen)
    G = torch.randn(f.spectrum_shape(), dtype=ct, device="cuda", generator=gen)
    tol = 2e-5 if dtype == "float32" else 1e-11
    # R2C and its adjoint
    Rx = torch.empty_like(G)
    f.forward(x, Rx)
    RtG = torch.empty_like(x)
    f.forward_adjoint(G.clone(), RtG)
    lhs, rhs = _rdot(Rx, G), _rdot(x, RtG)
    assert abs(lhs - rhs) <= tol * (abs(lhs) + abs(rhs) + 1.0), ("R2C", lhs, rhs)
    # C2R (unnormalised) and its adjoint, on an arbitrary (not Hermitian-consistent) spectrum
    CY = torch.empty_like(x)
    f.backward(Y.clone(), CY)
    CtG = torch.empty_like(G)
    f.backward_adjoint(g, CtG)
    lhs, rhs = _rdot(CY, g), _rdot(Y, CtG)
    assert abs(lhs - rhs) <= tol * (abs(lhs) + abs(rhs) + 1.0), ("C2R", lhs, rhs)


def _pipeline_fp64(torch, u64, sigma, sign):
    n = u64.shape
    X = torch.fft.rfftn(u64)
    kx = torch.fft.fftfreq(n[0], 1.0 / n[0], dtype=torch.float64, device=u64.device)[:, None, None]
    ky = torch.fft.fftfreq(n[1], 1.0 / n[1], dtype=torch.float64, device=u64.device)[None, :, None]
    kz = torch.arange(n[2] // 2 + 1, dtype=torch.float64, device=u64.device)[None, None, :]
    k2 = kx * kx + ky * ky + kz * kz
    G = torch.exp(-k2 / (2 * sigma ** 2))
    v = torch.fft.irfftn(X * G, s=n)
    P = torch.where(k2 == 0, torch.zeros_like(k2), sign / torch.where(k2 == 0, torch.ones_like(k2), k2))
    w = torch.fft.irfftn(torch.fft.rfftn(v) * P, s=n)
    return 0.5 * (w * w).sum()


def test_differentiable_pipeline_128(F, torch_cuda):
    torch = torch_cuda
    import fftm_b200.autograd as A
    n = (128, 128, 128)
    g = 2 * np.pi * np.arange(128) / 128
    u0 = (np.sin(g)[:, None, None] * np.cos(g)[None, :, None] * np.cos(g)[None, None, :]
          + 0.05 * np.random.default_rng(4).standard_normal(n))
    sigma, sign = 16.0, -1.0
    f = F.ffts("float32").init(*n)
    u = torch.tensor(u0, dtype=torch.float32, device="cuda", requires_grad=True)
    kx = torch.fft.fftfreq(128, 1.0 / 128, device="cuda")
    kz = torch.arange(65, device="cuda", dtype=torch.float32)
    k2 = kx[:, None, None] ** 2 + kx[None, :, None] ** 2 + kz[None, None, :] ** 2
    G = torch.exp(-k2 / (2 * sigma ** 2)).to(torch.complex64)
    spec = A.r2c(u, f)
    v = A.c2r(spec * G, f, normalized=True)
    w = A.poisson(v, f, sign)
    loss = 0.5 * (w.double() * w.double()).sum()
    loss.backward()
    grad = u.grad.double()

    # reference: torch autograd through torch.fft in float64
    u64 = torch.tensor(u0, dtype=torch.float64, device="cuda", requires_grad=True)
    L64 = _pipeline_fp64(torch, u64, sigma, sign)
    L64.backward()
    ref = u64.grad
    assert abs(loss.item() - L64.item()) <= 1e-5 * abs(L64.item())
    rel = float(torch.linalg.norm(grad - ref) / torch.linalg.norm(ref))
    assert rel <= 1e-5, rel

    # FP64 central differences on 64 random directions (the loss is quadratic, so the
    # central difference is exact up to rounding); the 64 directional derivatives are
    # compared as one vector, since a single random projection <grad, d> can be near zero
    gen = torch.Generator(device="cuda").manual_seed(64)
    with torch.no_grad():
        an, fd = [], []
        for _ in range(64):
            d = torch.randn(n, dtype=torch.float64, device="cuda", generator=gen)
            eps = 1e-3
            fd.append(float((_pipeline_fp64(torch, u64 + eps * d, sigma, sign) -
                             _pipeline_fp64(torch, u64 - eps * d, sigma, sign)) / (2 * eps)))
            an.append(float((grad * d).sum()))
        an, fd = np.array(an), np.array(fd)
        assert np.linalg.norm(an - fd) / np.linalg.norm(fd) <= 1e-5, np.linalg.norm(an - fd) / np.linalg.norm(fd)


def test_poisson_filter_autograd_self_adjoint(F, torch_cuda):
    torch = torch_cuda
    import fftm_b200.autograd as A
    for dims, layout in [((32, 24, 16), None), ((16, 8, 8, 12), "native_xzwy"), ((16, 8, 8, 12), "pencil")]:
        f = F.ffts("float64", strategy_4d=layout or "pencil").init(*dims)
        shape = f.real_shape()
        x = torch.randn(shape, dtype=torch.float64, device="cuda", requires_grad=True)
        y = torch.randn(shape, dtype=torch.float64, device="cuda")
        out = A.filter_poisson(A.poisson(x, f, -1.0), f, 3.0, 1.0)
        (out * y).sum().backward()
        # gradient of <A x, y> is A^T y = A y for the self-adjoint composition
        with torch.no_grad():
            t1 = torch.empty_like(y)
            f.filter(y, t1, 3.0, 1.0)
            t2 = torch.empty_like(y)
            f.poisson(t1, t2, -1.0)
        assert float(torch.linalg.norm(x.grad - t2) / torch.linalg.norm(t2)) <= 1e-12
