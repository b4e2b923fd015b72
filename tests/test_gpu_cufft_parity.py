"""Cross-check with torch.fft (cuFFT through torch's own plans) on the same GPU and the same
seeded inputs, beside the reference-plan harness of test_gpu_cufft_ffts.py: FP32 against
FP32, relative L2 <= 2e-6 for spectra and round trips, on the 3D layouts, the 4D native_xzwy
spectrum [ky][kz][kw][kx], and the Poisson solve."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 2e-6


@pytest.fixture(scope="module")
def F(torch_cuda):
    from fftm_b200 import build
    build.build()
    import fftm_b200
    return fftm_b200


def _rel(a, b):
    import torch
    a = a.to(torch.complex128) if a.is_complex() else a.double()
    b = b.to(torch.complex128) if b.is_complex() else b.double()
    return float(torch.linalg.norm(a - b) / torch.linalg.norm(b))


@pytest.mark.parametrize("shape", [(64, 64, 64), (256, 256, 256), (96, 48, 80), (128, 64, 32), (45, 27, 50)])
def test_3d_r2c_c2r_vs_cufft(F, torch_cuda, shape):
    torch = torch_cuda
    x = torch.from_numpy(np.random.default_rng(0).uniform(-1, 1, shape).astype(np.float32)).cuda()
    f = F.ffts("float32").init(*shape)
    X = torch.empty(f.spectrum_shape(), dtype=torch.complex64, device="cuda")
    f.forward(x, X)
    assert _rel(X, torch.fft.rfftn(x)) <= TOL
    y = torch.empty_like(x)
    f.backward(X.clone(), y)
    assert _rel(y, torch.fft.irfftn(X, s=shape) * x.numel()) <= TOL


def test_4d_native_xzwy_vs_cufft(F, torch_cuda):
    torch = torch_cuda
    d = (64, 64, 64, 64)
    x = torch.from_numpy(np.random.default_rng(1).standard_normal(d).astype(np.float32)).cuda()
    f = F.ffts("float32", strategy_4d="native_xzwy").init(*d)
    X = torch.empty(f.spectrum_shape(), dtype=torch.complex64, device="cuda")
    f.forward(x, X)
    ref = torch.fft.rfftn(x).permute(1, 2, 3, 0)        # [kx][ky][kz][kw] -> [ky][kz][kw][kx]
    assert _rel(X, ref) <= TOL
    y = torch.empty_like(x)
    f.backward(X, y, normalized=True)
    assert _rel(y, x) <= TOL


def test_poisson_256_vs_cufft(F, torch_cuda):
    torch = torch_cuda
    n = 256
    g = 2 * np.pi * np.arange(n) / n
    rhs = (np.sin(g)[:, None, None] * np.sin(2 * g)[None, :, None] * np.cos(3 * g)[None, None, :]
           + 0.1 * np.random.default_rng(0).uniform(-1, 1, (n, n, n)))
    rhs -= rhs.mean()
    x = torch.from_numpy(rhs.astype(np.float32)).cuda()
    f = F.ffts("float32").init(n, n, n)
    u = torch.empty_like(x)
    f.poisson(x, u, -1.0)
    k = torch.fft.fftfreq(n, 1.0 / n, device="cuda")
    kz = torch.arange(n // 2 + 1, device="cuda", dtype=torch.float32)
    k2 = k[:, None, None] ** 2 + k[None, :, None] ** 2 + kz[None, None, :] ** 2
    mult = torch.where(k2 == 0, torch.zeros_like(k2), -1.0 / k2)
    ref = torch.fft.irfftn(torch.fft.rfftn(x) * mult, s=(n, n, n))
    assert _rel(u, ref) <= TOL
