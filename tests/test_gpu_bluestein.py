"""GPU parity of the chirp-z (Bluestein) passes, which cover every line length up to
4096 that the radix kernels do not (large prime factors): 1D plans in both directions,
3D / 2D / 4D ffts with such axes (R2C on odd lengths and on even lengths whose half is
not covered, C2R with the Hermitian extension), the Poisson solve, and a batch that
contains such a shape.  Against numpy's FP64 FFT and the FP64 oracle."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def F(torch_cuda):
    from fftm_b200 import build
    build.build()
    import fftm_b200
    return fftm_b200


def _tol(dtype):
    return 2e-6 if dtype == "float32" else 1e-11


@pytest.mark.parametrize("dtype", ["float32", "float64"])
@pytest.mark.parametrize("n", [17, 19, 34, 97, 101, 257, 1009, 2310, 4093])
def test_1d_c2c_plans(F, torch_cuda, dtype, n):
    torch = torch_cuda
    ct = torch.complex64 if dtype == "float32" else torch.complex128
    batch = 6
    rng = np.random.default_rng(n)
    x = rng.standard_normal((batch, n)) + 1j * rng.standard_normal((batch, n))
    xd = torch.tensor(x, dtype=ct, device="cuda")
    X = torch.empty_like(xd)
    p = F.Plan(F.C2CF, [n], [n], 1, n, [n], 1, n, batch, dtype=dtype)
    p.exec(xd, X)
    torch.cuda.synchronize()
    assert O.rel_l2(X.cpu().numpy(), np.fft.fft(x, axis=1)) <= _tol(dtype)
    pi = F.Plan(F.C2CB, [n], [n], 1, n, [n], 1, n, batch, dtype=dtype)
    y = torch.empty_like(xd)
    pi.exec(X, y)
    torch.cuda.synchronize()
    assert O.rel_l2(y.cpu().numpy() / n, x) <= _tol(dtype)


@pytest.mark.parametrize("dtype,shape", [("float32", (17, 19, 23)), ("float64", (17, 19, 23)),
                                         ("float32", (34, 22, 26)), ("float32", (96, 17, 34)),
                                         ("float64", (11, 13, 38))])
def test_3d_prime_axes_vs_oracle(F, torch_cuda, dtype, shape):
    torch = torch_cuda
    rt = torch.float32 if dtype == "float32" else torch.float64
    ct = torch.complex64 if dtype == "float32" else torch.complex128
    x = O.random_3d(*shape, 23, single=(dtype == "float32"))
    f = F.ffts(dtype).init(*shape)
    xd = torch.tensor(x, dtype=rt, device="cuda")
    X = torch.empty(f.spectrum_shape(), dtype=ct, device="cuda")
    f.forward(xd, X)
    torch.cuda.synchronize()
    ref = O.ffts3d_forward(x.astype(np.float64))
    assert O.rel_l2(X.cpu().numpy(), ref) <= _tol(dtype)
    out = torch.empty_like(xd)
    f.backward(torch.tensor(ref, dtype=ct, device="cuda"), out, normalized=True)
    torch.cuda.synchronize()
    assert O.rel_l2(out.cpu().numpy(), x) <= _tol(dtype)
    f.poisson(xd, out, -1.0)
    torch.cuda.synchronize()
    assert O.rel_l2(out.cpu().numpy(), O.poisson3d_solve(x.astype(np.float64), -1.0)) <= _tol(dtype)


def test_2d_and_4d_prime_axes(F, torch_cuda):
    torch = torch_cuda
    # 2D with an odd prime R2C axis and an even length whose half is prime
    for dims in [(19, 17), (38, 34)]:
        f = F.ffts("float64").init(*dims)
        x = np.random.default_rng(1).standard_normal(dims)
        X = torch.empty(f.spectrum_shape(), dtype=torch.complex128, device="cuda")
        f.forward(torch.tensor(x, device="cuda"), X)
        torch.cuda.synchronize()
        assert O.rel_l2(X.cpu().numpy(), np.fft.rfftn(x)) <= 1e-11
    # 4D native_xzwy with prime axes
    dims = (6, 17, 5, 19)
    f = F.ffts("float64", strategy_4d="native_xzwy").init(*dims)
    x = O.random_4d(*dims, 3, layout=O.NATIVE_XZWY)
    X = torch.empty(f.spectrum_shape(), dtype=torch.complex128, device="cuda")
    f.forward(torch.tensor(x, device="cuda"), X)
    torch.cuda.synchronize()
    assert O.rel_l2(X.cpu().numpy(), O.ffts4d_forward(O.NATIVE_XZWY, x, dims)) <= 1e-11


def test_batch_with_prime_shape(F, torch_cuda):
    torch = torch_cuda
    import fftm_b200.batch as B
    shapes = [(32, 48, 64), (17, 20, 23), (64, 64, 32)]
    b = B.Batch(shapes)
    x = torch.rand(b.real_total, device="cuda") * 2 - 1
    out = torch.zeros_like(x)
    b.exec(B.ROUNDTRIP, x, out)       # falls back to sequential launches for the chirp-z passes
    torch.cuda.synchronize()
    for i, s in enumerate(shapes):
        o = b.real_offsets[i]
        n = int(np.prod(s))
        assert O.rel_l2(out[o:o + n].cpu().numpy(), x[o:o + n].cpu().numpy()) <= 2e-6
