"""GPU parity of lines longer than 4096 points (the reference's cuFFT plans take any
length, source/external_wrap/fft_wrap_many.h:137-186): the four-step long-line step
(n = L1 * L2, both pass-kernel lengths) and, for a large prime factor, chirp-z over a
power-of-two four-step convolution.  1D C2C plans both ways and R2C / C2R plans against
numpy's FP64 FFT, strided batches, and 3D ffts with a long axis against the FP64 oracle.
Tolerances: 2e-6 (f32) for the four-step form; the chirp-z form in f32 carries the
rounding of its two length-M convolution FFTs and is held to 5e-6; 1e-11 in f64."""
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


CHIRP = {10007, 8191 * 2, 4099}


def _tol(dtype, n):
    if dtype == "float64":
        return 1e-11
    return 5e-6 if n in CHIRP else 2e-6


@pytest.mark.parametrize("dtype", ["float32", "float64"])
@pytest.mark.parametrize("n", [8192, 3 * 4096, 5000, 10007, 4099])
def test_1d_c2c_long_lines(F, torch_cuda, dtype, n):
    torch = torch_cuda
    ct = torch.complex64 if dtype == "float32" else torch.complex128
    batch = 3
    rng = np.random.default_rng(n)
    x = rng.standard_normal((batch, n)) + 1j * rng.standard_normal((batch, n))
    xd = torch.tensor(x, dtype=ct, device="cuda")
    X = torch.empty_like(xd)
    p = F.Plan(F.C2CF, [n], [n], 1, n, [n], 1, n, batch, dtype=dtype)
    p.exec(xd, X)
    torch.cuda.synchronize()
    assert O.rel_l2(X.cpu().numpy(), np.fft.fft(x, axis=1)) <= _tol(dtype, n)
    pi = F.Plan(F.C2CB, [n], [n], 1, n, [n], 1, n, batch, dtype=dtype)
    y = torch.empty_like(xd)
    pi.exec(X, y)
    torch.cuda.synchronize()
    assert O.rel_l2(y.cpu().numpy() / n, x) <= _tol(dtype, n)


@pytest.mark.parametrize("dtype", ["float32", "float64"])
@pytest.mark.parametrize("n", [16384, 12000, 10007, 8191 * 2])
def test_r2c_c2r_long_lines(F, torch_cuda, dtype, n):
    torch = torch_cuda
    rt = torch.float32 if dtype == "float32" else torch.float64
    ct = torch.complex64 if dtype == "float32" else torch.complex128
    batch = 2
    nh = n // 2 + 1
    x = np.random.default_rng(n + 1).uniform(-1, 1, (batch, n))
    xd = torch.tensor(x, dtype=rt, device="cuda")
    X = torch.empty((batch, nh), dtype=ct, device="cuda")
    F.Plan(F.R2C, [n], [n], 1, n, [nh], 1, nh, batch, dtype=dtype).exec(xd, X)
    torch.cuda.synchronize()
    assert O.rel_l2(X.cpu().numpy(), np.fft.rfft(x, axis=1)) <= _tol(dtype, n)
    y = torch.empty_like(xd)
    F.Plan(F.C2R, [n], [nh], 1, nh, [n], 1, n, batch, dtype=dtype).exec(X, y)
    torch.cuda.synchronize()
    assert O.rel_l2(y.cpu().numpy() / n, x) <= _tol(dtype, n)


def test_strided_batched_long_line(F, torch_cuda):
    # lines of 8192 points with stride 3 and distance 1 (interleaved), as advanced layouts allow
    torch = torch_cuda
    n, batch = 8192, 3
    rng = np.random.default_rng(5)
    x = rng.standard_normal((n, batch)) + 1j * rng.standard_normal((n, batch))
    xd = torch.tensor(x, dtype=torch.complex64, device="cuda")
    X = torch.empty_like(xd)
    F.Plan(F.C2CF, [n], [n], batch, 1, [n], batch, 1, batch, dtype="float32").exec(xd, X)
    torch.cuda.synchronize()
    assert O.rel_l2(X.cpu().numpy(), np.fft.fft(x, axis=0)) <= 2e-6


@pytest.mark.parametrize("dtype,shape", [("float32", (3, 4, 16384)), ("float64", (2, 3, 12288)),
                                         ("float32", (10000, 2, 4))])
def test_3d_ffts_with_a_long_axis_vs_oracle(F, torch_cuda, dtype, shape):
    torch = torch_cuda
    rt = torch.float32 if dtype == "float32" else torch.float64
    ct = torch.complex64 if dtype == "float32" else torch.complex128
    x = O.random_3d(*shape, 31, single=(dtype == "float32"))
    f = F.ffts(dtype).init(*shape)
    xd = torch.tensor(x, dtype=rt, device="cuda")
    X = torch.empty(f.spectrum_shape(), dtype=ct, device="cuda")
    f.forward(xd, X)
    torch.cuda.synchronize()
    tol = 2e-6 if dtype == "float32" else 1e-11
    assert O.rel_l2(X.cpu().numpy(), O.ffts3d_forward(x.astype(np.float64))) <= tol
    y = torch.empty_like(xd)
    f.backward(X.clone(), y)
    torch.cuda.synchronize()
    assert O.rel_l2(y.cpu().numpy() / x.size, x) <= tol


@pytest.mark.parametrize("shape,tol", [((10000, 2, 4), 2e-6), ((4, 3, 10007), 5e-6)])
def test_poisson_with_a_long_axis_vs_oracle(F, torch_cuda, shape, tol):
    # a long x axis runs the sandwich (forward, -1/|k|^2, inverse) on the long line; a long
    # prime z axis runs chirp-z R2C / C2R
    torch = torch_cuda
    x = O.random_3d(*shape, 41, single=True)
    f = F.ffts("float32").init(*shape)
    xd = torch.tensor(x, dtype=torch.float32, device="cuda")
    u = torch.empty_like(xd)
    f.poisson(xd, u, -1.0)
    torch.cuda.synchronize()
    assert O.rel_l2(u.cpu().numpy(), O.poisson3d_solve(x.astype(np.float64), -1.0)) <= tol
