"""GPU tests of the spectral derivative (the reference's derivative_spectra_functor,
source/tests/test_3D_poisson.cu:113-145: multiply by i k with k = index on the half axis
and index or index - n on the full axes): the whole derivative du/d(axis) against the
FP64 oracle pipeline and against analytic derivatives, and the standalone spectrum
multiply on the 2D, 3D and 4D layouts against numpy."""
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


def _k(n, half=False):
    i = np.arange(n // 2 + 1 if half else n)
    return i.astype(np.float64) if half else np.where(i <= n // 2, i, i - n).astype(np.float64)


def _oracle_derivative(u, axis):
    nx, ny, nz = u.shape
    X = O.ffts3d_forward(u)
    k = [_k(nx)[:, None, None], _k(ny)[None, :, None], _k(nz, True)[None, None, :]][axis]
    return O.ffts3d_backward(1j * k * X, nz) / u.size


@pytest.mark.parametrize("dtype,shape", [("float32", (64, 64, 64)), ("float32", (24, 20, 18)),
                                         ("float64", (16, 12, 10)), ("float32", (32, 128, 256))])
def test_derivative_vs_oracle(F, torch_cuda, dtype, shape):
    torch = torch_cuda
    rt = torch.float32 if dtype == "float32" else torch.float64
    tol = 2e-6 if dtype == "float32" else 1e-12
    u = O.random_3d(*shape, 17, single=(dtype == "float32"))
    f = F.ffts(dtype).init(*shape)
    ud = torch.tensor(u, dtype=rt, device="cuda")
    out = torch.empty_like(ud)
    for axis in range(3):
        f.derivative(ud, out, axis)
        torch.cuda.synchronize()
        got = out.cpu().numpy().astype(np.float64)
        assert O.rel_l2(got, _oracle_derivative(u.astype(np.float64), axis)) <= tol, axis


@pytest.mark.parametrize("dtype", ["float32", "float64"])
def test_derivative_analytic(F, torch_cuda, dtype):
    torch = torch_cuda
    n = 32
    g = 2 * np.pi * np.arange(n) / n
    x, y, z = np.meshgrid(g, g, g, indexing="ij")
    u = np.sin(x) * np.cos(2 * y) * np.sin(3 * z)
    exact = [np.cos(x) * np.cos(2 * y) * np.sin(3 * z), -2 * np.sin(x) * np.sin(2 * y) * np.sin(3 * z),
             3 * np.sin(x) * np.cos(2 * y) * np.cos(3 * z)]
    rt = torch.float32 if dtype == "float32" else torch.float64
    f = F.ffts(dtype).init(n, n, n)
    ud = torch.tensor(u, dtype=rt, device="cuda")
    out = torch.empty_like(ud)
    for axis in range(3):
        f.derivative(ud, out, axis)
        torch.cuda.synchronize()
        err = O.rel_l2(out.cpu().numpy().astype(np.float64), exact[axis])
        assert err <= (2e-6 if dtype == "float32" else 1e-12), (axis, err)


@pytest.mark.parametrize("dims,layout", [((12, 20), "pencil"), ((8, 6, 10, 12), "native_xzwy"),
                                         ((8, 6, 10, 12), "slab"), ((8, 6, 10, 12), "pencil")])
def test_spectrum_derivative_layouts(F, torch_cuda, dims, layout):
    torch = torch_cuda
    f = F.ffts("float64", strategy_4d=layout).init(*dims)
    rng = np.random.default_rng(5)
    X = rng.standard_normal(f.spectrum_shape()) + 1j * rng.standard_normal(f.spectrum_shape())
    Xd = torch.tensor(X, dtype=torch.complex128, device="cuda")
    out = torch.empty_like(Xd)
    d = len(dims)
    # logical axis -> (physical axis of the spectrum, its length n, half axis?)
    if d == 2:
        phys = {0: (0, dims[0], False), 1: (1, dims[1], True)}
    elif layout == "slab":
        phys = {0: (0, dims[0], False), 1: (1, dims[1], False), 2: (2, dims[2], False), 3: (3, dims[3], True)}
    else:  # [ky][kz][kw][kx]
        phys = {0: (3, dims[0], False), 1: (0, dims[1], False), 2: (1, dims[2], False), 3: (2, dims[3], True)}
    for axis in range(d):
        f.spectrum_derivative(Xd, out, axis, 0.5)
        torch.cuda.synchronize()
        p, n, half = phys[axis]
        shape = [1] * d
        shape[p] = -1
        ref = 0.5j * _k(n, half).reshape(shape) * X
        assert O.rel_l2(out.cpu().numpy(), ref) <= 1e-14, axis


@pytest.mark.parametrize("dims,layout", [((24, 18, 30), "pencil"), ((8, 6, 10, 12), "native_xzwy"),
                                         ((12, 20), "pencil")])
@pytest.mark.parametrize("rule,cutoff", [("two_thirds", 0), ("box", 3), ("box", 0)])
def test_spectrum_truncate(F, torch_cuda, dims, layout, rule, cutoff):
    torch = torch_cuda
    f = F.ffts("float32", strategy_4d=layout).init(*dims)
    rng = np.random.default_rng(9)
    X = (rng.standard_normal(f.spectrum_shape()) + 1j * rng.standard_normal(f.spectrum_shape())).astype(np.complex64)
    Xd = torch.tensor(X, device="cuda")
    f.spectrum_truncate(Xd, rule, cutoff)
    torch.cuda.synchronize()
    d = len(dims)
    if d == 2:
        axes = [(0, dims[0], False), (1, dims[1], True)]
    elif d == 3:
        axes = [(0, dims[0], False), (1, dims[1], False), (2, dims[2], True)]
    else:  # [ky][kz][kw][kx]
        axes = [(3, dims[0], False), (0, dims[1], False), (1, dims[2], False), (2, dims[3], True)]
    keep = np.ones(f.spectrum_shape(), bool)
    for p, n, half in axes:
        shape = [1] * d
        shape[p] = -1
        ak = np.abs(_k(n, half)).reshape(shape)
        if rule == "two_thirds":
            keep &= ak <= n // 3
        elif cutoff > 0:
            keep &= ak <= cutoff
    np.testing.assert_array_equal(Xd.cpu().numpy(), np.where(keep, X, 0))


@pytest.mark.parametrize("dtype,shape,layout", [("float32", (64, 64, 64), "pencil"), ("float64", (15, 12, 17), "pencil"),
                                                ("float64", (6, 8, 10, 12), "native_xzwy")])
def test_gradient_matches_derivatives(F, torch_cuda, dtype, shape, layout):
    torch = torch_cuda
    rt = torch.float32 if dtype == "float32" else torch.float64
    f = F.ffts(dtype, strategy_4d=layout).init(*shape)
    u = torch.randn(f.real_shape(), dtype=rt, device="cuda")
    outs = [torch.empty_like(u) for _ in shape]
    f.gradient(u, outs)
    tol = 2e-6 if dtype == "float32" else 1e-12
    for a in range(len(shape)):
        ref = torch.empty_like(u)
        f.derivative(u, ref, a)       # on the fused path the multiply rides in the column pass
        torch.cuda.synchronize()
        err = float(torch.linalg.norm((outs[a] - ref).double()) / torch.linalg.norm(ref.double()))
        assert err <= tol, (a, err)


@pytest.mark.parametrize("shape", [(64, 64, 64), (32, 128, 256), (24, 20, 18)])
def test_gradient_vs_oracle_fused_and_staged(F, torch_cuda, shape):
    # the fused gradient (planes' R2C once, per axis the column sandwich with i k into a
    # second buffer and the inverse planes) and the staged one, both against the oracle
    torch = torch_cuda
    u = O.random_3d(*shape, 29, single=True)
    ud = torch.tensor(u, dtype=torch.float32, device="cuda")
    for strategy in ("auto", "staged"):
        f = F.ffts("float32").init(*shape)
        f.set_strategy(strategy)
        outs = [torch.empty_like(ud) for _ in range(3)]
        f.gradient(ud, outs)
        torch.cuda.synchronize()
        for a in range(3):
            got = outs[a].cpu().numpy().astype(np.float64)
            assert O.rel_l2(got, _oracle_derivative(u.astype(np.float64), a)) <= 2e-6, (strategy, a)
