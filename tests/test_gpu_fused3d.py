"""GPU parity of the specialised fused 3D path (plane kernels with clusters of 1, 2,
4 and 8 CTAs per plane, x column kernels) against the FP64 oracle, f32 tolerance 2e-6."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu
TOL = 2e-6

# (nx, ny, nz): sizes with a specialised path (the default picks the smallest plane
# cluster that fits: one CTA per plane, two for 256 x 256 planes)
FUSED = [
    (64, 64, 64),
    (256, 64, 64),
    (32, 128, 256),    # nx = 32
    (64, 256, 128),
    (128, 128, 128),
    (256, 128, 64),
    (256, 256, 256),   # 2-CTA clusters, the benchmark size
]
# every plane cluster size, forced
CLUSTERS = [((64, 64, 64), 1), ((64, 64, 64), 2), ((64, 64, 64), 4), ((32, 128, 256), 1), ((32, 128, 256), 2),
            ((32, 128, 256), 4), ((32, 128, 256), 8), ((32, 256, 256), 2), ((32, 256, 256), 4),
            ((32, 256, 256), 8), ((32, 256, 128), 8), ((32, 128, 128), 8)]


@pytest.fixture(scope="module")
def F(torch_cuda):
    from fftm_b200 import build
    build.build()
    import fftm_b200
    return fftm_b200


def _dev(torch, a):
    return torch.tensor(np.ascontiguousarray(a), dtype=torch.float32, device="cuda")


def _host(t):
    import torch
    torch.cuda.synchronize()
    return t.cpu().numpy().astype(np.complex128 if t.is_complex() else np.float64)


@pytest.mark.parametrize("shape", FUSED)
def test_fused_forward_backward(F, torch_cuda, shape):
    torch = torch_cuda
    f = F.ffts("float32").init(*shape)
    assert f.num_launches("forward") == 2 and f.num_launches("poisson") == 3
    x = O.random_3d(*shape, 0x1234ABCDEF987654, single=True)
    xin = _dev(torch, x)
    spec = torch.empty(f.spectrum_shape(), dtype=torch.complex64, device="cuda")
    f.forward(xin, spec)
    ref = O.ffts3d_forward(x)
    assert O.rel_l2(_host(spec), ref) <= TOL
    out = torch.empty_like(xin)
    f.backward(spec, out)
    assert O.rel_l2(_host(out) / x.size, x) <= TOL
    spec2 = torch.tensor(ref, dtype=torch.complex64, device="cuda")
    f.backward(spec2, out, normalized=True)
    assert O.rel_l2(_host(out), x) <= TOL


@pytest.mark.parametrize("shape,cl", CLUSTERS)
def test_every_plane_cluster(F, torch_cuda, shape, cl):
    torch = torch_cuda
    f = F.ffts("float32").init(*shape)
    f.set_strategy("fused", cl)
    assert f.strategy() == ("fused", cl)
    x = O.random_3d(*shape, 77 + cl, single=True)
    spec = torch.empty(f.spectrum_shape(), dtype=torch.complex64, device="cuda")
    f.forward(_dev(torch, x), spec)
    ref = O.ffts3d_forward(x)
    assert O.rel_l2(_host(spec), ref) <= TOL
    out = torch.empty(shape, dtype=torch.float32, device="cuda")
    f.backward(torch.tensor(ref, dtype=torch.complex64, device="cuda"), out, normalized=True)
    assert O.rel_l2(_host(out), x) <= TOL
    f.poisson(_dev(torch, x), out, -1.0)
    assert O.rel_l2(_host(out), O.poisson3d_solve(x, -1.0)) <= TOL


@pytest.mark.parametrize("shape", FUSED)
def test_fused_poisson_and_filter(F, torch_cuda, shape):
    torch = torch_cuda
    f = F.ffts("float32").init(*shape)
    rhs = O.random_3d(*shape, 99, single=True)
    sol = torch.empty(shape, dtype=torch.float32, device="cuda")
    f.poisson(_dev(torch, rhs), sol, -1.0)
    assert O.rel_l2(_host(sol), O.poisson3d_solve(rhs, -1.0)) <= TOL
    f.poisson(_dev(torch, rhs), sol, +1.0)
    assert O.rel_l2(_host(sol), O.poisson3d_solve(rhs, +1.0)) <= TOL
    sigma = 6.0
    f.filter(_dev(torch, rhs), sol, sigma, poisson_sign=-1.0)
    X = O.ffts3d_forward(rhs)
    nx, ny, nz = shape
    kx = np.fft.fftfreq(nx, 1.0 / nx)[:, None, None]
    ky = np.fft.fftfreq(ny, 1.0 / ny)[None, :, None]
    kz = np.arange(nz // 2 + 1)[None, None, :]
    k2 = kx ** 2 + ky ** 2 + kz ** 2
    with np.errstate(divide="ignore", invalid="ignore"):
        P = np.where(k2 == 0, 0.0, -1.0 / k2)
    ref = O.ffts3d_backward(X * np.exp(-k2 / (2 * sigma ** 2)) * P, nz) / rhs.size
    assert O.rel_l2(_host(sol), ref) <= TOL


def test_fused_poisson_manufactured_256(F, torch_cuda):
    torch = torch_cuda
    n = 256
    g = 2 * np.pi * np.arange(n) / n
    u = (np.sin(g)[:, None, None] * np.cos(2 * g)[None, :, None] * np.sin(3 * g)[None, None, :])
    f = F.ffts("float32").init(n, n, n)
    sol = torch.empty((n, n, n), dtype=torch.float32, device="cuda")
    f.poisson(_dev(torch, 14 * u), sol, +1.0)
    assert O.rel_l2(_host(sol), u) <= TOL


def test_fused_round_trip_criterion_256(F, torch_cuda):
    # the reference benchmarks' pin: RMS(C2R(R2C(x))/N - x) <= 10 eps_f32
    torch = torch_cuda
    shape = (256, 256, 256)
    f = F.ffts("float32").init(*shape)
    x = torch.rand(shape, device="cuda") * 2 - 1
    spec = torch.empty(f.spectrum_shape(), dtype=torch.complex64, device="cuda")
    out = torch.empty_like(x)
    f.forward(x, spec)
    f.backward(spec, out, normalized=True)
    rms = torch.sqrt(torch.mean((out - x) ** 2)).item()
    assert rms <= 10 * np.finfo(np.float32).eps


TC_TOL = 5e-6


@pytest.mark.parametrize("shape", [(64, 64, 64), (32, 128, 256), (128, 128, 64), (256, 256, 256)])
def test_fused_tensor_core_form(F, torch_cuda, shape):
    """Split-FP16 tensor-core x column kernel: relative L2 vs the FP64 oracle <= 5e-6."""
    torch = torch_cuda
    f = F.ffts("float32").init(*shape)
    f.set_strategy("fused_tc")
    assert f.strategy()[0] == "fused_tc"
    x = O.random_3d(*shape, 0x5EED, single=True)
    spec = torch.empty(f.spectrum_shape(), dtype=torch.complex64, device="cuda")
    f.forward(_dev(torch, x), spec)
    err_f = O.rel_l2(_host(spec), O.ffts3d_forward(x))
    out = torch.empty(shape, dtype=torch.float32, device="cuda")
    f.backward(spec, out, normalized=True)
    err_rt = O.rel_l2(_host(out), x)
    f.poisson(_dev(torch, x), out, -1.0)
    err_p = O.rel_l2(_host(out), O.poisson3d_solve(x, -1.0))
    print(f"tensor-core form {shape}: forward {err_f:.2e}, round trip {err_rt:.2e}, Poisson {err_p:.2e}")
    assert err_f <= TC_TOL and err_rt <= TC_TOL and err_p <= TC_TOL


def _offset(torch, n, dtype, shape):
    """A contiguous tensor of `shape` that starts one element past a 16-byte boundary."""
    buf = torch.empty(n + 4, dtype=dtype, device="cuda")
    t = buf[1:1 + n].view(shape)
    assert t.data_ptr() % 16 != 0
    return t


@pytest.mark.parametrize("shape", [(64, 64, 64), (128, 64, 128), (256, 256, 256)])
def test_fused_unaligned_buffers(F, torch_cuda, shape):
    """User buffers that start 4 (real) or 8 (complex) bytes past a 16-byte boundary: the
    kernels take their staged paths instead of bulk and tensor copies, with the same results."""
    torch = torch_cuda
    nx, ny, nz = shape
    n, nh = nx * ny * nz, nx * ny * (nz // 2 + 1)
    x = O.random_3d(*shape, 21, single=True)
    f = F.ffts("float32").init(*shape)
    xin = _offset(torch, n, torch.float32, shape)
    xin.copy_(_dev(torch, x))
    spec = _offset(torch, nh, torch.complex64, (nx, ny, nz // 2 + 1))
    out = _offset(torch, n, torch.float32, shape)
    f.forward(xin, spec)
    assert O.rel_l2(_host(spec), O.ffts3d_forward(x.astype(np.float64))) <= TOL
    f.backward(spec, out, normalized=True)
    assert O.rel_l2(_host(out), x) <= TOL
    f.poisson(xin, out, -1.0)
    assert O.rel_l2(_host(out), O.poisson3d_solve(x.astype(np.float64), -1.0)) <= TOL
