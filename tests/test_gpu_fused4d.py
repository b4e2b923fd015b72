"""GPU parity of the specialised 4D path (slab and native_xzwy; (z,w) plane kernels,
batched y and x column kernels, transposed x pass for native_xzwy) against the FP64
oracle, f32 tolerance 2e-6."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu
TOL = 2e-6
LAYOUTS = [("slab", O.SLAB), ("native_xzwy", O.NATIVE_XZWY)]
FUSED4 = [(32, 32, 64, 64), (64, 32, 64, 128), (32, 64, 128, 64), (64, 64, 64, 64)]


@pytest.fixture(scope="module")
def F(torch_cuda):
    from fftm_b200 import build
    build.build()
    import fftm_b200
    return fftm_b200


def _dev(torch, a, dt=None):
    return torch.tensor(np.ascontiguousarray(a), dtype=dt or torch.float32, device="cuda")


def _host(t):
    import torch
    torch.cuda.synchronize()
    return t.cpu().numpy().astype(np.complex128 if t.is_complex() else np.float64)


@pytest.mark.parametrize("name,layout", LAYOUTS)
@pytest.mark.parametrize("dims", FUSED4)
def test_fused4d_forward_backward(F, torch_cuda, name, layout, dims):
    torch = torch_cuda
    f = F.ffts("float32", strategy_4d=name).init(*dims)
    assert f.num_launches("forward") == 3 and f.num_launches("poisson") == 5
    x = O.random_4d(*dims, 1, layout=layout, single=True)
    xin = _dev(torch, x)
    spec = torch.empty(f.spectrum_shape(), dtype=torch.complex64, device="cuda")
    f.forward(xin, spec)
    ref = O.ffts4d_forward(layout, x, dims)
    assert O.rel_l2(_host(spec), ref) <= TOL
    out = torch.empty_like(xin)
    f.backward(spec, out)
    assert O.rel_l2(_host(out) / x.size, x) <= TOL
    f.backward(_dev(torch, ref, torch.complex64), out, normalized=True)
    assert O.rel_l2(_host(out), x) <= TOL


@pytest.mark.parametrize("name,layout", LAYOUTS)
@pytest.mark.parametrize("dims", FUSED4[:3])
def test_fused4d_poisson_filter(F, torch_cuda, name, layout, dims):
    torch = torch_cuda
    f = F.ffts("float32", strategy_4d=name).init(*dims)
    rhs = O.random_4d(*dims, 7, layout=layout, single=True)
    sol = torch.empty(rhs.shape, dtype=torch.float32, device="cuda")
    for sign in (-1.0, 1.0):
        f.poisson(_dev(torch, rhs), sol, sign)
        assert O.rel_l2(_host(sol), O.poisson4d_solve(layout, rhs, dims, sign)) <= TOL
    sigma = 5.0
    f.filter(_dev(torch, rhs), sol, sigma, poisson_sign=-1.0)
    nx, ny, nz, nw = dims
    X = O.ffts4d_forward(O.SLAB, rhs, dims)        # [kx][ky][kz][kw]
    kx = np.fft.fftfreq(nx, 1.0 / nx)[:, None, None, None]
    ky = np.fft.fftfreq(ny, 1.0 / ny)[None, :, None, None]
    kz = np.fft.fftfreq(nz, 1.0 / nz)[None, None, :, None]
    kw = np.arange(nw // 2 + 1)[None, None, None, :]
    k2 = kx ** 2 + ky ** 2 + kz ** 2 + kw ** 2
    with np.errstate(divide="ignore", invalid="ignore"):
        P = np.where(k2 == 0, 0.0, -1.0 / k2)
    ref = O.ffts4d_backward(O.SLAB, X * np.exp(-k2 / (2 * sigma ** 2)) * P, dims) / rhs.size
    assert O.rel_l2(_host(sol), ref) <= TOL


def test_fused4d_poisson_manufactured_64(F, torch_cuda):
    torch = torch_cuda
    dims = (64, 64, 64, 64)
    g = [2 * np.pi * np.arange(d) / d for d in dims]
    u = (np.sin(g[0])[:, None, None, None] * np.cos(2 * g[1])[None, :, None, None] *
         np.sin(3 * g[2])[None, None, :, None] * np.cos(g[3])[None, None, None, :])
    for name in ("slab", "native_xzwy"):
        f = F.ffts("float32", strategy_4d=name).init(*dims)
        sol = torch.empty(dims, dtype=torch.float32, device="cuda")
        f.poisson(_dev(torch, 15 * u), sol, +1.0)
        assert O.rel_l2(_host(sol), u) <= TOL


TC_TOL = 5e-6


@pytest.mark.parametrize("dims", [(32, 64, 128, 64), (64, 64, 64, 64)])
def test_fused4d_tensor_core_form(F, torch_cuda, dims):
    """Split-FP16 tensor-core column kernels: relative L2 vs the FP64 oracle <= 5e-6."""
    torch = torch_cuda
    f = F.ffts("float32", strategy_4d="native_xzwy").init(*dims)
    f.set_strategy("fused_tc")
    assert f.strategy()[0] == "fused_tc"
    x = O.random_4d(*dims, 1, layout=O.NATIVE_XZWY, single=True)
    spec = torch.empty(f.spectrum_shape(), dtype=torch.complex64, device="cuda")
    f.forward(_dev(torch, x), spec)
    err_f = O.rel_l2(_host(spec), O.ffts4d_forward(O.NATIVE_XZWY, x, dims))
    out = torch.empty(f.real_shape(), dtype=torch.float32, device="cuda")
    f.backward(spec, out, normalized=True)
    err_rt = O.rel_l2(_host(out), x)
    f.poisson(_dev(torch, x), out, -1.0)
    err_p = O.rel_l2(_host(out), O.poisson4d_solve(O.NATIVE_XZWY, x, dims, -1.0))
    print(f"tensor-core form {dims}: forward {err_f:.2e}, round trip {err_rt:.2e}, Poisson {err_p:.2e}")
    assert err_f <= TC_TOL and err_rt <= TC_TOL and err_p <= TC_TOL


def test_fused4d_unaligned_buffers(F, torch_cuda):
    """64^4 native_xzwy with user buffers one element past a 16-byte boundary (the plane
    kernels' and column kernels' staged paths)."""
    torch = torch_cuda
    dims = (64, 64, 64, 64)
    f = F.ffts("float32", strategy_4d="native_xzwy").init(*dims)
    x = O.random_4d(*dims, 23, layout=O.NATIVE_XZWY, single=True)
    n = x.size
    rb = torch.empty(n + 4, dtype=torch.float32, device="cuda")
    xin = rb[1:1 + n].view(x.shape)
    xin.copy_(_dev(torch, x))
    sshape = f.spectrum_shape()
    ns = int(np.prod(sshape))
    sb = torch.empty(ns + 2, dtype=torch.complex64, device="cuda")
    spec = sb[1:1 + ns].view(sshape)
    ob = torch.empty(n + 4, dtype=torch.float32, device="cuda")
    out = ob[1:1 + n].view(x.shape)
    assert xin.data_ptr() % 16 and spec.data_ptr() % 16 and out.data_ptr() % 16
    f.forward(xin, spec)
    assert O.rel_l2(_host(spec), O.ffts4d_forward(O.NATIVE_XZWY, x, dims)) <= TOL
    f.backward(spec, out, normalized=True)
    assert O.rel_l2(_host(out), x) <= TOL
