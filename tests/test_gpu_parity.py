"""GPU parity tests: the CUDA library (through the C ABI) against the FP64 oracle.

Tolerances (relative L2 against the FP64 oracle): float32 <= 2e-6, float64 <= 1e-12.
"""
import os

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

TOL = {"float32": 2e-6, "float64": 1e-12}
GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden_small.npz"))


@pytest.fixture(scope="module")
def F(torch_cuda):
    from fftm_b200 import build
    build.build()
    import fftm_b200
    return fftm_b200


def dev_real(torch, a, dtype):
    return torch.tensor(np.ascontiguousarray(a), dtype=getattr(torch, dtype), device="cuda")


def dev_cplx(torch, a, dtype):
    ct = torch.complex64 if dtype == "float32" else torch.complex128
    return torch.tensor(np.ascontiguousarray(a), dtype=ct, device="cuda")


def empty_c(torch, shape, dtype):
    ct = torch.complex64 if dtype == "float32" else torch.complex128
    return torch.empty(shape, dtype=ct, device="cuda")


def host(t):
    t.device.type == "cuda" and __import__("torch").cuda.synchronize()
    return t.detach().cpu().numpy().astype(np.complex128 if t.is_complex() else np.float64)


SHAPES_3D = [(8, 8, 8), (6, 10, 12), (5, 7, 9), (16, 12, 10), (32, 32, 32), (64, 64, 64), (48, 96, 32),
             (4, 2, 2), (1, 8, 16), (3, 5, 7)]


@pytest.mark.parametrize("dtype", ["float32", "float64"])
@pytest.mark.parametrize("shape", SHAPES_3D)
def test_ffts3d_forward_backward(F, torch_cuda, dtype, shape):
    torch = torch_cuda
    x = O.random_3d(*shape, 0x1234ABCDEF987654, single=(dtype == "float32"))
    f = F.ffts(dtype).init(*shape)
    xin = dev_real(torch, x, dtype)
    spec = empty_c(torch, f.spectrum_shape(), dtype)
    f.forward(xin, spec)
    ref = O.ffts3d_forward(x)
    assert O.rel_l2(host(spec), ref) <= TOL[dtype]
    out = torch.empty_like(xin)
    f.backward(spec, out)
    assert O.rel_l2(host(out) / x.size, x) <= TOL[dtype]
    # normalised variant (1/N fused into the last pass)
    spec2 = dev_cplx(torch, ref, dtype)
    f.backward(spec2, out, normalized=True)
    assert O.rel_l2(host(out), O.ffts3d_backward(ref, shape[2]) / x.size) <= TOL[dtype]


@pytest.mark.parametrize("shape", [(8, 8, 8), (6, 10, 12), (5, 7, 9), (16, 12, 10)])
def test_ffts3d_against_golden_fixture(F, torch_cuda, shape):
    torch = torch_cuda
    key = "r3d_" + "x".join(map(str, shape))
    f = F.ffts("float64").init(*shape)
    spec = empty_c(torch, f.spectrum_shape(), "float64")
    f.forward(dev_real(torch, GOLD[key + "_in"], "float64"), spec)
    assert O.rel_l2(host(spec), GOLD[key + "_spec"]) <= 1e-13


@pytest.mark.parametrize("dtype", ["float32", "float64"])
@pytest.mark.parametrize("shape", [(12, 20), (16, 16), (7, 9), (64, 128)])
def test_ffts2d(F, torch_cuda, dtype, shape):
    torch = torch_cuda
    rng = np.random.default_rng(1)
    x = rng.uniform(-1, 1, shape)
    f = F.ffts(dtype).init(*shape)
    spec = empty_c(torch, f.spectrum_shape(), dtype)
    f.forward(dev_real(torch, x, dtype), spec)
    ref = O.ffts2d_forward(x)
    assert O.rel_l2(host(spec), ref) <= TOL[dtype]
    out = dev_real(torch, np.zeros(shape), dtype)
    f.backward(spec, out, normalized=True)
    assert O.rel_l2(host(out), x) <= TOL[dtype]


LAYOUTS = [("pencil", O.PENCIL), ("slab", O.SLAB), ("native_xzwy", O.NATIVE_XZWY)]


@pytest.mark.parametrize("dtype", ["float32", "float64"])
@pytest.mark.parametrize("name,layout", LAYOUTS)
@pytest.mark.parametrize("dims", [(6, 4, 8, 10), (8, 8, 8, 8), (16, 12, 10, 6), (5, 3, 7, 9)])
def test_ffts4d_layouts(F, torch_cuda, dtype, name, layout, dims):
    torch = torch_cuda
    x = O.random_4d(*dims, 0xABCDEF0123456789, layout=layout, single=(dtype == "float32"))
    f = F.ffts(dtype, strategy_4d=name).init(*dims)
    assert f.real_shape() == x.shape
    xin = dev_real(torch, x, dtype)
    spec = empty_c(torch, f.spectrum_shape(), dtype)
    f.forward(xin, spec)
    ref = O.ffts4d_forward(layout, x, dims)
    assert O.rel_l2(host(spec), ref) <= TOL[dtype]
    out = torch.empty_like(xin)
    f.backward(spec, out)
    assert O.rel_l2(host(out) / x.size, x) <= TOL[dtype]


def test_ffts4d_golden(F, torch_cuda):
    torch = torch_cuda
    dims = (6, 4, 8, 10)
    xl = GOLD["r4d_in_xyzw"]
    for name, layout in LAYOUTS:
        x = np.ascontiguousarray(xl.transpose(3, 2, 1, 0)) if layout == O.PENCIL else xl
        f = F.ffts("float64", strategy_4d=name).init(*dims)
        spec = empty_c(torch, f.spectrum_shape(), "float64")
        f.forward(dev_real(torch, x, "float64"), spec)
        ref = GOLD["r4d_spec_slab"] if layout == O.SLAB else GOLD["r4d_spec_yzwx"]
        assert O.rel_l2(host(spec), ref) <= 1e-13


def _grid(n):
    return 2 * np.pi * np.arange(n) / n


@pytest.mark.parametrize("dtype", ["float32", "float64"])
def test_poisson3d_manufactured(F, torch_cuda, dtype):
    torch = torch_cuda
    n = 32
    x, y, z = np.meshgrid(_grid(n), _grid(n), _grid(n), indexing="ij")
    u = np.sin(x) * np.cos(2 * y) * np.sin(3 * z)
    f = F.ffts(dtype).init(n, n, n)
    sol = dev_real(torch, np.zeros_like(u), dtype)
    f.poisson(dev_real(torch, 14 * u, dtype), sol, sign=+1.0)
    tol = 1e-10 if dtype == "float64" else 2e-6
    assert O.rel_l2(host(sol), u) <= tol


@pytest.mark.parametrize("dtype", ["float32", "float64"])
@pytest.mark.parametrize("shape", [(16, 12, 10), (32, 32, 32), (9, 6, 5)])
def test_poisson3d_random_vs_oracle(F, torch_cuda, dtype, shape):
    torch = torch_cuda
    rhs = O.random_3d(*shape, 77, single=(dtype == "float32"))
    f = F.ffts(dtype).init(*shape)
    sol = dev_real(torch, np.zeros(shape), dtype)
    f.poisson(dev_real(torch, rhs, dtype), sol, sign=-1.0)
    assert O.rel_l2(host(sol), O.poisson3d_solve(rhs, -1.0)) <= TOL[dtype]
    # aliasing rhs and solution is allowed
    buf = dev_real(torch, rhs, dtype)
    f.poisson(buf, buf, sign=-1.0)
    assert O.rel_l2(host(buf), O.poisson3d_solve(rhs, -1.0)) <= TOL[dtype]


@pytest.mark.parametrize("name,layout", LAYOUTS)
def test_poisson4d_manufactured_and_oracle(F, torch_cuda, name, layout):
    torch = torch_cuda
    dims = (16, 16, 16, 8)
    X, Y, Z, W = np.meshgrid(*[_grid(d) for d in dims], indexing="ij")
    u = np.sin(X) * np.cos(2 * Y) * np.sin(3 * Z) * np.cos(W)
    if layout == O.PENCIL:
        u = np.ascontiguousarray(u.transpose(3, 2, 1, 0))
    f = F.ffts("float64", strategy_4d=name).init(*dims)
    sol = dev_real(torch, np.zeros_like(u), "float64")
    f.poisson(dev_real(torch, 15 * u, "float64"), sol, sign=+1.0)
    assert O.rel_l2(host(sol), u) <= 1e-10
    rhs = O.random_4d(*dims, 9, layout=layout)
    f32 = F.ffts("float32", strategy_4d=name).init(*dims)
    sol32 = dev_real(torch, np.zeros_like(rhs), "float32")
    f32.poisson(dev_real(torch, rhs, "float32"), sol32, sign=-1.0)
    assert O.rel_l2(host(sol32), O.poisson4d_solve(layout, rhs, dims, -1.0)) <= 2e-6


@pytest.mark.parametrize("dtype", ["float32", "float64"])
def test_filter_then_poisson_vs_oracle(F, torch_cuda, dtype):
    torch = torch_cuda
    shape = (32, 24, 16)
    rhs = O.random_3d(*shape, 5, single=(dtype == "float32"))
    sigma = 4.0
    f = F.ffts(dtype).init(*shape)
    out = dev_real(torch, np.zeros(shape), dtype)
    f.filter(dev_real(torch, rhs, dtype), out, sigma, poisson_sign=-1.0)
    X = O.ffts3d_forward(rhs)
    kx = np.fft.fftfreq(shape[0], 1.0 / shape[0])
    ky = np.fft.fftfreq(shape[1], 1.0 / shape[1])
    kz = np.arange(shape[2] // 2 + 1)
    k2 = kx[:, None, None] ** 2 + ky[None, :, None] ** 2 + kz[None, None, :] ** 2
    G = np.exp(-k2 / (2 * sigma ** 2))
    with np.errstate(divide="ignore", invalid="ignore"):
        P = np.where(k2 == 0, 0.0, -1.0 / k2)
    ref = O.ffts3d_backward(X * G * P, shape[2]) / rhs.size
    assert O.rel_l2(host(out), ref) <= TOL[dtype]
    # filter only
    f.filter(dev_real(torch, rhs, dtype), out, sigma)
    ref2 = O.ffts3d_backward(X * G, shape[2]) / rhs.size
    assert O.rel_l2(host(out), ref2) <= TOL[dtype]


def test_spectrum_poisson_standalone(F, torch_cuda):
    torch = torch_cuda
    shape = (12, 10, 8)
    x = O.random_3d(*shape, 3)
    X = O.ffts3d_forward(x)
    f = F.ffts("float64").init(*shape)
    s = dev_cplx(torch, X, "float64")
    f.spectrum_poisson(s, sign=-1.0, scale=0.5)
    assert O.rel_l2(host(s), 0.5 * O.poisson3d(X, shape[2], -1.0)) <= 1e-13
    dims = (6, 4, 8, 10)
    for name, layout in LAYOUTS:
        x4 = O.random_4d(*dims, 4, layout=layout)
        X4 = O.ffts4d_forward(layout, x4, dims)
        f4 = F.ffts("float64", strategy_4d=name).init(*dims)
        s4 = dev_cplx(torch, X4, "float64")
        f4.spectrum_poisson(s4, sign=1.0)
        assert O.rel_l2(host(s4), O.poisson4d(layout, X4, dims, 1.0)) <= 1e-13


# ---------------------------------------------------------------------- plans
def _exec_plan_gpu(F, torch, direction, n, inembed, istride, idist, onembed, ostride, odist, batch, inp, out_size,
                   dtype):
    p = F.Plan(direction, n, inembed, istride, idist, onembed, ostride, odist, batch, dtype)
    if direction == F.R2C:
        xin = dev_real(torch, inp, dtype)
    else:
        xin = dev_cplx(torch, inp, dtype)
    if direction == F.C2R:
        out = dev_real(torch, np.zeros(out_size), dtype)
    else:
        out = empty_c(torch, (out_size,), dtype)
    p.exec(xin, out)
    return host(out), p


@pytest.mark.parametrize("dtype", ["float32", "float64"])
@pytest.mark.parametrize("n", [2, 3, 5, 7, 8, 11, 12, 13, 16, 30, 48, 64, 96, 100, 128, 256, 243, 512, 1024, 2048,
                               4096])
def test_plan_1d_all_directions(F, torch_cuda, dtype, n):
    torch = torch_cuda
    rng = np.random.default_rng(n)
    B = 3
    nh = n // 2 + 1
    x = rng.normal(size=(B, n))
    X, _ = _exec_plan_gpu(F, torch, F.R2C, [n], None, 1, 0, None, 1, 0, B, x.ravel(), B * nh, dtype)
    assert O.rel_l2(X, np.fft.rfft(x, axis=1).ravel()) <= TOL[dtype]
    Y = np.fft.rfft(x, axis=1)
    xb, _ = _exec_plan_gpu(F, torch, F.C2R, [n], None, 1, 0, None, 1, 0, B, Y.ravel(), B * n, dtype)
    assert O.rel_l2(xb / n, x.ravel()) <= TOL[dtype]
    z = rng.normal(size=(B, n)) + 1j * rng.normal(size=(B, n))
    Z, p = _exec_plan_gpu(F, torch, F.C2CF, [n], None, 1, 0, None, 1, 0, B, z.ravel(), B * n, dtype)
    assert O.rel_l2(Z, np.fft.fft(z, axis=1).ravel()) <= TOL[dtype]
    zi = dev_cplx(torch, z.ravel(), dtype)
    zo = empty_c(torch, (B * n,), dtype)
    p.exec_direction(F.C2CB, zi, zo)
    assert O.rel_l2(host(zo), (np.fft.ifft(z, axis=1) * n).ravel()) <= TOL[dtype]


@pytest.mark.parametrize("dtype", ["float32", "float64"])
def test_plan_advanced_layouts_match_oracle(F, torch_cuda, dtype):
    torch = torch_cuda
    rng = np.random.default_rng(11)
    cases = [
        # 4D pencil stage plans (source/ffts.hpp:709-741) at nx,ny,nz,nw = 6,4,5,8
        (F.R2C, [8], [1], 120, 1, [1], 120, 1, 120),
        (F.C2CF, [5], [1], 6 * 4 * 5, 1, [1], 6 * 4 * 5, 1, 6 * 4 * 5),
        (F.C2CB, [6], [6], 1, 6, [6], 1, 6, 4 * 5 * 5),
        # 4D slab plans (source/ffts.hpp:751-775) at nx,ny,nz,nw = 4,6,5,8
        (F.R2C, [5, 8], [5, 8], 1, 40, [5, 5], 1, 25, 24),
        (F.C2R, [5, 8], [5, 5], 1, 25, [5, 8], 1, 40, 24),
        (F.C2CF, [4, 6], [4, 6], 25, 1, [4, 6], 25, 1, 25),
        # native_xzwy plan (source/fftm.hpp:2941-2961) at x,y,z,wh = 4,6,3,5
        (F.C2CF, [6, 4], [6, 4 * 3 * 5], 1, 4, [6, 4 * 3 * 5], 1, 4, 15),
        # 3D with padded embeds, stride 2 and distance
        (F.C2CF, [4, 6, 8], [4, 7, 9], 2, 4 * 7 * 9 * 2 + 3, [4, 6, 8], 1, 192, 2),
        (F.R2C, [4, 6, 8], [4, 6, 10], 1, 240, [4, 6, 5], 1, 120, 2),
    ]
    for d, n, ie, istr, idist, oe, ostr, odist, batch in cases:
        rank = len(n)
        full_in = [n[j] if j < rank - 1 or d != F.C2R else n[j] // 2 + 1 for j in range(rank)]
        in_size = (batch - 1) * idist + 1
        for j in range(rank):
            in_size += (full_in[j] - 1) * istr * int(np.prod(ie[j + 1:]))
        full_out = [n[j] if j < rank - 1 or d != F.R2C else n[j] // 2 + 1 for j in range(rank)]
        out_size = (batch - 1) * odist + 1
        for j in range(rank):
            out_size += (full_out[j] - 1) * ostr * int(np.prod(oe[j + 1:]))
        if d == F.R2C:
            inp = rng.normal(size=in_size)
        else:
            inp = rng.normal(size=in_size) + 1j * rng.normal(size=in_size)
        ref = O.exec_plan(d, n, ie, istr, idist, oe, ostr, odist, batch, inp, out_size)
        got, _ = _exec_plan_gpu(F, torch, d, n, ie, istr, idist, oe, ostr, odist, batch, inp, out_size, dtype)
        # compare only the addressed output elements (others untouched / undefined)
        mask = np.zeros(out_size, bool)
        for b in range(batch):
            for idx in np.ndindex(*full_out):
                off = b * odist
                lin = 0
                for j in range(rank):
                    lin = lin * (oe[j] if j > 0 else 1) + idx[j]
                mask[off + lin * ostr] = True
        assert O.rel_l2(got[mask], ref[mask]) <= TOL[dtype], (d, n)


def test_plan_in_place_c2c_and_descriptor(F, torch_cuda):
    torch = torch_cuda
    rng = np.random.default_rng(2)
    z = rng.normal(size=(64, 32)) + 1j * rng.normal(size=(64, 32))
    p = F.Plan(F.C2CF, [64, 32], dtype="float32")
    t = dev_cplx(torch, z, "float32")
    p.exec(t, t)
    assert O.rel_l2(host(t), np.fft.fft2(z)) <= 2e-6
    d = p.descriptor()
    assert d["rank"] == 2 and d["n"] == [64, 32] and d["dir"] == F.C2CF and d["batch"] == 1
    assert p.num_launches() == 2


def test_plan_unsupported_size_is_reported(F, torch_cuda):
    # every length up to 4096 runs one pass kernel (radix or chirp-z) and longer lines a
    # long-line step (four-step, or chirp-z for a large prime factor: 17 * 257 here); lines
    # past 2^24 points are reported as unsupported
    torch = torch_cuda
    n = 17 * 257
    x = np.random.default_rng(9).standard_normal(n) + 1j * np.random.default_rng(10).standard_normal(n)
    xd = torch.tensor(x, dtype=torch.complex64, device="cuda")
    X = torch.empty_like(xd)
    F.Plan(F.C2CF, [n], dtype="float32").exec(xd, X)
    torch.cuda.synchronize()
    assert O.rel_l2(X.cpu().numpy(), np.fft.fft(x)) <= 5e-6
    with pytest.raises(F.FftbError) as e:
        F.Plan(F.C2CF, [(1 << 24) + 2], dtype="float32")
    assert e.value.status == -2


def test_fft_wrap_many_registry(F, torch_cuda):
    torch = torch_cuda
    w = F.fft_wrap_many("float64")
    nx, ny, nz = 8, 6, 10
    nzh = nz // 2 + 1
    # exactly the 3D plans of source/ffts.hpp:680-694
    w.add_plan_3D(F.R2C, "forward_3d", nx, ny, nz, nx, ny, nz, 1, nx * ny * nz, nx, ny, nzh, 1, nx * ny * nzh, 1)
    w.add_plan_3D(F.C2R, "inverse_3d", nx, ny, nz, nx, ny, nzh, 1, nx * ny * nzh, nx, ny, nz, 1, nx * ny * nz, 1)
    assert w.activate_work_size() == 0
    x = O.random_3d(nx, ny, nz, 1)
    xin = dev_real(torch, x, "float64")
    spec = empty_c(torch, (nx, ny, nzh), "float64")
    w.exec("forward_3d", xin, spec)
    assert O.rel_l2(host(spec), O.ffts3d_forward(x)) <= 1e-13
    w.exec("inverse_3d", spec, xin)
    assert O.rel_l2(host(xin) / x.size, x) <= 1e-13
    with pytest.raises(KeyError):
        w.exec("forward_w", xin, spec)


def test_errors_follow_reference_semantics(F, torch_cuda):
    torch = torch_cuda
    f = F.ffts("float32")
    with pytest.raises(F.LogicError):
        f.forward(torch.zeros(4, 4, 4, device="cuda"), torch.zeros(4, 4, 3, dtype=torch.complex64, device="cuda"))
    f.init(8, 8, 8)
    with pytest.raises(F.LogicError):
        f.init(8, 8, 8)
    with pytest.raises(F.LogicError):
        f.forward(torch.zeros(8, 8, 8, 8, device="cuda"), torch.zeros(8, 8, 8, 5, dtype=torch.complex64,
                                                                         device="cuda"))
    assert f.dimension() == 3
