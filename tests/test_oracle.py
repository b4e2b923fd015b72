"""CPU tests: pin the FP64 oracle before it is trusted as the checker.

Pins used (the reference stores no golden vectors for this path):
  * the committed golden fixtures (numpy pocketfft FP64, an independent FFT, on the
    reference tests' splitmix64 inputs) -- tests/golden/make_golden.py;
  * the reference's analytic tests: the Poisson examples (u = sin x cos 2y sin 3z,
    f = 14u, rel-L2 <= 1e-10, examples/poisson/source/poisson_periodic_3d_autotuned.cpp:64-71,
    :409-410; 4D f = 15u, examples/poisson/source/poisson_periodic_4d_autotuned.cpp:225-249),
    the periodic Laplacian v4 (u = sin x sin y sin z, f = -3u,
    source/tests/detail/versioned_ffts_3d_test_driver.h:186-210);
  * the reference benchmarks' round-trip criterion RMS(C2R(R2C(x))/N - x) <= 10 eps
    (source/tests/test_benchmark_ffts_3D.cu:100-120, fft_benchmark_common.h:28-32);
  * the reference Poisson test problems, Gaussian-modulated sines with closed-form
    solutions (source/tests/detail/poisson_3d_problem.h:22-50 with its gradient,
    poisson_4d_problem.h:14-55), whose L2 and H1 errors the reference reports
    (source/tests/test_3D_poisson.cu:247-280).
"""
import os

import numpy as np
import pytest

import oracle as O

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden_small.npz"))


def test_splitmix_generator_matches_fixture():
    x = O.random_3d(4, 4, 4, 0x1234ABCDEF987654)
    np.testing.assert_array_equal(x.ravel()[:8], GOLD["splitmix_first_values"])


@pytest.mark.parametrize("shape", [(8, 8, 8), (6, 10, 12), (5, 7, 9), (16, 12, 10)])
def test_oracle_3d_against_golden(shape):
    key = "r3d_" + "x".join(map(str, shape))
    x = O.random_3d(*shape, 0x1234ABCDEF987654)
    np.testing.assert_array_equal(x, GOLD[key + "_in"])
    X = O.ffts3d_forward(x)
    assert O.rel_l2(X, GOLD[key + "_spec"]) < 1e-14
    back = O.ffts3d_backward(X, shape[2]) / x.size
    assert O.rel_l2(back, x) < 1e-14


@pytest.mark.parametrize("layout", [O.PENCIL, O.SLAB, O.NATIVE_XZWY])
def test_oracle_4d_layouts_against_golden(layout):
    dims = (6, 4, 8, 10)
    xl = GOLD["r4d_in_xyzw"]
    x = np.ascontiguousarray(xl.transpose(3, 2, 1, 0)) if layout == O.PENCIL else xl
    xo = O.random_4d(*dims, 0xABCDEF0123456789, layout=layout)
    np.testing.assert_array_equal(xo, x)
    X = O.ffts4d_forward(layout, x, dims)
    ref = GOLD["r4d_spec_slab"] if layout == O.SLAB else GOLD["r4d_spec_yzwx"]
    assert O.rel_l2(X, ref) < 1e-14
    assert O.rel_l2(O.ffts4d_backward(layout, X, dims) / x.size, x) < 1e-14


def test_oracle_2d_and_c2c_against_golden():
    X = O.ffts2d_forward(GOLD["r2d_in"])
    assert O.rel_l2(X, GOLD["r2d_spec"]) < 1e-14
    z = GOLD["c1d_in"]
    f = O.exec_plan(O.C2CF, [48], None, 1, 0, None, 1, 0, 3, z, z.size)
    b = O.exec_plan(O.C2CB, [48], None, 1, 0, None, 1, 0, 3, z, z.size)
    assert O.rel_l2(f, GOLD["c1d_fwd"].ravel()) < 1e-14
    assert O.rel_l2(b, GOLD["c1d_inv"].ravel()) < 1e-14


def _grid(n):
    return 2 * np.pi * np.arange(n) / n


def test_oracle_poisson_example_3d():
    # -lap u = f with f = 14 u, u = sin x cos 2y sin 3z; sign +1 (example convention)
    n = 32
    x, y, z = np.meshgrid(_grid(n), _grid(n), _grid(n), indexing="ij")
    u = np.sin(x) * np.cos(2 * y) * np.sin(3 * z)
    sol = O.poisson3d_solve(14 * u, sign=+1.0)
    assert O.rel_l2(sol, u) <= 1e-10


def test_oracle_laplacian_v4():
    # lap u = f with u = sin x sin y sin z, f = -3u; sign -1 (test-driver convention)
    n = 16
    x, y, z = np.meshgrid(_grid(n), _grid(n), _grid(n), indexing="ij")
    u = np.sin(x) * np.sin(y) * np.sin(z)
    sol = O.poisson3d_solve(-3 * u, sign=-1.0)
    assert np.sqrt(np.mean((sol - u) ** 2)) < 1e-13


def _gaussian_sine_problem(n):
    # u = 100 g sin x sin y sin z with g = exp(-|r - pi|^2) on [0, 2 pi)^3; f = lap u and
    # du/dx in closed form (the reference's poisson_3d_problem<T>::evaluate)
    x, y, z = np.meshgrid(_grid(n), _grid(n), _grid(n), indexing="ij")
    dx, dy, dz = x - np.pi, y - np.pi, z - np.pi
    g = np.exp(-(dx * dx + dy * dy + dz * dz))
    sx, cx, sy, cy, sz, cz = np.sin(x), np.cos(x), np.sin(y), np.cos(y), np.sin(z), np.cos(z)
    u = 100 * g * sx * sy * sz
    ux = 100 * g * (cx - 2 * dx * sx) * sy * sz
    f = 100 * g * ((4 * (dx * dx + dy * dy + dz * dz) - 9) * sx * sy * sz
                   - 4 * dx * cx * sy * sz - 4 * dy * sx * cy * sz - 4 * dz * sx * sy * cz)
    return u, ux, f


def test_oracle_gaussian_sine_poisson_problem():
    # lap u = f (sign -1).  The Gaussian's tails leave a periodicity defect of order
    # exp(-pi^2), so the spectral error is small but not at rounding level, and it falls
    # as the grid is refined; the x derivative of the solution (the H1 part) likewise
    errs = []
    for n in (32, 64):
        u, ux, f = _gaussian_sine_problem(n)
        sol = O.poisson3d_solve(f, sign=-1.0)
        kx = np.fft.fftfreq(n, 1.0 / n)[:, None, None]
        dsol = O.ffts3d_backward(1j * kx * O.ffts3d_forward(sol), n) / sol.size
        errs.append((O.rel_l2(sol, u), O.rel_l2(dsol, ux)))
    assert errs[0][0] < 1e-4 and errs[1][0] < errs[0][0]
    assert errs[0][1] < 1e-3 and errs[1][1] < errs[0][1]


def _gaussian_sine_problem_4d(n):
    # the 4D problem of the reference (poisson_4d_problem<T>::evaluate,
    # source/tests/detail/poisson_4d_problem.h:14-55): u = 100 g sin x sin y sin z sin w
    g1 = _grid(n)
    x, y, z, w = np.meshgrid(g1, g1, g1, g1, indexing="ij")
    d = [x - np.pi, y - np.pi, z - np.pi, w - np.pi]
    s = [np.sin(x), np.sin(y), np.sin(z), np.sin(w)]
    c = [np.cos(x), np.cos(y), np.cos(z), np.cos(w)]
    g = np.exp(-sum(a * a for a in d))
    prod = s[0] * s[1] * s[2] * s[3]
    f = (4 * sum(a * a for a in d) - 12) * prod
    for a in range(4):
        others = np.prod([s[b] for b in range(4) if b != a], axis=0)
        f = f - 4 * d[a] * c[a] * others
    return 100 * g * prod, 100 * g * f


@pytest.mark.parametrize("layout", [O.PENCIL, O.SLAB, O.NATIVE_XZWY])
def test_oracle_gaussian_sine_poisson_problem_4d(layout):
    errs = []
    for n in (16, 24):
        u, f = _gaussian_sine_problem_4d(n)
        if layout == O.PENCIL:   # pencil real arrays are stored [w][z][y][x]
            u, f = (np.ascontiguousarray(a.transpose(3, 2, 1, 0)) for a in (u, f))
        errs.append(O.rel_l2(O.poisson4d_solve(layout, f, (n,) * 4, sign=-1.0), u))
    assert errs[0] < 2e-4 and errs[1] < errs[0], errs


@pytest.mark.parametrize("layout", [O.PENCIL, O.SLAB, O.NATIVE_XZWY])
def test_oracle_poisson_example_4d(layout):
    dims = (16, 16, 16, 8)
    X, Y, Z, W = np.meshgrid(*[_grid(d) for d in dims], indexing="ij")
    u = np.sin(X) * np.cos(2 * Y) * np.sin(3 * Z) * np.cos(W)
    if layout == O.PENCIL:
        u = np.ascontiguousarray(u.transpose(3, 2, 1, 0))
    sol = O.poisson4d_solve(layout, 15 * u, dims, sign=+1.0)
    assert O.rel_l2(sol, u) <= 1e-10


def test_oracle_round_trip_criterion():
    x = O.random_3d(12, 10, 8, 0xABCDEF0123456789)
    back = O.ffts3d_backward(O.ffts3d_forward(x), 8) / x.size
    rms = np.sqrt(np.mean((back - x) ** 2))
    assert rms <= 10 * np.finfo(np.float64).eps


def test_oracle_c2r_ignores_dc_and_nyquist_imag():
    rng = np.random.default_rng(3)
    X = np.fft.rfft(rng.normal(size=16))
    Xb = X.copy()
    Xb[0] += 0.5j
    Xb[-1] -= 0.25j
    a = O.exec_plan(O.C2R, [16], None, 1, 0, None, 1, 0, 1, X, 16)
    b = O.exec_plan(O.C2R, [16], None, 1, 0, None, 1, 0, 1, Xb, 16)
    np.testing.assert_allclose(a, b, atol=1e-14)
    np.testing.assert_allclose(a / 16, np.fft.irfft(X, 16), atol=1e-14)


def test_oracle_advanced_layout_strided_batch():
    # 1D R2C with stride and distance, as the 4D pencil w-plan uses them (source/ffts.hpp:709-711)
    rng = np.random.default_rng(5)
    nw, B = 10, 6
    x = rng.normal(size=(nw, B))           # element (w, b) at w*B + b -> istride B, idist 1
    X = O.exec_plan(O.R2C, [nw], [1], B, 1, [1], B, 1, B, x.ravel(), (nw // 2 + 1) * B)
    ref = np.fft.rfft(x, axis=0)
    assert O.rel_l2(X, ref.ravel()) < 1e-14
