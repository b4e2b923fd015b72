"""GPU test of fftb_poisson3d_f32_noalloc, the Poisson solve that allocates no
device memory (for callers that cannot call cudaMalloc, e.g. when a framework's
memory pool owns the device).

It is called through the C ABI twice in a row over a set of fields and sizes (mixed
sizes, a power-of-two cube that the regular entry point runs through its fused plane
and column kernels, and an odd z length whose R2C/C2R run full complex lines), and each
result is compared with the FP64 oracle and with the regular entry point
(fftb_ffts_poisson via the ffts object) at the float32 tolerance of the other GPU tests
(relative L2 2e-6).  The file is named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

TOL = 2e-6


@pytest.fixture(scope="module")
def lib(torch_cuda):
    from fftm_b200 import build
    build.build()
    from fftm_b200 import _lib
    L = _lib.load()
    L.fftb_poisson3d_f32_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_longlong,
                                             ctypes.c_longlong, ctypes.c_longlong, ctypes.c_double,
                                             ctypes.c_void_p]
    L.fftb_poisson3d_f32_noalloc.restype = ctypes.c_int
    return L


def _noalloc(L, torch, rhs, sol, sign):
    nx, ny, nz = rhs.shape
    st = L.fftb_poisson3d_f32_noalloc(rhs.data_ptr(), sol.data_ptr(), nx, ny, nz, sign,
                                      torch.cuda.current_stream().cuda_stream)
    assert st == 0, st


def _regular(torch, rhs, sign):
    import fftm_b200 as F
    f = F.ffts("float32").init(*rhs.shape)
    out = torch.empty_like(rhs)
    f.poisson(rhs, out, sign)
    torch.cuda.synchronize()
    return out


def test_noalloc_matches_regular_entry_point_on_two_calls(lib, torch_cuda):
    torch = torch_cuda
    cases = [((32, 24, 16), 11, -1.0), ((64, 48, 40), 12, 1.0), ((64, 64, 64), 13, -1.0),
             ((16, 12, 15), 14, -1.0)]
    rhs = [torch.tensor(O.random_3d(*shape, seed, single=True), dtype=torch.float32, device="cuda")
           for shape, seed, _ in cases]
    sol = [torch.empty_like(r) for r in rhs]
    # the first call on the device does the one-time set-up (scratch address lookup); one
    # call per size also makes CUDA load those kernels' code (lazy module loading), which
    # is not an allocation of the entry point
    for (shape, seed, sign), r, s in zip(cases, rhs, sol):
        _noalloc(lib, torch, r, s, sign)
    for s in sol:
        s.zero_()
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    for (shape, seed, sign), r, s in zip(cases, rhs, sol):
        _noalloc(lib, torch, r, s, sign)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before      # the two calls allocated nothing
    for (shape, seed, sign), r, s in zip(cases, rhs, sol):
        got = s.cpu().numpy().astype(np.float64)
        exact = O.poisson3d_solve(r.cpu().numpy().astype(np.float64), sign)
        err = O.rel_l2(got, exact)
        assert err <= TOL, (shape, "vs FP64 oracle", err)
        ref = _regular(torch, r, sign)
        err = O.rel_l2(got, ref.cpu().numpy().astype(np.float64))
        assert err <= TOL, (shape, "vs fftb_ffts_poisson", err)


def test_noalloc_rejects_sizes_beyond_its_scratch(lib, torch_cuda):
    torch = torch_cuda
    x = torch.zeros(8, device="cuda")
    # 256 x 256 x 128 needs a 33.8 MB spectrum, more than the 16 MiB static scratch
    assert lib.fftb_poisson3d_f32_noalloc(x.data_ptr(), x.data_ptr(), 256, 256, 128, -1.0, None) == -1
    assert lib.fftb_poisson3d_f32_noalloc(x.data_ptr(), x.data_ptr(), 1, 8, 8, -1.0, None) == -1
