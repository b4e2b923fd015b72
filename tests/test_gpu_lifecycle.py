"""GPU resource life cycle (the role of the reference's
source/tests/test_fftm_resource_lifecycle.cu for this path): creating and destroying
ffts objects, plans and batches repeatedly -- with their work areas, derivative
buffers, timing events, captured CUDA graphs and persistent / grouped plans -- returns
the device memory it took."""
import gc

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def F(torch_cuda):
    from fftm_b200 import build
    build.build()
    import fftm_b200
    return fftm_b200


def _free_bytes(torch):
    gc.collect()
    torch.cuda.synchronize()
    return torch.cuda.mem_get_info()[0]


def _cycle(F, torch):
    import fftm_b200.batch as B
    for dims, layout in [((64, 64, 64), "pencil"), ((24, 20, 18), "pencil"), ((16, 16, 16, 16), "native_xzwy")]:
        f = F.ffts("float32", strategy_4d=layout).init(*dims)
        x = torch.randn(f.real_shape(), device="cuda")
        y = torch.empty_like(x)
        s = torch.empty(f.spectrum_shape(), dtype=torch.complex64, device="cuda")
        f.timing_enable(16)
        f.forward(x, s)
        f.backward(s, y, normalized=True)
        f.poisson(x, y, -1.0)
        f.derivative(x, y, 0)
        f.timing_read()
        del f
    b = B.Batch(B.draw_shapes(6, seed=2))
    xb = torch.rand(b.real_total, device="cuda")
    yb = torch.empty_like(xb)
    for mode in (B.SEQUENTIAL, B.PERSISTENT, B.GRAPH, B.GROUPED, B.GROUPED_GRAPH):
        b.exec(B.ROUNDTRIP, xb, yb, mode=mode)
    torch.cuda.synchronize()
    del b


def test_create_destroy_returns_memory(F, torch_cuda):
    torch = torch_cuda
    torch.cuda.empty_cache()
    _cycle(F, torch)                      # first use: twiddle tables and module loading
    torch.cuda.empty_cache()
    base = _free_bytes(torch)
    for _ in range(5):
        _cycle(F, torch)
        torch.cuda.empty_cache()
    after = _free_bytes(torch)
    # torch's caching allocator is emptied each cycle; what remains is the library's
    assert base - after <= 8 * 1024 * 1024, (base - after)


def test_plan_and_wrap_many_release(F, torch_cuda):
    torch = torch_cuda
    torch.cuda.empty_cache()
    base = _free_bytes(torch)
    for _ in range(10):
        w = F.fft_wrap_many("float32")
        w.add_plan_3D(F.R2C, "forward_3d", 32, 32, 32, 32, 32, 32, 1, 32 * 32 * 32, 32, 32, 17, 1, 32 * 32 * 17, 1)
        w.add_plan_3D(F.C2R, "inverse_3d", 32, 32, 32, 32, 32, 17, 1, 32 * 32 * 17, 32, 32, 32, 1, 32 * 32 * 32, 1)
        w.activate()
        x = torch.randn(32, 32, 32, device="cuda")
        X = torch.empty(32, 32, 17, dtype=torch.complex64, device="cuda")
        w.exec("forward_3d", x, X)
        w.exec("inverse_3d", X, x)
        torch.cuda.synchronize()
        w.release()
        del w, x, X
        torch.cuda.empty_cache()
    after = _free_bytes(torch)
    assert base - after <= 8 * 1024 * 1024, (base - after)
