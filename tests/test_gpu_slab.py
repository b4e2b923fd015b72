"""The x-slab distributed 3D transform's rank-local GPU plans on one GPU (one rank, so
the exchange is a copy): forward against the FP64 oracle, backward round trip."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype,dims", [("float32", (32, 24, 40)), ("float64", (12, 10, 14))])
def test_slab_local_plans_one_rank(torch_cuda, dtype, dims):
    torch = torch_cuda
    from fftm_b200 import build
    build.build()
    from fftm_b200.slab import SlabFFT3D
    rt = torch.float32 if dtype == "float32" else torch.float64
    tol = 2e-6 if dtype == "float32" else 1e-12
    x = O.random_3d(*dims, 31, single=(dtype == "float32"))
    f = SlabFFT3D(*dims, dtype=dtype)
    assert f.P == 1
    xd = torch.tensor(x, dtype=rt, device="cuda")
    spec = f.forward(xd)
    torch.cuda.synchronize()
    assert O.rel_l2(spec.cpu().numpy(), O.ffts3d_forward(x.astype(np.float64))) <= tol
    back = f.backward(spec)
    torch.cuda.synchronize()
    assert O.rel_l2(back.cpu().numpy() / x.size, x) <= tol


@pytest.mark.parametrize("layout,dtype,dims", [("native_xzwy", "float32", (16, 12, 20, 24)),
                                               ("slab", "float32", (16, 12, 20, 24)),
                                               ("native_xzwy", "float64", (6, 10, 8, 12))])
def test_slab4d_local_plans_one_rank(torch_cuda, layout, dtype, dims):
    torch = torch_cuda
    from fftm_b200 import build
    build.build()
    from fftm_b200.slab import SlabFFT4D
    rt = torch.float32 if dtype == "float32" else torch.float64
    tol = 2e-6 if dtype == "float32" else 1e-12
    lay = O.NATIVE_XZWY if layout == "native_xzwy" else O.SLAB
    x = O.random_4d(*dims, 37, layout=lay, single=(dtype == "float32"))
    f = SlabFFT4D(*dims, dtype=dtype, layout=layout)
    assert f.P == 1
    xd = torch.tensor(x, dtype=rt, device="cuda")
    spec = f.forward(xd)
    torch.cuda.synchronize()
    ref = O.ffts4d_forward(lay, x.astype(np.float64), dims)
    assert tuple(spec.shape) == f.spectrum_slab_shape()
    assert O.rel_l2(spec.cpu().numpy(), ref.reshape(spec.shape)) <= tol
    back = f.backward(spec)
    torch.cuda.synchronize()
    assert O.rel_l2(back.cpu().numpy() / x.size, x) <= tol
