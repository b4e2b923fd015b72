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
