"""The slab-distributed 3D / 4D transforms' rank-local library passes on one GPU: one rank
(the exchange is nothing), and two ranks emulated on the one GPU -- with the exchange as
block copies (the all-to-all's data movement) and with the pack pass storing straight into
the other rank's receive buffer (the peer-store form) -- forward against the FP64 oracle,
backward round trip."""
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


def _two_ranks(torch, dims, dtype, layout, peer):
    """Two ranks of the slab transform emulated on one GPU: each rank's library passes on its
    own buffers; the exchange is block copies (NCCL's all-to-all between GPUs), or with
    `peer` nothing at all: each rank's pack pass stores straight into the other rank's
    receive buffer through set_peers.  The passes run one after another on one stream, so
    nothing waits on anything."""
    from fftm_b200.slab import _LibraryLocal
    P = 2
    loc = [_LibraryLocal(dims, P, r, dtype, layout) for r in range(P)]
    cdt = torch.complex64 if dtype == "float32" else torch.complex128
    n_ex = loc[0].exchange_elems
    blk = n_ex // P
    send = [torch.zeros(n_ex, dtype=cdt, device="cuda") for _ in range(P)]
    recv = [torch.zeros(n_ex, dtype=cdt, device="cuda") for _ in range(P)]
    if peer:
        esz = recv[0].element_size()
        for r in range(P):
            loc[r].set_peers([recv[q].data_ptr() + r * blk * esz for q in range(P)])
    return loc, send, recv, blk


def _exchange(send, recv, blk):
    P = len(send)
    for r in range(P):
        for q in range(P):
            recv[q][r * blk:(r + 1) * blk].copy_(send[r][q * blk:(q + 1) * blk])


@pytest.mark.parametrize("peer", [False, True])
@pytest.mark.parametrize("dtype,dims", [("float32", (32, 24, 40)), ("float64", (12, 10, 14))])
def test_slab3d_two_ranks_on_one_gpu(torch_cuda, dtype, dims, peer):
    torch = torch_cuda
    from fftm_b200 import build
    build.build()
    rt = torch.float32 if dtype == "float32" else torch.float64
    tol = 2e-6 if dtype == "float32" else 1e-12
    nx, ny, nz = dims
    x = O.random_3d(*dims, 43, single=(dtype == "float32"))
    ref = O.ffts3d_forward(x.astype(np.float64))
    loc, send, recv, blk = _two_ranks(torch, dims, dtype, "slab", peer)
    nxl, nyl = nx // 2, ny // 2
    for r in range(2):
        xs = torch.tensor(x[r * nxl:(r + 1) * nxl], dtype=rt, device="cuda")
        loc[r].forward_local(xs, send[r])
    if not peer:
        _exchange(send, recv, blk)
    for r in range(2):
        loc[r].forward_finish(recv[r], recv[r])
    torch.cuda.synchronize()
    for r in range(2):
        got = recv[r].view(nx, nyl, nz // 2 + 1).cpu().numpy()
        assert O.rel_l2(got, ref[:, r * nyl:(r + 1) * nyl, :]) <= tol
    # backward: spectrum slabs -> (x blocks exchanged) -> real slabs
    for r in range(2):
        loc[r].backward_local(recv[r], recv[r])
    spec_as_send = [t.clone() for t in recv]
    _exchange(spec_as_send, recv, blk)
    for r in range(2):
        out = torch.empty((nxl, ny, nz), dtype=rt, device="cuda")
        loc[r].backward_finish(recv[r], out)
        torch.cuda.synchronize()
        assert O.rel_l2(out.cpu().numpy() / x.size, x[r * nxl:(r + 1) * nxl]) <= tol


@pytest.mark.parametrize("peer", [False, True])
@pytest.mark.parametrize("layout", ["native_xzwy", "slab"])
def test_slab4d_two_ranks_on_one_gpu(torch_cuda, layout, peer):
    torch = torch_cuda
    from fftm_b200 import build
    build.build()
    dims = (16, 12, 20, 24)
    nx, ny, nz, nw = dims
    lay = O.NATIVE_XZWY if layout == "native_xzwy" else O.SLAB
    x = O.random_4d(*dims, 47, layout=O.SLAB, single=True)          # real [x][y][z][w]
    full = O.ffts4d_forward(O.SLAB, x.astype(np.float64), dims)      # [kx][ky][kz][kw]
    loc, send, recv, blk = _two_ranks(torch, dims, "float32", layout, peer)
    nxl, nzl, nwh = nx // 2, nz // 2, nw // 2 + 1
    for r in range(2):
        xs = torch.tensor(x[r * nxl:(r + 1) * nxl], dtype=torch.float32, device="cuda")
        loc[r].forward_local(xs, send[r])
    if not peer:
        _exchange(send, recv, blk)
    specs = []
    for r in range(2):
        if layout == "native_xzwy":
            sp = torch.empty((ny, nzl, nwh, nx), dtype=torch.complex64, device="cuda")
            loc[r].forward_finish(recv[r], sp)
        else:
            loc[r].forward_finish(recv[r], recv[r])
            sp = recv[r].view(nx, ny, nzl, nwh)
        specs.append(sp)
    torch.cuda.synchronize()
    for r in range(2):
        ref = full[:, :, r * nzl:(r + 1) * nzl, :]
        if layout == "native_xzwy":
            ref = ref.transpose(1, 2, 3, 0)
        assert O.rel_l2(specs[r].cpu().numpy(), ref) <= 2e-6
    sends = []
    for r in range(2):
        sd = torch.empty_like(send[r])
        loc[r].backward_local(specs[r].contiguous(), sd)
        sends.append(sd)
    _exchange(sends, recv, blk)
    for r in range(2):
        out = torch.empty((nxl, ny, nz, nw), dtype=torch.float32, device="cuda")
        loc[r].backward_finish(recv[r], out)
        torch.cuda.synchronize()
        assert O.rel_l2(out.cpu().numpy() / x.size, x[r * nxl:(r + 1) * nxl]) <= 2e-6
