"""Host logic of the x-slab distributed 3D and 4D transforms (fftm_b200.slab) with
world-size-2 `gloo` process groups on CPU: the slab decomposition and the all-to-all
exchange of the send blocks, checked against numpy's full 3D / 4D transform (4D in both the
slab [kx][ky][kz][kw] and fftm's native [ky][kz][kw][kx] spectrum orders).  The rank-local
passes are the numpy stand-in of fftm_b200.slab (the same send / receive block semantics as
the library's GPU passes, which replace it on GPUs; one GPU per test box means the NCCL
exchange itself is not run)."""
import json
import os
import socket

import numpy as np
import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, outdir, dims):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import torch
    import torch.distributed as dist
    from fftm_b200.slab import SlabFFT3D, numpy_local
    dist.init_process_group("gloo", rank=rank, world_size=world)
    nx, ny, nz = dims
    g = np.random.default_rng(7).standard_normal(dims)
    f = SlabFFT3D(nx, ny, nz, local=numpy_local(dims, world))
    assert f.real_slab_shape() == (nx // world, ny, nz)
    xs = torch.from_numpy(np.ascontiguousarray(g[rank * f.nxl:(rank + 1) * f.nxl])).double()
    spec = f.forward(xs)
    ref = np.fft.rfftn(g)[:, rank * f.nyl:(rank + 1) * f.nyl, :]
    err_f = float(np.linalg.norm(spec.numpy() - ref) / np.linalg.norm(ref))
    back = f.backward(spec.clone())
    err_b = float(np.linalg.norm(back.numpy() / g.size - xs.numpy()) / np.linalg.norm(xs.numpy()))
    with open(os.path.join(outdir, f"r{rank}.json"), "w") as fh:
        json.dump({"forward": err_f, "backward": err_b, "shape": list(spec.shape)}, fh)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("dims", [(8, 6, 10), (4, 12, 7)])
def test_slab_fft_two_ranks(tmp_path, dims):
    import torch.multiprocessing as mp
    mp.start_processes(_rank_main, args=(2, _free_port(), str(tmp_path), dims), nprocs=2, join=True,
                       start_method="spawn")
    for r in range(2):
        with open(tmp_path / f"r{r}.json") as fh:
            d = json.load(fh)
        assert d["forward"] < 1e-12 and d["backward"] < 1e-12, (r, d)
        assert d["shape"] == [dims[0], dims[1] // 2, dims[2] // 2 + 1]


def test_slab_rejects_indivisible():
    from fftm_b200.slab import SlabFFT3D, numpy_local
    f = SlabFFT3D(6, 4, 8, local=numpy_local((6, 4, 8), 1))      # no process group: one rank
    assert f.P == 1 and f.spectrum_slab_shape() == (6, 4, 5)
    # one rank: the exchange is nothing, and the host logic still transforms
    import torch
    g = np.random.default_rng(3).standard_normal((6, 4, 8))
    spec = f.forward(torch.from_numpy(g))
    assert np.linalg.norm(spec.numpy() - np.fft.rfftn(g)) / np.linalg.norm(np.fft.rfftn(g)) < 1e-12


def _rank_main_4d(rank, world, port, outdir, dims, layout):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import torch
    import torch.distributed as dist
    from fftm_b200.slab import SlabFFT4D, numpy_local
    dist.init_process_group("gloo", rank=rank, world_size=world)
    nx, ny, nz, nw = dims
    g = np.random.default_rng(11).standard_normal(dims)
    f = SlabFFT4D(nx, ny, nz, nw, layout=layout, local=numpy_local(dims, world, layout))
    assert f.real_slab_shape() == (nx // world, ny, nz, nw)
    xs = torch.from_numpy(np.ascontiguousarray(g[rank * f.nxl:(rank + 1) * f.nxl])).double()
    spec = f.forward(xs)
    ref = np.fft.rfftn(g)[:, :, rank * f.nzl:(rank + 1) * f.nzl, :]
    if layout == "native_xzwy":
        ref = ref.transpose(1, 2, 3, 0)
    err_f = float(np.linalg.norm(spec.numpy() - ref) / np.linalg.norm(ref))
    back = f.backward(spec.clone())
    err_b = float(np.linalg.norm(back.numpy() / g.size - xs.numpy()) / np.linalg.norm(xs.numpy()))
    with open(os.path.join(outdir, f"r{rank}.json"), "w") as fh:
        json.dump({"forward": err_f, "backward": err_b, "shape": list(spec.shape),
                   "expected": list(f.spectrum_slab_shape())}, fh)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("layout", ["native_xzwy", "slab"])
@pytest.mark.parametrize("dims", [(4, 6, 8, 10), (6, 5, 4, 7)])
def test_slab_fft_4d_two_ranks(tmp_path, dims, layout):
    import torch.multiprocessing as mp
    mp.start_processes(_rank_main_4d, args=(2, _free_port(), str(tmp_path), dims, layout), nprocs=2, join=True,
                       start_method="spawn")
    for r in range(2):
        with open(tmp_path / f"r{r}.json") as fh:
            d = json.load(fh)
        assert d["forward"] < 1e-12 and d["backward"] < 1e-12, (r, d)
        assert d["shape"] == d["expected"]


def test_slab_4d_rejects_indivisible_and_bad_layout():
    from fftm_b200.slab import SlabFFT4D, numpy_local
    f = SlabFFT4D(6, 4, 5, 8, local=numpy_local((6, 4, 5, 8), 1, "native_xzwy"))   # one rank
    assert f.P == 1 and f.spectrum_slab_shape() == (4, 5, 5, 6)
    with pytest.raises(ValueError):
        SlabFFT4D(6, 4, 5, 8, layout="pencil", local=object())
