"""Host logic of the x-slab distributed 3D and 4D transforms (fftm_b200.slab) with
world-size-2 `gloo` process groups on CPU: the slab decomposition, the all-to-all
exchange and its packing, checked against numpy's full 3D / 4D transform (4D in both
the slab [kx][ky][kz][kw] and fftm's native [ky][kz][kw][kx] spectrum orders).  The rank-local transforms are
numpy stand-ins here (the library's GPU plans replace them on GPUs; one GPU per test
box means the NCCL exchange itself is not run)."""
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


class _NumpyLocal:
    def __init__(self, ny, nz, nx):
        self.ny, self.nz, self.nx = ny, nz, nx

    def r2c_yz(self, x, out):
        import torch
        out.copy_(torch.from_numpy(np.fft.rfftn(x.numpy(), axes=(1, 2))))

    def c2r_yz(self, spec, out):
        import torch
        r = np.fft.irfftn(spec.numpy(), s=(self.ny, self.nz), axes=(1, 2)) * (self.ny * self.nz)
        out.copy_(torch.from_numpy(r))

    def fft_x(self, t, inverse=False):
        import torch
        a = t.numpy()
        r = np.fft.ifft(a, axis=0) * self.nx if inverse else np.fft.fft(a, axis=0)
        t.copy_(torch.from_numpy(r))


def _rank_main(rank, world, port, outdir, dims):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import torch
    import torch.distributed as dist
    from fftm_b200.slab import SlabFFT3D
    dist.init_process_group("gloo", rank=rank, world_size=world)
    nx, ny, nz = dims
    g = np.random.default_rng(7).standard_normal(dims)
    f = SlabFFT3D(nx, ny, nz, local=_NumpyLocal(ny, nz, nx))
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
    from fftm_b200.slab import SlabFFT3D
    f = SlabFFT3D(6, 4, 8, local=_NumpyLocal(4, 8, 6))      # no process group: one rank
    assert f.P == 1 and f.spectrum_slab_shape() == (6, 4, 5)


class _NumpyLocal4D:
    def __init__(self, nz, nw, nx, ny, layout):
        self.nz, self.nw, self.nx, self.ny, self.layout = nz, nw, nx, ny, layout

    def r2c_zw(self, x, out):
        import torch
        out.copy_(torch.from_numpy(np.fft.rfftn(x.numpy(), axes=(2, 3))))

    def c2r_zw(self, spec, out):
        import torch
        r = np.fft.irfftn(spec.numpy(), s=(self.nz, self.nw), axes=(2, 3)) * (self.nz * self.nw)
        out.copy_(torch.from_numpy(r))

    def fft_xy(self, t, inverse=False):
        import torch
        axes = (0, 3) if self.layout == "native_xzwy" else (0, 1)
        a = t.numpy()
        r = np.fft.ifftn(a, axes=axes) * (self.nx * self.ny) if inverse else np.fft.fftn(a, axes=axes)
        t.copy_(torch.from_numpy(r))


def _rank_main_4d(rank, world, port, outdir, dims, layout):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import torch
    import torch.distributed as dist
    from fftm_b200.slab import SlabFFT4D
    dist.init_process_group("gloo", rank=rank, world_size=world)
    nx, ny, nz, nw = dims
    g = np.random.default_rng(11).standard_normal(dims)
    f = SlabFFT4D(nx, ny, nz, nw, layout=layout, local=_NumpyLocal4D(nz, nw, nx, ny, layout))
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
    from fftm_b200.slab import SlabFFT4D
    f = SlabFFT4D(6, 4, 5, 8, local=_NumpyLocal4D(5, 8, 6, 4, "native_xzwy"))   # one rank
    assert f.P == 1 and f.spectrum_slab_shape() == (4, 5, 5, 6)
    with pytest.raises(ValueError):
        SlabFFT4D(6, 4, 5, 8, layout="pencil", local=object())
