"""3D and 4D R2C / C2R transforms of a field distributed over the ranks of a process group
(one process per GPU on one node), by x slabs: the multi-GPU form of the reference's fftm
slab paths, whose MPI redistributions (`source/detail/mpi_transpose_3d_same_x.h`,
`source/detail/mpi_transpose_4d_same_xw.h:437-497`) pack, exchange and unpack around the
FFTs.

The rank-local passes run in the library (``fftb_slab_*``, fftm_b200/csrc/fftb_slab.cu):
the last FFT pass before the exchange stores its output in send-buffer order (one
contiguous block per destination rank) and the first pass after it loads the received
blocks in place, so no pack or unpack copy touches the data.  The exchange is one
``all_to_all_single`` over the process group (NCCL between GPUs); with one rank it is
nothing (send and receive are one buffer).

3D, rank r of P (nx, ny divisible by P; nxl = nx/P, nyl = ny/P, nzh = nz/2+1):
real slab ``[nxl][ny][nz]`` -> z R2C -> y FFT storing ky block q to send block q ->
exchange -> x FFT in place -> spectrum slab ``[kx][nyl][nzh]`` (ky block r).

4D slab-slab (fftm's ``strategy_4d_slab_slab_mpi``; nx, nz divisible by P; nzl = nz/P,
nwh = nw/2+1): real ``[nxl][ny][nz][nw]`` -> w R2C -> z FFT storing kz block q to send
block q -> exchange -> (y, x) FFTs on ``[nx][ny][nzl][nwh]``, the x pass writing fftm's native
spectrum ``[ky][nzl][nwh][kx]`` (``layout="native_xzwy"``, the plan of
`source/fftm.hpp:2941-2961`) or keeping ``[kx][ky][nzl][nwh]`` (``layout="slab"``).

Backward is the mirror image (unnormalised C2R, as the reference's).
"""
from __future__ import annotations

import ctypes


class _LibraryLocal:
    """The rank-local passes of the library on the current GPU."""

    def __init__(self, dims, P, rank, dtype, layout):
        import torch

        from . import NATIVE_XZWY, SLAB, _check, _dtype_code, _lib
        self._torch = torch
        L = _lib.load()
        nx, ny, nz = dims[:3]
        nw = dims[3] if len(dims) == 4 else 0
        lay = NATIVE_XZWY if layout == "native_xzwy" else SLAB
        h = ctypes.c_void_p()
        _check(L.fftb_slab_create(_dtype_code(dtype), nx, ny, nz, nw, lay, P, rank, ctypes.byref(h)), "slab create")
        self._h = h
        v = [ctypes.c_longlong() for _ in range(4)]
        _check(L.fftb_slab_sizes(h, *[ctypes.byref(x) for x in v]), "slab sizes")
        self.real_elems, self.spec_elems, self.exchange_elems, work_elems = (x.value for x in v)
        self.cdt = torch.complex64 if dtype in ("float32", torch.float32) else torch.complex128
        self.work = torch.empty(work_elems, dtype=self.cdt, device="cuda")
        self.P = P

    def _bind(self):
        from . import _check, _lib
        _check(_lib.load().fftb_slab_set_stream(self._h, self._torch.cuda.current_stream().cuda_stream), "stream")

    def set_peers(self, blocks):
        """blocks[q]: device address of this rank's block in rank q's receive buffer (or None)."""
        from . import _check, _lib
        arr = (ctypes.c_void_p * 8)(*([b for b in blocks] + [None] * (8 - len(blocks))))
        _check(_lib.load().fftb_slab_set_peers(self._h, arr if any(blocks) else None), "set_peers")

    def forward_local(self, x, send):
        from . import _check, _lib
        self._bind()
        _check(_lib.load().fftb_slab_forward_local(self._h, x.data_ptr(), send.data_ptr(), self.work.data_ptr()),
               "forward_local")

    def forward_finish(self, recv, out):
        from . import _check, _lib
        self._bind()
        _check(_lib.load().fftb_slab_forward_finish(self._h, recv.data_ptr(), out.data_ptr()), "forward_finish")

    def backward_local(self, spec, send):
        from . import _check, _lib
        self._bind()
        _check(_lib.load().fftb_slab_backward_local(self._h, spec.data_ptr(), send.data_ptr()), "backward_local")

    def backward_finish(self, recv, out):
        from . import _check, _lib
        self._bind()
        _check(_lib.load().fftb_slab_backward_finish(self._h, recv.data_ptr(), out.data_ptr(), self.work.data_ptr()),
               "backward_finish")

    def __del__(self):
        try:
            from . import _lib
            if getattr(self, "_h", None):
                _lib.load().fftb_slab_destroy(self._h)
                self._h = None
        except Exception:
            pass


class _Slab:
    def __init__(self, dims, group, dtype, layout, local):
        import torch.distributed as dist
        self.dist = dist if dist.is_available() and dist.is_initialized() else None
        self.group = group
        self.P = self.dist.get_world_size(group) if self.dist else 1
        self.rank = self.dist.get_rank(group) if self.dist else 0
        self.dims = tuple(int(d) for d in dims)
        self.layout = layout
        split = (0, 1) if len(dims) == 3 else (0, 2)
        for a in split:
            if self.dims[a] % self.P:
                raise ValueError(f"axis {a} ({self.dims[a]}) must be divisible by the {self.P} ranks")
        self.local = local if local is not None else _LibraryLocal(self.dims, self.P, self.rank, dtype, layout)

    def _exchange(self, send, recv):
        """Block q of send to rank q; block q of recv from rank q (equal blocks)."""
        import torch
        if self.P == 1:
            if recv.data_ptr() != send.data_ptr():
                recv.copy_(send)
            return
        self.dist.all_to_all_single(torch.view_as_real(recv), torch.view_as_real(send), group=self.group)

    def _cdt(self, real):
        import torch
        return torch.complex64 if real.dtype == torch.float32 else torch.complex128

    def forward(self, x, out=None):
        """Real slab -> spectrum slab (unnormalised)."""
        import torch
        cdt = self._cdt(x)
        send = torch.empty(self._exchange_shape(), dtype=cdt, device=x.device)
        recv = send if self.P == 1 else torch.empty_like(send)
        self.local.forward_local(x, send)
        self._exchange(send, recv)
        if len(self.dims) == 4 and self.layout == "native_xzwy":
            spec = out if out is not None else torch.empty(self.spectrum_slab_shape(), dtype=cdt, device=x.device)
            self.local.forward_finish(recv, spec)
            return spec
        self.local.forward_finish(recv, recv)
        spec = recv.view(self.spectrum_slab_shape())
        if out is not None:
            out.copy_(spec)
            return out
        return spec

    def backward(self, spec, out=None):
        """Spectrum slab -> real slab (unnormalised C2R; spec is overwritten)."""
        import torch
        rdt = torch.float32 if spec.dtype == torch.complex64 else torch.float64
        if len(self.dims) == 3:
            send = spec.reshape(self._exchange_shape())
            self.local.backward_local(spec, spec)
        else:
            send = torch.empty(self._exchange_shape(), dtype=spec.dtype, device=spec.device)
            self.local.backward_local(spec, send)
        recv = send if self.P == 1 else torch.empty_like(send)
        self._exchange(send, recv)
        x = out if out is not None else torch.empty(self.real_slab_shape(), dtype=rdt, device=spec.device)
        self.local.backward_finish(recv, x)
        return x


class SlabFFT3D(_Slab):
    """x-slab distributed 3D R2C / C2R over a process group (see the module notes).

    ``local`` replaces the rank-local passes (an object with ``forward_local``,
    ``forward_finish``, ``backward_local`` and ``backward_finish`` of the library's
    semantics); the default runs the library on the current GPU."""

    def __init__(self, nx, ny, nz, group=None, dtype="float32", local=None):
        super().__init__((nx, ny, nz), group, dtype, "slab", local)
        self.nx, self.ny, self.nz = nx, ny, nz
        self.nxl, self.nyl, self.nzh = nx // self.P, ny // self.P, nz // 2 + 1

    def real_slab_shape(self):
        return (self.nxl, self.ny, self.nz)

    def spectrum_slab_shape(self):
        return (self.nx, self.nyl, self.nzh)

    def _exchange_shape(self):
        return (self.P, self.nxl, self.nyl, self.nzh)


class SlabFFT4D(_Slab):
    """x-slab distributed 4D R2C / C2R over a process group, spectrum by kz blocks (see
    the module notes)."""

    def __init__(self, nx, ny, nz, nw, group=None, dtype="float32", layout="native_xzwy", local=None):
        if layout not in ("native_xzwy", "slab"):
            raise ValueError(f"layout must be 'native_xzwy' or 'slab', not {layout!r}")
        super().__init__((nx, ny, nz, nw), group, dtype, layout, local)
        self.nx, self.ny, self.nz, self.nw = nx, ny, nz, nw
        self.nxl, self.nzl, self.nwh = nx // self.P, nz // self.P, nw // 2 + 1

    def real_slab_shape(self):
        return (self.nxl, self.ny, self.nz, self.nw)

    def spectrum_slab_shape(self):
        if self.layout == "native_xzwy":
            return (self.ny, self.nzl, self.nwh, self.nx)
        return (self.nx, self.ny, self.nzl, self.nwh)

    def _exchange_shape(self):
        return (self.P, self.nxl, self.ny, self.nzl, self.nwh)


def numpy_local(dims, P, layout="slab"):
    """A CPU stand-in of the library's rank-local passes with the same buffer semantics
    (send blocks in destination order, received blocks in source order), for host-logic
    tests without a GPU."""
    return _NumpyLocal(tuple(dims), P, layout)


class _NumpyLocal:
    def __init__(self, dims, P, layout):
        self.dims, self.P, self.layout = dims, P, layout

    def forward_local(self, x, send):
        import numpy as np
        import torch
        P = self.P
        if len(self.dims) == 3:
            _, ny, nz = self.dims
            s = np.fft.rfftn(x.numpy(), axes=(1, 2))                         # [nxl][ny][nzh]
            nxl, nyl = s.shape[0], ny // P
            blocks = s.reshape(nxl, P, nyl, -1).transpose(1, 0, 2, 3)         # [q][nxl][nyl][nzh]
        else:
            _, ny, nz, nw = self.dims
            s = np.fft.fft(np.fft.rfft(x.numpy(), axis=3), axis=2)            # [nxl][ny][nz][nwh]
            nxl, nzl = s.shape[0], nz // P
            blocks = s.reshape(nxl, ny, P, nzl, -1).transpose(2, 0, 1, 3, 4)  # [q][nxl][ny][nzl][nwh]
        send.copy_(torch.from_numpy(np.ascontiguousarray(blocks)).reshape(send.shape))

    def forward_finish(self, recv, out):
        import numpy as np
        import torch
        a = recv.numpy()
        if len(self.dims) == 3:
            nx, ny, nz = self.dims
            t = np.fft.fft(a.reshape(nx, ny // self.P, -1), axis=0)
        else:
            nx, ny, nz, nw = self.dims
            t = np.fft.fft2(a.reshape(nx, ny, nz // self.P, -1), axes=(0, 1))
            if self.layout == "native_xzwy":
                t = t.transpose(1, 2, 3, 0)
        out.copy_(torch.from_numpy(np.ascontiguousarray(t)).reshape(out.shape))

    def backward_local(self, spec, send):
        import numpy as np
        import torch
        a = spec.numpy()
        if len(self.dims) == 3:
            nx = self.dims[0]
            t = np.fft.ifft(a.reshape(nx, -1), axis=0) * nx
        else:
            nx, ny = self.dims[:2]
            if self.layout == "native_xzwy":
                a = a.transpose(3, 0, 1, 2)
            t = np.fft.ifft2(a.reshape(nx, ny, *a.shape[2:]), axes=(0, 1)) * (nx * ny)
        send.copy_(torch.from_numpy(np.ascontiguousarray(t)).reshape(send.shape))

    def backward_finish(self, recv, out):
        import numpy as np
        import torch
        a = recv.numpy()
        P = self.P
        if len(self.dims) == 3:
            nx, ny, nz = self.dims
            nxl, nyl = nx // P, ny // P
            s = a.reshape(P, nxl, nyl, -1).transpose(1, 0, 2, 3).reshape(nxl, ny, -1)
            r = np.fft.irfftn(s, s=(ny, nz), axes=(1, 2)) * (ny * nz)
        else:
            nx, ny, nz, nw = self.dims
            nxl, nzl = nx // P, nz // P
            s = a.reshape(P, nxl, ny, nzl, -1).transpose(1, 2, 0, 3, 4).reshape(nxl, ny, nz, -1)
            r = np.fft.irfft(np.fft.ifft(s, axis=2) * nz, n=nw, axis=3) * nw
        out.copy_(torch.from_numpy(np.ascontiguousarray(r)))
