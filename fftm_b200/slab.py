"""3D R2C / C2R transforms of a field distributed over the ranks of a process group
(one process per GPU on one node), by x slabs: the multi-GPU form of the reference's
fftm slab path (`source/fftm.hpp` slab-pencil with the `same_x` redistribution,
`source/detail/mpi_transpose_3d_same_x.h`), with its MPI exchange replaced by one
all-to-all over the process group (NCCL between GPUs).

Forward, on rank r of P (nx and ny divisible by P, nxl = nx/P, nyl = ny/P):

1. real slab ``[nxl][ny][nz]`` (planes x = r*nxl ...) -> 2D R2C over (y, z) of every
   local plane (one batched library plan) -> ``[nxl][ny][nz/2+1]``;
2. all-to-all: rank q receives ky block q of every rank; the blocks arrive ordered by
   source rank, which is x order, so they form ``[nx][nyl][nz/2+1]`` without unpacking;
3. the x FFT of every (ky, kz) column (one strided library plan) -> the spectrum slab
   ``[kx][nyl][nz/2+1]``: rank r holds ky in [r*nyl, (r+1)*nyl).

Backward is the mirror image (unnormalised C2R, as the reference's).  The library plans
run on the rank's GPU; the exchange is `torch.distributed.all_to_all_single`.

:class:`SlabFFT4D` is the 4D slab-slab form (fftm's ``strategy_4d_slab_slab_mpi`` with the
``same_xw`` redistribution, `source/detail/mpi_transpose_4d_same_xw.h`, real array
``arranger_3210`` = ``[x][y][z][w]``, `source/fftm.hpp:218-228`), nx and nz divisible by P,
nxl = nx/P, nzl = nz/P, nwh = nw/2+1:

1. real slab ``[nxl][ny][nz][nw]`` -> 2D R2C over (z, w) of every (x, y) plane ->
   ``[nxl][ny][nz][nwh]``;
2. all-to-all: rank q receives kz block q of every rank, ordered by source rank (x
   order) -> ``[nx][ny][nzl][nwh]``;
3. the 2D C2C over (x, y) of every (kz, kw) column -> the spectrum slab: ``layout="slab"``
   keeps ``[kx][ky][kzl][kw]`` (ffts' slab spectrum order); ``layout="native_xzwy"``
   first moves x innermost and gives fftm's native ``[ky][kzl][kw][kx]`` (the plan of
   `source/fftm.hpp:2941-2961` with z_size = nzl).
"""
from __future__ import annotations


class _LocalPlans:
    """The rank-local transforms on the GPU: fftb plans with cuFFT advanced layouts."""

    def __init__(self, nx, ny, nz, P, dtype):
        from . import C2CB, C2CF, C2R, R2C, Plan
        nxl, nyl, nzh = nx // P, ny // P, nz // 2 + 1
        self.r2c = Plan(R2C, [ny, nz], [ny, nz], 1, ny * nz, [ny, nzh], 1, ny * nzh, nxl, dtype=dtype)
        self.c2r = Plan(C2R, [ny, nz], [ny, nzh], 1, ny * nzh, [ny, nz], 1, ny * nz, nxl, dtype=dtype)
        cols = nyl * nzh
        self.xf = Plan(C2CF, [nx], [nx], cols, 1, [nx], cols, 1, cols, dtype=dtype)
        self.xb = Plan(C2CB, [nx], [nx], cols, 1, [nx], cols, 1, cols, dtype=dtype)
        import torch
        self._work = []
        for p in (self.r2c, self.c2r, self.xf, self.xb):
            if p.get_work_size() > 0:
                w = torch.empty(p.get_work_size() // 8 + 1, dtype=torch.complex64, device="cuda")
                p.set_work_area(w)
                self._work.append(w)

    def r2c_yz(self, x, out):
        self.r2c.exec(x, out)

    def c2r_yz(self, spec, out):
        self.c2r.exec(spec, out)

    def fft_x(self, t, inverse=False):
        (self.xb if inverse else self.xf).exec(t, t)


class SlabFFT3D:
    """x-slab distributed 3D R2C / C2R over a process group (see the module notes).

    ``local`` replaces the rank-local transforms (an object with ``r2c_yz``, ``c2r_yz``
    and ``fft_x``); the default runs the library's plans on the current GPU."""

    def __init__(self, nx, ny, nz, group=None, dtype="float32", local=None):
        import torch.distributed as dist
        self.dist = dist if dist.is_available() and dist.is_initialized() else None
        self.group = group
        self.P = self.dist.get_world_size(group) if self.dist else 1
        self.rank = self.dist.get_rank(group) if self.dist else 0
        if nx % self.P or ny % self.P:
            raise ValueError(f"nx ({nx}) and ny ({ny}) must be divisible by the {self.P} ranks")
        self.nx, self.ny, self.nz = nx, ny, nz
        self.nxl, self.nyl, self.nzh = nx // self.P, ny // self.P, nz // 2 + 1
        self.local = local if local is not None else _LocalPlans(nx, ny, nz, self.P, dtype)

    # ------------------------------------------------------------------ shapes
    def real_slab_shape(self):
        return (self.nxl, self.ny, self.nz)

    def spectrum_slab_shape(self):
        return (self.nx, self.nyl, self.nzh)

    def _exchange(self, send, recv):
        import torch
        if self.P == 1:
            recv.copy_(send)
            return
        self.dist.all_to_all_single(torch.view_as_real(recv), torch.view_as_real(send), group=self.group)

    # ------------------------------------------------------------------ transforms
    def forward(self, x, out=None):
        """Real slab [nxl][ny][nz] -> spectrum slab [kx][nyl][nz/2+1] (unnormalised)."""
        import torch
        P, nxl, nyl, nzh = self.P, self.nxl, self.nyl, self.nzh
        cdt = torch.complex64 if x.dtype == torch.float32 else torch.complex128
        s = torch.empty((nxl, self.ny, nzh), dtype=cdt, device=x.device)
        self.local.r2c_yz(x, s)
        send = s.view(nxl, P, nyl, nzh).permute(1, 0, 2, 3).contiguous()    # [dest][nxl][nyl][nzh]
        t = out if out is not None else torch.empty((self.nx, nyl, nzh), dtype=cdt, device=x.device)
        self._exchange(send, t.view(P, nxl, nyl, nzh))                       # arrives in x order
        self.local.fft_x(t, inverse=False)
        return t

    def backward(self, spec, out=None):
        """Spectrum slab [kx][nyl][nz/2+1] -> real slab [nxl][ny][nz] (unnormalised C2R;
        spec is overwritten)."""
        import torch
        P, nxl, nyl, nzh = self.P, self.nxl, self.nyl, self.nzh
        self.local.fft_x(spec, inverse=True)
        recv = torch.empty((P, nxl, nyl, nzh), dtype=spec.dtype, device=spec.device)
        self._exchange(spec.view(P, nxl, nyl, nzh).contiguous(), recv)     # [source ky block][nxl][nyl][nzh]
        s = recv.permute(1, 0, 2, 3).contiguous().view(nxl, self.ny, nzh)
        rdt = torch.float32 if spec.dtype == torch.complex64 else torch.float64
        x = out if out is not None else torch.empty((nxl, self.ny, self.nz), dtype=rdt, device=spec.device)
        self.local.c2r_yz(s, x)
        return x


class _LocalPlans4D:
    """The rank-local 4D transforms on the GPU: fftb plans with cuFFT advanced layouts."""

    def __init__(self, nx, ny, nz, nw, P, dtype, layout):
        from . import C2CB, C2CF, C2R, R2C, Plan
        nxl, nzl, nwh = nx // P, nz // P, nw // 2 + 1
        planes = nxl * ny
        self.r2c = Plan(R2C, [nz, nw], [nz, nw], 1, nz * nw, [nz, nwh], 1, nz * nwh, planes, dtype=dtype)
        self.c2r = Plan(C2R, [nz, nw], [nz, nwh], 1, nz * nwh, [nz, nw], 1, nz * nw, planes, dtype=dtype)
        cols = nzl * nwh
        if layout == "native_xzwy":
            # [ky][kzl][kw][kx]: y stride nzl*nwh*nx, x contiguous, batch (kz, kw) nx apart
            emb = [ny, cols * nx]
            args = ([ny, nx], emb, 1, nx, emb, 1, nx, cols)
        else:
            # [kx][ky][kzl][kw]: x stride ny*cols, y stride cols, batch (kz, kw) contiguous
            args = ([nx, ny], [nx, ny], cols, 1, [nx, ny], cols, 1, cols)
        self.xyf = Plan(C2CF, *args, dtype=dtype)
        self.xyb = Plan(C2CB, *args, dtype=dtype)
        import torch
        self._work = []
        for p in (self.r2c, self.c2r, self.xyf, self.xyb):
            if p.get_work_size() > 0:
                w = torch.empty(p.get_work_size() // 8 + 1, dtype=torch.complex64, device="cuda")
                p.set_work_area(w)
                self._work.append(w)

    def r2c_zw(self, x, out):
        self.r2c.exec(x, out)

    def c2r_zw(self, spec, out):
        self.c2r.exec(spec, out)

    def fft_xy(self, t, inverse=False):
        (self.xyb if inverse else self.xyf).exec(t, t)


class SlabFFT4D:
    """x-slab distributed 4D R2C / C2R over a process group, spectrum by kz blocks (see
    the module notes).  ``local`` replaces the rank-local transforms (an object with
    ``r2c_zw``, ``c2r_zw`` and ``fft_xy``)."""

    def __init__(self, nx, ny, nz, nw, group=None, dtype="float32", layout="native_xzwy", local=None):
        import torch.distributed as dist
        if layout not in ("native_xzwy", "slab"):
            raise ValueError(f"layout must be 'native_xzwy' or 'slab', not {layout!r}")
        self.dist = dist if dist.is_available() and dist.is_initialized() else None
        self.group = group
        self.P = self.dist.get_world_size(group) if self.dist else 1
        self.rank = self.dist.get_rank(group) if self.dist else 0
        if nx % self.P or nz % self.P:
            raise ValueError(f"nx ({nx}) and nz ({nz}) must be divisible by the {self.P} ranks")
        self.nx, self.ny, self.nz, self.nw = nx, ny, nz, nw
        self.nxl, self.nzl, self.nwh = nx // self.P, nz // self.P, nw // 2 + 1
        self.layout = layout
        self.local = local if local is not None else _LocalPlans4D(nx, ny, nz, nw, self.P, dtype, layout)

    def real_slab_shape(self):
        return (self.nxl, self.ny, self.nz, self.nw)

    def spectrum_slab_shape(self):
        if self.layout == "native_xzwy":
            return (self.ny, self.nzl, self.nwh, self.nx)
        return (self.nx, self.ny, self.nzl, self.nwh)

    def _exchange(self, send, recv):
        import torch
        if self.P == 1:
            recv.copy_(send)
            return
        self.dist.all_to_all_single(torch.view_as_real(recv), torch.view_as_real(send), group=self.group)

    def forward(self, x):
        """Real slab [nxl][ny][nz][nw] -> spectrum slab (unnormalised)."""
        import torch
        P, nxl, ny, nzl, nwh = self.P, self.nxl, self.ny, self.nzl, self.nwh
        cdt = torch.complex64 if x.dtype == torch.float32 else torch.complex128
        s = torch.empty((nxl, ny, self.nz, nwh), dtype=cdt, device=x.device)
        self.local.r2c_zw(x, s)
        send = s.view(nxl, ny, P, nzl, nwh).permute(2, 0, 1, 3, 4).contiguous()   # [dest][nxl][ny][nzl][nwh]
        t = torch.empty((self.nx, ny, nzl, nwh), dtype=cdt, device=x.device)
        self._exchange(send, t.view(P, nxl, ny, nzl, nwh))                       # arrives in x order
        if self.layout == "native_xzwy":
            t = t.permute(1, 2, 3, 0).contiguous()                               # [ky][kzl][kw][x]
        self.local.fft_xy(t, inverse=False)
        return t

    def backward(self, spec):
        """Spectrum slab -> real slab [nxl][ny][nz][nw] (unnormalised C2R; spec is
        overwritten)."""
        import torch
        P, nxl, ny, nzl, nwh = self.P, self.nxl, self.ny, self.nzl, self.nwh
        self.local.fft_xy(spec, inverse=True)
        t = spec.permute(3, 0, 1, 2).contiguous() if self.layout == "native_xzwy" else spec   # [x][y][zl][wh]
        recv = torch.empty((P, nxl, ny, nzl, nwh), dtype=spec.dtype, device=spec.device)
        self._exchange(t.contiguous().view(P, nxl, ny, nzl, nwh), recv)          # [source kz block][nxl]...
        s = recv.permute(1, 2, 0, 3, 4).contiguous().view(nxl, ny, self.nz, nwh)
        rdt = torch.float32 if spec.dtype == torch.complex64 else torch.float64
        x = torch.empty((nxl, ny, self.nz, self.nw), dtype=rdt, device=spec.device)
        self.local.c2r_zw(s, x)
        return x
