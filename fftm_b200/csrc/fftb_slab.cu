// fftb_slab.cu -- the rank-local part of the slab-distributed 3D and 4D transforms (one
// process per GPU): the multi-GPU form of fftm's slab paths, whose MPI redistributions
// (source/detail/mpi_transpose_3d_same_x.h for 3D, source/detail/mpi_transpose_4d_same_xw.h:
// 437-497 for 4D) pack a send buffer, exchange, and unpack around the FFTs.  Here the pack is
// the store of the last FFT pass before the exchange and the unpack the load of the first
// FFT pass after it (blocked point indices, fftb_pass.cuh), so the exchange moves the
// pass outputs as they are: one contiguous block per destination rank.  The exchange itself
// is the caller's (an NCCL all-to-all, or nothing at all when the pack pass stores straight
// into the peers' receive buffers through the pointer table of set_peers).
//
// 3D (x slabs; nx, ny divisible by P; nxl = nx/P, nyl = ny/P, nzh = nz/2+1), rank r:
//   forward_local:  real [nxl][ny][nz] -> z R2C -> work [nxl][ny][nzh] -> y FFT whose store
//                   writes block q = ky / nyl to send[q][nxl][nyl][nzh] (or peer q's receive
//                   buffer at block r);
//   (exchange: block q to rank q; the received blocks, ordered by source, are [nx][nyl][nzh])
//   forward_finish: x FFT in place on the receive buffer -> spectrum slab [kx][nyl][nzh].
//   backward_local: x FFT^-1 in place on the spectrum slab (its x blocks are the send blocks);
//   (exchange)
//   backward_finish: y FFT^-1 reading ky = q nyl + kyl from receive block q -> work -> z C2R.
// 4D (nx, nz divisible by P; nzl = nz/P, nwh = nw/2+1), same_xw: forward_local w R2C and a z
// FFT storing kz blocks to the ranks; forward_finish the (x, y) FFTs on [nx][ny][nzl][nwh],
// with the x pass writing fftm's native spectrum [ky][kzl][kw][kx] when asked; backward the
// mirror image.
#include <cuda_runtime.h>

#include <cstring>
#include <new>

#include "../../include/fftb.h"
#include "fftb_engine.h"

using namespace fftb;

struct fftb_slab_s {
    int dtype = 0, dim = 3, layout = 0, P = 1, rank = 0;
    long long nx = 0, ny = 0, nz = 0, nw = 0;
    Program fwd_local, fwd_finish, bwd_local, bwd_finish;
    long long real_elems = 0, spec_elems = 0, buf_elems = 0, work_elems = 0;
    void *peers[8] = {nullptr};
    cudaStream_t stream = 0;
};

namespace {

AxisPass mk(int kind, long long n, long long is, long long os, std::vector<Dim> batch, int in_buf, int out_buf)
{
    AxisPass p;
    p.kind = kind;
    p.n = (int)n;
    p.is = is;
    p.os = os;
    p.batch = std::move(batch);
    p.in_buf = in_buf;
    p.out_buf = out_buf;
    return p;
}

// buffers of each program: B_IN, B_OUT, B_WORK as noted per call
int build3d(fftb_slab_s *o)
{
    const long long P = o->P, nx = o->nx, ny = o->ny, nz = o->nz;
    const long long nxl = nx / P, nyl = ny / P, nzh = nz / 2 + 1;
    const int dt = o->dtype;
    int st;
    // forward_local(in = real slab, out = send buffer, work)
    if ((st = program_add(o->fwd_local, dt,
                          mk(K_R2C, nz, 1, 1, {Dim{ny, nz, nzh, 1}, Dim{nxl, ny * nz, ny * nzh, 0}}, B_IN, B_WORK))) !=
        FFTB_SUCCESS)
        return st;
    AxisPass y = mk(K_C2C_FWD, ny, nzh, nzh, {Dim{nzh, 1, 1, 2}, Dim{nxl, ny * nzh, nyl * nzh, 0}}, B_WORK, B_OUT);
    y.out_blk = (int)nyl;
    y.out_hi = nxl * nyl * nzh;
    if ((st = program_add(o->fwd_local, dt, y)) != FFTB_SUCCESS) return st;
    // forward_finish(in = out = receive buffer): x FFT in place
    if ((st = program_add(o->fwd_finish, dt,
                          mk(K_C2C_FWD, nx, nyl * nzh, nyl * nzh, {Dim{nzh, 1, 1, 2}, Dim{nyl, nzh, nzh, 1}}, B_IN,
                             B_IN))) != FFTB_SUCCESS)
        return st;
    // backward_local(in = out = spectrum slab): x FFT^-1 in place
    if ((st = program_add(o->bwd_local, dt,
                          mk(K_C2C_INV, nx, nyl * nzh, nyl * nzh, {Dim{nzh, 1, 1, 2}, Dim{nyl, nzh, nzh, 1}}, B_IN,
                             B_IN))) != FFTB_SUCCESS)
        return st;
    // backward_finish(in = receive buffer, out = real slab, work)
    AxisPass yi = mk(K_C2C_INV, ny, nzh, nzh, {Dim{nzh, 1, 1, 2}, Dim{nxl, nyl * nzh, ny * nzh, 0}}, B_IN, B_WORK);
    yi.in_blk = (int)nyl;
    yi.in_hi = nxl * nyl * nzh;
    if ((st = program_add(o->bwd_finish, dt, yi)) != FFTB_SUCCESS) return st;
    if ((st = program_add(o->bwd_finish, dt,
                          mk(K_C2R, nz, 1, 1, {Dim{ny, nzh, nz, 1}, Dim{nxl, ny * nzh, ny * nz, 0}}, B_WORK, B_OUT))) !=
        FFTB_SUCCESS)
        return st;
    o->real_elems = nxl * ny * nz;
    o->spec_elems = nx * nyl * nzh;
    o->buf_elems = nxl * ny * nzh;  // = nx * nyl * nzh
    o->work_elems = nxl * ny * nzh;
    return FFTB_SUCCESS;
}

int build4d(fftb_slab_s *o)
{
    const long long P = o->P, nx = o->nx, ny = o->ny, nz = o->nz, nw = o->nw;
    const long long nxl = nx / P, nzl = nz / P, nwh = nw / 2 + 1;
    const long long C = nzl * nwh;  // (kzl, kw) columns of a receive block row
    const int dt = o->dtype;
    const bool native = o->layout == FFTB_4D_NATIVE_XZWY;
    int st;
    // forward_local: w R2C of [nxl][ny][nz][nw] -> work [nxl][ny][nz][nwh]; z FFT storing kz
    // blocks: block q is [nxl][ny][nzl][nwh]
    if ((st = program_add(o->fwd_local, dt,
                          mk(K_R2C, nw, 1, 1, {Dim{nz, nw, nwh, 2}, Dim{nxl * ny, nz * nw, nz * nwh, 1}}, B_IN,
                             B_WORK))) != FFTB_SUCCESS)
        return st;
    AxisPass z = mk(K_C2C_FWD, nz, nwh, nwh, {Dim{nwh, 1, 1, 3}, Dim{nxl * ny, nz * nwh, C, 1}}, B_WORK, B_OUT);
    z.out_blk = (int)nzl;
    z.out_hi = nxl * ny * C;
    if ((st = program_add(o->fwd_local, dt, z)) != FFTB_SUCCESS) return st;
    // forward_finish: on the receive buffer [nx][ny][nzl][nwh]: y FFT in place, then the x FFT
    // in place (slab) or into out as [ky][kzl][kw][kx] (native)
    if ((st = program_add(o->fwd_finish, dt,
                          mk(K_C2C_FWD, ny, C, C, {Dim{C, 1, 1, 3}, Dim{nx, ny * C, ny * C, 0}}, B_IN, B_IN))) !=
        FFTB_SUCCESS)
        return st;
    if (native) {
        if ((st = program_add(o->fwd_finish, dt,
                              mk(K_C2C_FWD, nx, ny * C, 1, {Dim{C, 1, nx, 3}, Dim{ny, C, C * nx, 1}}, B_IN, B_OUT))) !=
            FFTB_SUCCESS)
            return st;
    } else if ((st = program_add(o->fwd_finish, dt,
                                 mk(K_C2C_FWD, nx, ny * C, ny * C, {Dim{C, 1, 1, 3}, Dim{ny, C, C, 1}}, B_IN, B_IN))) !=
               FFTB_SUCCESS) {
        return st;
    }
    // backward_local(in = spectrum slab, out = send buffer [nx][ny][nzl][nwh]): x FFT^-1 (from
    // the native layout, or in place), then y FFT^-1 in place on the send buffer
    if (native) {
        if ((st = program_add(o->bwd_local, dt,
                              mk(K_C2C_INV, nx, 1, ny * C, {Dim{C, nx, 1, 3}, Dim{ny, C * nx, C, 1}}, B_IN, B_OUT))) !=
            FFTB_SUCCESS)
            return st;
    } else if ((st = program_add(o->bwd_local, dt,
                                 mk(K_C2C_INV, nx, ny * C, ny * C, {Dim{C, 1, 1, 3}, Dim{ny, C, C, 1}}, B_IN, B_OUT))) !=
               FFTB_SUCCESS) {
        return st;
    }
    if ((st = program_add(o->bwd_local, dt,
                          mk(K_C2C_INV, ny, C, C, {Dim{C, 1, 1, 3}, Dim{nx, ny * C, ny * C, 0}}, B_OUT, B_OUT))) !=
        FFTB_SUCCESS)
        return st;
    // backward_finish(in = receive buffer [q][nxl][ny][nzl][nwh], out = real slab, work):
    // z FFT^-1 reading kz = q nzl + kzl from block q, then w C2R
    AxisPass zi = mk(K_C2C_INV, nz, nwh, nwh, {Dim{nwh, 1, 1, 3}, Dim{nxl * ny, C, nz * nwh, 1}}, B_IN, B_WORK);
    zi.in_blk = (int)nzl;
    zi.in_hi = nxl * ny * C;
    if ((st = program_add(o->bwd_finish, dt, zi)) != FFTB_SUCCESS) return st;
    if ((st = program_add(o->bwd_finish, dt,
                          mk(K_C2R, nw, 1, 1, {Dim{nz, nwh, nw, 2}, Dim{nxl * ny, nz * nwh, nz * nw, 1}}, B_WORK,
                             B_OUT))) != FFTB_SUCCESS)
        return st;
    o->real_elems = nxl * ny * nz * nw;
    o->spec_elems = nx * ny * C;
    o->buf_elems = nx * ny * C;  // = nxl * ny * nz * nwh
    o->work_elems = nxl * ny * nz * nwh;
    return FFTB_SUCCESS;
}

// the pack pass's block bases: the peers' receive buffers (block `rank` of each), if set
int exec_with_peers(fftb_slab_s *o, const Program &prog, void *in, void *out, void *work)
{
    bool any = false;
    for (int q = 0; q < o->P; ++q) any = any || o->peers[q];
    if (!any) return program_exec(prog, in, out, work, o->stream);
    Program p = prog;  // the pack pass reads its bases from the launch arguments
    for (Launch &L : p.launches)
        if (L.args.out_blk)
            for (int q = 0; q < o->P; ++q) L.args.out_peer[q] = o->peers[q];
    return program_exec(p, in, out, work, o->stream);
}

} // namespace

extern "C" {

int fftb_slab_create(int dtype, long long nx, long long ny, long long nz, long long nw, int layout4d, int nranks,
                     int rank, fftb_slab *obj)
{
    if (!obj) return FFTB_ERROR_INVALID_VALUE;
    *obj = nullptr;
    if ((dtype != FFTB_F32 && dtype != FFTB_F64) || nranks < 1 || nranks > 8 || rank < 0 || rank >= nranks ||
        nx < 2 || ny < 2 || nz < 2 || nw < 0 || nw == 1)
        return FFTB_ERROR_INVALID_VALUE;
    const int dim = nw ? 4 : 3;
    if (nx % nranks || (dim == 3 ? ny % nranks : nz % nranks)) {
        set_last_error("the slab axes must be divisible by the rank count");
        return FFTB_ERROR_INVALID_VALUE;
    }
    if (dim == 4 && layout4d != FFTB_4D_SLAB && layout4d != FFTB_4D_NATIVE_XZWY) return FFTB_ERROR_INVALID_VALUE;
    fftb_slab_s *o = new (std::nothrow) fftb_slab_s();
    if (!o) return FFTB_ERROR_ALLOC;
    o->dtype = dtype;
    o->dim = dim;
    o->layout = layout4d;
    o->P = nranks;
    o->rank = rank;
    o->nx = nx;
    o->ny = ny;
    o->nz = nz;
    o->nw = nw;
    const int st = dim == 3 ? build3d(o) : build4d(o);
    if (st != FFTB_SUCCESS) {
        delete o;
        return st;
    }
    *obj = o;
    return FFTB_SUCCESS;
}

int fftb_slab_destroy(fftb_slab o)
{
    if (!o) return FFTB_ERROR_INVALID_HANDLE;
    delete o;
    return FFTB_SUCCESS;
}

int fftb_slab_sizes(fftb_slab o, long long *real_elems, long long *spectrum_elems, long long *exchange_elems,
                    long long *work_elems)
{
    if (!o) return FFTB_ERROR_INVALID_HANDLE;
    if (real_elems) *real_elems = o->real_elems;
    if (spectrum_elems) *spectrum_elems = o->spec_elems;
    if (exchange_elems) *exchange_elems = o->buf_elems;
    if (work_elems) *work_elems = o->work_elems;
    return FFTB_SUCCESS;
}

int fftb_slab_set_stream(fftb_slab o, void *stream)
{
    if (!o) return FFTB_ERROR_INVALID_HANDLE;
    o->stream = (cudaStream_t)stream;
    return FFTB_SUCCESS;
}

int fftb_slab_set_peers(fftb_slab o, void *const *receive_blocks)
{
    if (!o) return FFTB_ERROR_INVALID_HANDLE;
    for (int q = 0; q < 8; ++q) o->peers[q] = (receive_blocks && q < o->P) ? receive_blocks[q] : nullptr;
    return FFTB_SUCCESS;
}

int fftb_slab_forward_local(fftb_slab o, const void *in, void *send, void *work)
{
    if (!o) return FFTB_ERROR_INVALID_HANDLE;
    if (!in || !send || !work) return FFTB_ERROR_INVALID_VALUE;
    return exec_with_peers(o, o->fwd_local, const_cast<void *>(in), send, work);
}

int fftb_slab_forward_finish(fftb_slab o, void *recv, void *out)
{
    if (!o) return FFTB_ERROR_INVALID_HANDLE;
    if (!recv || (o->dim == 4 && o->layout == FFTB_4D_NATIVE_XZWY && !out)) return FFTB_ERROR_INVALID_VALUE;
    return program_exec(o->fwd_finish, recv, out ? out : recv, nullptr, o->stream);
}

int fftb_slab_backward_local(fftb_slab o, void *spec, void *send)
{
    if (!o) return FFTB_ERROR_INVALID_HANDLE;
    if (!spec || (o->dim == 4 && !send)) return FFTB_ERROR_INVALID_VALUE;
    return program_exec(o->bwd_local, spec, send ? send : spec, nullptr, o->stream);
}

int fftb_slab_backward_finish(fftb_slab o, void *recv, void *out, void *work)
{
    if (!o) return FFTB_ERROR_INVALID_HANDLE;
    if (!recv || !out || !work) return FFTB_ERROR_INVALID_VALUE;
    return program_exec(o->bwd_finish, recv, out, work, o->stream);
}

} // extern "C"
