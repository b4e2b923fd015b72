// fftb_ffts.cu -- the `ffts` transform objects (replacement for fftm::ffts,
// reference source/ffts.hpp:159-383) on the pass engine.
//
// Every stage of the reference pipeline (cuFFT plan + SCFD transpose functor)
// becomes one pass of the engine whose load/store geometry absorbs the
// transpose; the Poisson / filter multiply becomes the epilogue of a
// forward-multiply-inverse "sandwich" pass on the last axis, and the 1/N scale
// the epilogue of the final C2R pass.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <new>
#include <string>

#include "../../include/fftb.h"
#include "fftb_device.cuh"
#include "fftb_engine.h"
#include "fftb_fused3d.h"
#include "fftb_profile.h"

using namespace fftb;

struct fftb_ffts_s {
    int dtype = 0, dim = 0, layout = 0;
    long long nx = 0, ny = 0, nz = 0, nw = 0;
    Program fwd, bwd, bwd_norm, poisson, filter;
    Program fwd_adj, bwd_adj;  // adjoints of forward (weighted C2R) and of backward (weighted R2C)
    size_t work_bytes = 0;
    void *work = nullptr;
    bool own_work = false;
    cudaStream_t stream = 0;
    Fused3D fused;   // specialised 3D kernels (when the size has them)
    Fused4D fused4;  // specialised 4D slab / native_xzwy kernels
    LaunchTimer timer;
    bool timing = false;
    void *dspec = nullptr;  // spectrum buffers of the derivative calls (allocated on first use)
    void *dspec2 = nullptr;
    size_t dspec_bytes = 0;
    // profiling (ffts_init_options): scopes per API call, memory entries, print flags
    Profiler prof;
    MemProfiler mem;
    int print_flags = 0;  // bit 0 profile summary, 1 profile totals, 2 memory profile, 3 memory totals
};

namespace {

AxisPass mkpass(int kind, long long n, long long is, long long os, std::vector<Dim> batch, int in_buf, int out_buf)
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

AxisPass with_scale(AxisPass p, double s)
{
    p.ep_mode |= EP_SCALE;
    p.ep_scale = s;
    return p;
}

AxisPass sandwich(AxisPass p, std::vector<EpAxis> axes)
{
    p.kind = K_SANDWICH;
    p.ep_mode = EP_SCALE | EP_POISSON;
    p.ep_axes = std::move(axes);
    p.ep_dynamic = 1;
    return p;
}

// EP_HALFW epilogue: interior bins of the half axis (batch dim `dim_id`, full length n) times w
AxisPass halfw(AxisPass p, int dim_id, long long n, double w)
{
    p.ep_mode |= EP_HALFW;
    p.ep_hw = w;
    p.ep_axes = {EpAxis{0, dim_id, (int)n, 1}};
    return p;
}

#define TRY(x)                                                                                                        \
    do {                                                                                                              \
        int _s = (x);                                                                                                 \
        if (_s != FFTB_SUCCESS) return _s;                                                                            \
    } while (0)

int build_2d(fftb_ffts_s *o)
{
    const long long nx = o->nx, ny = o->ny, nyh = ny / 2 + 1;
    const double invN = 1.0 / (double)(nx * ny);
    const int d = o->dtype;
    AxisPass r2c = mkpass(K_R2C, ny, 1, 1, {Dim{nx, ny, nyh, 0}}, B_IN, B_OUT);
    AxisPass xf = mkpass(K_C2C_FWD, nx, nyh, nyh, {Dim{nyh, 1, 1, 1}}, B_OUT, B_OUT);
    TRY(program_add(o->fwd, d, r2c));
    TRY(program_add(o->fwd, d, xf));
    AxisPass xi = mkpass(K_C2C_INV, nx, nyh, nyh, {Dim{nyh, 1, 1, 1}}, B_IN, B_IN);
    AxisPass c2r = mkpass(K_C2R, ny, 1, 1, {Dim{nx, nyh, ny, 0}}, B_IN, B_OUT);
    TRY(program_add(o->bwd, d, xi));
    TRY(program_add(o->bwd, d, c2r));
    TRY(program_add(o->bwd_norm, d, xi));
    TRY(program_add(o->bwd_norm, d, with_scale(c2r, invN)));
    TRY(program_add(o->fwd_adj, d, halfw(xi, 1, ny, 0.5)));
    TRY(program_add(o->fwd_adj, d, c2r));
    TRY(program_add(o->bwd_adj, d, r2c));
    TRY(program_add(o->bwd_adj, d, halfw(xf, 1, ny, 2.0)));
    for (int f = 0; f < 2; ++f) {
        Program &pr = f ? o->filter : o->poisson;
        AxisPass a = r2c;
        a.out_buf = B_WORK;
        AxisPass s = xf;
        s.in_buf = s.out_buf = B_WORK;
        s = sandwich(s, {EpAxis{1, -1, (int)nx, 0}, EpAxis{0, 1, (int)ny, 1}});
        AxisPass c = with_scale(c2r, invN);
        c.in_buf = B_WORK;
        TRY(program_add(pr, d, a));
        TRY(program_add(pr, d, s));
        TRY(program_add(pr, d, c));
    }
    o->work_bytes = complex_bytes(d) * (size_t)(nx * nyh);
    return FFTB_SUCCESS;
}

int build_3d(fftb_ffts_s *o)
{
    const long long nx = o->nx, ny = o->ny, nz = o->nz, nzh = nz / 2 + 1, C3 = ny * nzh;
    const double invN = 1.0 / (double)(nx * ny * nz);
    const int d = o->dtype;
    // forward_3d: source/ffts.hpp:680-686
    AxisPass zr = mkpass(K_R2C, nz, 1, 1, {Dim{ny, nz, nzh, 1}, Dim{nx, ny * nz, C3, 0}}, B_IN, B_OUT);
    AxisPass yf = mkpass(K_C2C_FWD, ny, nzh, nzh, {Dim{nzh, 1, 1, 2}, Dim{nx, C3, C3, 0}}, B_OUT, B_OUT);
    AxisPass xf = mkpass(K_C2C_FWD, nx, C3, C3, {Dim{nzh, 1, 1, 2}, Dim{ny, nzh, nzh, 1}}, B_OUT, B_OUT);
    TRY(program_add(o->fwd, d, zr));
    TRY(program_add(o->fwd, d, yf));
    TRY(program_add(o->fwd, d, xf));
    // inverse_3d: source/ffts.hpp:688-694 (destructive on the spectrum, like cuFFT C2R)
    AxisPass xi = mkpass(K_C2C_INV, nx, C3, C3, {Dim{nzh, 1, 1, 2}, Dim{ny, nzh, nzh, 1}}, B_IN, B_IN);
    AxisPass yi = mkpass(K_C2C_INV, ny, nzh, nzh, {Dim{nzh, 1, 1, 2}, Dim{nx, C3, C3, 0}}, B_IN, B_IN);
    AxisPass zc = mkpass(K_C2R, nz, 1, 1, {Dim{ny, nzh, nz, 1}, Dim{nx, C3, ny * nz, 0}}, B_IN, B_OUT);
    TRY(program_add(o->bwd, d, xi));
    TRY(program_add(o->bwd, d, yi));
    TRY(program_add(o->bwd, d, zc));
    TRY(program_add(o->bwd_norm, d, xi));
    TRY(program_add(o->bwd_norm, d, yi));
    TRY(program_add(o->bwd_norm, d, with_scale(zc, invN)));
    TRY(program_add(o->fwd_adj, d, halfw(xi, 2, nz, 0.5)));
    TRY(program_add(o->fwd_adj, d, yi));
    TRY(program_add(o->fwd_adj, d, zc));
    TRY(program_add(o->bwd_adj, d, zr));
    TRY(program_add(o->bwd_adj, d, yf));
    TRY(program_add(o->bwd_adj, d, halfw(xf, 2, nz, 2.0)));
    for (int f = 0; f < 2; ++f) {
        Program &pr = f ? o->filter : o->poisson;
        AxisPass a = zr;
        a.out_buf = B_WORK;
        AxisPass y1 = yf;
        y1.in_buf = y1.out_buf = B_WORK;
        AxisPass s = xf;
        s.in_buf = s.out_buf = B_WORK;
        s = sandwich(s, {EpAxis{1, -1, (int)nx, 0}, EpAxis{0, 1, (int)ny, 0}, EpAxis{0, 2, (int)nz, 1}});
        AxisPass y2 = yi;
        y2.in_buf = y2.out_buf = B_WORK;
        AxisPass c = with_scale(zc, invN);
        c.in_buf = B_WORK;
        TRY(program_add(pr, d, a));
        TRY(program_add(pr, d, y1));
        TRY(program_add(pr, d, s));
        TRY(program_add(pr, d, y2));
        TRY(program_add(pr, d, c));
    }
    o->work_bytes = complex_bytes(d) * (size_t)(nx * C3);
    return FFTB_SUCCESS;
}

int build_4d(fftb_ffts_s *o)
{
    const long long nx = o->nx, ny = o->ny, nz = o->nz, nw = o->nw, nwh = nw / 2 + 1;
    const double invN = 1.0 / (double)(nx * ny * nz * nw);
    const int d = o->dtype;
    o->work_bytes = complex_bytes(d) * (size_t)(nx * ny * nz * nwh);
    if (o->layout == FFTB_4D_SLAB || o->layout == FFTB_4D_NATIVE_XZWY) {
        const long long C = nz * nwh;
        // slab stage 0: 2D R2C over (z,w) per (x,y) (source/ffts.hpp:751-763), split into w then z
        AxisPass wr = mkpass(K_R2C, nw, 1, 1,
                             {Dim{nz, nw, nwh, 2}, Dim{ny, nz * nw, C, 1}, Dim{nx, ny * nz * nw, ny * C, 0}}, B_IN,
                             B_OUT);
        AxisPass zf = mkpass(K_C2C_FWD, nz, nwh, nwh, {Dim{nwh, 1, 1, 3}, Dim{ny, C, C, 1}, Dim{nx, ny * C, ny * C, 0}},
                             B_OUT, B_OUT);
        AxisPass yf = mkpass(K_C2C_FWD, ny, C, C, {Dim{nwh, 1, 1, 3}, Dim{nz, nwh, nwh, 2}, Dim{nx, ny * C, ny * C, 0}},
                             B_OUT, B_OUT);
        AxisPass xf = mkpass(K_C2C_FWD, nx, ny * C, ny * C, {Dim{nwh, 1, 1, 3}, Dim{nz, nwh, nwh, 2}, Dim{ny, C, C, 1}},
                             B_OUT, B_OUT);
        AxisPass wc = mkpass(K_C2R, nw, 1, 1,
                             {Dim{nz, nwh, nw, 2}, Dim{ny, C, nz * nw, 1}, Dim{nx, ny * C, ny * nz * nw, 0}}, B_IN,
                             B_OUT);
        auto on = [](AxisPass p, int ib, int ob) { p.in_buf = ib; p.out_buf = ob; return p; };
        auto inv = [](AxisPass p) { p.kind = K_C2C_INV; return p; };
        if (o->layout == FFTB_4D_SLAB) {
            TRY(program_add(o->fwd, d, wr));
            TRY(program_add(o->fwd, d, zf));
            TRY(program_add(o->fwd, d, yf));
            TRY(program_add(o->fwd, d, xf));
            TRY(program_add(o->fwd_adj, d, halfw(on(inv(xf), B_IN, B_IN), 3, nw, 0.5)));
            TRY(program_add(o->fwd_adj, d, on(inv(yf), B_IN, B_IN)));
            TRY(program_add(o->fwd_adj, d, on(inv(zf), B_IN, B_IN)));
            TRY(program_add(o->fwd_adj, d, wc));
            TRY(program_add(o->bwd_adj, d, wr));
            TRY(program_add(o->bwd_adj, d, zf));
            TRY(program_add(o->bwd_adj, d, yf));
            TRY(program_add(o->bwd_adj, d, halfw(xf, 3, nw, 2.0)));
            for (int nrm = 0; nrm < 2; ++nrm) {
                Program &pr = nrm ? o->bwd_norm : o->bwd;
                TRY(program_add(pr, d, on(inv(xf), B_IN, B_IN)));
                TRY(program_add(pr, d, on(inv(yf), B_IN, B_IN)));
                TRY(program_add(pr, d, on(inv(zf), B_IN, B_IN)));
                TRY(program_add(pr, d, nrm ? with_scale(wc, invN) : wc));
            }
        } else {
            // native_xzwy: the (y,x) C2C of source/fftm.hpp:2941-2961 with the local permute to
            // [ky][kz][kw][kx] fused into the x pass
            TRY(program_add(o->fwd, d, on(wr, B_IN, B_WORK)));
            TRY(program_add(o->fwd, d, on(zf, B_WORK, B_WORK)));
            TRY(program_add(o->fwd, d, on(yf, B_WORK, B_WORK)));
            AxisPass xp = mkpass(K_C2C_FWD, nx, ny * C, 1,
                                 {Dim{nwh, 1, nx, 3}, Dim{nz, nwh, nwh * nx, 2}, Dim{ny, C, C * nx, 1}}, B_WORK, B_OUT);
            TRY(program_add(o->fwd, d, xp));
            AxisPass xq = mkpass(K_C2C_INV, nx, 1, ny * C,
                                 {Dim{nwh, nx, 1, 3}, Dim{nz, nwh * nx, nwh, 2}, Dim{ny, C * nx, C, 1}}, B_IN, B_WORK);
            TRY(program_add(o->fwd_adj, d, halfw(xq, 3, nw, 0.5)));
            TRY(program_add(o->fwd_adj, d, on(inv(yf), B_WORK, B_WORK)));
            TRY(program_add(o->fwd_adj, d, on(inv(zf), B_WORK, B_WORK)));
            TRY(program_add(o->fwd_adj, d, on(wc, B_WORK, B_OUT)));
            TRY(program_add(o->bwd_adj, d, on(wr, B_IN, B_WORK)));
            TRY(program_add(o->bwd_adj, d, on(zf, B_WORK, B_WORK)));
            TRY(program_add(o->bwd_adj, d, on(yf, B_WORK, B_WORK)));
            TRY(program_add(o->bwd_adj, d, halfw(xp, 3, nw, 2.0)));
            for (int nrm = 0; nrm < 2; ++nrm) {
                Program &pr = nrm ? o->bwd_norm : o->bwd;
                TRY(program_add(pr, d, xq));
                TRY(program_add(pr, d, on(inv(yf), B_WORK, B_WORK)));
                TRY(program_add(pr, d, on(inv(zf), B_WORK, B_WORK)));
                TRY(program_add(pr, d, on(nrm ? with_scale(wc, invN) : wc, B_WORK, B_OUT)));
            }
        }
        for (int f = 0; f < 2; ++f) {
            Program &pr = f ? o->filter : o->poisson;
            TRY(program_add(pr, d, on(wr, B_IN, B_WORK)));
            TRY(program_add(pr, d, on(zf, B_WORK, B_WORK)));
            TRY(program_add(pr, d, on(yf, B_WORK, B_WORK)));
            TRY(program_add(pr, d, sandwich(on(xf, B_WORK, B_WORK),
                                            {EpAxis{1, -1, (int)nx, 0}, EpAxis{0, 1, (int)ny, 0},
                                             EpAxis{0, 2, (int)nz, 0}, EpAxis{0, 3, (int)nw, 1}})));
            TRY(program_add(pr, d, on(inv(yf), B_WORK, B_WORK)));
            TRY(program_add(pr, d, on(inv(zf), B_WORK, B_WORK)));
            TRY(program_add(pr, d, on(with_scale(wc, invN), B_WORK, B_OUT)));
        }
    } else if (o->layout == FFTB_4D_PENCIL) {
        const long long Vs = nx * ny * nz;
        // forward_w .. forward_x with the three transposes of source/ffts.hpp:809-825 fused
        AxisPass wr = mkpass(K_R2C, nw, Vs, Vs, {Dim{nx, 1, 1, 0}, Dim{ny, nx, nx, 1}, Dim{nz, nx * ny, nx * ny, 2}},
                             B_IN, B_WORK);
        AxisPass zf = mkpass(K_C2C_FWD, nz, nx * ny, nx * ny,
                             {Dim{nx, 1, 1, 0}, Dim{ny, nx, nx, 1}, Dim{nwh, Vs, Vs, 3}}, B_WORK, B_WORK);
        AxisPass yf = mkpass(K_C2C_FWD, ny, nx, nx,
                             {Dim{nx, 1, 1, 0}, Dim{nz, nx * ny, nx * ny, 2}, Dim{nwh, Vs, Vs, 3}}, B_WORK, B_WORK);
        AxisPass xp = mkpass(K_C2C_FWD, nx, 1, 1,
                             {Dim{ny, nx, nz * nwh * nx, 1}, Dim{nz, nx * ny, nwh * nx, 2}, Dim{nwh, Vs, nx, 3}},
                             B_WORK, B_OUT);
        AxisPass xq = mkpass(K_C2C_INV, nx, 1, 1,
                             {Dim{ny, nz * nwh * nx, nx, 1}, Dim{nz, nwh * nx, nx * ny, 2}, Dim{nwh, nx, Vs, 3}},
                             B_IN, B_WORK);
        AxisPass wc = mkpass(K_C2R, nw, Vs, Vs, {Dim{nx, 1, 1, 0}, Dim{ny, nx, nx, 1}, Dim{nz, nx * ny, nx * ny, 2}},
                             B_WORK, B_OUT);
        auto inv = [](AxisPass p) { p.kind = K_C2C_INV; return p; };
        TRY(program_add(o->fwd, d, wr));
        TRY(program_add(o->fwd, d, zf));
        TRY(program_add(o->fwd, d, yf));
        TRY(program_add(o->fwd, d, xp));
        TRY(program_add(o->fwd_adj, d, halfw(xq, 3, nw, 0.5)));
        TRY(program_add(o->fwd_adj, d, inv(yf)));
        TRY(program_add(o->fwd_adj, d, inv(zf)));
        TRY(program_add(o->fwd_adj, d, wc));
        TRY(program_add(o->bwd_adj, d, wr));
        TRY(program_add(o->bwd_adj, d, zf));
        TRY(program_add(o->bwd_adj, d, yf));
        TRY(program_add(o->bwd_adj, d, halfw(xp, 3, nw, 2.0)));
        for (int nrm = 0; nrm < 2; ++nrm) {
            Program &pr = nrm ? o->bwd_norm : o->bwd;
            TRY(program_add(pr, d, xq));
            TRY(program_add(pr, d, inv(yf)));
            TRY(program_add(pr, d, inv(zf)));
            TRY(program_add(pr, d, nrm ? with_scale(wc, invN) : wc));
        }
        AxisPass xs = mkpass(K_C2C_FWD, nx, 1, 1, {Dim{ny, nx, nx, 1}, Dim{nz, nx * ny, nx * ny, 2}, Dim{nwh, Vs, Vs, 3}},
                             B_WORK, B_WORK);
        for (int f = 0; f < 2; ++f) {
            Program &pr = f ? o->filter : o->poisson;
            TRY(program_add(pr, d, wr));
            TRY(program_add(pr, d, zf));
            TRY(program_add(pr, d, yf));
            TRY(program_add(pr, d, sandwich(xs, {EpAxis{1, -1, (int)nx, 0}, EpAxis{0, 1, (int)ny, 0},
                                                 EpAxis{0, 2, (int)nz, 0}, EpAxis{0, 3, (int)nw, 1}})));
            TRY(program_add(pr, d, inv(yf)));
            TRY(program_add(pr, d, inv(zf)));
            TRY(program_add(pr, d, with_scale(wc, invN)));
        }
    } else {
        return FFTB_ERROR_INVALID_VALUE;
    }
    return FFTB_SUCCESS;
}

bool aligned16(const void *a, const void *b) { return ((uintptr_t)a % 16 == 0) && ((uintptr_t)b % 16 == 0); }

int ensure_work(fftb_ffts_s *o)
{
    if (o->work || o->work_bytes == 0) return FFTB_SUCCESS;
    void *p = nullptr;
    cudaError_t e = cudaMalloc(&p, o->work_bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return FFTB_ERROR_ALLOC;
    }
    o->work = p;
    o->own_work = true;
    o->mem.set_bytes("ffts/shared_work_buffer", (long long)o->work_bytes);
    return FFTB_SUCCESS;
}

bool needs_work(const Program &p)
{
    for (const Launch &L : p.launches)
        if (L.in_buf == B_WORK || L.out_buf == B_WORK) return true;
    return false;
}

int run(fftb_ffts_s *o, const Program &p, const void *in, void *out, const EpValues *ep)
{
    if (needs_work(p)) {
        int st = ensure_work(o);
        if (st != FFTB_SUCCESS) return st;
    }
    return program_exec(p, const_cast<void *>(in), out, o->work, o->stream, ep, o->timing ? &o->timer : nullptr);
}

// ---------------------------------------------------------------- standalone spectral multiply
template <typename R>
__global__ void spectrum_poisson_kernel(cpx<R> *s, long long total, int4 dims, int4 ns, int half_axis, R sign,
                                        R scale)
{
    const int d[4] = {dims.x, dims.y, dims.z, dims.w};
    const int n[4] = {ns.x, ns.y, ns.z, ns.w};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        long long r = i;
        R k2 = R(0);
#pragma unroll
        for (int a = 3; a >= 0; --a) {
            const int idx = (int)(r % d[a]);
            r /= d[a];
            const int k = (a == half_axis) ? idx : (idx <= n[a] / 2 ? idx : idx - n[a]);
            k2 += R(k) * R(k);
        }
        cpx<R> v = s[i];
        const R f = (k2 == R(0)) ? R(0) : scale * sign / k2;
        v.x *= f;
        v.y *= f;
        s[i] = v;
    }
}

// out = i k_slot * in * scale: the spectral derivative of the reference's
// derivative_spectra_functor (source/tests/test_3D_poisson.cu:113-145), with k = idx on
// the half axis and k = idx <= n/2 ? idx : idx - n on the full axes (Nyquist kept, as there).
template <typename R>
__global__ void spectrum_derivative_kernel(const cpx<R> *in, cpx<R> *out, long long total, int4 dims, int4 ns,
                                           int half_axis, int slot, R scale)
{
    const int d[4] = {dims.x, dims.y, dims.z, dims.w};
    const int n[4] = {ns.x, ns.y, ns.z, ns.w};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        long long r = i;
        int k = 0;
#pragma unroll
        for (int a = 3; a >= 0; --a) {
            const int idx = (int)(r % d[a]);
            r /= d[a];
            if (a == slot) k = (a == half_axis) ? idx : (idx <= n[a] / 2 ? idx : idx - n[a]);
        }
        const cpx<R> v = in[i];
        const R f = R(k) * scale;
        cpx<R> w;
        w.x = -f * v.y;
        w.y = f * v.x;
        out[i] = w;
    }
}

// Zeroes the modes outside a box (the turbulence example's spectral truncations,
// examples/turbulence/source/taylor_green_kernels.h:41-44, 186-200): rule 0 keeps
// |k_a| <= n_a / 3 on every axis (two-thirds dealiasing), rule 1 keeps |k_a| <= cutoff
// (cutoff <= 0 keeps everything).  k as in the derivative (signed on full axes).
template <typename R>
__global__ void spectrum_truncate_kernel(cpx<R> *s, long long total, int4 dims, int4 ns, int half_axis, int rule,
                                         int cutoff)
{
    const int d[4] = {dims.x, dims.y, dims.z, dims.w};
    const int n[4] = {ns.x, ns.y, ns.z, ns.w};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        long long r = i;
        bool keep = true;
#pragma unroll
        for (int a = 3; a >= 0; --a) {
            const int idx = (int)(r % d[a]);
            r /= d[a];
            if (n[a] <= 1) continue;  // unused slot
            const int k = (a == half_axis) ? idx : (idx <= n[a] / 2 ? idx : idx - n[a]);
            const int ak = k < 0 ? -k : k;
            if (rule == 0 ? ak > n[a] / 3 : (cutoff > 0 && ak > cutoff)) keep = false;
        }
        if (!keep) {
            cpx<R> z;
            z.x = R(0);
            z.y = R(0);
            s[i] = z;
        }
    }
}

// index geometry of the object's spectrum: slot extents, axis lengths, the half axis
// slot, and the slot of each logical axis x, y, z, w
void spectrum_geometry(const fftb_ffts_s *o, int4 &dims, int4 &ns, int &half_axis, int (&slot)[4])
{
    if (o->dim == 2) {
        dims = make_int4(1, 1, (int)o->nx, (int)(o->ny / 2 + 1));
        ns = make_int4(1, 1, (int)o->nx, (int)o->ny);
        half_axis = 3;
        slot[0] = 2; slot[1] = 3; slot[2] = slot[3] = -1;
    } else if (o->dim == 3) {
        dims = make_int4(1, (int)o->nx, (int)o->ny, (int)(o->nz / 2 + 1));
        ns = make_int4(1, (int)o->nx, (int)o->ny, (int)o->nz);
        half_axis = 3;
        slot[0] = 1; slot[1] = 2; slot[2] = 3; slot[3] = -1;
    } else if (o->layout == FFTB_4D_SLAB) {
        dims = make_int4((int)o->nx, (int)o->ny, (int)o->nz, (int)(o->nw / 2 + 1));
        ns = make_int4((int)o->nx, (int)o->ny, (int)o->nz, (int)o->nw);
        half_axis = 3;
        slot[0] = 0; slot[1] = 1; slot[2] = 2; slot[3] = 3;
    } else {
        dims = make_int4((int)o->ny, (int)o->nz, (int)(o->nw / 2 + 1), (int)o->nx);
        ns = make_int4((int)o->ny, (int)o->nz, (int)o->nw, (int)o->nx);
        half_axis = 2;
        slot[0] = 3; slot[1] = 0; slot[2] = 1; slot[3] = 2;
    }
}

} // namespace

namespace {
// "ffts::<what><D>" scope names of the profiler (built only when profiling is on)
std::string scope_name(const fftb_ffts_s *o, const char *what)
{
    return std::string("ffts::") + what + "<" + std::to_string(o->dim) + ">";
}
} // namespace
#define FFTB_PROFILE_SCOPE(o, what)                                                                                   \
    ProfScope _prof_scope((o)->prof, (o)->prof.enabled ? scope_name((o), (what)) : std::string(), (o)->stream)

extern "C" {

void fftb_init_options_default(fftb_init_options *opt)
{
    if (!opt) return;
    opt->profiling_key = "ffts_prof";
    opt->memory_profiling_key = "ffts_mem";
    opt->print_profile_summary_on_destroy = 1;
    opt->print_profile_totals_on_destroy = 1;
    opt->print_memory_profile_on_destroy = 1;
    opt->print_memory_totals_on_destroy = 1;
}

int fftb_ffts_create(int dtype, long long nx, long long ny, long long nz, long long nw, int layout4d, fftb_ffts *obj)
{
    fftb_init_options off = {nullptr, nullptr, 0, 0, 0, 0};
    return fftb_ffts_create_ex(dtype, nx, ny, nz, nw, layout4d, &off, obj);
}

int fftb_ffts_create_ex(int dtype, long long nx, long long ny, long long nz, long long nw, int layout4d,
                        const fftb_init_options *options, fftb_ffts *obj)
{
    if (!obj) return FFTB_ERROR_INVALID_VALUE;
    *obj = nullptr;
    if (dtype != FFTB_F32 && dtype != FFTB_F64) return FFTB_ERROR_INVALID_VALUE;
    if (nx < 1 || ny < 1 || nz < 0 || nw < 0 || (nz == 0 && nw > 0)) return FFTB_ERROR_INVALID_VALUE;
    fftb_ffts_s *o = new (std::nothrow) fftb_ffts_s();
    if (!o) return FFTB_ERROR_ALLOC;
    o->dtype = dtype;
    o->nx = nx;
    o->ny = ny;
    o->nz = nz;
    o->nw = nw;
    o->layout = layout4d;
    o->dim = nz == 0 ? 2 : (nw == 0 ? 3 : 4);
    fftb_init_options defaults;
    fftb_init_options_default(&defaults);
    const fftb_init_options &op = options ? *options : defaults;
    if (op.profiling_key && op.profiling_key[0]) {
        o->prof.enabled = true;
        o->prof.key = op.profiling_key;
    }
    if (op.memory_profiling_key && op.memory_profiling_key[0]) {
        o->mem.enabled = true;
        o->mem.key = op.memory_profiling_key;
        o->mem.set_bytes("ffts/shared_work_buffer", 0);
    }
    o->print_flags = (op.print_profile_summary_on_destroy ? 1 : 0) | (op.print_profile_totals_on_destroy ? 2 : 0) |
                     (op.print_memory_profile_on_destroy ? 4 : 0) | (op.print_memory_totals_on_destroy ? 8 : 0);
    int st;
    {
        FFTB_PROFILE_SCOPE(o, "init");
        if (o->dim == 2) st = build_2d(o);
        else if (o->dim == 3) st = build_3d(o);
        else st = build_4d(o);
        if (st == FFTB_SUCCESS && o->dim == 3) st = fused3d_init(o->fused, dtype, nx, ny, nz);
        if (st == FFTB_SUCCESS && o->dim == 4) st = fused4d_init(o->fused4, dtype, layout4d, nx, ny, nz, nw);
    }
    if (st != FFTB_SUCCESS) {
        o->prof.clear_events();
        delete o;
        return st;
    }
    *obj = o;
    return FFTB_SUCCESS;
}

int fftb_ffts_destroy(fftb_ffts o)
{
    if (!o) return FFTB_ERROR_INVALID_HANDLE;
    // print-on-destroy of the profiles (source/ffts.hpp:199-208, :449-476)
    if (o->prof.enabled && (o->print_flags & 1)) std::fputs(o->prof.summary().c_str(), stdout);
    if (o->prof.enabled && (o->print_flags & 2)) std::fputs(o->prof.totals().c_str(), stdout);
    if (o->mem.enabled && (o->print_flags & 4)) std::fputs(o->mem.summary().c_str(), stdout);
    if (o->mem.enabled && (o->print_flags & 8)) std::fputs(o->mem.totals().c_str(), stdout);
    if (o->print_flags) std::fflush(stdout);
    o->prof.clear_events();
    if (o->own_work && o->work) cudaFree(o->work);
    if (o->dspec) cudaFree(o->dspec);
    if (o->dspec2) cudaFree(o->dspec2);
    delete o;
    return FFTB_SUCCESS;
}

int fftb_ffts_profile_report(fftb_ffts o, int which, char *text, size_t capacity, size_t *needed)
{
    if (!o) return FFTB_ERROR_INVALID_HANDLE;
    if (which < 0 || which > 3) return FFTB_ERROR_INVALID_VALUE;
    std::string r;
    if (which == 0) r = o->prof.enabled ? o->prof.summary() : std::string();
    else if (which == 1) r = o->prof.enabled ? o->prof.totals() : std::string();
    else if (which == 2) r = o->mem.enabled ? o->mem.summary() : std::string();
    else r = o->mem.enabled ? o->mem.totals() : std::string();
    if (needed) *needed = r.size() + 1;
    if (text && capacity > 0) {
        const size_t n = r.size() < capacity - 1 ? r.size() : capacity - 1;
        std::memcpy(text, r.data(), n);
        text[n] = 0;
    }
    return FFTB_SUCCESS;
}

int fftb_ffts_dimension(fftb_ffts o, int *dim)
{
    if (!o || !dim) return FFTB_ERROR_INVALID_HANDLE;
    *dim = o->dim;
    return FFTB_SUCCESS;
}

int fftb_ffts_work_size(fftb_ffts o, size_t *bytes)
{
    if (!o || !bytes) return FFTB_ERROR_INVALID_HANDLE;
    *bytes = o->work_bytes;
    return FFTB_SUCCESS;
}

int fftb_ffts_set_work_area(fftb_ffts o, void *work)
{
    if (!o) return FFTB_ERROR_INVALID_HANDLE;
    if ((uintptr_t)work % 256 != 0) return FFTB_ERROR_MISALIGNED;
    if (o->own_work && o->work) cudaFree(o->work);
    o->own_work = false;
    o->work = work;
    o->mem.set_bytes("ffts/shared_work_buffer", 0);  // an external work area is the caller's
    return FFTB_SUCCESS;
}

int fftb_ffts_set_stream(fftb_ffts o, void *stream)
{
    if (!o) return FFTB_ERROR_INVALID_HANDLE;
    o->stream = (cudaStream_t)stream;
    return FFTB_SUCCESS;
}

int fftb_ffts_forward(fftb_ffts o, const void *in, void *out)
{
    if (!o) return FFTB_ERROR_INVALID_HANDLE;
    FFTB_PROFILE_SCOPE(o, "forward");
    if (!in || !out) return FFTB_ERROR_INVALID_VALUE;
    LaunchTimer *tm = o->timing ? &o->timer : nullptr;
    if (o->fused.enabled && aligned16(in, out)) return fused3d_forward(o->fused, in, out, o->stream, tm);
    if (o->fused4.enabled && aligned16(in, out)) {
        int st = ensure_work(o);
        if (st != FFTB_SUCCESS) return st;
        return fused4d_forward(o->fused4, in, out, o->work, o->stream, tm);
    }
    return run(o, o->fwd, in, out, nullptr);
}

int fftb_ffts_backward(fftb_ffts o, void *in, void *out)
{
    if (!o) return FFTB_ERROR_INVALID_HANDLE;
    FFTB_PROFILE_SCOPE(o, "backward");
    if (!in || !out) return FFTB_ERROR_INVALID_VALUE;
    LaunchTimer *tm = o->timing ? &o->timer : nullptr;
    if (o->fused.enabled && aligned16(in, out)) return fused3d_backward(o->fused, in, out, 1.0, o->stream, tm);
    if (o->fused4.enabled && aligned16(in, out)) {
        int st = ensure_work(o);
        if (st != FFTB_SUCCESS) return st;
        return fused4d_backward(o->fused4, in, out, o->work, 1.0, o->stream, tm);
    }
    return run(o, o->bwd, in, out, nullptr);
}

int fftb_ffts_backward_normalized(fftb_ffts o, void *in, void *out)
{
    if (!o) return FFTB_ERROR_INVALID_HANDLE;
    FFTB_PROFILE_SCOPE(o, "backward_normalized");
    if (!in || !out) return FFTB_ERROR_INVALID_VALUE;
    LaunchTimer *tm = o->timing ? &o->timer : nullptr;
    if (o->fused.enabled && aligned16(in, out))
        return fused3d_backward(o->fused, in, out, 1.0 / (double)(o->nx * o->ny * o->nz), o->stream, tm);
    if (o->fused4.enabled && aligned16(in, out)) {
        int st = ensure_work(o);
        if (st != FFTB_SUCCESS) return st;
        return fused4d_backward(o->fused4, in, out, o->work, 1.0 / (double)(o->nx * o->ny * o->nz * o->nw),
                                o->stream, tm);
    }
    return run(o, o->bwd_norm, in, out, nullptr);
}

int fftb_ffts_poisson(fftb_ffts o, const void *rhs, void *sol, double sign)
{
    if (!o) return FFTB_ERROR_INVALID_HANDLE;
    FFTB_PROFILE_SCOPE(o, "poisson");
    if (!rhs || !sol) return FFTB_ERROR_INVALID_VALUE;
    EpValues ep;
    ep.scale = 1.0;
    ep.sign = sign;
    ep.mode = EP_SCALE | EP_POISSON;
    if ((o->fused.enabled || o->fused4.enabled) && aligned16(rhs, sol)) {
        int st = ensure_work(o);
        if (st != FFTB_SUCCESS) return st;
        LaunchTimer *tm = o->timing ? &o->timer : nullptr;
        if (o->fused.enabled) return fused3d_spectral(o->fused, rhs, sol, o->work, ep, o->stream, tm);
        return fused4d_spectral(o->fused4, rhs, sol, o->work, ep, o->stream, tm);
    }
    return run(o, o->poisson, rhs, sol, &ep);
}

int fftb_ffts_filter(fftb_ffts o, const void *in, void *out, double sigma, double poisson_sign)
{
    if (!o) return FFTB_ERROR_INVALID_HANDLE;
    FFTB_PROFILE_SCOPE(o, "filter");
    if (!in || !out || !(sigma > 0.0)) return FFTB_ERROR_INVALID_VALUE;
    EpValues ep;
    ep.scale = 1.0;
    ep.sign = poisson_sign;
    ep.gauss = 1.0 / (2.0 * sigma * sigma);
    ep.mode = EP_SCALE | EP_GAUSS | (poisson_sign != 0.0 ? EP_POISSON : 0);
    if ((o->fused.enabled || o->fused4.enabled) && aligned16(in, out)) {
        int st = ensure_work(o);
        if (st != FFTB_SUCCESS) return st;
        LaunchTimer *tm = o->timing ? &o->timer : nullptr;
        if (o->fused.enabled) return fused3d_spectral(o->fused, in, out, o->work, ep, o->stream, tm);
        return fused4d_spectral(o->fused4, in, out, o->work, ep, o->stream, tm);
    }
    return run(o, o->filter, in, out, &ep);
}

int fftb_ffts_forward_adjoint(fftb_ffts o, void *grad_spectrum, void *grad_real)
{
    if (!o) return FFTB_ERROR_INVALID_HANDLE;
    FFTB_PROFILE_SCOPE(o, "forward_adjoint");
    if (!grad_spectrum || !grad_real) return FFTB_ERROR_INVALID_VALUE;
    LaunchTimer *tm = o->timing ? &o->timer : nullptr;
    if (o->fused.enabled && aligned16(grad_spectrum, grad_real))
        return fused3d_forward_adjoint(o->fused, grad_spectrum, grad_real, o->stream, tm);
    if (o->fused4.enabled && aligned16(grad_spectrum, grad_real)) {
        int st = ensure_work(o);
        if (st != FFTB_SUCCESS) return st;
        return fused4d_forward_adjoint(o->fused4, grad_spectrum, grad_real, o->work, o->stream, tm);
    }
    return run(o, o->fwd_adj, grad_spectrum, grad_real, nullptr);
}

int fftb_ffts_backward_adjoint(fftb_ffts o, const void *grad_real, void *grad_spectrum)
{
    if (!o) return FFTB_ERROR_INVALID_HANDLE;
    FFTB_PROFILE_SCOPE(o, "backward_adjoint");
    if (!grad_spectrum || !grad_real) return FFTB_ERROR_INVALID_VALUE;
    LaunchTimer *tm = o->timing ? &o->timer : nullptr;
    if (o->fused.enabled && aligned16(grad_spectrum, grad_real))
        return fused3d_backward_adjoint(o->fused, grad_real, grad_spectrum, o->stream, tm);
    if (o->fused4.enabled && aligned16(grad_spectrum, grad_real)) {
        int st = ensure_work(o);
        if (st != FFTB_SUCCESS) return st;
        return fused4d_backward_adjoint(o->fused4, grad_real, grad_spectrum, o->work, o->stream, tm);
    }
    return run(o, o->bwd_adj, grad_real, grad_spectrum, nullptr);
}

int fftb_ffts_spectrum_poisson(fftb_ffts o, void *spec, double sign, double scale)
{
    if (!o) return FFTB_ERROR_INVALID_HANDLE;
    if (!spec) return FFTB_ERROR_INVALID_VALUE;
    int4 dims, ns;
    int half_axis, slot[4];
    spectrum_geometry(o, dims, ns, half_axis, slot);
    const long long total = (long long)dims.x * dims.y * dims.z * dims.w;
    const int bs = 256;
    const long long gs = std::min<long long>((total + bs - 1) / bs, 148LL * 16);
    if (o->dtype == FFTB_F32)
        spectrum_poisson_kernel<float><<<(unsigned)gs, bs, 0, o->stream>>>((float2 *)spec, total, dims, ns, half_axis,
                                                                           (float)sign, (float)scale);
    else
        spectrum_poisson_kernel<double><<<(unsigned)gs, bs, 0, o->stream>>>((double2 *)spec, total, dims, ns,
                                                                            half_axis, sign, scale);
    return set_status_from_cuda(cudaGetLastError());
}

int fftb_ffts_spectrum_derivative(fftb_ffts o, const void *spec_in, void *spec_out, int axis, double scale)
{
    if (!o) return FFTB_ERROR_INVALID_HANDLE;
    if (!spec_in || !spec_out || axis < 0 || axis >= o->dim) return FFTB_ERROR_INVALID_VALUE;
    int4 dims, ns;
    int half_axis, slot[4];
    spectrum_geometry(o, dims, ns, half_axis, slot);
    const long long total = (long long)dims.x * dims.y * dims.z * dims.w;
    const int bs = 256;
    const long long gs = std::min<long long>((total + bs - 1) / bs, 148LL * 16);
    if (o->dtype == FFTB_F32)
        spectrum_derivative_kernel<float><<<(unsigned)gs, bs, 0, o->stream>>>(
            (const float2 *)spec_in, (float2 *)spec_out, total, dims, ns, half_axis, slot[axis], (float)scale);
    else
        spectrum_derivative_kernel<double><<<(unsigned)gs, bs, 0, o->stream>>>(
            (const double2 *)spec_in, (double2 *)spec_out, total, dims, ns, half_axis, slot[axis], scale);
    return set_status_from_cuda(cudaGetLastError());
}

int fftb_ffts_spectrum_truncate(fftb_ffts o, void *spec, int rule, int cutoff)
{
    if (!o) return FFTB_ERROR_INVALID_HANDLE;
    if (!spec || (rule != FFTB_TRUNCATE_TWO_THIRDS && rule != FFTB_TRUNCATE_BOX)) return FFTB_ERROR_INVALID_VALUE;
    int4 dims, ns;
    int half_axis, slot[4];
    spectrum_geometry(o, dims, ns, half_axis, slot);
    const long long total = (long long)dims.x * dims.y * dims.z * dims.w;
    const int bs = 256;
    const long long gs = std::min<long long>((total + bs - 1) / bs, 148LL * 16);
    if (o->dtype == FFTB_F32)
        spectrum_truncate_kernel<float><<<(unsigned)gs, bs, 0, o->stream>>>((float2 *)spec, total, dims, ns,
                                                                            half_axis, rule, cutoff);
    else
        spectrum_truncate_kernel<double><<<(unsigned)gs, bs, 0, o->stream>>>((double2 *)spec, total, dims, ns,
                                                                             half_axis, rule, cutoff);
    return set_status_from_cuda(cudaGetLastError());
}

} // extern "C"

namespace {
int ensure_spectrum(fftb_ffts_s *o, void **buf)
{
    if (*buf) return FFTB_SUCCESS;
    int4 dims, ns;
    int half_axis, slot[4];
    spectrum_geometry(o, dims, ns, half_axis, slot);
    const size_t bytes = (size_t)dims.x * dims.y * dims.z * dims.w * complex_bytes(o->dtype);
    if (cudaMalloc(buf, bytes) != cudaSuccess) {
        cudaGetLastError();
        *buf = nullptr;
        return FFTB_ERROR_ALLOC;
    }
    o->dspec_bytes = bytes;
    o->mem.set_bytes(buf == &o->dspec ? "ffts/derivative_spectrum" : "ffts/gradient_spectrum", (long long)bytes);
    return FFTB_SUCCESS;
}

double points(const fftb_ffts_s *o)
{
    double n = (double)o->nx * (double)o->ny;
    if (o->dim >= 3) n *= (double)o->nz;
    if (o->dim == 4) n *= (double)o->nw;
    return n;
}
} // namespace

extern "C" {

int fftb_ffts_derivative(fftb_ffts o, const void *in, void *out, int axis)
{
    if (!o) return FFTB_ERROR_INVALID_HANDLE;
    FFTB_PROFILE_SCOPE(o, "derivative");
    if (!in || !out || axis < 0 || axis >= o->dim) return FFTB_ERROR_INVALID_VALUE;
    int st = ensure_spectrum(o, &o->dspec);
    if (st != FFTB_SUCCESS) return st;
    if (o->fused.enabled && aligned16(in, out))  // the multiply rides in the x column pass
        return fused3d_derivative(o->fused, in, o->dspec, out, axis, o->stream, o->timing ? &o->timer : nullptr);
    st = fftb_ffts_forward(o, in, o->dspec);
    if (st == FFTB_SUCCESS) st = fftb_ffts_spectrum_derivative(o, o->dspec, o->dspec, axis, 1.0 / points(o));
    if (st == FFTB_SUCCESS) st = fftb_ffts_backward(o, o->dspec, out);
    return st;
}

int fftb_ffts_gradient(fftb_ffts o, const void *in, void *const *outs)
{
    if (!o) return FFTB_ERROR_INVALID_HANDLE;
    FFTB_PROFILE_SCOPE(o, "gradient");
    if (!in || !outs) return FFTB_ERROR_INVALID_VALUE;
    for (int a = 0; a < o->dim; ++a)
        if (!outs[a]) return FFTB_ERROR_INVALID_VALUE;
    int st = ensure_spectrum(o, &o->dspec);
    if (st == FFTB_SUCCESS) st = ensure_spectrum(o, &o->dspec2);
    if (st != FFTB_SUCCESS) return st;
    bool outs_aligned = true;
    for (int a = 0; a < o->dim; ++a) outs_aligned = outs_aligned && aligned16(in, outs[a]);
    if (o->fused.enabled && outs_aligned)  // 7 launches: the multiply rides in the column pass
        return fused3d_gradient(o->fused, in, o->dspec, o->dspec2, outs, o->stream, o->timing ? &o->timer : nullptr);
    // one forward transform; per axis the i k multiply into the second buffer (the
    // backward transform consumes its input) and the backward transform
    st = fftb_ffts_forward(o, in, o->dspec);
    for (int a = 0; a < o->dim && st == FFTB_SUCCESS; ++a) {
        st = fftb_ffts_spectrum_derivative(o, o->dspec, o->dspec2, a, 1.0 / points(o));
        if (st == FFTB_SUCCESS) st = fftb_ffts_backward(o, o->dspec2, outs[a]);
    }
    return st;
}

int fftb_ffts_timing_enable(fftb_ffts o, int max_launches)
{
    if (!o) return FFTB_ERROR_INVALID_HANDLE;
    if (max_launches <= 0) {
        o->timer.release();
        o->timing = false;
        return FFTB_SUCCESS;
    }
    int st = o->timer.reserve((size_t)max_launches * 2 + 2);
    o->timing = (st == FFTB_SUCCESS);
    return st;
}

int fftb_ffts_timing_read(fftb_ffts o, float *ms, double *bytes, char *names, int name_stride, int cap, int *count)
{
    if (!o || !count) return FFTB_ERROR_INVALID_HANDLE;
    LaunchTimer &t = o->timer;
    *count = 0;
    if (t.used == 0) return FFTB_SUCCESS;
    cudaError_t e = cudaEventSynchronize(t.ev[t.used - 1]);
    if (e != cudaSuccess) return set_status_from_cuda(e);
    int n = 0;
    for (size_t i = 0; i + 1 < t.used; ++i) {
        if (t.owner[i] != 1) continue;
        if (n < cap) {
            float v = 0.f;
            e = cudaEventElapsedTime(&v, t.ev[i], t.ev[i + 1]);
            if (e != cudaSuccess) return set_status_from_cuda(e);
            if (ms) ms[n] = v;
            if (bytes) bytes[n] = t.bytes[i];
            if (names && name_stride > 0) {
                strncpy(names + (size_t)n * name_stride, t.names[i].c_str(), (size_t)name_stride - 1);
                names[(size_t)n * name_stride + name_stride - 1] = 0;
            }
        }
        ++n;
    }
    *count = n < cap ? n : cap;
    t.used = 0;
    return FFTB_SUCCESS;
}

int fftb_ffts_num_launches(fftb_ffts o, int which, int *launches)
{
    if (!o || !launches) return FFTB_ERROR_INVALID_HANDLE;
    if (o->fused.enabled) {
        *launches = fused3d_num_launches(o->fused, which);
        return FFTB_SUCCESS;
    }
    if (o->fused4.enabled) {
        *launches = fused4d_num_launches(o->fused4, which);
        return FFTB_SUCCESS;
    }
    const Program *p = which == 0 ? &o->fwd : which == 1 ? &o->bwd : which == 2 ? &o->poisson : &o->filter;
    *launches = (int)p->launches.size();
    return FFTB_SUCCESS;
}

int fftb_ffts_set_strategy(fftb_ffts o, int strategy, int plane_cluster)
{
    if (!o) return FFTB_ERROR_INVALID_HANDLE;
    if (strategy < FFTB_STRATEGY_AUTO || strategy > FFTB_STRATEGY_FUSED_TC) return FFTB_ERROR_INVALID_VALUE;
    const bool tc = strategy == FFTB_STRATEGY_FUSED_TC;
    if (tc) strategy = FFTB_STRATEGY_FUSED;
    if (plane_cluster != 0 && plane_cluster != 1 && plane_cluster != 2 && plane_cluster != 4 && plane_cluster != 8)
        return FFTB_ERROR_INVALID_VALUE;
    if (o->dim == 2) {
        if (strategy == FFTB_STRATEGY_FUSED) {
            set_last_error("2D transforms have no fused kernels");
            return FFTB_ERROR_UNSUPPORTED_SIZE;
        }
        return FFTB_SUCCESS;
    }
    int st = FFTB_SUCCESS;
    if (o->dim == 3) {
        Fused3D f;
        if (strategy != FFTB_STRATEGY_STAGED)
            st = fused3d_init(f, o->dtype, o->nx, o->ny, o->nz, plane_cluster);
        if (st != FFTB_SUCCESS) return st;
        if (strategy == FFTB_STRATEGY_FUSED && !f.enabled) {
            set_last_error("no fused 3D kernels for this size / dtype / plane cluster");
            return FFTB_ERROR_UNSUPPORTED_SIZE;
        }
        f.tc = tc;
        o->fused = f;
    } else {
        Fused4D f;
        if (plane_cluster > 1) {
            set_last_error("4D plane kernels run one CTA per plane");
            return FFTB_ERROR_UNSUPPORTED_SIZE;
        }
        if (strategy != FFTB_STRATEGY_STAGED)
            st = fused4d_init(f, o->dtype, o->layout, o->nx, o->ny, o->nz, o->nw);
        if (st != FFTB_SUCCESS) return st;
        if (strategy == FFTB_STRATEGY_FUSED && !f.enabled) {
            set_last_error("no fused 4D kernels for this size / dtype / layout");
            return FFTB_ERROR_UNSUPPORTED_SIZE;
        }
        f.tc = tc;
        o->fused4 = f;
    }
    return FFTB_SUCCESS;
}

int fftb_ffts_get_strategy(fftb_ffts o, int *strategy, int *plane_cluster)
{
    if (!o || !strategy || !plane_cluster) return FFTB_ERROR_INVALID_HANDLE;
    if (o->fused.enabled) {
        *strategy = o->fused.tc ? FFTB_STRATEGY_FUSED_TC : FFTB_STRATEGY_FUSED;
        *plane_cluster = o->fused.cluster;
    } else if (o->fused4.enabled) {
        *strategy = o->fused4.tc ? FFTB_STRATEGY_FUSED_TC : FFTB_STRATEGY_FUSED;
        *plane_cluster = 1;
    } else {
        *strategy = FFTB_STRATEGY_STAGED;
        *plane_cluster = 0;
    }
    return FFTB_SUCCESS;
}

} // extern "C"
