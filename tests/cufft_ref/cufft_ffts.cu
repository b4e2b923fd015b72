// cufft_ffts.cu -- the reference's cuFFT-backed `ffts` transform path, restated as a small
// C library for the parity tests and the benchmark (never linked into fftb).
//
// The reference binds `fftm::ffts<BaseFFT, ...>` to cuFFT through `cufft::fft<T, D>`
// (source/external_wrap/cufft_wrap.h:456-1282): every plan is made with
// cufftMakePlanMany64 with auto-allocation off (cufft_wrap.h:1237-1259) and runs in one
// external work area that fft_wrap_many sizes to the largest plan
// (source/external_wrap/fft_wrap_many.h:264-292).  The plans restated here carry exactly the
// advanced-layout parameters of
//   3D:            source/ffts.hpp:677-695   (forward_3d R2C, inverse_3d C2R)
//   4D pencil:     source/ffts.hpp:697-742   (1D w R2C/C2R, z/y strided C2C, x contiguous C2C)
//   4D slab:       source/ffts.hpp:744-776   (2D (z,w) R2C/C2R, 2D (x,y) strided C2C)
//   4D native:     source/fftm.hpp:2941-2961 (2D (y,x) C2C over the [y][kz][kw][x] spectrum)
// and run in the stage order of source/ffts.hpp:809-867.  The 4D stages move between
// layouts with the reference's direct transpose (one thread per element,
// source/detail/direct_transpose_4d.h:17-211, followed by a wait, :204).  The Poisson solve is
// the example's sequence (examples/poisson/source/poisson_periodic_3d_autotuned.cpp:348-375):
// forward, a separate -1/|k|^2 multiply kernel (:74-103, k = 0 -> 0), backward, a separate
// 1/N scale kernel (:105-115).
#include <cuda_runtime.h>
#include <cufft.h>

#include <cstdint>
#include <cstring>
#include <new>
#include <string>
#include <vector>

namespace {

enum { REF_F32 = 0, REF_F64 = 1 };
enum { REF_PENCIL = 0, REF_SLAB = 1, REF_NATIVE_XZWY = 2 };
enum { R2C = 1, C2R = 2, C2CF = 3, C2CB = 4 };  // source/fft_direction.h:9-15

struct Plan {
    cufftHandle h = 0;
    int dir = 0;
    size_t work = 0;
};

struct Ref {
    int dtype = REF_F32, dim = 3, layout = 0;
    long long nx = 0, ny = 0, nz = 0, nw = 0;
    std::vector<Plan> plans;  // 3D: forward, inverse; 4D: see make_4d
    size_t work_bytes = 0, stage_bytes = 0;
    void *work = nullptr, *stage0 = nullptr, *stage1 = nullptr;
    cudaStream_t stream = nullptr;
};

thread_local std::string g_err;

int fail(const std::string &m)
{
    g_err = m;
    return -1;
}

cufftType fft_type(int dtype, int dir)
{
    if (dtype == REF_F32) return dir == R2C ? CUFFT_R2C : dir == C2R ? CUFFT_C2R : CUFFT_C2C;
    return dir == R2C ? CUFFT_D2Z : dir == C2R ? CUFFT_Z2D : CUFFT_Z2Z;
}

int add_plan(Ref &r, int dir, int rank, long long *n, long long *inembed, long long istride, long long idist,
             long long *onembed, long long ostride, long long odist, long long batch)
{
    Plan p;
    p.dir = dir;
    if (cufftCreate(&p.h) != CUFFT_SUCCESS) return fail("cufftCreate failed");
    if (cufftSetAutoAllocation(p.h, 0) != CUFFT_SUCCESS ||
        cufftMakePlanMany64(p.h, rank, n, inembed, istride, idist, onembed, ostride, odist, fft_type(r.dtype, dir),
                            batch, &p.work) != CUFFT_SUCCESS) {
        cufftDestroy(p.h);
        return fail("cufftMakePlanMany64 failed");
    }
    r.plans.push_back(p);
    if (p.work > r.work_bytes) r.work_bytes = p.work;
    return 0;
}

int exec(const Ref &r, int i, void *in, void *out)
{
    const Plan &p = r.plans[i];
    cufftResult e;
    if (r.dtype == REF_F32) {
        if (p.dir == R2C) e = cufftExecR2C(p.h, (cufftReal *)in, (cufftComplex *)out);
        else if (p.dir == C2R) e = cufftExecC2R(p.h, (cufftComplex *)in, (cufftReal *)out);
        else e = cufftExecC2C(p.h, (cufftComplex *)in, (cufftComplex *)out, p.dir == C2CF ? CUFFT_FORWARD : CUFFT_INVERSE);
    } else {
        if (p.dir == R2C) e = cufftExecD2Z(p.h, (cufftDoubleReal *)in, (cufftDoubleComplex *)out);
        else if (p.dir == C2R) e = cufftExecZ2D(p.h, (cufftDoubleComplex *)in, (cufftDoubleReal *)out);
        else
            e = cufftExecZ2Z(p.h, (cufftDoubleComplex *)in, (cufftDoubleComplex *)out,
                             p.dir == C2CF ? CUFFT_FORWARD : CUFFT_INVERSE);
    }
    return e == CUFFT_SUCCESS ? 0 : fail("cufftExec failed");
}

// ------------------------------------------------------------------ element kernels
// direct_transpose_4d: out(o) = in(c), o[j] = c[D[j]], over the source's logical range;
// offsets follow the arrangers (order[0] = fastest logical index).
struct Perm {
    long long sd[4], dd[4];
    int so[4], dor[4], D[4];
};

__device__ __forceinline__ long long arr_off(const long long *idx, const long long *d, const int *order)
{
    long long off = 0, mult = 1;
    for (int j = 0; j < 4; ++j) {
        off += idx[order[j]] * mult;
        mult *= d[order[j]];
    }
    return off;
}

template <typename C> __global__ void permute_kernel(const C *__restrict__ src, C *__restrict__ dst, Perm p, long long n)
{
    const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (e >= n) return;
    long long c[4], o[4], rem = e;
    c[3] = rem % p.sd[3]; rem /= p.sd[3];
    c[2] = rem % p.sd[2]; rem /= p.sd[2];
    c[1] = rem % p.sd[1]; rem /= p.sd[1];
    c[0] = rem;
    for (int j = 0; j < 4; ++j) o[j] = c[p.D[j]];
    dst[arr_off(o, p.dd, p.dor)] = src[arr_off(c, p.sd, p.so)];
}

// solve_negative_laplacian_functor on [kx][ky][kz < nz/2+1], times sign (the example has +1)
template <typename R, typename C>
__global__ void poisson3d_kernel(C *spec, long long nx, long long ny, long long nzh, R sign)
{
    const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (e >= nx * ny * nzh) return;
    const long long z = e % nzh, y = (e / nzh) % ny, x = e / (nzh * ny);
    const long long kx = x <= nx / 2 ? x : x - nx, ky = y <= ny / 2 ? y : y - ny, kz = z;
    const R k2 = R(kx * kx + ky * ky + kz * kz);
    if (k2 == R(0)) {
        spec[e].x = R(0);
        spec[e].y = R(0);
        return;
    }
    const R s = sign / k2;
    spec[e].x *= s;
    spec[e].y *= s;
}

template <typename R> __global__ void scale_kernel(R *a, long long n, R s)
{
    const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (e < n) a[e] *= s;
}

int permute(const Ref &r, const void *src, const long long *sd, const int *so, void *dst, const long long *dd,
            const int *dor, const int *D)
{
    Perm p;
    for (int j = 0; j < 4; ++j) {
        p.sd[j] = sd[j];
        p.dd[j] = dd[j];
        p.so[j] = so[j];
        p.dor[j] = dor[j];
        p.D[j] = D[j];
    }
    const long long n = sd[0] * sd[1] * sd[2] * sd[3];
    const unsigned blocks = (unsigned)((n + 255) / 256);
    if (r.dtype == REF_F32) permute_kernel<float2><<<blocks, 256, 0, r.stream>>>((const float2 *)src, (float2 *)dst, p, n);
    else permute_kernel<double2><<<blocks, 256, 0, r.stream>>>((const double2 *)src, (double2 *)dst, p, n);
    if (cudaGetLastError() != cudaSuccess) return fail("transpose launch failed");
    // the reference waits for its for_each after every transpose (direct_transpose_4d.h:204)
    return cudaStreamSynchronize(r.stream) == cudaSuccess ? 0 : fail("transpose failed");
}

const int A0123[4] = {0, 1, 2, 3}, A0213[4] = {0, 2, 1, 3}, A3210[4] = {3, 2, 1, 0}, A1032[4] = {1, 0, 3, 2},
          A2103[4] = {2, 1, 0, 3};

int make_4d(Ref &r)
{
    const long long nx = r.nx, ny = r.ny, nz = r.nz, nw = r.nw, nwh = nw / 2 + 1;
    int st = 0;
    if (r.layout == REF_PENCIL) {  // source/ffts.hpp:697-742
        const long long rb = nx * ny * nz, zb = nx * ny * nwh, yb = nx * nz * nwh, xb = ny * nz * nwh;
        const long long ws = nx * ny * nz, zs = nx * ny * nwh, ys = nx * nz * nwh;
        long long n, e1 = 1, ex = nx;
        n = nw; st |= add_plan(r, R2C, 1, &n, &e1, ws, 1, &e1, ws, 1, rb);   // 0 forward_w
        n = nw; st |= add_plan(r, C2R, 1, &n, &e1, ws, 1, &e1, ws, 1, rb);   // 1 inverse_w
        n = nz; st |= add_plan(r, C2CF, 1, &n, &e1, zs, 1, &e1, zs, 1, zb);  // 2 forward_z
        n = nz; st |= add_plan(r, C2CB, 1, &n, &e1, zs, 1, &e1, zs, 1, zb);  // 3 inverse_z
        n = ny; st |= add_plan(r, C2CF, 1, &n, &e1, ys, 1, &e1, ys, 1, yb);  // 4 forward_y
        n = ny; st |= add_plan(r, C2CB, 1, &n, &e1, ys, 1, &e1, ys, 1, yb);  // 5 inverse_y
        n = nx; st |= add_plan(r, C2CF, 1, &n, &ex, 1, nx, &ex, 1, nx, xb);  // 6 forward_x
        n = nx; st |= add_plan(r, C2CB, 1, &n, &ex, 1, nx, &ex, 1, nx, xb);  // 7 inverse_x
    } else if (r.layout == REF_SLAB) {  // source/ffts.hpp:744-776
        long long n2[2] = {nz, nw}, ie[2] = {nz, nw}, oe[2] = {nz, nwh};
        st |= add_plan(r, R2C, 2, n2, ie, 1, nz * nw, oe, 1, nz * nwh, nx * ny);  // 0 forward_zw
        long long ie2[2] = {nz, nwh}, oe2[2] = {nz, nw};
        st |= add_plan(r, C2R, 2, n2, ie2, 1, nz * nwh, oe2, 1, nz * nw, nx * ny);  // 1 inverse_zw
        long long nxy[2] = {nx, ny};
        st |= add_plan(r, C2CF, 2, nxy, nxy, nz * nwh, 1, nxy, nz * nwh, 1, nz * nwh);  // 2 forward_xy
        st |= add_plan(r, C2CB, 2, nxy, nxy, nz * nwh, 1, nxy, nz * nwh, 1, nz * nwh);  // 3 inverse_xy
    } else {  // fftm slab with the native_xzwy spectrum: (z,w) as the slab plans, (y,x) per fftm.hpp:2941-2961
        long long n2[2] = {nz, nw}, ie[2] = {nz, nw}, oe[2] = {nz, nwh};
        st |= add_plan(r, R2C, 2, n2, ie, 1, nz * nw, oe, 1, nz * nwh, nx * ny);
        long long ie2[2] = {nz, nwh}, oe2[2] = {nz, nw};
        st |= add_plan(r, C2R, 2, n2, ie2, 1, nz * nwh, oe2, 1, nz * nw, nx * ny);
        long long nyx[2] = {ny, nx}, e2[2] = {ny, nx * nz * nwh};
        st |= add_plan(r, C2CF, 2, nyx, e2, 1, nx, e2, 1, nx, nz * nwh);
        st |= add_plan(r, C2CB, 2, nyx, e2, 1, nx, e2, 1, nx, nz * nwh);
    }
    r.stage_bytes = (size_t)(nx * ny * nz * nwh) * (r.dtype == REF_F32 ? 8 : 16);
    return st;
}

int forward_4d(Ref &r, void *in, void *out)
{
    const long long nx = r.nx, ny = r.ny, nz = r.nz, nwh = r.nw / 2 + 1;
    void *s0 = r.stage0, *s1 = r.stage1;
    int st = 0;
    if (r.layout == REF_PENCIL) {  // source/ffts.hpp:809-825
        st |= exec(r, 0, in, s0);
        { const long long sd[4] = {nx, ny, nz, nwh}, dd[4] = {nx, ny, nwh, nz}; const int D[4] = {0, 1, 3, 2};
          st |= permute(r, s0, sd, A0123, s1, dd, A0123, D); }
        st |= exec(r, 2, s1, s1);
        { const long long sd[4] = {nx, ny, nwh, nz}, dd[4] = {nx, nz, nwh, ny}; const int D[4] = {0, 3, 2, 1};
          st |= permute(r, s1, sd, A0123, s0, dd, A0213, D); }
        st |= exec(r, 4, s0, s0);
        { const long long sd[4] = {nx, nz, nwh, ny}, dd[4] = {ny, nz, nwh, nx}; const int D[4] = {3, 1, 2, 0};
          st |= permute(r, s0, sd, A0213, out, dd, A3210, D); }
        st |= exec(r, 6, out, out);
    } else if (r.layout == REF_SLAB) {  // :827-837
        st |= exec(r, 0, in, s0);
        { const long long sd[4] = {nx, ny, nz, nwh}, dd[4] = {nz, nwh, nx, ny}; const int D[4] = {2, 3, 0, 1};
          st |= permute(r, s0, sd, A3210, s1, dd, A1032, D); }
        st |= exec(r, 2, s1, s1);
        { const long long sd[4] = {nz, nwh, nx, ny}, dd[4] = {ny, nz, nwh, nx}; const int D[4] = {3, 0, 1, 2};
          st |= permute(r, s1, sd, A1032, out, dd, A2103, D); }
    } else {  // fftm native_xzwy: (z,w) R2C, local permute to [y][kz][kw][x], (y,x) C2C in place
        st |= exec(r, 0, in, s0);
        { const long long sd[4] = {nx, ny, nz, nwh}, dd[4] = {nx, nz, nwh, ny}; const int D[4] = {0, 2, 3, 1};
          st |= permute(r, s0, sd, A3210, out, dd, A0213, D); }
        st |= exec(r, 2, out, out);
    }
    return st;
}

int backward_4d(Ref &r, void *in, void *out)
{
    const long long nx = r.nx, ny = r.ny, nz = r.nz, nwh = r.nw / 2 + 1;
    void *s0 = r.stage0, *s1 = r.stage1;
    int st = 0;
    if (r.layout == REF_PENCIL) {  // source/ffts.hpp:839-855
        st |= exec(r, 7, in, in);
        { const long long sd[4] = {ny, nz, nwh, nx}, dd[4] = {nx, nz, nwh, ny}; const int D[4] = {3, 1, 2, 0};
          st |= permute(r, in, sd, A3210, s0, dd, A0213, D); }
        st |= exec(r, 5, s0, s0);
        { const long long sd[4] = {nx, nz, nwh, ny}, dd[4] = {nx, ny, nwh, nz}; const int D[4] = {0, 3, 2, 1};
          st |= permute(r, s0, sd, A0213, s1, dd, A0123, D); }
        st |= exec(r, 3, s1, s1);
        { const long long sd[4] = {nx, ny, nwh, nz}, dd[4] = {nx, ny, nz, nwh}; const int D[4] = {0, 1, 3, 2};
          st |= permute(r, s1, sd, A0123, s0, dd, A0123, D); }
        st |= exec(r, 1, s0, out);
    } else if (r.layout == REF_SLAB) {  // :857-867
        { const long long sd[4] = {ny, nz, nwh, nx}, dd[4] = {nz, nwh, nx, ny}; const int D[4] = {1, 2, 3, 0};
          st |= permute(r, in, sd, A2103, s1, dd, A1032, D); }
        st |= exec(r, 3, s1, s1);
        { const long long sd[4] = {nz, nwh, nx, ny}, dd[4] = {nx, ny, nz, nwh}; const int D[4] = {2, 3, 0, 1};
          st |= permute(r, s1, sd, A1032, s0, dd, A3210, D); }
        st |= exec(r, 1, s0, out);
    } else {
        st |= exec(r, 3, in, in);
        { const long long sd[4] = {nx, nz, nwh, ny}, dd[4] = {nx, ny, nz, nwh}; const int D[4] = {0, 3, 1, 2};
          st |= permute(r, in, sd, A0213, s0, dd, A3210, D); }
        st |= exec(r, 1, s0, out);
    }
    return st;
}

} // namespace

extern "C" {

const char *ref_last_error() { return g_err.c_str(); }

// dim 3: (nx, ny, nz), layout ignored; dim 4: (nx, ny, nz, nw) with layout 0 pencil, 1 slab,
// 2 native_xzwy.  *work_bytes: the shared cuFFT work area; *stage_bytes: each of the two 4D
// stage buffers (0 in 3D).  Buffers are bound with ref_set_buffers before any exec.
int ref_create(int dtype, int dim, int layout, long long nx, long long ny, long long nz, long long nw, void **handle,
               size_t *work_bytes, size_t *stage_bytes)
{
    if (!handle || (dtype != REF_F32 && dtype != REF_F64) || (dim != 3 && dim != 4)) return fail("bad arguments");
    Ref *r = new (std::nothrow) Ref;
    if (!r) return fail("out of host memory");
    r->dtype = dtype;
    r->dim = dim;
    r->layout = layout;
    r->nx = nx;
    r->ny = ny;
    r->nz = nz;
    r->nw = nw;
    int st;
    if (dim == 3) {  // source/ffts.hpp:677-695
        const long long nzh = nz / 2 + 1;
        long long n[3] = {nx, ny, nz}, e[3] = {nx, ny, nz}, eh[3] = {nx, ny, nzh};
        st = add_plan(*r, R2C, 3, n, e, 1, nx * ny * nz, eh, 1, nx * ny * nzh, 1);
        if (st == 0) st = add_plan(*r, C2R, 3, n, eh, 1, nx * ny * nzh, e, 1, nx * ny * nz, 1);
    } else {
        st = make_4d(*r);
    }
    if (st != 0) {
        for (Plan &p : r->plans) cufftDestroy(p.h);
        delete r;
        return -1;
    }
    *handle = r;
    if (work_bytes) *work_bytes = r->work_bytes;
    if (stage_bytes) *stage_bytes = r->stage_bytes;
    return 0;
}

int ref_set_buffers(void *handle, void *work, void *stage0, void *stage1)
{
    Ref *r = (Ref *)handle;
    if (!r) return fail("null handle");
    r->work = work;
    r->stage0 = stage0;
    r->stage1 = stage1;
    for (Plan &p : r->plans)
        if (cufftSetWorkArea(p.h, work) != CUFFT_SUCCESS) return fail("cufftSetWorkArea failed");
    return 0;
}

int ref_set_stream(void *handle, void *stream)
{
    Ref *r = (Ref *)handle;
    if (!r) return fail("null handle");
    r->stream = (cudaStream_t)stream;
    for (Plan &p : r->plans)
        if (cufftSetStream(p.h, r->stream) != CUFFT_SUCCESS) return fail("cufftSetStream failed");
    return 0;
}

// ffts::forward: in real, out complex (in is not modified)
int ref_forward(void *handle, void *in, void *out)
{
    Ref *r = (Ref *)handle;
    if (!r) return fail("null handle");
    return r->dim == 3 ? exec(*r, 0, in, out) : forward_4d(*r, in, out);
}

// ffts::backward, unnormalised; destroys `in` as the reference's does
int ref_backward(void *handle, void *in, void *out)
{
    Ref *r = (Ref *)handle;
    if (!r) return fail("null handle");
    return r->dim == 3 ? exec(*r, 1, in, out) : backward_4d(*r, in, out);
}

// The periodic Poisson solve of the example: forward into spec, spec *= sign/|k|^2 (k = 0 -> 0),
// backward into out, out *= 1/N.  3D only.
int ref_poisson3d(void *handle, void *rhs, void *spec, void *out, double sign)
{
    Ref *r = (Ref *)handle;
    if (!r || r->dim != 3) return fail("ref_poisson3d needs a 3D handle");
    const long long nzh = r->nz / 2 + 1, nc = r->nx * r->ny * nzh, n = r->nx * r->ny * r->nz;
    int st = exec(*r, 0, rhs, spec);
    if (st) return st;
    const unsigned bc = (unsigned)((nc + 255) / 256), br = (unsigned)((n + 255) / 256);
    if (r->dtype == REF_F32) poisson3d_kernel<float, float2><<<bc, 256, 0, r->stream>>>((float2 *)spec, r->nx, r->ny, nzh, (float)sign);
    else poisson3d_kernel<double, double2><<<bc, 256, 0, r->stream>>>((double2 *)spec, r->nx, r->ny, nzh, sign);
    if (cudaGetLastError() != cudaSuccess) return fail("multiply launch failed");
    if ((st = exec(*r, 1, spec, out)) != 0) return st;
    if (r->dtype == REF_F32) scale_kernel<float><<<br, 256, 0, r->stream>>>((float *)out, n, 1.0f / (float)n);
    else scale_kernel<double><<<br, 256, 0, r->stream>>>((double *)out, n, 1.0 / (double)n);
    return cudaGetLastError() == cudaSuccess ? 0 : fail("scale launch failed");
}

// a *= s over n reals: the separate 1/N kernel the reference's callers run after backward
// (source/tests/test_benchmark_ffts_3D.cu:100-104)
int ref_scale(void *handle, void *a, long long n, double s)
{
    Ref *r = (Ref *)handle;
    if (!r) return fail("null handle");
    const unsigned b = (unsigned)((n + 255) / 256);
    if (r->dtype == REF_F32) scale_kernel<float><<<b, 256, 0, r->stream>>>((float *)a, n, (float)s);
    else scale_kernel<double><<<b, 256, 0, r->stream>>>((double *)a, n, s);
    return cudaGetLastError() == cudaSuccess ? 0 : fail("scale launch failed");
}

void ref_destroy(void *handle)
{
    Ref *r = (Ref *)handle;
    if (!r) return;
    for (Plan &p : r->plans) cufftDestroy(p.h);
    delete r;
}

} // extern "C"
