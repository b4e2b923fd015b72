// fftb_noalloc.cu -- a 3D periodic Poisson solve that allocates no device memory.
//
// Who needs it: callers that cannot call cudaMalloc -- code that runs while a
// memory pool owns every byte of the device (a framework allocator, a serving
// process with a fixed arena), code that must not allocate between steps of a
// long-running job, or code that must avoid the implicit device synchronisation
// a cudaMalloc/cudaFree can cause.  The regular ffts object (fftb_ffts_poisson)
// needs a spectrum-sized work area and device twiddle tables, which it
// allocates itself unless the caller supplies the work area.
//
// This entry point keeps its scratch -- the twiddle tables and the spectrum of
// the solve -- in one file-scope __device__ array of fixed size, which every GPU
// that loads the library holds until the process exits.  The kernels it runs are
// the same pass kernels as the regular path (R2C on z, C2C on y, the x pass with
// the -1/|k|^2 multiply between its forward and inverse FFT, C2C^-1 on y, C2R on
// z with 1/N).
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "../../include/fftb.h"
#include "fftb_device.cuh"
#include "fftb_engine.h"

namespace fftb {
namespace {

constexpr size_t kTwBytes = 3u * 4096u * sizeof(float2);  // three root tables of up to 4096 entries
constexpr size_t kSpecBytes = (size_t)FFTB_NOALLOC_MAX_SPECTRUM_BYTES;

// The scratch.  In host code `g_noalloc_scratch` names a host-side stand-in, not
// device memory: its device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kTwBytes + kSpecBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void *g_scratch_addr[kMaxDevices] = {nullptr};

// Device address of the scratch on the current device, looked up once per device.
int scratch_address(void **out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return set_status_from_cuda(e);
    if (dev < 0 || dev >= kMaxDevices) return FFTB_ERROR_INVALID_VALUE;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return set_status_from_cuda(e);
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return FFTB_SUCCESS;
}

__global__ void noalloc_roots_kernel(float2 *w, int n0, int n1, int n2)
{
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    const int ns[3] = {n0, n1, n2};
#pragma unroll
    for (int t = 0; t < 3; ++t) {
        if (m < ns[t]) {
            double s, c;
            sincospi(-2.0 * (double)m / (double)ns[t], &s, &c);
            w[t * 4096 + m] = make_float2((float)c, (float)s);
        }
    }
}

int floor_pow2(int v)
{
    int p = 1;
    while (p * 2 <= v) p *= 2;
    return p;
}

// One pass launch with its geometry.  Batch dims are given already ordered
// (dim 0 the most contiguous on the input side); counts are >= 2.
struct NaPass {
    int kind, n;
    long long is, os;
    int nb;
    long long cnt[2], ibs[2], obs[2];
    const void *in;
    void *out;
    const float2 *tw;
    int ep_mode;
    double ep_scale, ep_sign;
};

int launch_pass(const NaPass &p, cudaStream_t stream)
{
    const bool realk = (p.kind == K_R2C || p.kind == K_C2R);
    bool half = realk && (p.n % 2 == 0);
    int nf = half ? p.n / 2 : p.n;
    PassKernelInfo k;
    if (half && !lookup_kernel(FFTB_F32, nf, &k)) {
        // no half-length kernel: the real line runs as a full complex line of length n,
        // as the regular pass programs do (its root table, [0], has length n)
        half = false;
        nf = p.n;
    }
    if (!lookup_kernel(FFTB_F32, nf, &k)) return FFTB_ERROR_UNSUPPORTED_SIZE;
    PassArgs a;
    memset(&a, 0, sizeof(a));
    a.in = p.in;
    a.out = p.out;
    a.kind = p.kind;
    a.half = half ? 1 : 0;
    a.is = p.is;
    a.os = p.os;
    a.c0 = p.cnt[0];
    a.c1 = p.nb > 1 ? p.cnt[1] : 1;
    a.nlines = a.c0 * a.c1;
    a.ib0 = p.ibs[0];
    a.ob0 = p.obs[0];
    a.ib1 = p.nb > 1 ? p.ibs[1] : 0;
    a.ob1 = p.nb > 1 ? p.obs[1] : 0;
    a.in_pts_fast = (p.is == 1) || (p.ibs[0] != 1 && p.is < p.ibs[0]);
    a.out_pts_fast = (p.os == 1) || (p.obs[0] != 1 && p.os < p.obs[0]);
    a.tw = p.tw;
    a.ntw = half ? 2 * nf : nf;
    a.tw_smem = ((size_t)a.ntw * sizeof(float2) <= 16384) ? 1 : 0;
    a.ep_mode = p.ep_mode;
    a.ep_scale = p.ep_scale;
    a.ep_sign = p.ep_sign;
    if (p.kind == K_SANDWICH) {
        // x pass of the 3D solve: kx = point index, kz = b0 (half axis, count nz/2+1), ky = b1
        a.ep_naxes = 3;
        a.ep_src[0] = 0; a.ep_n[0] = p.n;                        a.ep_half[0] = 0; a.ep_kscale[0] = 1.0;
        a.ep_src[1] = 2; a.ep_n[1] = (int)p.cnt[1];              a.ep_half[1] = 0; a.ep_kscale[1] = 1.0;
        a.ep_src[2] = 1; a.ep_n[2] = (int)(2 * (p.cnt[0] - 1));  a.ep_half[2] = 1; a.ep_kscale[2] = 1.0;
    }
    if (p.kind == K_R2C && half)
        a.pair_io = ((uintptr_t)p.in % 8 == 0) && p.ibs[0] % 2 == 0 && (p.nb < 2 || p.ibs[1] % 2 == 0);
    if (p.kind == K_C2R && half)
        a.pair_io = ((uintptr_t)p.out % 8 == 0) && p.obs[0] % 2 == 0 && (p.nb < 2 || p.obs[1] % 2 == 0);
    const int T = k.threads_per_line;
    int G = 256 / T > 1 ? 256 / T : 1;
    if (!a.in_pts_fast || !a.out_pts_fast) G = G > 16 ? G : 16;
    const int gmax = 512 / T > 1 ? 512 / T : 1;
    G = floor_pow2(G < gmax ? G : gmax);
    while (G > 1 && G / 2 >= a.nlines) G /= 2;
    const size_t smem_tw = a.tw_smem ? (size_t)a.ntw * sizeof(float2) : 0;
    size_t smem = smem_tw + (size_t)G * 32 + (size_t)G * (size_t)k.line_pitch * sizeof(float2);
    while (G > 1 && smem > 48 * 1024) {
        G /= 2;
        smem = smem_tw + (size_t)G * 32 + (size_t)G * (size_t)k.line_pitch * sizeof(float2);
    }
    if (smem > 48 * 1024) return FFTB_ERROR_UNSUPPORTED_SIZE;
    a.G = G;
    int gs = 0;
    while ((1 << gs) < G) ++gs;
    a.gshift = gs;
    const long long ncta = (a.nlines + G - 1) / G;
    void *args[] = {&a};
    return set_status_from_cuda(cudaLaunchKernel(k.fn, dim3((unsigned)ncta), dim3(G * T), args, smem, stream));
}

} // namespace
} // namespace fftb

using namespace fftb;

extern "C" int fftb_poisson3d_f32_noalloc(const float *rhs, float *solution, long long nx, long long ny,
                                          long long nz, double sign, void *stream)
{
    if (!rhs || !solution) return FFTB_ERROR_INVALID_VALUE;
    if (nx < 2 || ny < 2 || nz < 2 || nx > 4096 || ny > 4096 || nz > 4096) return FFTB_ERROR_INVALID_VALUE;
    const long long nzh = nz / 2 + 1, C3 = ny * nzh;
    if ((size_t)(nx * C3) * sizeof(float2) > kSpecBytes) {
        set_last_error("spectrum larger than the static scratch of fftb_poisson3d_f32_noalloc");
        return FFTB_ERROR_INVALID_VALUE;
    }
    // every line length must have a pass kernel of its own (R2C/C2R of even nz run nz/2, or
    // nz as a full complex line when nz/2 has none); lengths that need the chirp-z passes do
    // not, since those need a padded work line of their own
    const bool zok = has_kernel(FFTB_F32, (int)nz) || (nz % 2 == 0 && has_kernel(FFTB_F32, (int)(nz / 2)));
    if (!zok || !has_kernel(FFTB_F32, (int)ny) || !has_kernel(FFTB_F32, (int)nx)) {
        set_last_error("fftb_poisson3d_f32_noalloc: a line length has no direct pass kernel");
        return FFTB_ERROR_UNSUPPORTED_SIZE;
    }
    if ((uintptr_t)rhs % sizeof(float) || (uintptr_t)solution % sizeof(float)) return FFTB_ERROR_MISALIGNED;
    void *base = nullptr;
    int st = scratch_address(&base);
    if (st != FFTB_SUCCESS) return st;
    cudaStream_t s = (cudaStream_t)stream;
    float2 *tw = (float2 *)base;
    float2 *spec = (float2 *)((char *)base + kTwBytes);
    // root tables: [0] length nz (the z pass: 2*(nz/2) for even nz, nz for odd), [1] ny, [2] nx
    const int mx = (int)(nx > ny ? (nx > nz ? nx : nz) : (ny > nz ? ny : nz));
    noalloc_roots_kernel<<<(mx + 255) / 256, 256, 0, s>>>(tw, (int)nz, (int)ny, (int)nx);
    st = set_status_from_cuda(cudaGetLastError());
    if (st != FFTB_SUCCESS) return st;

    // the spectrum [kx][ky][kz < nz/2+1] lives in the scratch; batch dims listed most contiguous first
    NaPass zr = {K_R2C, (int)nz, 1, 1, 2, {ny, nx}, {nz, ny * nz}, {nzh, C3}, rhs, spec, tw, 0, 1.0, 0.0};
    NaPass yf = {K_C2C_FWD, (int)ny, nzh, nzh, 2, {nzh, nx}, {1, C3}, {1, C3}, spec, spec, tw + 4096, 0, 1.0, 0.0};
    NaPass xs = {K_SANDWICH, (int)nx, C3, C3, 2, {nzh, ny}, {1, nzh}, {1, nzh}, spec, spec, tw + 2 * 4096,
                 EP_SCALE | EP_POISSON, 1.0, sign};
    NaPass yi = yf;
    yi.kind = K_C2C_INV;
    NaPass zc = {K_C2R, (int)nz, 1, 1, 2, {ny, nx}, {nzh, C3}, {nz, ny * nz}, spec, solution, tw, EP_SCALE,
                 1.0 / (double)(nx * ny * nz), 0.0};
    if ((st = launch_pass(zr, s)) != FFTB_SUCCESS) return st;
    if ((st = launch_pass(yf, s)) != FFTB_SUCCESS) return st;
    if ((st = launch_pass(xs, s)) != FFTB_SUCCESS) return st;
    if ((st = launch_pass(yi, s)) != FFTB_SUCCESS) return st;
    return launch_pass(zc, s);
}
