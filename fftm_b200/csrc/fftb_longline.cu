// fftb_longline.cu -- lines longer than one pass kernel holds in shared memory (more
// than 4096 points, the reference's cuFFT plans accept any length,
// source/external_wrap/fft_wrap_many.h:137-186).
//
// A long line is transformed through a contiguous complex work line of length L:
//   gather   the input line into the work line (C2C: copied; R2C: real parts; C2R: the
//            Hermitian extension of the half spectrum), zero padded to L;
//   FFT_L    four-step: L = L1 * L2 with X[k1 + L1 k2] = sum_j2 w_L2^(j2 k2) w_L^(j2 k1)
//            sum_j1 x[j2 + L2 j1] w_L1^(j1 k1), as two pass-engine passes over the work
//            lines (length L1 with stride L2, the w_L^(j2 k1) twiddle fused into its
//            store; then length L2), each factor a pass kernel of its own;
//   scatter  the work line to the output (C2C: all points; R2C: the half spectrum; C2R:
//            the real parts), times the pass's epilogue factor (scale, Poisson, Gaussian,
//            half-axis weights: the same rules as the pass kernel's store).
// A sandwich pass (forward FFT, spectral multiply, inverse FFT) runs FFT_L, the multiply,
// and FFT_L^-1 on the work line.
// When n has no split into two pass-kernel lengths (a large prime factor), the line runs
// Bluestein's chirp-z (Bluestein 1970): L = M, a power of two >= 2n - 1; the gather
// multiplies by the chirp c_j = exp(-i pi j^2 / n), FFT_M, a multiply by B = FFT_M(b) / M
// with b the wrapped conj chirp (FP64 on the host), FFT_M^-1, and the scatter multiplies by
// the chirp again.  Inverse directions run as the conjugate of the forward transform of
// the conjugated input.  The work lines are owned by the step (two buffers of
// lines x L complex values).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <vector>

#include "../../include/fftb.h"
#include "fftb_device.cuh"
#include "fftb_longline.h"

namespace fftb {

struct LongLine {
    int dtype = 0, kind = 0, n = 0;
    long long nlines = 0, c0 = 1, c1 = 1;
    long long ib[3] = {0, 0, 0}, ob[3] = {0, 0, 0};
    long long is = 1, os = 1;
    int in_buf = B_IN, out_buf = B_OUT;
    size_t in_off = 0, out_off = 0;
    double scale = 1.0;
    // epilogue, resolved as the pass kernel's (src 0: point index, 1..3: batch index b0..b2)
    int ep_mode = 0, ep_naxes = 0;
    int ep_src[4] = {0, 0, 0, 0}, ep_n[4] = {0, 0, 0, 0}, ep_half[4] = {0, 0, 0, 0};
    double ep_sign = -1.0, ep_gauss = 0.0, ep_hw = 1.0;
    bool chirp = false;
    bool inverse = false;
    int L = 0, L1 = 0, L2 = 0;
    Program fwd, inv;                  // the two four-step passes, each direction
    void *w0 = nullptr, *w1 = nullptr;  // work lines: nlines * L complex each
    const void *chirp_t = nullptr;      // chirp-z: c_j (n entries)
    void *bhat = nullptr;               // chirp-z: B (L entries)
    ~LongLine()
    {
        if (w0) cudaFree(w0);
        if (w1) cudaFree(w1);
        if (chirp_t) cudaFree(const_cast<void *>(chirp_t));
        if (bhat) cudaFree(bhat);
    }
};

namespace {

struct Geom {
    long long nlines, c0, c1, ib0, ib1, ib2, ob0, ob1, ob2, is, os;
    int n, L, kind;
    // epilogue
    int ep_mode, ep_naxes;
    int ep_src[4], ep_n[4], ep_half[4];
    double ep_scale, ep_sign, ep_gauss, ep_hw;
};

__device__ __forceinline__ void line_idx(long long l, const Geom &g, long long b[3])
{
    b[0] = l % g.c0;
    const long long r = l / g.c0;
    b[1] = r % g.c1;
    b[2] = r / g.c1;
}

__device__ __forceinline__ long long line_off(long long l, const Geom &g, bool out)
{
    long long b[3];
    line_idx(l, g, b);
    return out ? b[0] * g.ob0 + b[1] * g.ob1 + b[2] * g.ob2 : b[0] * g.ib0 + b[1] * g.ib1 + b[2] * g.ib2;
}

// the pass kernel's epilogue factor (fftb_pass.cuh ep_factor) for point p of line l
template <typename R> __device__ R ll_factor(const Geom &g, int p, long long l)
{
    long long b[3];
    line_idx(l, g, b);
    R k2 = R(0), hw = R(1);
    for (int ax = 0; ax < g.ep_naxes; ++ax) {
        const long long i = g.ep_src[ax] == 0 ? p : b[g.ep_src[ax] - 1];
        const long long n = g.ep_n[ax];
        const long long k = g.ep_half[ax] ? i : (i <= n / 2 ? i : i - n);
        k2 += R(k) * R(k);
        if (g.ep_half[ax] && i != 0 && 2 * i != n) hw = R(g.ep_hw);
    }
    R f = R(g.ep_scale);
    if (g.ep_mode & EP_HALFW) f *= hw;
    if (g.ep_mode & EP_POISSON) f = (k2 == R(0)) ? R(0) : f * R(g.ep_sign) / k2;
    if (g.ep_mode & EP_GAUSS) f *= exp(-k2 * R(g.ep_gauss));
    return f;
}

// work[l][p] for p < L: the input line as a complex line, zero past n
template <typename R> __global__ void ll_gather(const void *in, cpx<R> *w, Geom g)
{
    using C = cpx<R>;
    const long long total = g.nlines * g.L;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const long long l = e / g.L;
        const int p = (int)(e - l * g.L);
        C v = mk<R>(R(0), R(0));
        if (p < g.n) {
            const long long off = line_off(l, g, false);
            if (g.kind == K_R2C) {
                v.x = reinterpret_cast<const R *>(in)[off + p * g.is];
            } else if (g.kind == K_C2R) {
                const C *X = reinterpret_cast<const C *>(in) + off;
                if (2 * p <= g.n) {
                    v = X[p * g.is];
                    if (p == 0 || 2 * p == g.n) v.y = R(0);  // DC / Nyquist taken real
                } else {
                    v = cconj(X[(g.n - p) * g.is]);
                }
            } else {
                v = reinterpret_cast<const C *>(in)[off + p * g.is];
            }
        }
        w[e] = v;
    }
}

// chirp-z: before the convolution w = (conj?) w * c over the n points, zero past n;
// after it w = (conj?)(c * w) over the n points
template <typename R>
__global__ void ll_chirp(cpx<R> *w, const cpx<R> *c, long long nlines, int n, int L, int conj, int pre)
{
    const long long total = nlines * L;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int p = (int)(e % L);
        if (p >= n) {
            if (pre) w[e] = mk<R>(R(0), R(0));
            continue;
        }
        cpx<R> v = w[e];
        if (pre) {
            if (conj) v = cconj(v);
            v = cmul(v, c[p]);
        } else {
            v = cmul(v, c[p]);
            if (conj) v = cconj(v);
        }
        w[e] = v;
    }
}

template <typename R> __global__ void ll_mul_table(cpx<R> *w, const cpx<R> *t, long long nlines, int L)
{
    const long long total = nlines * L;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x)
        w[e] = cmul(w[e], t[e % L]);
}

// the sandwich's spectral multiply on the n points of every work line
template <typename R> __global__ void ll_multiply(cpx<R> *w, Geom g)
{
    const long long total = g.nlines * g.n;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const long long l = e / g.n;
        const int p = (int)(e - l * g.n);
        w[l * g.L + p] = cscale(w[l * g.L + p], ll_factor<R>(g, p, l));
    }
}

template <typename R> __global__ void ll_scatter(const cpx<R> *w, void *out, Geom g, int factor)
{
    using C = cpx<R>;
    const int nout = g.kind == K_R2C ? g.n / 2 + 1 : g.n;
    const long long total = g.nlines * nout;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const long long l = e / nout;
        const int k = (int)(e - l * nout);
        C v = w[l * g.L + k];
        const long long off = line_off(l, g, true);
        if (g.kind == K_C2R) {
            reinterpret_cast<R *>(out)[off + k * g.os] = v.x * (factor ? R(g.ep_scale) : R(1));
        } else {
            if (factor) v = cscale(v, ll_factor<R>(g, k, l));
            reinterpret_cast<C *>(out)[off + k * g.os] = v;
        }
    }
}

unsigned grid_for(long long total)
{
    const long long b = (total + 255) / 256;
    return (unsigned)std::max(1LL, std::min(b, 148LL * 32));
}

// L1 * L2 = L with both factors pass-kernel lengths (not chirp-z), the split closest to
// the square root; 0 if none
int split(int dtype, int L)
{
    int best = 0;
    for (int a = 2; a <= 4096; ++a) {
        if (L % a) continue;
        const int b = L / a;
        if (b < 2 || b > 4096 || !has_kernel(dtype, a) || !has_kernel(dtype, b)) continue;
        if (!best || std::abs(std::log((double)a / b)) < std::abs(std::log((double)best / (L / best)))) best = a;
    }
    return best;
}

// iterative radix-2 FFT in FP64 with an exact root table (the chirp-z kernel spectrum)
void host_fft_pow2(std::vector<std::complex<double>> &x)
{
    const size_t N = x.size();
    std::vector<std::complex<double>> root(N / 2);
    for (size_t k = 0; k < N / 2; ++k) {
        const double ang = -2.0 * M_PI * (double)k / (double)N;
        root[k] = std::complex<double>(std::cos(ang), std::sin(ang));
    }
    for (size_t i = 1, j = 0; i < N; ++i) {
        size_t bit = N >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) std::swap(x[i], x[j]);
    }
    for (size_t len = 2; len <= N; len <<= 1) {
        const size_t step = N / len;
        for (size_t i = 0; i < N; i += len)
            for (size_t k = 0; k < len / 2; ++k) {
                const std::complex<double> u = x[i + k], v = x[i + k + len / 2] * root[k * step];
                x[i + k] = u + v;
                x[i + k + len / 2] = u - v;
            }
    }
}

template <typename T> int upload(const std::vector<std::complex<double>> &h, int dtype, T **dst)
{
    const size_t n = h.size(), cb = complex_bytes(dtype);
    void *p = nullptr;
    if (cudaMalloc(&p, n * cb) != cudaSuccess) {
        cudaGetLastError();
        return FFTB_ERROR_ALLOC;
    }
    cudaError_t e;
    if (dtype == FFTB_F32) {
        std::vector<float2> v(n);
        for (size_t i = 0; i < n; ++i) v[i] = make_float2((float)h[i].real(), (float)h[i].imag());
        e = cudaMemcpy(p, v.data(), n * cb, cudaMemcpyHostToDevice);
    } else {
        std::vector<double2> v(n);
        for (size_t i = 0; i < n; ++i) v[i] = make_double2(h[i].real(), h[i].imag());
        e = cudaMemcpy(p, v.data(), n * cb, cudaMemcpyHostToDevice);
    }
    if (e != cudaSuccess) {
        cudaFree(p);
        return set_status_from_cuda(e);
    }
    *dst = (T *)p;
    return FFTB_SUCCESS;
}

// the four-step passes of one direction over nlines contiguous work lines of length L
int four_step(int dtype, int kind, int L, int L1, long long nlines, const void *roots, Program &prog)
{
    const int L2 = L / L1;
    AxisPass a;
    a.kind = kind;
    a.n = L1;
    a.is = L2;
    a.os = L2;
    a.batch = {Dim{L2, 1, 1, 1}, Dim{nlines, L, L, 2}};
    a.in_buf = B_IN;
    a.out_buf = B_OUT;
    a.ep_mode = EP_TWIDDLE;
    a.ep_axes = {EpAxis{0, 1, L, 0}};
    a.ep_tw = roots;
    int st = program_add(prog, dtype, a);
    if (st != FFTB_SUCCESS) return st;
    AxisPass b;
    b.kind = kind;
    b.n = L2;
    b.is = 1;
    b.os = L1;
    b.batch = {Dim{L1, L2, 1, 1}, Dim{nlines, L, L, 2}};
    b.in_buf = B_OUT;  // the first pass's output
    b.out_buf = B_IN;  // back into the first work line
    return program_add(prog, dtype, b);
}

} // namespace

int longline_create(int dtype, const AxisPass &p, std::shared_ptr<LongLine> &out)
{
    if (p.kind < K_C2C_FWD || p.kind > K_SANDWICH || (p.ep_mode & ~(EP_SCALE | EP_POISSON | EP_GAUSS | EP_HALFW))) {
        set_last_error("long lines take the scale, Poisson, Gaussian and half-axis weight epilogues only");
        return FFTB_ERROR_UNSUPPORTED_SIZE;
    }
    if (p.n < 2 || p.n > (1 << 24)) {
        set_last_error("line length out of range");
        return FFTB_ERROR_UNSUPPORTED_SIZE;
    }
    std::vector<Dim> b;
    for (const Dim &d : p.batch)
        if (d.count > 1) b.push_back(d);
    if (b.size() > 3) return FFTB_ERROR_INVALID_VALUE;
    while (b.size() < 3) b.push_back(Dim{1, 0, 0, -1});
    auto L = std::make_shared<LongLine>();
    L->dtype = dtype;
    L->kind = p.kind;
    L->n = p.n;
    L->nlines = b[0].count * b[1].count * b[2].count;
    L->c0 = b[0].count;
    L->c1 = b[1].count;
    for (int i = 0; i < 3; ++i) {
        L->ib[i] = b[i].is;
        L->ob[i] = b[i].os;
    }
    L->is = p.is;
    L->os = p.os;
    L->in_buf = p.in_buf;
    L->out_buf = p.out_buf;
    const size_t in_el = (p.kind == K_R2C) ? real_bytes(dtype) : complex_bytes(dtype);
    const size_t out_el = (p.kind == K_C2R) ? real_bytes(dtype) : complex_bytes(dtype);
    L->in_off = (size_t)p.in_base * in_el;
    L->out_off = (size_t)p.out_base * out_el;
    L->scale = p.ep_scale;
    L->ep_mode = p.ep_mode;
    L->ep_sign = p.ep_sign;
    L->ep_gauss = p.ep_gauss;
    L->ep_hw = p.ep_hw;
    // epilogue axes to point / batch slots, as program_add resolves them
    if (p.ep_axes.size() > 4) return FFTB_ERROR_INVALID_VALUE;
    L->ep_naxes = (int)p.ep_axes.size();
    for (int i = 0; i < L->ep_naxes; ++i) {
        const EpAxis &e = p.ep_axes[i];
        int src = 0;
        if (!e.from_point) {
            src = -1;
            for (int j = 0; j < 3; ++j)
                if (b[j].id == e.dim_id && b[j].count > 1) src = j + 1;
            if (src < 0)  // a dimension of count 1: index 0, read from an unused slot
                for (int j = 2; j >= 0; --j)
                    if (b[j].count == 1) {
                        src = j + 1;
                        break;
                    }
            if (src < 0) return FFTB_ERROR_INVALID_VALUE;
        }
        L->ep_src[i] = src;
        L->ep_n[i] = e.n;
        L->ep_half[i] = e.half;
    }
    L->inverse = (p.kind == K_C2C_INV || p.kind == K_C2R);
    int L1 = split(dtype, p.n);
    if (L1) {
        L->L = p.n;
    } else {
        if (p.n > (1 << 21)) {
            set_last_error("chirp-z long lines are limited to 2^21 points");
            return FFTB_ERROR_UNSUPPORTED_SIZE;
        }
        L->chirp = true;
        int M = 1;
        while (M < 2 * p.n - 1) M *= 2;
        L->L = M;
        L1 = split(dtype, M);
    }
    if (!L1) {
        set_last_error("no four-step split for line length " + std::to_string(p.n));
        return FFTB_ERROR_UNSUPPORTED_SIZE;
    }
    L->L1 = L1;
    L->L2 = L->L / L1;
    void *roots = nullptr;
    int st = engine_roots(dtype, L->L, &roots);
    if (st != FFTB_SUCCESS) return st;
    if ((st = four_step(dtype, K_C2C_FWD, L->L, L1, L->nlines, roots, L->fwd)) != FFTB_SUCCESS) return st;
    if ((st = four_step(dtype, K_C2C_INV, L->L, L1, L->nlines, roots, L->inv)) != FFTB_SUCCESS) return st;
    const size_t bytes = (size_t)L->nlines * (size_t)L->L * complex_bytes(dtype);
    if (cudaMalloc(&L->w0, bytes) != cudaSuccess || cudaMalloc(&L->w1, bytes) != cudaSuccess) {
        cudaGetLastError();
        set_last_error("cudaMalloc of the long-line work lines failed");
        return FFTB_ERROR_ALLOC;
    }
    if (L->chirp) {
        const int n = p.n, M = L->L;
        std::vector<std::complex<double>> c(n), bb(M, std::complex<double>(0.0, 0.0));
        for (int j = 0; j < n; ++j) {
            const long long q = ((long long)j * j) % (2LL * n);  // j^2 mod 2n: the angle stays exact
            const double ang = -M_PI * (double)q / (double)n;
            c[j] = std::complex<double>(std::cos(ang), std::sin(ang));
        }
        for (int j = 0; j < n; ++j) {
            bb[j] = std::conj(c[j]);
            if (j > 0) bb[M - j] = std::conj(c[j]);
        }
        host_fft_pow2(bb);
        for (auto &v : bb) v /= (double)M;
        void *ct = nullptr;
        if ((st = upload(c, dtype, &ct)) != FFTB_SUCCESS) return st;
        L->chirp_t = ct;
        if ((st = upload(bb, dtype, &L->bhat)) != FFTB_SUCCESS) return st;
    }
    out = L;
    return FFTB_SUCCESS;
}

namespace {
// the DFT of every work line in w0, in place: four-step, or chirp-z around a
// power-of-two four-step convolution (inverse as the conjugate of the forward)
template <typename R> int line_dft(const LongLine &L, bool inverse, cudaStream_t s)
{
    using C = cpx<R>;
    const long long tot = L.nlines * L.L;
    if (!L.chirp) return program_exec(inverse ? L.inv : L.fwd, L.w0, L.w1, nullptr, s);
    ll_chirp<R><<<grid_for(tot), 256, 0, s>>>((C *)L.w0, (const C *)L.chirp_t, L.nlines, L.n, L.L, inverse, 1);
    int st = set_status_from_cuda(cudaGetLastError());
    if (st == FFTB_SUCCESS) st = program_exec(L.fwd, L.w0, L.w1, nullptr, s);
    if (st != FFTB_SUCCESS) return st;
    ll_mul_table<R><<<grid_for(tot), 256, 0, s>>>((C *)L.w0, (const C *)L.bhat, L.nlines, L.L);
    if ((st = set_status_from_cuda(cudaGetLastError())) != FFTB_SUCCESS) return st;
    if ((st = program_exec(L.inv, L.w0, L.w1, nullptr, s)) != FFTB_SUCCESS) return st;
    ll_chirp<R><<<grid_for(tot), 256, 0, s>>>((C *)L.w0, (const C *)L.chirp_t, L.nlines, L.n, L.L, inverse, 0);
    return set_status_from_cuda(cudaGetLastError());
}

template <typename R> int run(const LongLine &L, const void *in, void *out, const Geom &g, cudaStream_t s)
{
    using C = cpx<R>;
    const long long tot = L.nlines * L.L;
    ll_gather<R><<<grid_for(tot), 256, 0, s>>>(in, (C *)L.w0, g);
    int st = set_status_from_cuda(cudaGetLastError());
    if (st != FFTB_SUCCESS) return st;
    if (L.kind == K_SANDWICH) {
        if ((st = line_dft<R>(L, false, s)) != FFTB_SUCCESS) return st;
        ll_multiply<R><<<grid_for(L.nlines * L.n), 256, 0, s>>>((C *)L.w0, g);
        if ((st = set_status_from_cuda(cudaGetLastError())) != FFTB_SUCCESS) return st;
        if ((st = line_dft<R>(L, true, s)) != FFTB_SUCCESS) return st;
    } else if ((st = line_dft<R>(L, L.inverse, s)) != FFTB_SUCCESS) {
        return st;
    }
    const long long nout = L.nlines * (L.kind == K_R2C ? L.n / 2 + 1 : L.n);
    const int factor = (L.kind != K_SANDWICH && g.ep_mode != 0) ? 1 : 0;
    ll_scatter<R><<<grid_for(nout), 256, 0, s>>>((const C *)L.w0, out, g, factor);
    return set_status_from_cuda(cudaGetLastError());
}
} // namespace

int longline_exec(const LongLine &L, void *const bufs[3], cudaStream_t s, const EpValues *ep)
{
    if (!bufs[L.in_buf] || !bufs[L.out_buf]) {
        set_last_error("missing buffer");
        return L.in_buf == B_WORK || L.out_buf == B_WORK ? FFTB_ERROR_NO_WORK_AREA : FFTB_ERROR_INVALID_VALUE;
    }
    const void *in = (const char *)bufs[L.in_buf] + L.in_off;
    void *out = (char *)bufs[L.out_buf] + L.out_off;
    Geom g;
    g.nlines = L.nlines;
    g.c0 = L.c0;
    g.c1 = L.c1;
    g.ib0 = L.ib[0]; g.ib1 = L.ib[1]; g.ib2 = L.ib[2];
    g.ob0 = L.ob[0]; g.ob1 = L.ob[1]; g.ob2 = L.ob[2];
    g.is = L.is;
    g.os = L.os;
    g.n = L.n;
    g.L = L.L;
    g.kind = L.kind;
    g.ep_mode = L.ep_mode;
    g.ep_naxes = L.ep_naxes;
    for (int i = 0; i < 4; ++i) {
        g.ep_src[i] = L.ep_src[i];
        g.ep_n[i] = L.ep_n[i];
        g.ep_half[i] = L.ep_half[i];
    }
    g.ep_scale = L.scale;
    g.ep_sign = L.ep_sign;
    g.ep_gauss = L.ep_gauss;
    g.ep_hw = L.ep_hw;
    if (ep) {  // the dynamic epilogue values of this execution
        g.ep_scale = ep->scale;
        g.ep_sign = ep->sign;
        g.ep_gauss = ep->gauss;
        if (ep->mode >= 0) g.ep_mode = ep->mode;
    }
    return L.dtype == FFTB_F32 ? run<float>(L, in, out, g, s) : run<double>(L, in, out, g, s);
}

int longline_launches(const LongLine &L)
{
    const int dft = L.chirp ? 7 : 2;
    return 2 + (L.kind == K_SANDWICH ? 2 * dft + 1 : dft);
}

double longline_alg_bytes(const LongLine &L)
{
    const size_t in_el = (L.kind == K_R2C) ? real_bytes(L.dtype) : complex_bytes(L.dtype);
    const size_t out_el = (L.kind == K_C2R) ? real_bytes(L.dtype) : complex_bytes(L.dtype);
    const double pin = L.kind == K_C2R ? L.n / 2 + 1 : L.n, pout = L.kind == K_R2C ? L.n / 2 + 1 : L.n;
    return (double)L.nlines * (pin * in_el + pout * out_el);
}

} // namespace fftb
