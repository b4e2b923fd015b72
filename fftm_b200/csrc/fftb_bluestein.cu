// fftb_bluestein.cu -- lines of any length n <= 4096 that the radix kernels do not
// cover (large prime factors: 17, 19, 34, 70, 1000, ...), through Bluestein's chirp-z
// identity (L. I. Bluestein, "A linear filtering approach to the computation of the
// discrete Fourier transform", 1970):
//   with c_j = exp(-i pi j^2 / n) and mk = (m^2 + k^2 - (k - m)^2) / 2,
//   X_k = sum_m x_m exp(-2 pi i m k / n) = c_k sum_m (x_m c_m) conj(c_{k-m}),
// a linear convolution evaluated as a circular one of power-of-two length M >= 2n - 1:
//   a = (x c, zero padded), b_j = conj(c_|j|) for |j| < n (wrapped), X = c * IFFT_M(FFT_M(a) B),
// with B = FFT_M(b) / M precomputed on the host in FP64.  The inverse transform is
// conj(Bluestein(conj x)).  One CTA holds G lines of M points in shared memory and runs
// the two length-M FFTs with the Stockham core; the pass geometry (strides, batch
// dimensions, epilogues, the R2C / C2R forms on the full line) is the generic pass's.
#include <cuda_runtime.h>

#include <cmath>
#include <complex>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "../../include/fftb.h"
#include "fftb_bluestein.h"
#include "fftb_pass.cuh"

namespace fftb {
namespace {

template <typename R, int M>
__global__ void __launch_bounds__(512) fftb_bluestein_kernel(PassArgs a)
{
    using C = cpx<R>;
    constexpr int T = threads_per_line(M);
    constexpr int LP = pad16(M) + 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *stw_s = reinterpret_cast<C *>(smem_raw);
    const int ntw_s = a.tw_smem ? a.ntw : 0;
    long long *offs = reinterpret_cast<long long *>(stw_s + ntw_s);  // [G][2] in/out offsets
    int *bidx = reinterpret_cast<int *>(offs + 2 * a.G);            // [G][4] batch indices, valid
    C *lines = reinterpret_cast<C *>(bidx + 4 * a.G);               // [G][LP]

    const int tid = threadIdx.x;
    const int G = a.G;
    const int g = tid / T, t = tid - (tid / T) * T;
    const long long line0 = (long long)blockIdx.x * G;
    const C *twg = reinterpret_cast<const C *>(a.tw);
    for (int i = tid; i < ntw_s; i += blockDim.x) stw_s[i] = twg[i];
    const C *stw = a.tw_smem ? stw_s : twg;
    for (int gg = tid; gg < G; gg += blockDim.x) {
        const long long l = line0 + gg;
        const bool v = l < a.nlines;
        const long long ll = v ? l : 0;
        const long long b0 = ll % a.c0, r = ll / a.c0, b1 = r % a.c1, b2 = r / a.c1;
        offs[2 * gg] = b0 * a.ib0 + b1 * a.ib1 + b2 * a.ib2;
        offs[2 * gg + 1] = b0 * a.ob0 + b1 * a.ob1 + b2 * a.ob2;
        bidx[4 * gg] = (int)b0;
        bidx[4 * gg + 1] = (int)b1;
        bidx[4 * gg + 2] = (int)b2;
        bidx[4 * gg + 3] = v ? 1 : 0;
    }
    __syncthreads();

    const int n = a.bs_n;
    const int kind = a.kind;
    const C *chirp = reinterpret_cast<const C *>(a.bs_chirp);
    const C *bhat = reinterpret_cast<const C *>(a.bs_bhat);
    const bool has = g < G;                        // this thread belongs to a line of the CTA
    const bool valid = has && bidx[4 * g + 3];     // ... that exists
    C *ln = lines + (has ? g : 0) * LP;
    const long long io = has ? offs[2 * g] : 0, oo = has ? offs[2 * g + 1] : 0;
    const C zero = mk<R>(R(0), R(0));

    // X = c * IFFT_M(FFT_M(a) B) on the line, a[m] = u[m] c[m] already staged
    auto convolve = [&]() {
        fft_line<R, M, -1>(ln, stw, a.ntw, t, has);
        if (has)
            for (int m = t; m < M; m += T) ln[pad16(m)] = cmul(ln[pad16(m)], bhat[m]);
        __syncthreads();
        fft_line<R, M, +1>(ln, stw, a.ntw, t, has);
    };

    // ---- stage u c, zero padded; the inverse direction conjugates in and out
    const bool inv = (kind == K_C2C_INV || kind == K_C2R);
    if (has) {
        for (int m = t; m < M; m += T) {
            C v = zero;
            if (m < n && valid) {
                if (kind == K_R2C) {
                    v = mk<R>(reinterpret_cast<const R *>(a.in)[io + (long long)m * a.is], R(0));
                } else if (kind == K_C2R) {
                    // Hermitian extension of the half spectrum; the imaginary parts of the
                    // DC and (even n) Nyquist bins are ignored, as a C2R transform does
                    const int k = m <= n / 2 ? m : n - m;
                    v = reinterpret_cast<const C *>(a.in)[io + (long long)k * a.is];
                    if (m > n / 2) v = cconj(v);
                    if (m == 0 || 2 * m == n) v.y = R(0);
                } else {
                    v = reinterpret_cast<const C *>(a.in)[io + (long long)m * a.is];
                }
                if (inv) v = cconj(v);
                v = cmul(v, chirp[m]);
            }
            ln[pad16(m)] = v;
        }
    }
    __syncthreads();
    convolve();
    if (has)
        for (int k = t; k < n; k += T) {
            C y = cmul(ln[pad16(k)], chirp[k]);
            ln[pad16(k)] = inv ? cconj(y) : y;
        }
    __syncthreads();

    // ---- sandwich: spectral multiply, then the inverse transform of the line
    if (kind == K_SANDWICH) {
        if (has) {
            for (int m = t; m < M; m += T) {
                C v = zero;
                if (m < n && valid) v = cmul(cconj(cscale(ln[pad16(m)], ep_factor<R>(a, m, bidx + 4 * g))), chirp[m]);
                ln[pad16(m)] = v;
            }
        }
        __syncthreads();
        convolve();
        if (has)
            for (int k = t; k < n; k += T) ln[pad16(k)] = cconj(cmul(ln[pad16(k)], chirp[k]));
        __syncthreads();
    }

    // ---- store (epilogue as in the generic pass: scale for C2R, the spectral factor otherwise)
    if (!valid) return;
    const bool ep_store = (a.ep_mode != 0) && kind != K_SANDWICH;
    if (kind == K_C2R) {
        R *out = reinterpret_cast<R *>(a.out);
        const R sc = ep_store ? R(a.ep_scale) : R(1);
        for (int m = t; m < n; m += T) out[oo + (long long)m * a.os] = ln[pad16(m)].x * sc;
    } else {
        C *out = reinterpret_cast<C *>(a.out);
        const int nout = kind == K_R2C ? n / 2 + 1 : n;
        for (int k = t; k < nout; k += T) {
            C v = ln[pad16(k)];
            if (ep_store) v = cscale(v, ep_factor<R>(a, k, bidx + 4 * g));
            out[oo + (long long)k * a.os] = v;
        }
    }
}

template <typename R, int M> PassKernelInfo bluestein_info()
{
    PassKernelInfo k;
    k.nf = M;
    k.threads_per_line = threads_per_line(M);
    k.line_pitch = pad16(M) + 1;
    k.fn = (const void *)&fftb_bluestein_kernel<R, M>;
    return k;
}

template <typename R> bool bluestein_lookup(int M, PassKernelInfo *k)
{
    switch (M) {
    case 32: *k = bluestein_info<R, 32>(); return true;
    case 64: *k = bluestein_info<R, 64>(); return true;
    case 128: *k = bluestein_info<R, 128>(); return true;
    case 256: *k = bluestein_info<R, 256>(); return true;
    case 512: *k = bluestein_info<R, 512>(); return true;
    case 1024: *k = bluestein_info<R, 1024>(); return true;
    case 2048: *k = bluestein_info<R, 2048>(); return true;
    case 4096: *k = bluestein_info<R, 4096>(); return true;
    case 8192: *k = bluestein_info<R, 8192>(); return true;
    default: return false;
    }
}

// in-place iterative radix-2 FFT (forward, unnormalised) of a power-of-two vector, FP64
void host_fft(std::vector<std::complex<double>> &x)
{
    const size_t N = x.size();
    for (size_t i = 1, j = 0; i < N; ++i) {
        size_t bit = N >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) std::swap(x[i], x[j]);
    }
    for (size_t len = 2; len <= N; len <<= 1) {
        for (size_t i = 0; i < N; i += len) {
            for (size_t k = 0; k < len / 2; ++k) {
                // exp(-2 pi i k / len) with the angle reduced exactly
                const double ang = -2.0 * M_PI * (double)k / (double)len;
                const std::complex<double> w(std::cos(ang), std::sin(ang));
                const std::complex<double> u = x[i + k], v = x[i + k + len / 2] * w;
                x[i + k] = u + v;
                x[i + k + len / 2] = u - v;
            }
        }
    }
}

struct Tables {
    void *chirp = nullptr, *bhat = nullptr;
};

} // namespace

int bluestein_size(int n)
{
    if (n < 2 || n > 4096) return 0;
    int M = 32;
    while (M < 2 * n - 1) M *= 2;
    return M;
}

bool bluestein_kernel(int dtype, int n, PassKernelInfo *k)
{
    const int M = bluestein_size(n);
    if (!M) return false;
    return dtype == FFTB_F32 ? bluestein_lookup<float>(M, k) : bluestein_lookup<double>(M, k);
}

int bluestein_tables(int dtype, int n, const void **chirp, const void **bhat)
{
    static std::mutex mu;
    static std::map<std::tuple<int, int, int>, Tables> cache;
    const int M = bluestein_size(n);
    if (!M) return FFTB_ERROR_UNSUPPORTED_SIZE;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return set_status_from_cuda(e);
    std::lock_guard<std::mutex> lk(mu);
    auto key = std::make_tuple(dev, dtype, n);
    auto it = cache.find(key);
    if (it != cache.end()) {
        *chirp = it->second.chirp;
        *bhat = it->second.bhat;
        return FFTB_SUCCESS;
    }
    // c_j = exp(-i pi j^2 / n), with j^2 reduced mod 2n so the angle is exact
    std::vector<std::complex<double>> c(n), b(M, std::complex<double>(0.0, 0.0));
    for (int j = 0; j < n; ++j) {
        const long long q = ((long long)j * j) % (2LL * n);
        const double ang = -M_PI * (double)q / (double)n;
        c[j] = std::complex<double>(std::cos(ang), std::sin(ang));
    }
    for (int j = 0; j < n; ++j) {
        b[j] = std::conj(c[j]);
        if (j > 0) b[M - j] = std::conj(c[j]);
    }
    host_fft(b);
    for (auto &v : b) v /= (double)M;
    Tables t;
    const size_t cb = complex_bytes(dtype);
    e = cudaMalloc(&t.chirp, cb * n);
    if (e == cudaSuccess) e = cudaMalloc(&t.bhat, cb * M);
    if (e != cudaSuccess) {
        cudaGetLastError();
        if (t.chirp) cudaFree(t.chirp);
        set_last_error("cudaMalloc of Bluestein tables failed");
        return FFTB_ERROR_ALLOC;
    }
    if (dtype == FFTB_F32) {
        std::vector<float2> hc(n), hb(M);
        for (int j = 0; j < n; ++j) hc[j] = make_float2((float)c[j].real(), (float)c[j].imag());
        for (int j = 0; j < M; ++j) hb[j] = make_float2((float)b[j].real(), (float)b[j].imag());
        e = cudaMemcpy(t.chirp, hc.data(), cb * n, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(t.bhat, hb.data(), cb * M, cudaMemcpyHostToDevice);
    } else {
        std::vector<double2> hc(n), hb(M);
        for (int j = 0; j < n; ++j) hc[j] = make_double2(c[j].real(), c[j].imag());
        for (int j = 0; j < M; ++j) hb[j] = make_double2(b[j].real(), b[j].imag());
        e = cudaMemcpy(t.chirp, hc.data(), cb * n, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(t.bhat, hb.data(), cb * M, cudaMemcpyHostToDevice);
    }
    if (e != cudaSuccess) return set_status_from_cuda(e);
    cache[key] = t;
    *chirp = t.chirp;
    *bhat = t.bhat;
    return FFTB_SUCCESS;
}

} // namespace fftb
