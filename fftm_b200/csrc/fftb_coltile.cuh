// fftb_coltile.cuh -- the register-resident column tile of the x column kernels and the
// row-pair tile of the grouped z rows, shared by the fused 3D / 4D kernels and the batch
// kernels (device templates and the column epilogue parameters).
#pragma once

#include <cuda_runtime.h>

#include "fftb_device.cuh"
#include "fftb_fused3d.h"
#include "fftb_internal.h"
#include "fftb_regfft.cuh"
#include "fftb_tc.cuh"

namespace fftb {

// ------------------------------------------------------------------ x column kernel
// Columns c in [0, ncols) of a spectrum whose x rows are `stride` apart.  Thread
// (t, col) = (tid / W, tid % W) holds rows t + T*r of column col, so every load
// and store instruction of a warp touches W (or 32) consecutive columns.
struct XColEp {
    int mode;  // EpMode bits (0: none)
    float scale_f, sign_f, gauss_f;
    double scale, sign, gauss;
    // column -> wavenumbers: 3D col = ky*nzh + kz (kz half axis); 4D (nd4) col = (ky*nz + kz)*nwh + kw
    int nzh, ny, nz;
    int nd4, nwh;
    // EP_HALFW: interior bins of the half axis (column index mod (hn/2+1)) times hw
    int hn;
    float hw_f;
    double hw;
    int tc;  // host side: launch the tensor-core variant of the kernel
    // EP_DERIV (3D, inverse mode): multiply by i k_daxis * dscale before the x FFT
    int daxis;
    float dscale_f;
    double dscale;
};

template <int NX> struct XColShape {
    static constexpr int T = RegFFTShape<NX>::T;
    static constexpr int W = 256 / T;      // columns per CTA (48, 96 points: T = 3, 6, and the
    static constexpr int NT = 256;         // threads past T * W idle)
};

// TC: the first radix-16 stage runs on the tensor cores (fftb_tc.cuh, float only)
template <typename R, int NX, int SIGN, bool TC>
__device__ __forceinline__ void xcol_fft(cpx<R> (&v)[16], cpx<R> *scr, const cpx<R> *tw, int t, int col,
                                         unsigned char *stage, const TcDft16 &F)
{
    using C = cpx<R>;
    constexpr int T = XColShape<NX>::T, W = XColShape<NX>::W;
    if constexpr (16 % T != 0) {
        // T = 3 or 6 threads per column (48 or 96 points): thread t runs the second-stage DFTs
        // of k1 = t, t + T, ... < 16, and one more exchange brings the results back to the
        // layout v[j] = X[t + T j]; threads past T * W (t = T) take part in the barriers only
        static_assert(!TC, "tensor-core form: power-of-two columns only");
        const bool act = t < T;
        const int tt = act ? t : 0;
        dft16<SIGN, C, R>(v);
#pragma unroll
        for (int k1 = 1; k1 < 16; ++k1) v[k1] = twiddle_mul<SIGN>(v[k1], tw, tt * k1);
        __syncthreads();
        if (act) {
#pragma unroll
            for (int k1 = 0; k1 < 16; ++k1) scr[(k1 * T + t) * W + col] = v[k1];
        }
        __syncthreads();
        constexpr int A = (16 + T - 1) / T;
        C res[A][T];
#pragma unroll
        for (int a = 0; a < A; ++a) {
            const int k1 = tt + T * a;
            const bool valid = act && k1 < 16;
#pragma unroll
            for (int q = 0; q < T; ++q) res[a][q] = valid ? scr[(k1 * T + q) * W + col] : mk<R>(R(0), R(0));
            dft_small<SIGN, T, C, R>(res[a]);
        }
        __syncthreads();
#pragma unroll
        for (int a = 0; a < A; ++a) {
            const int k1 = tt + T * a;
            if (act && k1 < 16) {
#pragma unroll
                for (int k2 = 0; k2 < T; ++k2) scr[(k1 + 16 * k2) * W + col] = res[a][k2];
            }
        }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < 16; ++j) v[j] = act ? scr[(t + T * j) * W + col] : mk<R>(R(0), R(0));
        return;
    }
    if constexpr (TC) tc_dft16<SIGN>(v, stage, F, (int)(threadIdx.x & 31));
    else dft16<SIGN, C, R>(v);
#pragma unroll
    for (int k1 = 1; k1 < 16; ++k1) v[k1] = twiddle_mul<SIGN>(v[k1], tw, t * k1);
    __syncthreads();
#pragma unroll
    for (int k1 = 0; k1 < 16; ++k1) scr[(k1 * T + t) * W + col] = v[k1];
    __syncthreads();
    constexpr int A = 16 / T;
#pragma unroll
    for (int a = 0; a < A; ++a) {
        C u[T];
#pragma unroll
        for (int q = 0; q < T; ++q) u[q] = scr[((t + T * a) * T + q) * W + col];
        dft_small<SIGN, T, C, R>(u);
#pragma unroll
        for (int k2 = 0; k2 < T; ++k2) v[a + A * k2] = u[k2];
    }
}

// The spectral multiply of the column sandwich (MODE 2): v holds rows kx = t + T*j of column
// cg0; ky, kz (and kw in 4D) follow from the column index.
template <typename R, int NX>
__device__ __forceinline__ void xcol_multiply(cpx<R> (&v)[16], int t, int cg0, const XColEp &ep)
{
    constexpr int T = XColShape<NX>::T;
    // wavenumbers: kx = t + T*j (output row); ky, kz, kw from the column
    int ky_i, kz, kw = 0;
    if (ep.nd4) {
        const int cc = cg0 % (ep.nz * ep.nwh);
        ky_i = cg0 / (ep.nz * ep.nwh);
        const int kz_i = cc / ep.nwh;
        kw = cc - kz_i * ep.nwh;
        kz = kz_i <= ep.nz / 2 ? kz_i : kz_i - ep.nz;
    } else {
        ky_i = cg0 / ep.nzh;
        kz = cg0 - (cg0 / ep.nzh) * ep.nzh;
    }
    const int ky = ky_i <= ep.ny / 2 ? ky_i : ky_i - ep.ny;
    const R kyz = R(ky * ky + kz * kz + kw * kw);
    const R sc = sizeof(R) == 4 ? R(ep.scale_f) : R(ep.scale);
    const R sg = sizeof(R) == 4 ? R(ep.sign_f) : R(ep.sign);
    if (ep.mode & EP_DERIV) {
        // i k v * scale with k = kx (row), ky or kz (the column); 3D only.  kz is the half
        // axis: its Nyquist bin carries the real cosine part, whose derivative the C2R
        // drops with the imaginary part, the same as a separate multiply does
        const R ds = sizeof(R) == 4 ? R(ep.dscale_f) : R(ep.dscale);
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const int kxi = t + T * j;
            const int k = ep.daxis == 0 ? (kxi <= NX / 2 ? kxi : kxi - NX) : (ep.daxis == 1 ? ky : kz);
            const R fct = R(k) * ds;
            v[j] = mk<R>(-fct * v[j].y, fct * v[j].x);
        }
    } else if ((ep.mode & (EP_POISSON | EP_GAUSS)) == EP_POISSON) {
        const R ss = sc * sg;
        const R tr = R(t);
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            // kx = t + T j, or t + T j - NX past the Nyquist row (T j = NX/2 is the Nyquist row
            // itself only for t = 0); the offsets are compile-time constants
            R kx;
            if (T * j < NX / 2) kx = tr + R(T * j);
            else if (T * j > NX / 2) kx = tr + R(T * j - NX);
            else kx = t == 0 ? R(NX / 2) : tr + R(T * j - NX);
            const R k2 = kx * kx + kyz;
            R fct;
            if constexpr (sizeof(R) == 4) fct = ss * rcp_approx(k2);  // relative error below 2^-22
            else fct = ss / k2;
            if (j == 0 && k2 == R(0)) fct = R(0);  // only row kx = 0 can hold the zero mode
            v[j] = cscale(v[j], fct);
        }
    } else {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const int kxi = t + T * j;
            const int kx = kxi <= NX / 2 ? kxi : kxi - NX;
            const R k2 = R(kx * kx) + kyz;
            R fct = sc;
            if (ep.mode & EP_POISSON) fct = (k2 == R(0)) ? R(0) : fct * sg / k2;
            if (ep.mode & EP_GAUSS) fct *= exp(-k2 * (sizeof(R) == 4 ? R(ep.gauss_f) : R(ep.gauss)));
            v[j] = cscale(v[j], fct);
        }
    }
}

// EP_HALFW: interior bins of the half axis times hw (the adjoint weights)
template <typename R> __device__ __forceinline__ void xcol_halfw(cpx<R> (&v)[16], int cg0, const XColEp &ep)
{
    const int ih = cg0 % (ep.hn / 2 + 1);
    if (ih != 0 && 2 * ih != ep.hn) {
        const R w = sizeof(R) == 4 ? R(ep.hw_f) : R(ep.hw);
#pragma unroll
        for (int j = 0; j < 16; ++j) v[j] = cscale(v[j], w);
    }
}

// MODE 0: forward, 1: inverse, 2: forward -> spectral multiply -> inverse (in place, or
// into tdata, laid out like data, when tdata is given),
// 3: forward, written transposed: column col becomes the contiguous row tout[col][kx],
// 4: inverse of 3: reads the rows tin[col][kx], writes the columns in place of `data`.
// blockIdx.y selects a batch of column sets `bstride` elements apart (the transposed
// side has NX * ncols elements per batch).
// The body of one column tile (blockIdx.x of xcol_kernel): tile `tile` of batch `batch`.
template <typename R, int NX, int MODE, bool TC>
__device__ __forceinline__ void xcol_tile(cpx<R> *__restrict__ data, long long stride, int ncols, long long bstride,
                                          cpx<R> *__restrict__ tdata, const cpx<R> *__restrict__ roots,
                                          const XColEp &ep, int tile, int batch)
{
    using C = cpx<R>;
    constexpr int T = XColShape<NX>::T, W = XColShape<NX>::W;
    constexpr int RP = NX + 1;  // row pitch of the transposing stage
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *scr = reinterpret_cast<C *>(smem_raw);
    C *tw = scr + (16 * T * W > W * RP ? 16 * T * W : W * RP);
    // TC: each warp's tensor-core staging area follows the twiddles
    unsigned char *stage = reinterpret_cast<unsigned char *>(tw + NX) + (threadIdx.x >> 5) * kTcWarpBytes;
    TcDft16 F;
    if constexpr (TC) tc_build_dft16(F, (int)(threadIdx.x & 31));
    const int tid = threadIdx.x;
    const int t = tid / W, col = tid - (tid / W) * W;
    for (int i = tid; i < NX; i += 256) tw[i] = roots[i];
    const int cg0 = tile * W + col;
    const bool act = t < T;  // false only for the idle threads of 48- and 96-point columns
    const bool ok = act && cg0 < ncols;
    data += (size_t)batch * bstride;
    C *p = data + (ok ? cg0 : 0);
    C v[16];
    if (MODE == 4) {
        // rows of the transposed input -> shared memory -> columns in registers
        const C *src = tdata + (size_t)batch * NX * ncols + (size_t)tile * W * NX;
        const int nrow = (ncols - tile * W) < W ? (ncols - tile * W) : W;
        // all of the tile's row loads in flight at once
        for (int e = tid; e < nrow * NX; e += 256) {
            const int rr = e / NX, kx = e - (e / NX) * NX;
            cp_async<sizeof(C)>(&scr[rr * RP + kx], src + (size_t)rr * NX + kx, true);
        }
        cp_async_wait_all();
        __syncthreads();
#pragma unroll
        for (int r = 0; r < 16; ++r) v[r] = scr[col * RP + t + T * r];
    } else {
#pragma unroll
        for (int r = 0; r < 16; ++r) v[r] = act ? p[(size_t)(t + T * r) * stride] : mk<R>(R(0), R(0));
    }
    __syncthreads();
    if (MODE == 1 || MODE == 4) xcol_fft<R, NX, +1, TC>(v, scr, tw, t, col, stage, F);
    else xcol_fft<R, NX, -1, TC>(v, scr, tw, t, col, stage, F);
    if (MODE == 2) {
        xcol_multiply<R, NX>(v, t, cg0, ep);
        xcol_fft<R, NX, +1, TC>(v, scr, tw, t, col, stage, F);
    }
    if (MODE != 2 && (ep.mode & EP_HALFW)) xcol_halfw<R>(v, cg0, ep);
    if (MODE == 3) {
        // columns in registers -> shared memory -> contiguous rows of the transposed output
        __syncthreads();
#pragma unroll
        for (int j = 0; j < 16; ++j) scr[col * RP + t + T * j] = v[j];
        __syncthreads();
        C *dstp = tdata + (size_t)batch * NX * ncols + (size_t)tile * W * NX;
        const int nrow = (ncols - tile * W) < W ? (ncols - tile * W) : W;
        for (int e = tid; e < nrow * NX; e += 256) {
            const int rr = e / NX, kx = e - (e / NX) * NX;
            dstp[(size_t)rr * NX + kx] = scr[rr * RP + kx];
        }
    } else if (ok) {
        C *q = (MODE == 2 && tdata) ? tdata + (size_t)batch * bstride + cg0 : p;
#pragma unroll
        for (int j = 0; j < 16; ++j) q[(size_t)(t + T * j) * stride] = v[j];
    }
}

// The y FFT (MODE 0 forward, 1 inverse) of one tile of lines (x, kz) of a 3D spectrum
// [nx][ny][nzh], kz fastest, W lines per tile, so a warp reads 32 consecutive lines of a y row
// (contiguous within each x).  it.ncols holds nx * nzh, it.tile the tile, it.ny / it.nz the
// spectrum's sizes, it.off its offset from data.
template <int NY, int MODE>
__device__ __forceinline__ void ycol_tile(const XGroupItem &it, float2 *__restrict__ data,
                                          const float2 *__restrict__ roots)
{
    using C = float2;
    constexpr int T = XColShape<NY>::T, W = XColShape<NY>::W;
    constexpr int RP = NY + 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *scr = reinterpret_cast<C *>(smem_raw);
    C *tw = scr + (16 * T * W > W * RP ? 16 * T * W : W * RP);
    const int tid = threadIdx.x;
    const int t = tid / W, col = tid - (tid / W) * W;
    for (int i = tid; i < NY; i += 256) tw[i] = roots[i];
    const int nzh = it.nz / 2 + 1;
    const int l = it.tile * W + col;
    const bool act = t < T;  // false only for the idle threads of 48- and 96-point lines
    const bool ok = act && l < it.ncols;
    const int lc = ok ? l : 0;
    const int x = lc / nzh, kz = lc - (lc / nzh) * nzh;
    C *p = data + it.off + (long long)x * it.ny * nzh + kz;
    C v[16];
#pragma unroll
    for (int r = 0; r < 16; ++r) v[r] = act ? p[(size_t)(t + T * r) * nzh] : mk<float>(0.f, 0.f);
    __syncthreads();
    TcDft16 F;
    xcol_fft<float, NY, MODE == 1 ? +1 : -1, false>(v, scr, tw, t, col, nullptr, F);
    if (ok) {
#pragma unroll
        for (int j = 0; j < 16; ++j) p[(size_t)(t + T * j) * nzh] = v[j];
    }
}

// The R2C (DIR 0) or C2R (DIR 1) of one tile of row pairs of the contiguous z rows of a 3D
// transform, two real rows per complex NZ-point FFT (the plane kernels' z stage without the
// plane): a group of TZ = NZ / 16 threads holds the row pair in registers.  R2C: z = a + i b,
// X_a[k] = (Z[k] + conj Z[-k]) / 2, X_b[k] = (Z[k] - conj Z[-k]) / 2i, DC and Nyquist real.
// C2R: Z = X_a + i X_b over the Hermitian extension (the imaginary parts of DC and Nyquist
// ignored, as the C2R pass does), a = Re IFFT(Z), b = Im IFFT(Z), times it.scale.  Rows at
// real offset it.roff, spectra at it.soff.
template <int NZ, int DIR>
__device__ __forceinline__ void row_tile(const RowGroupItem &it, const void *__restrict__ in, void *__restrict__ out,
                                         const float2 *__restrict__ roots)
{
    using C = float2;
    constexpr int TZ = NZ / 16, FZ = 256 / TZ, NH = NZ / 2 + 1;
    static_assert(NZ >= 32 && NZ <= 256 && (NZ & (NZ - 1)) == 0, "power-of-two rows of 32-256 points");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int tid = threadIdx.x;
    const int f = tid / TZ, t = tid - (tid / TZ) * TZ;
    C *reg = reinterpret_cast<C *>(smem_raw) + f * RegFFTShape<NZ>::REGION;
    C tw[16];
    load_stage_twiddles<float, NZ>(tw, roots, NZ, t);
    const long long p = (long long)it.tile * FZ + f;  // row pair
    const bool ok = 2 * p < it.nrows;
    const bool hasb = 2 * p + 1 < it.nrows;
    const long long pa = ok ? 2 * p : 0, pb = hasb ? 2 * p + 1 : pa;
    C v[16];
    if constexpr (DIR == 0) {
        const float *rin = reinterpret_cast<const float *>(in) + it.roff;
        const float *ra = rin + pa * NZ, *rb = rin + pb * NZ;
#pragma unroll
        for (int r = 0; r < 16; ++r) v[r] = mk<float>(ra[t + TZ * r], hasb ? rb[t + TZ * r] : 0.f);
        regfft_warp_rt<float, NZ, -1>(v, reg, tw, t);
        // Z[t + TZ j] sits in lane t, register j; Z[NZ - (t + TZ j)] in lane (TZ - t) mod TZ,
        // register 15 - j (t > 0), or in this lane, register (16 - j) mod 16 (t = 0)
        const int lane = threadIdx.x & 31;
        const int src = (lane - t) + ((TZ - t) & (TZ - 1));
        const C zn = mk<float>(__shfl_sync(0xffffffffu, v[8].x, lane - t),
                               __shfl_sync(0xffffffffu, v[8].y, lane - t));  // Z[NZ/2]
        C *sout = reinterpret_cast<C *>(out) + it.soff;
        C *oa = sout + pa * NH, *ob = sout + pb * NH;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int k = t + TZ * j;  // k < NZ/2
            const C zk = v[j];
            C zp;
            zp.x = __shfl_sync(0xffffffffu, v[15 - j].x, src);
            zp.y = __shfl_sync(0xffffffffu, v[15 - j].y, src);
            if (t == 0) zp = v[(16 - j) & 15];
            const C zm = cconj(zp);
            C A = cscale(cadd(zk, zm), 0.5f);
            C B = cscale(mul_si<-1>(csub(zk, zm)), 0.5f);
            if (k == 0) {
                A = mk<float>(zk.x, 0.f);
                B = mk<float>(zk.y, 0.f);
            }
            if (ok) {
                oa[k] = A;
                if (hasb) ob[k] = B;
            }
        }
        if (ok && t == 0) {
            oa[NZ / 2] = mk<float>(zn.x, 0.f);
            if (hasb) ob[NZ / 2] = mk<float>(zn.y, 0.f);
        }
    } else {
        const C *sin_ = reinterpret_cast<const C *>(in) + it.soff;
        const C *ha = sin_ + pa * NH, *hb = sin_ + pb * NH;
        // n = t + TZ r: registers r < 8 hold n < NZ/2 (X[n]); r >= 8 hold n >= NZ/2, X[n] =
        // conj X[NZ - n]; DC (r = 0) and Nyquist (r = 8) of lane t = 0 keep their real parts
#pragma unroll
        for (int r = 0; r < 16; ++r) {
            const int k = r < 8 ? t + TZ * r : TZ * (16 - r) - t;
            C xa = ha[k], xb = hasb ? hb[k] : mk<float>(0.f, 0.f);
            if (r >= 8) {
                xa = cconj(xa);
                xb = cconj(xb);
            }
            if ((r == 0 || r == 8) && t == 0) {
                xa.y = 0.f;
                xb.y = 0.f;
            }
            v[r] = mk<float>(xa.x - xb.y, xa.y + xb.x);  // X_a + i X_b
        }
        regfft_warp_rt<float, NZ, +1>(v, reg, tw, t);
        float *rout = reinterpret_cast<float *>(out) + it.roff;
        float *ra = rout + pa * NZ, *rb = rout + pb * NZ;
        if (ok) {
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                ra[t + TZ * j] = v[j].x * it.scale;
                if (hasb) rb[t + TZ * j] = v[j].y * it.scale;
            }
        }
    }
}

} // namespace fftb
