// fftb_pass.cuh -- the generic strided/batched 1D FFT pass kernel.
//
// One launch transforms L independent lines of one axis.  A CTA owns G
// consecutive lines (G a power of two), stages them in shared memory with
// coalesced loads (points-fastest when the axis is contiguous, lines-fastest when
// the lines are), runs the Stockham core on each line with T threads, applies
// the fused spectral epilogue and writes the lines back with coalesced stores.
// Input and output geometries are independent, so a pass can also permute the
// array (this is how the 4D layout changes of the reference's transposes,
// source/detail/direct_transpose_4d.h:17-32, are fused into the FFT passes).
#pragma once

#include "fftb_device.cuh"
#include "fftb_internal.h"
#include "fftb_regfft.cuh"

namespace fftb {

// Lines of 16 T points (T = 2..16 a power of two, or T = 3, 5, 6: 48, 80 and 96 points) run
// the register-resident two-stage FFT (fftb_regfft.cuh) on their staged line instead of the
// Stockham passes: one read of the line into registers, radix-16 in registers, one exchange
// through the line's own buffer, T-point DFTs in registers, one write back.
template <int NF> constexpr bool pass_regfft()
{
    return (NF >= 32 && NF <= 256 && (NF & (NF - 1)) == 0) || NF == 48 || NF == 80 || NF == 96;
}

// pitch of a staged line: the padded line, or the register FFT's exchange region if larger
template <int NF> constexpr int pass_line_pitch()
{
    return pass_regfft<NF>() && RegFFTShape<NF>::REGION > pad16(NF) + 1 ? RegFFTShape<NF>::REGION : pad16(NF) + 1;
}

// In-order FFT of the staged line `ln` (padded indices) by its T threads.  Every
// thread of the block calls it; threads without a line (act == false) touch no shared
// memory.  Ends with a block barrier.  tw: forward roots of length ntw (a multiple of NF).
template <typename R, int NF, int SIGN>
__device__ __forceinline__ void line_fft(cpx<R> *ln, cpx<R> *lnp, const cpx<R> *tw, int ntw, int t, bool act)
{
    if constexpr (pass_regfft<NF>() && 16 % RegFFTShape<NF>::T != 0) {
        // T = 3, 5, 6 threads per line: a line's threads may straddle two warps, so the
        // exchange is ordered by block barriers; thread t runs the second-stage DFTs of
        // k1 = t, t + T, ... < 16 and holds their results until every thread has read the
        // exchange region, then writes X[k1 + 16 k2]
        using C = cpx<R>;
        using S = RegFFTShape<NF>;
        constexpr int T = S::T;
        constexpr int A = (16 + T - 1) / T;
        const int rs = ntw / NF;
        C v[16];
#pragma unroll
        for (int r = 0; r < 16; ++r) v[r] = act ? ln[pad16(t + T * r)] : mk<R>(R(0), R(0));
        __syncthreads();  // every line is read before the exchanges overwrite it
        dft16<SIGN, C, R>(v);
#pragma unroll
        for (int k1 = 1; k1 < 16; ++k1) v[k1] = twiddle_mul<SIGN>(v[k1], tw, (t * k1) * rs);
        if (act) {
#pragma unroll
            for (int k1 = 0; k1 < 16; ++k1) ln[k1 * S::ROWP + t] = v[k1];
        }
        __syncthreads();
        C res[A][T];
#pragma unroll
        for (int a = 0; a < A; ++a) {
            const int k1 = t + T * a;
#pragma unroll
            for (int q = 0; q < T; ++q) res[a][q] = (act && k1 < 16) ? ln[k1 * S::ROWP + q] : mk<R>(R(0), R(0));
            dft_small<SIGN, T, C, R>(res[a]);
        }
        __syncthreads();  // the exchange regions are read before the results overwrite them
        if (act) {
#pragma unroll
            for (int a = 0; a < A; ++a) {
                const int k1 = t + T * a;
                if (k1 < 16) {
#pragma unroll
                    for (int k2 = 0; k2 < T; ++k2) ln[pad16(k1 + 16 * k2)] = res[a][k2];
                }
            }
        }
        __syncthreads();
    } else if constexpr (pass_regfft<NF>()) {
        using C = cpx<R>;
        using S = RegFFTShape<NF>;
        constexpr int T = S::T;
        const unsigned mask = __activemask();
        const int rs = ntw / NF;
        C v[16];
#pragma unroll
        for (int r = 0; r < 16; ++r) v[r] = act ? ln[pad16(t + T * r)] : mk<R>(R(0), R(0));
        __syncwarp(mask);  // the line is read before the exchange overwrites it
        dft16<SIGN, C, R>(v);
#pragma unroll
        for (int k1 = 1; k1 < 16; ++k1) v[k1] = twiddle_mul<SIGN>(v[k1], tw, (t * k1) * rs);
        if (act) {
#pragma unroll
            for (int k1 = 0; k1 < 16; ++k1) ln[k1 * S::ROWP + t] = v[k1];
        }
        __syncwarp(mask);
        constexpr int A = 16 / T;
#pragma unroll
        for (int a = 0; a < A; ++a) {
            C u[T];
#pragma unroll
            for (int q = 0; q < T; ++q) u[q] = act ? ln[(t + T * a) * S::ROWP + q] : mk<R>(R(0), R(0));
            dft_small<SIGN, T, C, R>(u);
#pragma unroll
            for (int k2 = 0; k2 < T; ++k2) v[a + A * k2] = u[k2];
        }
        __syncwarp(mask);  // the exchange region is read before the results overwrite it
        if (act) {
#pragma unroll
            for (int j = 0; j < 16; ++j) ln[pad16(t + T * j)] = v[j];
        }
        __syncthreads();
    } else {
        fft_line<R, NF, SIGN>(lnp, tw, ntw, act ? t : 0, act);
    }
}

template <typename R> __device__ __forceinline__ R ep_factor(const PassArgs &a, int p, const int *bidx)
{
    R k2 = R(0);
    R hw = R(1);
#pragma unroll 4
    for (int ax = 0; ax < a.ep_naxes; ++ax) {
        const int src = a.ep_src[ax];
        const int i = src == 0 ? p : bidx[src - 1];
        const int n = a.ep_n[ax];
        const int k = a.ep_half[ax] ? i : (i <= n / 2 ? i : i - n);
        const R kk = R(k) * R(a.ep_kscale[ax]);
        k2 += kk * kk;
        if (a.ep_half[ax] && i != 0 && 2 * i != n) hw = R(a.ep_hw);
    }
    R f = R(a.ep_scale);
    if (a.ep_mode & EP_HALFW) f *= hw;
    if (a.ep_mode & EP_POISSON) f = (k2 == R(0)) ? R(0) : f * R(a.ep_sign) / k2;
    if (a.ep_mode & EP_GAUSS) f *= exp(-k2 * R(a.ep_gauss));
    return f;
}

// One CTA's share of a pass: the G lines starting at line0.  Any block size works;
// threads past G * threads_per_line(NF) only join the barriers.  EXT compiles in the
// blocked point indices (slab exchanges) and the four-step twiddle epilogue (long lines);
// callers that never use them (the batch kernels) leave them out, which keeps their
// register count and occupancy.
// The line buffers are in_ptr / out_ptr (a.in / a.out for a plain launch; the batch kernels
// bind theirs per item without copying the argument struct).
template <typename R, int NF, bool CG, bool EXT = true>
__device__ __forceinline__ void pass_body(const PassArgs &a, const void *in_ptr, void *out_ptr, long long line0,
                                          unsigned char *smem_raw)
{
    using C = cpx<R>;
    constexpr int T = threads_per_line(NF);
    constexpr int LP = pass_line_pitch<NF>();
    C *stw_s = reinterpret_cast<C *>(smem_raw);
    const int ntw_s = a.tw_smem ? a.ntw : 0;
    long long *offs = reinterpret_cast<long long *>(stw_s + ntw_s);  // [G][2] in/out offsets
    int *bidx = reinterpret_cast<int *>(offs + 2 * a.G);            // [G][3]
    C *lines = reinterpret_cast<C *>(bidx + 4 * a.G);               // [G][LP]

    const int tid = threadIdx.x;
    const int G = a.G;
    const int gshift = a.gshift;
    const int g = tid / T;
    const int t = tid - g * T;

    const C *twg = reinterpret_cast<const C *>(a.tw);
    for (int i = tid; i < ntw_s; i += blockDim.x) stw_s[i] = twg[i];
    const C *stw = a.tw_smem ? stw_s : twg;
    for (int gg = tid; gg < G; gg += blockDim.x) {
        const long long l = line0 + gg;
        if (l < a.nlines) {
            const long long b0 = l % a.c0;
            const long long r = l / a.c0;
            const long long b1 = r % a.c1;
            const long long b2 = r / a.c1;
            offs[2 * gg] = b0 * a.ib0 + b1 * a.ib1 + b2 * a.ib2;
            offs[2 * gg + 1] = b0 * a.ob0 + b1 * a.ob1 + b2 * a.ob2;
            bidx[4 * gg] = (int)b0;
            bidx[4 * gg + 1] = (int)b1;
            bidx[4 * gg + 2] = (int)b2;
            bidx[4 * gg + 3] = 1;
        } else {
            offs[2 * gg] = 0;
            offs[2 * gg + 1] = 0;
            bidx[4 * gg] = bidx[4 * gg + 1] = bidx[4 * gg + 2] = 0;
            bidx[4 * gg + 3] = 0;
        }
    }
    __syncthreads();

    const int kind = a.kind;
    const long long is = a.is, os = a.os;

    // ------------------------------------------------------------ load (asynchronous copies)
    const void *gdummy = in_ptr;
    if (kind == K_C2C_FWD || kind == K_C2C_INV || kind == K_SANDWICH) {
        const C *in = reinterpret_cast<const C *>(in_ptr);
        const int tot = G * NF;
        // the blocked point index (a slab exchange's unpack) gets a loop of its own, so the
        // plain loop carries none of its index arithmetic
        if (EXT && a.in_blk) {
            const int blk = a.in_blk;
            const long long hi = a.in_hi;
            for (int e = tid; e < tot; e += blockDim.x) {
                int gg, p;
                if (a.in_pts_fast) { gg = e / NF; p = e - gg * NF; }
                else { gg = e & (G - 1); p = e >> gshift; }
                const bool ok = bidx[4 * gg + 3] != 0;
                const int q = p / blk;
                const long long pi = (long long)q * hi + (long long)(p - q * blk) * is;
                stage_load<CG, sizeof(C)>(&lines[gg * LP + pad16(p)],
                                          ok ? (const void *)(in + offs[2 * gg] + pi) : gdummy, ok);
            }
        } else {
#pragma unroll 4
            for (int e = tid; e < tot; e += blockDim.x) {
                int gg, p;
                if (a.in_pts_fast) { gg = e / NF; p = e - gg * NF; }
                else { gg = e & (G - 1); p = e >> gshift; }
                const bool ok = bidx[4 * gg + 3] != 0;
                stage_load<CG, sizeof(C)>(&lines[gg * LP + pad16(p)],
                                          ok ? (const void *)(in + offs[2 * gg] + p * is) : gdummy, ok);
            }
        }
    } else if (kind == K_R2C) {
        const R *in = reinterpret_cast<const R *>(in_ptr);
        const int tot = G * NF;
#pragma unroll 4
        for (int e = tid; e < tot; e += blockDim.x) {
            int gg, p;
            if (a.in_pts_fast) { gg = e / NF; p = e - gg * NF; }
            else { gg = e & (G - 1); p = e >> gshift; }
            const bool ok = bidx[4 * gg + 3] != 0;
            C *dst = &lines[gg * LP + pad16(p)];
            const R *src = in + offs[2 * gg];
            if (a.half) {
                if (a.pair_io) {
                    stage_load<CG, sizeof(C)>(dst, ok ? (const void *)(src + 2 * p) : gdummy, ok);
                } else {
                    stage_load<CG, sizeof(R)>(&dst->x, ok ? (const void *)(src + (2 * p) * is) : gdummy, ok);
                    stage_load<CG, sizeof(R)>(&dst->y, ok ? (const void *)(src + (2 * p + 1) * is) : gdummy, ok);
                }
            } else {
                stage_load<CG, sizeof(R)>(&dst->x, ok ? (const void *)(src + p * is) : gdummy, ok);
                dst->y = R(0);
            }
        }
    } else { // K_C2R
        const C *in = reinterpret_cast<const C *>(in_ptr);
        const int nin = a.half ? NF + 1 : NF / 2 + 1;
        const int tot = G * nin;
#pragma unroll 4
        for (int e = tid; e < tot; e += blockDim.x) {
            int gg, p;
            if (a.in_pts_fast) { gg = e / nin; p = e - gg * nin; }
            else { gg = e & (G - 1); p = e >> gshift; }
            const bool ok = bidx[4 * gg + 3] != 0;
            stage_load<CG, sizeof(C)>(&lines[gg * LP + pad16(p)], ok ? (const void *)(in + offs[2 * gg] + p * is) : gdummy,
                                ok);
        }
    }
    cp_async_wait_all();
    __syncthreads();

    C *ln = lines + g * LP;
    const bool active_thread = g < G;

    // ------------------------------------------------------------ C2R pre-processing
    if (kind == K_C2R) {
        if (active_thread) {
            if (a.half) {
                // Z[k] = E + iO, Z[NF-k] = conj(E - iO) with E = X[k] + conj(X[NF-k]),
                // O = (X[k] - conj(X[NF-k])) * conj(w_{2NF}^k); DC and Nyquist taken real.
                for (int k = t; k <= NF / 2; k += T) {
                    C xk = ln[pad16(k)];
                    C xm = cconj(ln[pad16(NF - k)]);
                    if (k == 0) { xk.y = R(0); xm.y = R(0); }
                    const C e = cadd(xk, xm);
                    const C o = cmulc(csub(xk, xm), stw[k]);
                    const C io = mul_si<1>(o);
                    ln[pad16(k)] = cadd(e, io);
                    if (k != 0) ln[pad16(NF - k)] = cconj(csub(e, io));
                }
            } else {
                // full-length line: Hermitian extension of the half line (the imaginary
                // parts of the DC and, for even lengths, Nyquist bins are ignored)
                for (int k = t; k < NF; k += T) {
                    if (k == 0 || 2 * k == NF) { C v = ln[pad16(k)]; v.y = R(0); ln[pad16(k)] = v; }
                    else if (k > NF / 2) ln[pad16(k)] = cconj(ln[pad16(NF - k)]);
                }
            }
        }
        __syncthreads();
    }

    // ------------------------------------------------------------ FFT core
    C *lnp = active_thread ? ln : lines;  // threads without a line still join the barriers
    if (kind == K_C2C_INV || kind == K_C2R) {
        line_fft<R, NF, +1>(ln, lnp, stw, a.ntw, t, active_thread);
    } else {
        line_fft<R, NF, -1>(ln, lnp, stw, a.ntw, t, active_thread);
    }

    if (kind == K_SANDWICH) {
        if (active_thread && bidx[4 * g + 3]) {
            for (int p = t; p < NF; p += T) ln[pad16(p)] = cscale(ln[pad16(p)], ep_factor<R>(a, p, bidx + 4 * g));
        }
        __syncthreads();
        line_fft<R, NF, +1>(ln, lnp, stw, a.ntw, t, active_thread);
    }

    // ------------------------------------------------------------ R2C post-processing
    if (kind == K_R2C && a.half) {
        if (active_thread) {
            // X[k] = E + w^k O, X[NF-k] = conj(E - w^k O), E = (Z[k]+conj Z[NF-k])/2, O = -i(Z[k]-conj Z[NF-k])/2
            for (int k = t; k <= NF / 2; k += T) {
                const C zk = ln[pad16(k)];
                const C zm = cconj(ln[pad16(k == 0 ? 0 : NF - k)]);
                const C e = cscale(cadd(zk, zm), R(0.5));
                const C o = cscale(mul_si<-1>(csub(zk, zm)), R(0.5));
                const C w = cmul(o, stw[k]);
                ln[pad16(k)] = cadd(e, w);
                ln[pad16(NF - k)] = cconj(csub(e, w));
            }
        }
        __syncthreads();
    }

    // ------------------------------------------------------------ store
    const bool ep_store = (a.ep_mode != 0) && kind != K_SANDWICH;
    if (kind == K_C2R) {
        R *out = reinterpret_cast<R *>(out_ptr);
        const R sc = R(a.ep_scale);
        if (a.half) {
            const int tot = G * NF;
            for (int e = tid; e < tot; e += blockDim.x) {
                int gg, p;
                if (a.out_pts_fast) { gg = e / NF; p = e - gg * NF; }
                else { gg = e & (G - 1); p = e >> gshift; }
                if (!bidx[4 * gg + 3]) continue;
                C v = lines[gg * LP + pad16(p)];
                if (ep_store) v = cscale(v, sc);
                R *dst = out + offs[2 * gg + 1];
                if (a.pair_io) *reinterpret_cast<C *>(dst + 2 * p) = v;
                else { dst[(2 * p) * os] = v.x; dst[(2 * p + 1) * os] = v.y; }
            }
        } else {
            const int tot = G * NF;
            for (int e = tid; e < tot; e += blockDim.x) {
                int gg, p;
                if (a.out_pts_fast) { gg = e / NF; p = e - gg * NF; }
                else { gg = e & (G - 1); p = e >> gshift; }
                if (!bidx[4 * gg + 3]) continue;
                R v = lines[gg * LP + pad16(p)].x;
                if (ep_store) v *= sc;
                out[offs[2 * gg + 1] + p * os] = v;
            }
        }
    } else {
        C *out = reinterpret_cast<C *>(out_ptr);
        const int nout = (kind == K_R2C) ? (a.half ? NF + 1 : NF / 2 + 1) : NF;
        const int tot = G * nout;
        if (EXT && ((a.ep_mode & EP_TWIDDLE) || a.out_blk)) {
            // the four-step twiddle (long lines) and the blocked store (a slab exchange's
            // pack, optionally into peer buffers) in a loop of their own
            const bool twid = (a.ep_mode & EP_TWIDDLE) != 0;
            const bool fct = ep_store && (a.ep_mode & ~EP_TWIDDLE) != 0;
            const C *eptw = reinterpret_cast<const C *>(a.ep_tw);
            for (int e = tid; e < tot; e += blockDim.x) {
                int gg, p;
                if (a.out_pts_fast) { gg = e / nout; p = e - gg * nout; }
                else { gg = e & (G - 1); p = e >> gshift; }
                if (!bidx[4 * gg + 3]) continue;
                C v = lines[gg * LP + pad16(p)];
                if (twid) {
                    // p < L1 and j < L2, so p * j < L: no reduction needed
                    const C w = eptw[(long long)p * bidx[4 * gg + a.ep_src[0] - 1]];
                    v = kind == K_C2C_INV ? cmulc(v, w) : cmul(v, w);
                }
                if (fct) v = cscale(v, ep_factor<R>(a, p, bidx + 4 * gg));
                if (a.out_blk) {
                    const int q = p / a.out_blk;
                    // select the peer pointer with compile-time indices: a dynamic index into
                    // the argument struct would move the whole struct to local memory in the
                    // kernels that copy it
                    void *peer = nullptr;
#pragma unroll
                    for (int i = 0; i < 8; ++i)
                        if (i == q) peer = a.out_peer[i];
                    C *base = peer ? reinterpret_cast<C *>(peer) : out + (long long)q * a.out_hi;
                    base[offs[2 * gg + 1] + (long long)(p - q * a.out_blk) * os] = v;
                } else {
                    out[offs[2 * gg + 1] + p * os] = v;
                }
            }
        } else {
#pragma unroll 4
            for (int e = tid; e < tot; e += blockDim.x) {
                int gg, p;
                if (a.out_pts_fast) { gg = e / nout; p = e - gg * nout; }
                else { gg = e & (G - 1); p = e >> gshift; }
                if (!bidx[4 * gg + 3]) continue;
                C v = lines[gg * LP + pad16(p)];
                if (ep_store) v = cscale(v, ep_factor<R>(a, p, bidx + 4 * gg));
                out[offs[2 * gg + 1] + p * os] = v;
            }
        }
    }
}

template <typename R, int NF>
__global__ void __launch_bounds__(512) fftb_pass_kernel(PassArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    pass_body<R, NF, false>(a, a.in, a.out, (long long)blockIdx.x * a.G, smem_raw);
}

template <typename R, int NF> inline PassKernelInfo pass_kernel_info()
{
    PassKernelInfo k;
    k.nf = NF;
    k.threads_per_line = threads_per_line(NF);
    k.line_pitch = pass_line_pitch<NF>();
    k.fn = (const void *)&fftb_pass_kernel<R, NF>;
    return k;
}

} // namespace fftb
