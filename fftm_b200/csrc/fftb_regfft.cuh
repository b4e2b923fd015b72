// fftb_regfft.cuh -- register-resident two-stage FFTs for the specialised kernels.
//
// An N-point FFT (N = 16*T, T in {1, 2, 4, 8, 16}) is run by T threads, each
// holding 16 complex values.  Thread t starts with v[r] = x[t + T*r] and ends
// with v[j] = X[t + T*j]:
//   stage 1: radix-16 DFT over r in registers        -> Y_t[k1]
//   twiddle: Y_t[k1] *= w_N^(t*k1)
//   exchange through this FFT's shared-memory region  (one store, one load)
//   stage 2: 16/T DFTs of length T over t in registers -> X[k1 + 16*k2]
// (the four-step decomposition X[k1 + 16 k2] = sum_t w_T^(t k2) w_N^(t k1)
//  sum_r x[t + T r] w_16^(r k1)).
#pragma once

#include "fftb_device.cuh"

namespace fftb {

// Size of one FFT's exchange region (complex entries).  Regions of the FFTs that
// share a half-warp are offset by T (mod 16) so stores and loads are conflict-free.
template <int N> struct RegFFTShape {
    static constexpr int T = N >= 16 ? N / 16 : 1;
    static constexpr int ROWP = T + 1;                         // entries per k1 row
    static constexpr int REGION = (T == 1) ? 16 : 16 * ROWP + (T == 16 ? 0 : T);
};

// In-order DFT of 6 values: X[k] = E[k] + w6^k O[k], X[k + 3] = E[k] - w6^k O[k] with E, O the
// 3-point DFTs of the even and odd samples (Cooley-Tukey, 6 = 2 x 3).
template <int SIGN, typename C, typename R> __device__ __forceinline__ void dft6(C *u)
{
    C e[3] = {u[0], u[2], u[4]}, o[3] = {u[1], u[3], u[5]};
    dft3<SIGN, C, R>(e);
    dft3<SIGN, C, R>(o);
    const R h = R(0.5), s3 = kconst<R>::s3;
    // w6^1 = 1/2 + SIGN i s3, w6^2 = -1/2 + SIGN i s3
    const C o1 = mk<R>(h * o[1].x - SIGN * s3 * o[1].y, h * o[1].y + SIGN * s3 * o[1].x);
    const C o2 = mk<R>(-h * o[2].x - SIGN * s3 * o[2].y, -h * o[2].y + SIGN * s3 * o[2].x);
    u[0] = cadd(e[0], o[0]);
    u[3] = csub(e[0], o[0]);
    u[1] = cadd(e[1], o1);
    u[4] = csub(e[1], o1);
    u[2] = cadd(e[2], o2);
    u[5] = csub(e[2], o2);
}

template <int SIGN, int L, typename C, typename R> __device__ __forceinline__ void dft_small(C *u)
{
    if constexpr (L == 1) {
    } else if constexpr (L == 2) {
        dft2<SIGN>(u[0], u[1]);
    } else if constexpr (L == 3) {
        dft3<SIGN, C, R>(u);
    } else if constexpr (L == 5) {
        dft5<SIGN, C, R>(u);
    } else if constexpr (L == 6) {
        dft6<SIGN, C, R>(u);
    } else if constexpr (L == 4) {
        dft4<SIGN>(u[0], u[1], u[2], u[3]);
    } else if constexpr (L == 8) {
        dft8<SIGN, C, R>(u);
    } else {
        static_assert(L == 16, "length");
        dft16<SIGN, C, R>(u);
    }
}

// Multiplies v by w^e (SIGN<0) or conj(w)^e (SIGN>0) with w^e = tw[e*stride].
template <int SIGN, typename C> __device__ __forceinline__ C twiddle_mul(C v, const C *tw, int idx)
{
    const C w = tw[idx];
    return SIGN < 0 ? cmul(v, w) : cmulc(v, w);
}

// Stage twiddle table of an N-point register FFT: st[k1 * T + t] = w_N^(t * k1), so the
// 16 twiddle loads of the T threads of one FFT hit consecutive shared-memory words.
template <typename R, int N>
__device__ __forceinline__ void build_stage_table(cpx<R> *st, const cpx<R> *roots, int nroots, int tid, int nthreads)
{
    constexpr int T = RegFFTShape<N>::T;
    for (int i = tid; i < 16 * T; i += nthreads) {
        const int k1 = i / T, t = i - (i / T) * T;
        st[i] = roots[((t * k1) % N) * (nroots / N)];
    }
}

// The T threads of this FFT must be consecutive lanes of one warp (exchange with
// __syncwarp).  st: stage table of build_stage_table<R, N>; reg: exchange region.
template <typename R, int N, int SIGN>
__device__ __forceinline__ void regfft_warp(cpx<R> (&v)[16], cpx<R> *reg, const cpx<R> *st, int t)
{
    using C = cpx<R>;
    using S = RegFFTShape<N>;
    constexpr int T = S::T;
    if constexpr (N <= 16) {
        dft_small<SIGN, N, C, R>(v);
    } else {
        dft16<SIGN, C, R>(v);
#pragma unroll
        for (int k1 = 1; k1 < 16; ++k1) v[k1] = twiddle_mul<SIGN>(v[k1], st, k1 * T + t);
        __syncwarp();
#pragma unroll
        for (int k1 = 0; k1 < 16; ++k1) reg[k1 * S::ROWP + t] = v[k1];
        __syncwarp();
        constexpr int A = 16 / T;
#pragma unroll
        for (int a = 0; a < A; ++a) {
            C u[T];
#pragma unroll
            for (int q = 0; q < T; ++q) u[q] = reg[(t + T * a) * S::ROWP + q];
            dft_small<SIGN, T, C, R>(u);
#pragma unroll
            for (int k2 = 0; k2 < T; ++k2) v[a + A * k2] = u[k2];
        }
    }
}

// Stage twiddles of one thread in registers: tw[k1] = w_N^(t k1), k1 = 1..15 (tw[0] = 1), read
// from the forward root table `roots` of length nroots (a multiple of N).  A thread whose t
// is fixed for a whole kernel loads them once instead of reading a table every FFT.
template <typename R, int N>
__device__ __forceinline__ void load_stage_twiddles(cpx<R> (&tw)[16], const cpx<R> *roots, int nroots, int t)
{
    tw[0] = mk<R>(R(1), R(0));
#pragma unroll
    for (int k1 = 1; k1 < 16; ++k1) tw[k1] = roots[((t * k1) % N) * (nroots / N)];
}

// regfft_warp with the stage twiddles in registers (load_stage_twiddles<R, N> of this t).
template <typename R, int N, int SIGN>
__device__ __forceinline__ void regfft_warp_rt(cpx<R> (&v)[16], cpx<R> *reg, const cpx<R> (&tw)[16], int t)
{
    using C = cpx<R>;
    using S = RegFFTShape<N>;
    constexpr int T = S::T;
    if constexpr (N <= 16) {
        dft_small<SIGN, N, C, R>(v);
    } else {
        dft16<SIGN, C, R>(v);
#pragma unroll
        for (int k1 = 1; k1 < 16; ++k1) v[k1] = SIGN < 0 ? cmul(v[k1], tw[k1]) : cmulc(v[k1], tw[k1]);
        __syncwarp();
#pragma unroll
        for (int k1 = 0; k1 < 16; ++k1) reg[k1 * S::ROWP + t] = v[k1];
        __syncwarp();
        constexpr int A = 16 / T;
#pragma unroll
        for (int a = 0; a < A; ++a) {
            C u[T];
#pragma unroll
            for (int q = 0; q < T; ++q) u[q] = reg[(t + T * a) * S::ROWP + q];
            dft_small<SIGN, T, C, R>(u);
#pragma unroll
            for (int k2 = 0; k2 < T; ++k2) v[a + A * k2] = u[k2];
        }
    }
}

} // namespace fftb
