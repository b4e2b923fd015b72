// fftb_device.cuh -- device building blocks of the fftb sm_100a FFT engine.
//
// Complex arithmetic, in-register DFT butterflies (radix 2,3,4,5,7,8,16 and a
// generic odd radix through the twiddle table), the compile-time radix plan and
// the shared-memory Stockham core that every pass kernel runs.
//
// Conventions follow the reference's backend contract: forward = exp(-i*theta),
// inverse = exp(+i*theta), both unnormalised (reference
// source/external_wrap/cufft_wrap.h:356,386).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace fftb {

template <typename R> struct cpx_t;
template <> struct cpx_t<float> { using type = float2; };
template <> struct cpx_t<double> { using type = double2; };
template <typename R> using cpx = typename cpx_t<R>::type;

template <typename R> __host__ __device__ __forceinline__ cpx<R> mk(R x, R y) { cpx<R> c; c.x = x; c.y = y; return c; }
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { a.x += b.x; a.y += b.y; return a; }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { a.x -= b.x; a.y -= b.y; return a; }
template <typename C> __device__ __forceinline__ C cmul(C a, C b)
{
    C r;
    r.x = a.x * b.x - a.y * b.y;
    r.y = a.x * b.y + a.y * b.x;
    return r;
}
// a * conj(b)
template <typename C> __device__ __forceinline__ C cmulc(C a, C b)
{
    C r;
    r.x = a.x * b.x + a.y * b.y;
    r.y = a.y * b.x - a.x * b.y;
    return r;
}
template <typename C> __device__ __forceinline__ C cconj(C a) { a.y = -a.y; return a; }
template <typename C, typename R> __device__ __forceinline__ C cscale(C a, R s) { a.x *= s; a.y *= s; return a; }

// float2 forms on sm_100's paired FP32 instructions (FADD2 / FMUL2 / FFMA2: one
// instruction for both components, each rounded as the scalar operation would be).
// a - b is formed as fma(b, -1, a), which is exact in its product and so equals the
// rounded difference.
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return __fmul2_rn(a, make_float2(s, s)); }
// multiply by SIGN*i  (SIGN = -1: -i, SIGN = +1: +i)
template <int SIGN, typename C> __device__ __forceinline__ C mul_si(C a)
{
    C r;
    if (SIGN < 0) { r.x = a.y; r.y = -a.x; }
    else { r.x = -a.y; r.y = a.x; }
    return r;
}

// Asynchronous global->shared copy of BYTES (4, 8 or 16) bytes; zero-fills the
// destination when !valid (src-size 0 reads nothing from gsrc).
template <int BYTES> __device__ __forceinline__ void cp_async(void *sdst, const void *gsrc, bool valid)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
    const int src_size = valid ? BYTES : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(s), "l"(gsrc), "n"(BYTES), "r"(src_size)
                 : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// waits until at most N of this thread's committed cp.async groups are pending
template <int N> __device__ __forceinline__ void cp_async_wait_group()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// L2 eviction policies (createpolicy) and loads / stores that carry them: evict_first for
// data read or written once (the real fields), evict_last for data the next kernel of the
// same transform reads again (the spectrum), so the streaming fields do not push it out.
__device__ __forceinline__ unsigned long long l2_evict_first()
{
    unsigned long long p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;\n" : "=l"(p));
    return p;
}
__device__ __forceinline__ unsigned long long l2_evict_last()
{
    unsigned long long p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;\n" : "=l"(p));
    return p;
}
__device__ __forceinline__ float ld_hint(const float *g, unsigned long long pol)
{
    float v;
    asm volatile("ld.global.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;\n" : "=f"(v) : "l"(g), "l"(pol));
    return v;
}
__device__ __forceinline__ float2 ld_hint(const float2 *g, unsigned long long pol)
{
    float2 v;
    asm volatile("ld.global.L1::no_allocate.L2::cache_hint.v2.f32 {%0, %1}, [%2], %3;\n"
                 : "=f"(v.x), "=f"(v.y) : "l"(g), "l"(pol));
    return v;
}
__device__ __forceinline__ void st_hint(float *g, float v, unsigned long long pol)
{
    asm volatile("st.global.L1::no_allocate.L2::cache_hint.f32 [%0], %1, %2;\n" ::"l"(g), "f"(v), "l"(pol) : "memory");
}
__device__ __forceinline__ void st_hint(float2 *g, float2 v, unsigned long long pol)
{
    asm volatile("st.global.L1::no_allocate.L2::cache_hint.v2.f32 [%0], {%1, %2}, %3;\n" ::"l"(g), "f"(v.x), "f"(v.y),
                 "l"(pol)
                 : "memory");
}
// Asynchronous prefetch of BYTES (a multiple of 16, 16-byte aligned) of global memory into L2.
__device__ __forceinline__ void prefetch_l2(const void *g, unsigned bytes)
{
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(g), "r"(bytes) : "memory");
}

// ---------------------------------------------------------------- bulk copies (TMA)
// mbarrier-tracked tensor copies global -> shared (no multicast: every copy reads this
// GPU's own memory into this CTA's shared memory).
__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
// makes initialised barriers visible to the asynchronous (copy) proxy
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long *bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity)
{
    unsigned ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(ok)
                 : "r"(smem_u32(bar)), "r"(parity)
                 : "memory");
    return ok != 0;
}
// Bounded wait for the phase with the given parity: false after `limit` polls.
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity, int limit)
{
    for (int i = 0; i < limit; ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        if (i >= 16) __nanosleep(128);
    }
    return false;
}
// Orders this thread's generic-proxy shared-memory accesses before later bulk copies.
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
// 3D tiled tensor copy into this CTA's shared memory, completing on `bar` (byte count).
// The innermost coordinate x times the element size must be a multiple of 16 bytes.
__device__ __forceinline__ void tma_load_3d(void *dst, const void *tmap, unsigned long long *bar, int x, int y, int z)
{
    asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                 " [%0], [%1, {%3, %4, %5}], [%2];\n" ::"r"(smem_u32(dst)),
                 "l"(tmap), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
                 : "memory");
}

// Approximate reciprocal (one MUFU operation, relative error at most 2^-23 per the PTX
// specification of rcp.approx.f32): for factors whose rounding error is far below the
// transforms' own.
__device__ __forceinline__ float rcp_approx(float x)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;\n" : "=f"(r) : "f"(x));
    return r;
}

// Shared-memory index padding: one spare slot per 16 entries keeps the
// stride-R Stockham scatters free of bank conflicts.
__host__ __device__ constexpr int pad16(int a) { return a + (a >> 4); }

// ---------------------------------------------------------------- radix plan
// Powers of two are covered by radix 16 passes and one remainder pass (2, 4
// or 8); odd factors 3, 5, 7 and any other odd prime follow.  T (threads per
// line) is NF / (largest radix).
__host__ __device__ constexpr int fftb_ilog2(int n) { return n <= 1 ? 0 : 1 + fftb_ilog2(n >> 1); }
__host__ __device__ constexpr int pow2_part(int n) { return (n & 1) ? 1 : 2 * pow2_part(n >> 1); }
__host__ __device__ constexpr int smallest_odd_factor(int n, int p = 3)
{
    return n <= 1 ? 1 : (n % p == 0 ? p : (p * p > n ? n : smallest_odd_factor(n, p + 2)));
}
// number of passes
__host__ __device__ constexpr int odd_passes(int m) { return m <= 1 ? 0 : 1 + odd_passes(m / smallest_odd_factor(m)); }
__host__ __device__ constexpr int num_passes(int n)
{
    return (fftb_ilog2(pow2_part(n)) + 3) / 4 + odd_passes(n / pow2_part(n));
}
__host__ __device__ constexpr int odd_radix_at(int m, int i)
{
    return i == 0 ? smallest_odd_factor(m) : odd_radix_at(m / smallest_odd_factor(m), i - 1);
}
__host__ __device__ constexpr int radix_at(int n, int pass)
{
    // pow2 passes first: full radix-16 passes, then the remainder pass
    return pass < fftb_ilog2(pow2_part(n)) / 4
               ? 16
               : (pass < (fftb_ilog2(pow2_part(n)) + 3) / 4
                      ? (1 << (fftb_ilog2(pow2_part(n)) % 4))
                      : odd_radix_at(n / pow2_part(n), pass - (fftb_ilog2(pow2_part(n)) + 3) / 4));
}
__host__ __device__ constexpr int max_radix(int n, int p = 0)
{
    return p >= num_passes(n) ? 1 : (radix_at(n, p) > max_radix(n, p + 1) ? radix_at(n, p) : max_radix(n, p + 1));
}
__host__ __device__ constexpr int stride_before(int n, int pass) { return pass == 0 ? 1 : stride_before(n, pass - 1) * radix_at(n, pass - 1); }
__host__ __device__ constexpr int threads_per_line(int n) { return n <= 1 ? 1 : n / max_radix(n); }

// ---------------------------------------------------------------- butterflies
// In-order DFT of R values in registers: v[k] <- sum_r v[r] * exp(SIGN*2*pi*i*r*k/R).
template <int SIGN, typename C> __device__ __forceinline__ void dft2(C &a, C &b)
{
    C t = a;
    a = cadd(t, b);
    b = csub(t, b);
}

template <int SIGN, typename C> __device__ __forceinline__ void dft4(C &v0, C &v1, C &v2, C &v3)
{
    C t0 = cadd(v0, v2), t1 = csub(v0, v2), t2 = cadd(v1, v3), t3 = mul_si<SIGN>(csub(v1, v3));
    v0 = cadd(t0, t2);
    v2 = csub(t0, t2);
    v1 = cadd(t1, t3);
    v3 = csub(t1, t3);
}

template <typename R> struct kconst {
    static constexpr R r2 = R(0.70710678118654752440084436210485);   // sqrt(2)/2
    static constexpr R c8 = R(0.92387953251128675612818318939679);   // cos(pi/8)
    static constexpr R s8 = R(0.38268343236508977172845998403040);   // sin(pi/8)
    static constexpr R s3 = R(0.86602540378443864676372317075294);   // sin(2pi/3)
    static constexpr R c51 = R(0.30901699437494742410229341718282);  // cos(2pi/5)
    static constexpr R c52 = R(-0.80901699437494742410229341718282); // cos(4pi/5)
    static constexpr R s51 = R(0.95105651629515357211643933337938);  // sin(2pi/5)
    static constexpr R s52 = R(0.58778525229247312916870595463907);  // sin(4pi/5)
    static constexpr R c71 = R(0.62348980185873353052500488400424);  // cos(2pi/7)
    static constexpr R c72 = R(-0.22252093395631440428890256449680); // cos(4pi/7)
    static constexpr R c73 = R(-0.90096886790241912623610231950745); // cos(6pi/7)
    static constexpr R s71 = R(0.78183148246802980870844452667406);  // sin(2pi/7)
    static constexpr R s72 = R(0.97492791218182360701813168299393);  // sin(4pi/7)
    static constexpr R s73 = R(0.43388373911755812047576833284836);  // sin(6pi/7)
};

// multiply by exp(SIGN*i*pi/4), exp(SIGN*i*3pi/4) (the radix-8 twiddles)
template <int SIGN, typename C, typename R> __device__ __forceinline__ C mul_w8_1(C a)
{
    const R h = kconst<R>::r2;
    C r;
    // (x + i y)(h + SIGN i h)
    r.x = h * (a.x - SIGN * a.y);
    r.y = h * (a.y + SIGN * a.x);
    return r;
}
template <int SIGN, typename C, typename R> __device__ __forceinline__ C mul_w8_3(C a)
{
    const R h = kconst<R>::r2;
    C r;
    // (x + i y)(-h + SIGN i h)
    r.x = -h * (a.x + SIGN * a.y);
    r.y = h * (SIGN * a.x - a.y);
    return r;
}

template <int SIGN, typename C, typename R> __device__ __forceinline__ void dft8(C *v)
{
    C a0 = cadd(v[0], v[4]), b0 = csub(v[0], v[4]);
    C a1 = cadd(v[1], v[5]), b1 = mul_w8_1<SIGN, C, R>(csub(v[1], v[5]));
    C a2 = cadd(v[2], v[6]), b2 = mul_si<SIGN>(csub(v[2], v[6]));
    C a3 = cadd(v[3], v[7]), b3 = mul_w8_3<SIGN, C, R>(csub(v[3], v[7]));
    dft4<SIGN>(a0, a1, a2, a3);
    dft4<SIGN>(b0, b1, b2, b3);
    v[0] = a0; v[2] = a1; v[4] = a2; v[6] = a3;
    v[1] = b0; v[3] = b1; v[5] = b2; v[7] = b3;
}

// exp(SIGN*2*pi*i*e/16) for e in 1..9 applied to a
template <int SIGN, int E, typename C, typename R> __device__ __forceinline__ C mul_w16(C a)
{
    constexpr R c1 = kconst<R>::c8, s1 = kconst<R>::s8, h = kconst<R>::r2;
    // cos and sin of 2*pi*E/16
    constexpr R cs = (E == 0) ? R(1) : (E == 1) ? c1 : (E == 2) ? h : (E == 3) ? s1 : (E == 4) ? R(0)
                   : (E == 5) ? -s1 : (E == 6) ? -h : (E == 7) ? -c1 : (E == 8) ? R(-1) : -c1;
    constexpr R sn = (E == 0) ? R(0) : (E == 1) ? s1 : (E == 2) ? h : (E == 3) ? c1 : (E == 4) ? R(1)
                   : (E == 5) ? c1 : (E == 6) ? h : (E == 7) ? s1 : (E == 8) ? R(0) : -s1;
    C r;
    r.x = a.x * cs - SIGN * a.y * sn;
    r.y = a.y * cs + SIGN * a.x * sn;
    return r;
}

template <int SIGN, typename C, typename R> __device__ __forceinline__ void dft16(C *v)
{
    // DIF 4x4: u_{r0}[k0] = sum_{r1} v[r0+4r1] w4^{r1 k0}; twiddle w16^{r0 k0}; then DFT4 over r0.
    dft4<SIGN>(v[0], v[4], v[8], v[12]);
    dft4<SIGN>(v[1], v[5], v[9], v[13]);
    dft4<SIGN>(v[2], v[6], v[10], v[14]);
    dft4<SIGN>(v[3], v[7], v[11], v[15]);
    v[5] = mul_w16<SIGN, 1, C, R>(v[5]);
    v[9] = mul_w16<SIGN, 2, C, R>(v[9]);
    v[13] = mul_w16<SIGN, 3, C, R>(v[13]);
    v[6] = mul_w16<SIGN, 2, C, R>(v[6]);
    v[10] = mul_si<SIGN>(v[10]);
    v[14] = mul_w16<SIGN, 6, C, R>(v[14]);
    v[7] = mul_w16<SIGN, 3, C, R>(v[7]);
    v[11] = mul_w16<SIGN, 6, C, R>(v[11]);
    v[15] = mul_w16<SIGN, 9, C, R>(v[15]);
    dft4<SIGN>(v[0], v[1], v[2], v[3]);
    dft4<SIGN>(v[4], v[5], v[6], v[7]);
    dft4<SIGN>(v[8], v[9], v[10], v[11]);
    dft4<SIGN>(v[12], v[13], v[14], v[15]);
    // after the second stage, y[k0 + 4 k1] sits at v[4*k0 + k1]: transpose 4x4
    C t;
    t = v[1]; v[1] = v[4]; v[4] = t;
    t = v[2]; v[2] = v[8]; v[8] = t;
    t = v[3]; v[3] = v[12]; v[12] = t;
    t = v[6]; v[6] = v[9]; v[9] = t;
    t = v[7]; v[7] = v[13]; v[13] = t;
    t = v[11]; v[11] = v[14]; v[14] = t;
}

template <int SIGN, typename C, typename R> __device__ __forceinline__ void dft3(C *v)
{
    const R s3 = kconst<R>::s3;
    C t = cadd(v[1], v[2]);
    C d = csub(v[1], v[2]);
    C m;
    m.x = v[0].x - R(0.5) * t.x;
    m.y = v[0].y - R(0.5) * t.y;
    v[0] = cadd(v[0], t);
    C rot = mul_si<SIGN>(cscale(d, s3));
    v[1] = cadd(m, rot);
    v[2] = csub(m, rot);
}

template <int SIGN, typename C, typename R> __device__ __forceinline__ void dft5(C *v)
{
    const R c1 = kconst<R>::c51, c2 = kconst<R>::c52, s1 = kconst<R>::s51, s2 = kconst<R>::s52;
    C a1 = cadd(v[1], v[4]), b1 = csub(v[1], v[4]);
    C a2 = cadd(v[2], v[3]), b2 = csub(v[2], v[3]);
    C y0 = cadd(v[0], cadd(a1, a2));
    C m1, m2, n1, n2;
    m1.x = v[0].x + c1 * a1.x + c2 * a2.x; m1.y = v[0].y + c1 * a1.y + c2 * a2.y;
    m2.x = v[0].x + c2 * a1.x + c1 * a2.x; m2.y = v[0].y + c2 * a1.y + c1 * a2.y;
    n1.x = s1 * b1.x + s2 * b2.x; n1.y = s1 * b1.y + s2 * b2.y;
    n2.x = s2 * b1.x - s1 * b2.x; n2.y = s2 * b1.y - s1 * b2.y;
    n1 = mul_si<SIGN>(n1);
    n2 = mul_si<SIGN>(n2);
    v[0] = y0;
    v[1] = cadd(m1, n1);
    v[4] = csub(m1, n1);
    v[2] = cadd(m2, n2);
    v[3] = csub(m2, n2);
}

template <int SIGN, typename C, typename R> __device__ __forceinline__ void dft7(C *v)
{
    const R c1 = kconst<R>::c71, c2 = kconst<R>::c72, c3 = kconst<R>::c73;
    const R s1 = kconst<R>::s71, s2 = kconst<R>::s72, s3 = kconst<R>::s73;
    C a1 = cadd(v[1], v[6]), b1 = csub(v[1], v[6]);
    C a2 = cadd(v[2], v[5]), b2 = csub(v[2], v[5]);
    C a3 = cadd(v[3], v[4]), b3 = csub(v[3], v[4]);
    C y0 = cadd(v[0], cadd(a1, cadd(a2, a3)));
    C m1, m2, m3, n1, n2, n3;
    m1.x = v[0].x + c1 * a1.x + c2 * a2.x + c3 * a3.x; m1.y = v[0].y + c1 * a1.y + c2 * a2.y + c3 * a3.y;
    m2.x = v[0].x + c2 * a1.x + c3 * a2.x + c1 * a3.x; m2.y = v[0].y + c2 * a1.y + c3 * a2.y + c1 * a3.y;
    m3.x = v[0].x + c3 * a1.x + c1 * a2.x + c2 * a3.x; m3.y = v[0].y + c3 * a1.y + c1 * a2.y + c2 * a3.y;
    // sin(2pi*j*k/7) for (k,j): k=1: s1,s2,s3; k=2: s2,-s3,-s1; k=3: s3,-s1,s2
    n1.x = s1 * b1.x + s2 * b2.x + s3 * b3.x; n1.y = s1 * b1.y + s2 * b2.y + s3 * b3.y;
    n2.x = s2 * b1.x - s3 * b2.x - s1 * b3.x; n2.y = s2 * b1.y - s3 * b2.y - s1 * b3.y;
    n3.x = s3 * b1.x - s1 * b2.x + s2 * b3.x; n3.y = s3 * b1.y - s1 * b2.y + s2 * b3.y;
    n1 = mul_si<SIGN>(n1);
    n2 = mul_si<SIGN>(n2);
    n3 = mul_si<SIGN>(n3);
    v[0] = y0;
    v[1] = cadd(m1, n1); v[6] = csub(m1, n1);
    v[2] = cadd(m2, n2); v[5] = csub(m2, n2);
    v[3] = cadd(m3, n3); v[4] = csub(m3, n3);
}

// Generic odd radix through the forward root table tw (tw[m] = exp(-2 pi i m / NT)).
template <int SIGN, int RAD, typename C> __device__ __forceinline__ void dft_generic(C *v, const C *tw, int NT)
{
    C o[RAD];
    const int st = NT / RAD;
#pragma unroll
    for (int k = 0; k < RAD; ++k) {
        C acc = v[0];
#pragma unroll
        for (int r = 1; r < RAD; ++r) {
            C w = tw[((r * k) % RAD) * st];
            acc = cadd(acc, SIGN < 0 ? cmul(v[r], w) : cmulc(v[r], w));
        }
        o[k] = acc;
    }
#pragma unroll
    for (int k = 0; k < RAD; ++k) v[k] = o[k];
}

template <int SIGN, int RAD, typename C, typename R> __device__ __forceinline__ void dft_radix(C *v, const C *tw, int NT)
{
    if constexpr (RAD == 1) {
    } else if constexpr (RAD == 2) {
        dft2<SIGN>(v[0], v[1]);
    } else if constexpr (RAD == 3) {
        dft3<SIGN, C, R>(v);
    } else if constexpr (RAD == 4) {
        dft4<SIGN>(v[0], v[1], v[2], v[3]);
    } else if constexpr (RAD == 5) {
        dft5<SIGN, C, R>(v);
    } else if constexpr (RAD == 7) {
        dft7<SIGN, C, R>(v);
    } else if constexpr (RAD == 8) {
        dft8<SIGN, C, R>(v);
    } else if constexpr (RAD == 16) {
        dft16<SIGN, C, R>(v);
    } else {
        dft_generic<SIGN, RAD>(v, tw, NT);
    }
}

// ---------------------------------------------------------------- Stockham core
// One pass of the Stockham autosort FFT on a padded shared-memory line `s`
// (Govindaraju et al., "High performance discrete Fourier transforms on graphics
// processors", SC 2008):  butterfly b reads s[b + r*NF/R], twiddles by
// w_{Ns*R}^{(b mod Ns)*r}, runs a radix-R DFT and writes s[(b/Ns)*Ns*R + b%Ns + r*Ns].
// tw holds the forward roots of length NT (NT a multiple of NF).
template <typename R, int NF, int SIGN, int PASS, int T>
__device__ __forceinline__ void stockham_pass(cpx<R> *s, const cpx<R> *tw, int NT, int t, bool act)
{
    using C = cpx<R>;
    constexpr int RAD = radix_at(NF, PASS);
    constexpr int NS = stride_before(NF, PASS);
    constexpr int NB = NF / RAD;
    constexpr int PER = (NB + T - 1) / T;
    C v[PER][RAD];
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        const int b = t + k * T;
        if (act && (PER * T == NB || b < NB)) {
#pragma unroll
            for (int r = 0; r < RAD; ++r) v[k][r] = s[pad16(b + r * NB)];
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        const int b = t + k * T;
        if (act && (PER * T == NB || b < NB)) {
            if constexpr (NS > 1) {
                const int j = b % NS;
                const int step = (NT / (NS * RAD)) * j;
#pragma unroll
                for (int r = 1; r < RAD; ++r) {
                    const C w = tw[r * step];
                    v[k][r] = SIGN < 0 ? cmul(v[k][r], w) : cmulc(v[k][r], w);
                }
            }
            dft_radix<SIGN, RAD, C, R>(v[k], tw, NT);
            const int d = (b / NS) * NS * RAD + (b % NS);
#pragma unroll
            for (int r = 0; r < RAD; ++r) s[pad16(d + r * NS)] = v[k][r];
        }
    }
    __syncthreads();
}

template <typename R, int NF, int SIGN, int PASS, int T>
__device__ __forceinline__ void stockham_from(cpx<R> *s, const cpx<R> *tw, int NT, int t, bool act)
{
    if constexpr (PASS < num_passes(NF)) {
        stockham_pass<R, NF, SIGN, PASS, T>(s, tw, NT, t, act);
        stockham_from<R, NF, SIGN, PASS + 1, T>(s, tw, NT, t, act);
    }
}

// Full in-order FFT of length NF on the padded line s by T = threads_per_line(NF)
// threads (t in [0,T)).  Every thread of the block must call it (it synchronises
// the block); threads with act == false (no line of their own) only join the barriers.
template <typename R, int NF, int SIGN>
__device__ __forceinline__ void fft_line(cpx<R> *s, const cpx<R> *tw, int NT, int t, bool act = true)
{
    stockham_from<R, NF, SIGN, 0, threads_per_line(NF)>(s, tw, NT, t, act);
}

// Global -> shared staging of BYTES (4, 8 or 16) bytes.  CG = false: asynchronous
// cp.async (completed by cp_async_wait_all); CG = true: a synchronous load that
// bypasses L1 (ld.global.cg), for data other CTAs of the same launch wrote.
template <bool CG, int BYTES> __device__ __forceinline__ void stage_load(void *d, const void *s, bool ok)
{
    if constexpr (!CG) {
        cp_async<BYTES>(d, s, ok);
    } else if constexpr (BYTES == 4) {
        *reinterpret_cast<float *>(d) = ok ? __ldcg(reinterpret_cast<const float *>(s)) : 0.f;
    } else if constexpr (BYTES == 8) {
        *reinterpret_cast<float2 *>(d) = ok ? __ldcg(reinterpret_cast<const float2 *>(s)) : make_float2(0.f, 0.f);
    } else {
        *reinterpret_cast<float4 *>(d) =
            ok ? __ldcg(reinterpret_cast<const float4 *>(s)) : make_float4(0.f, 0.f, 0.f, 0.f);
    }
}

} // namespace fftb
