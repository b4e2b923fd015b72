// fftb_tc.cuh -- the radix-16 DFT of a register FFT stage as a 16x16 complex
// contraction on the tensor cores, in split FP16 with FP32 accumulation.
//
// One warp transforms 32 lines at once (lane = line, 16 complex values per lane, the
// same register layout as dft16).  With F = exp(-2 pi i k r / 16) split into
// F = Fr + i Fi and every operand split into an FP16 head and an FP16 tail,
//   Y = F X:  Yr = Fr Xr - Fi Xi,   Yi = Fr Xi + Fi Xr,
// each real product A B is computed as A_hi B_hi + A_hi B_lo + A_lo B_hi by
// mma.sync m16n8k16 (A = the 16x16 DFT block, B = 16 points x 8 lines) into FP32
// accumulators; only the A_lo B_lo term (relative 2^-22) is dropped.  The inverse uses
// the same fragments with the signs of the Fi terms flipped.  FP16's range is handled by
// scaling the warp's 32 lines by one power of two (exact) so their largest component
// sits in [2^14, 2^15).
//
// Data path per warp: the heads and tails are written line by line into a private
// staging area (32 rows of 144 bytes: the 16-byte pad makes the ldmatrix row reads
// conflict-free), read back as B fragments with ldmatrix (rows = lines, columns = k),
// and the accumulators (rows = k, columns = lines) are written back line by line and
// re-read so that each lane again holds its own line in natural order.
#pragma once

#include <cuda_fp16.h>

#include <cstdint>

namespace fftb {

constexpr int kTcRowBytes = 144;                      // one line in the staging area
constexpr int kTcWarpBytes = 32 * kTcRowBytes;        // one warp's staging area

struct TcDft16 {
    uint32_t fr_hi[4], fr_lo[4], fi_hi[4], fi_lo[4];  // A fragments of Re F and Im F (forward)
};

__device__ __forceinline__ uint32_t tc_h2_bits(__half2 h) { return *reinterpret_cast<uint32_t *>(&h); }

// head and tail of two floats as FP16 pairs
__device__ __forceinline__ void tc_split2(float a, float b, uint32_t &hi, uint32_t &lo)
{
    const __half2 h = __floats2half2_rn(a, b);
    const float2 f = __half22float2(h);
    hi = tc_h2_bits(h);
    lo = tc_h2_bits(__floats2half2_rn(a - f.x, b - f.y));
}

// The A fragments (m16n8k16, row major) of the forward 16-point DFT matrix for this lane:
// register q holds F[row][col], F[row][col+1] with row = lane/4 (+8 for q = 1, 3) and
// col = 2 (lane%4) (+8 for q = 2, 3).  The angles 2 pi (k r mod 16) / 16 are exact
// arguments of sincospif.
__device__ __forceinline__ void tc_build_dft16(TcDft16 &F, int lane)
{
    const int g = lane >> 2, c = lane & 3;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int row = g + ((q & 1) ? 8 : 0), col = 2 * c + ((q & 2) ? 8 : 0);
        float cr[2], ci[2];
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            float sn, cs;
            sincospif((float)((row * (col + e)) & 15) * 0.125f, &sn, &cs);
            cr[e] = cs;
            ci[e] = -sn;
        }
        tc_split2(cr[0], cr[1], F.fr_hi[q], F.fr_lo[q]);
        tc_split2(ci[0], ci[1], F.fi_hi[q], F.fi_lo[q]);
    }
}

__device__ __forceinline__ void tc_mma(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1)
{
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                 "{%0,%1,%2,%3};\n"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// split product A B ~ A_hi B_hi + A_hi B_lo + A_lo B_hi
__device__ __forceinline__ void tc_mma3(float (&d)[4], const uint32_t (&ahi)[4], const uint32_t (&alo)[4],
                                        uint32_t bh0, uint32_t bh1, uint32_t bl0, uint32_t bl1)
{
    tc_mma(d, ahi, bh0, bh1);
    tc_mma(d, ahi, bl0, bl1);
    tc_mma(d, alo, bh0, bh1);
}

__device__ __forceinline__ void tc_ldmatrix_x4(uint32_t saddr, uint32_t &r0, uint32_t &r1, uint32_t &r2, uint32_t &r3)
{
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"(saddr)
                 : "memory");
}

// v <- DFT16(v) (SIGN < 0: forward, SIGN > 0: inverse, unnormalised) for the 32 lines
// of this warp.  `stage` is this warp's private kTcWarpBytes of shared memory (16-byte
// aligned); all 32 lanes must call.
template <int SIGN>
__device__ __forceinline__ void tc_dft16(float2 (&v)[16], unsigned char *stage, const TcDft16 &F, int lane)
{
    // one power-of-two scale for the warp's lines
    float m = 0.f;
#pragma unroll
    for (int r = 0; r < 16; ++r) m = fmaxf(m, fmaxf(fabsf(v[r].x), fabsf(v[r].y)));
#pragma unroll
    for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    int e = 0;
    if (m > 0.f) e = 14 - (((__float_as_int(m) >> 23) & 0xff) - 127);
    e = e < -100 ? -100 : (e > 100 ? 100 : e);
    const float sc = __int_as_float((e + 127) << 23), inv = __int_as_float((127 - e) << 23);

    // heads and tails of this lane's line: [Re hi | Im hi | Re lo | Im lo], 16 halves each
    uint32_t rh[8], rl[8], ih[8], il[8];
#pragma unroll
    for (int p = 0; p < 8; ++p) {
        tc_split2(v[2 * p].x * sc, v[2 * p + 1].x * sc, rh[p], rl[p]);
        tc_split2(v[2 * p].y * sc, v[2 * p + 1].y * sc, ih[p], il[p]);
    }
    __syncwarp();
    uint4 *row = reinterpret_cast<uint4 *>(stage + lane * kTcRowBytes);
    row[0] = make_uint4(rh[0], rh[1], rh[2], rh[3]);
    row[1] = make_uint4(rh[4], rh[5], rh[6], rh[7]);
    row[2] = make_uint4(ih[0], ih[1], ih[2], ih[3]);
    row[3] = make_uint4(ih[4], ih[5], ih[6], ih[7]);
    row[4] = make_uint4(rl[0], rl[1], rl[2], rl[3]);
    row[5] = make_uint4(rl[4], rl[5], rl[6], rl[7]);
    row[6] = make_uint4(il[0], il[1], il[2], il[3]);
    row[7] = make_uint4(il[4], il[5], il[6], il[7]);
    __syncwarp();

    const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(stage);
    const int mat = lane >> 3, mrow = lane & 7;   // this lane's ldmatrix row address
    float2 y[4][4];                                // [group][c0..c3] outputs
#pragma unroll
    for (int grp = 0; grp < 4; ++grp) {
        const uint32_t a = sbase + (uint32_t)((8 * grp + mrow) * kTcRowBytes + 16 * mat);
        uint32_t xr_h0, xr_h1, xi_h0, xi_h1, xr_l0, xr_l1, xi_l0, xi_l1;
        tc_ldmatrix_x4(a, xr_h0, xr_h1, xi_h0, xi_h1);
        tc_ldmatrix_x4(a + 64, xr_l0, xr_l1, xi_l0, xi_l1);
        float prr[4] = {0.f, 0.f, 0.f, 0.f}, pii[4] = {0.f, 0.f, 0.f, 0.f};
        float pri[4] = {0.f, 0.f, 0.f, 0.f}, pir[4] = {0.f, 0.f, 0.f, 0.f};
        tc_mma3(prr, F.fr_hi, F.fr_lo, xr_h0, xr_h1, xr_l0, xr_l1);
        tc_mma3(pii, F.fi_hi, F.fi_lo, xi_h0, xi_h1, xi_l0, xi_l1);
        tc_mma3(pri, F.fr_hi, F.fr_lo, xi_h0, xi_h1, xi_l0, xi_l1);
        tc_mma3(pir, F.fi_hi, F.fi_lo, xr_h0, xr_h1, xr_l0, xr_l1);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            y[grp][q].x = (SIGN < 0 ? prr[q] - pii[q] : prr[q] + pii[q]) * inv;
            y[grp][q].y = (SIGN < 0 ? pri[q] + pir[q] : pri[q] - pir[q]) * inv;
        }
    }
    // accumulator element q of group grp: k = lane/4 (+8 for q >= 2), line = 8 grp + 2 (lane%4) + (q & 1)
    __syncwarp();
    const int g = lane >> 2, c = lane & 3;
#pragma unroll
    for (int grp = 0; grp < 4; ++grp) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int k = g + (q >= 2 ? 8 : 0), line = 8 * grp + 2 * c + (q & 1);
            *reinterpret_cast<float2 *>(stage + line * kTcRowBytes + 8 * k) = y[grp][q];
        }
    }
    __syncwarp();
    const float2 *mine = reinterpret_cast<const float2 *>(stage + lane * kTcRowBytes);
#pragma unroll
    for (int k = 0; k < 16; ++k) v[k] = mine[k];
    __syncwarp();
}

} // namespace fftb
