// fftb_internal.h -- host/device shared structures of the fftb engine.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace fftb {

// pass kinds
enum PassKind : int {
    K_C2C_FWD = 0,
    K_C2C_INV = 1,
    K_R2C = 2,
    K_C2R = 3,
    K_SANDWICH = 4,  // forward FFT, spectral multiply, inverse FFT in one pass
};

// epilogue (spectral multiplier) flags
enum EpMode : int {
    EP_SCALE = 1,    // multiply by ep_scale
    EP_POISSON = 2,  // multiply by ep_sign / |k|^2 (0 at k = 0)
    EP_GAUSS = 4,    // multiply by exp(-|k|^2 * ep_gauss)
    EP_HALFW = 8,    // multiply interior bins of the half (R2C) axis by ep_hw (adjoint weights)
    EP_DERIV = 16,   // multiply by i k_axis * scale (spectral derivative; fused column kernel)
    EP_TWIDDLE = 32, // multiply output point p by w_L^(p j), j the batch index of ep_src[0], L = ep_n[0]
                     // (the inter-step twiddle of a four-step long line; w from the table ep_tw)
};

// Everything one pass launch needs.  POD, passed by value.
struct PassArgs {
    const void *in;
    void *out;
    long long is, os;         // stride between the points of a line (elements of the in/out type)
    long long nlines;         // L
    long long c0, c1;         // batch dims: b0 = l % c0, b1 = (l / c0) % c1, b2 = l / (c0*c1)
    long long ib0, ib1, ib2;  // input offsets per batch index
    long long ob0, ob1, ob2;  // output offsets per batch index
    int kind;
    int half;                 // R2C/C2R through the half-length complex packing (even length)
    int in_pts_fast, out_pts_fast;
    int pair_io;              // real side accessed as aligned (even, odd) pairs
    int G, gshift;            // lines per CTA (power of two)
    const void *tw;           // forward roots exp(-2 pi i m / ntw), m in [0, ntw)
    int ntw;
    int tw_smem;              // stage the root table in shared memory
    // epilogue
    int ep_mode;
    int ep_naxes;
    int ep_src[4];            // 0: point index, 1..3: batch index b0..b2
    int ep_n[4];
    int ep_half[4];
    double ep_kscale[4];
    double ep_scale, ep_sign, ep_gauss, ep_hw;
    const void *ep_tw;        // EP_TWIDDLE: forward roots exp(-2 pi i m / L), m in [0, L)
    // chirp-z passes (bs_n > 0): line length n, chirp table (n) and convolution
    // kernel spectrum (M); tw / ntw are then the roots of the convolution length M
    int bs_n;
    const void *bs_chirp, *bs_bhat;
    // blocked point index (slab exchanges; C2C passes): in_blk > 0 loads point p from
    // (p / in_blk) * in_hi + (p % in_blk) * is; out_blk > 0 stores point p at
    // (p % out_blk) * os from the base of block q = p / out_blk: out_peer[q] when set (a
    // peer's receive buffer), else out + q * out_hi
    int in_blk, out_blk;
    long long in_hi, out_hi;
    void *out_peer[8];
};

struct PassKernelInfo {
    int nf;
    int threads_per_line;
    int line_pitch;
    const void *fn;
};

} // namespace fftb
