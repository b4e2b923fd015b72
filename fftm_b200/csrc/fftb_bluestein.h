// fftb_bluestein.h -- chirp-z (Bluestein) passes for line lengths the radix kernels
// do not cover (internal).
#pragma once

#include "fftb_engine.h"

namespace fftb {

// power-of-two convolution length for a line of n points (0 if n is out of range)
int bluestein_size(int n);
// the Bluestein pass kernel for (dtype, n): nf = its convolution length M
bool bluestein_kernel(int dtype, int n, PassKernelInfo *k);
// device tables of (dtype, n), cached per device: chirp c_j = exp(-i pi j^2 / n)
// (n entries) and B = FFT_M(conj c wrapped) / M (M entries)
int bluestein_tables(int dtype, int n, const void **chirp, const void **bhat);

} // namespace fftb
