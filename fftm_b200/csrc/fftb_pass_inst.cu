// fftb_pass_inst.cu -- explicit instantiations of the pass kernel.
//
// Compiled several times with -DFFTB_REAL=float|double and -DFFTB_PART=k
// (k in [0, FFTB_NPARTS)) so the instantiation work spreads over parallel
// compiler processes; each object exports one table of (NF, kernel) pairs.
#include "fftb_pass.cuh"

#ifndef FFTB_REAL
#define FFTB_REAL float
#endif
#ifndef FFTB_PART
#define FFTB_PART 0
#endif
#ifndef FFTB_NPARTS
#define FFTB_NPARTS 1
#endif

#define FFTB_CAT2(a, b) a##b
#define FFTB_CAT(a, b) FFTB_CAT2(a, b)
#define FFTB_CAT4(a, b, c, d) FFTB_CAT(FFTB_CAT(a, b), FFTB_CAT(c, d))

// The complex line lengths the engine supports directly (R2C/C2R of even n
// run NF = n/2, everything else NF = n).
#define FFTB_NF_LIST(X)                                                                            \
    X(1) X(2) X(4) X(8) X(16) X(32) X(64) X(128) X(256) X(512) X(1024) X(2048) X(4096)            \
    X(3) X(6) X(12) X(24) X(48) X(96) X(192) X(384) X(768) X(1536) X(3072)                         \
    X(5) X(10) X(20) X(40) X(80) X(160) X(320) X(640) X(1280) X(2560)                              \
    X(7) X(14) X(28) X(56) X(112) X(224) X(448) X(896) X(1792) X(3584)                             \
    X(9) X(18) X(36) X(72) X(144) X(288) X(576) X(1152) X(2304)                                    \
    X(15) X(30) X(60) X(120) X(240) X(480) X(960) X(1920) X(3840)                                  \
    X(25) X(50) X(100) X(200) X(400) X(800) X(1600) X(3200)                                        \
    X(27) X(54) X(108) X(216) X(432) X(864) X(1728) X(3456)                                        \
    X(21) X(42) X(84) X(168) X(336) X(672) X(1344) X(2688)                                         \
    X(35) X(45) X(49) X(63) X(75) X(81) X(105) X(125) X(135) X(147) X(175) X(189) X(225) X(243)   \
    X(11) X(13) X(22) X(26) X(44) X(52) X(88) X(104) X(176) X(208) X(352) X(416) X(704) X(832)

namespace {
constexpr int kNF[] = {
#define FFTB_ITEM(n) n,
    FFTB_NF_LIST(FFTB_ITEM)
#undef FFTB_ITEM
};
constexpr int kCount = (int)(sizeof(kNF) / sizeof(kNF[0]));

template <int I> void fill_table(fftb::PassKernelInfo *out, int cap, int &n)
{
    if constexpr (I < kCount) {
        if constexpr (I % FFTB_NPARTS == FFTB_PART) {
            if (n < cap) out[n] = fftb::pass_kernel_info<FFTB_REAL, kNF[I]>();
            ++n;
        }
        fill_table<I + 1>(out, cap, n);
    }
}
} // namespace

extern "C" int FFTB_CAT4(fftb_pass_table_, FFTB_REAL, _part, FFTB_PART)(fftb::PassKernelInfo *out, int cap)
{
    int n = 0;
    fill_table<0>(out, cap, n);
    return n;
}
