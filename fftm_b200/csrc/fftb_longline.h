// fftb_longline.h -- lines longer than the pass kernels hold in shared memory (internal).
#pragma once

#include <memory>

#include "fftb_engine.h"

namespace fftb {

struct LongLine;

// Builds the long-line step for pass `p` (C2C, R2C or C2R with at most a scale epilogue)
// whose length no single pass kernel covers.  Returns FFTB_ERROR_UNSUPPORTED_SIZE when the
// pass asks for something the long-line form does not do.
int longline_create(int dtype, const AxisPass &p, std::shared_ptr<LongLine> &out);
// Runs it with the program's buffers bound (in, out, work); ep: the dynamic scale, if any.
int longline_exec(const LongLine &L, void *const bufs[3], cudaStream_t s, const EpValues *ep);
// launches one execution issues
int longline_launches(const LongLine &L);
// bytes the step must read and write once
double longline_alg_bytes(const LongLine &L);

} // namespace fftb
