// fftb_engine.h -- host-side program builder and executor (internal).
//
// A "program" is the fixed sequence of kernel launches one transform call
// issues.  It is built once (plan creation / ffts init) and replayed on every
// call with the caller's buffers bound in; execution never allocates and never
// synchronises the host.
#pragma once

#include <cuda_runtime.h>

#include <memory>
#include <string>
#include <vector>

#include "fftb_internal.h"

namespace fftb {

enum Buf : int { B_IN = 0, B_OUT = 1, B_WORK = 2 };

// One batch dimension of an axis pass: count, input stride, output stride
// (strides in elements of the input / output element type).
struct Dim {
    long long count;
    long long is;
    long long os;
    int id;  // stable id for epilogue axis mapping (-1: none)
};

// Which index supplies each spectral axis of a fused epilogue.
struct EpAxis {
    int from_point;  // 1: the pass's point index; 0: batch dim with `dim_id`
    int dim_id;
    int n;           // full axis length (wavenumber wrap)
    int half;        // half (R2C) axis: k = index
};

struct AxisPass {
    int kind = K_C2C_FWD;
    int n = 0;                  // logical line length (real length for R2C/C2R)
    long long is = 1, os = 1;   // point strides
    std::vector<Dim> batch;
    int in_buf = B_IN, out_buf = B_OUT;
    long long in_base = 0, out_base = 0;  // element offsets inside the buffers
    int ep_mode = 0;
    double ep_scale = 1.0, ep_sign = -1.0, ep_gauss = 0.0, ep_hw = 1.0;
    std::vector<EpAxis> ep_axes;
    int ep_dynamic = 0;         // epilogue parameters supplied at execution
    const void *ep_tw = nullptr;  // EP_TWIDDLE root table
    // blocked point index of a C2C pass (PassArgs in_blk / out_blk): the slab exchanges'
    // pack (store) and unpack (load); strides in elements
    int in_blk = 0, out_blk = 0;
    long long in_hi = 0, out_hi = 0;
};

struct LongLine;

struct Launch {
    PassArgs args;
    PassKernelInfo k;
    int in_buf, out_buf;
    size_t in_off_bytes, out_off_bytes;
    int pair_candidate;  // real side contiguous with even strides
    size_t real_align;   // required alignment of the real side for pair access
    int real_side;       // 0: none, 1: input real, 2: output real
    dim3 grid;
    int block;
    size_t smem;
    int ep_dynamic;
    std::string name;   // kernel + geometry, for timing reports
    double alg_bytes;   // bytes the launch must read and write once (its algorithmic traffic)
    std::shared_ptr<LongLine> longline;  // set: a long-line step (fftb_longline.cu) instead of one pass
};

struct Program {
    int dtype = 0;
    std::vector<Launch> launches;
};

// Dynamic epilogue values for one execution.
struct EpValues {
    double scale = 1.0, sign = -1.0, gauss = 0.0, hw = 1.0;
    int mode = -1;  // -1: keep the built mode
};

// Appends the launch for `p` to prog.  Returns an FFTB status.
int program_add(Program &prog, int dtype, const AxisPass &p);

// Optional per-launch event recorder (profiling hook).  When attached to an
// execution, an event is recorded on the stream before every launch and after
// the last one; read() converts consecutive pairs into per-launch milliseconds.
struct LaunchTimer {
    std::vector<cudaEvent_t> ev;      // pool, created by reserve()
    std::vector<int> owner;           // launch index of each begin event (-1: end marker)
    std::vector<std::string> names;
    std::vector<double> bytes;
    size_t used = 0;
    int reserve(size_t n);
    void release();
    ~LaunchTimer() { release(); }
};

// Runs every launch of prog on `stream` with buffers bound.  Returns an FFTB status.
int program_exec(const Program &prog, void *in, void *out, void *work, cudaStream_t stream,
                 const EpValues *ep = nullptr, LaunchTimer *timer = nullptr);

// record helpers shared with the specialised kernels
int timer_mark(LaunchTimer *t, cudaStream_t s, const std::string &name, double bytes);
int timer_end(LaunchTimer *t, cudaStream_t s);

// device table of the forward roots exp(-2 pi i m / ntw), shared per (device, dtype, ntw)
int engine_roots(int dtype, int ntw, void **out);

// true if a line of complex length nf has a compiled kernel for dtype
bool has_kernel(int dtype, int nf);
// copies the registry entry of the pass kernel for (dtype, nf); false if none
bool lookup_kernel(int dtype, int nf, PassKernelInfo *out);

// element size of the complex type
inline size_t complex_bytes(int dtype) { return dtype == 0 ? 8 : 16; }
inline size_t real_bytes(int dtype) { return dtype == 0 ? 4 : 8; }

int set_status_from_cuda(cudaError_t e);
void set_last_error(const std::string &msg);
const char *last_error();

} // namespace fftb
