// fftb_api.cu -- the C ABI: plan objects (cufft::fft<T,D> replacement) and
// ffts transform objects (fftm::ffts replacement), built on the pass engine.
#include <cuda_runtime.h>

#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/fftb.h"
#include "fftb_device.cuh"
#include "fftb_engine.h"

using namespace fftb;

// ================================================================== plans
struct fftb_plan_s {
    int dir = 0, dtype = 0, rank = 0;
    long long n[3] = {0, 0, 0}, ie[3] = {0, 0, 0}, oe[3] = {0, 0, 0};
    long long istride = 0, idist = 0, ostride = 0, odist = 0, batch = 0;
    bool default_layout = false;
    Program prog;      // the plan's own direction
    Program prog_alt;  // C2C plans: the opposite sign (exec_direction)
    void *work = nullptr;
    cudaStream_t stream = 0;
};

namespace {

bool valid_dtype(int d) { return d == FFTB_F32 || d == FFTB_F64; }

// Axis strides of an advanced layout: axis j stride = stride * prod_{i>j} embed[i].
void axis_strides(int rank, const long long *embed, long long stride, long long *out)
{
    long long m = stride;
    for (int j = rank - 1; j >= 0; --j) {
        out[j] = m;
        m *= embed[j];
    }
}

// Builds the pass list of one advanced-layout plan (cuFFT semantics: R2C = last
// axis real-to-half-complex then the other axes in place on the output; C2R =
// the leading axes inverted in place on the input, then the last axis C2R).
int build_plan_program(fftb_plan_s *p, int dir, Program &prog)
{
    const int r = p->rank;
    long long is_ax[3], os_ax[3];
    axis_strides(r, p->ie, p->istride, is_ax);
    axis_strides(r, p->oe, p->ostride, os_ax);
    const long long nh = p->n[r - 1] / 2 + 1;
    auto count_of = [&](int j, bool half_last) { return (j == r - 1 && half_last) ? nh : p->n[j]; };
    int st;
    if (dir == FFTB_R2C) {
        AxisPass a;
        a.kind = K_R2C;
        a.n = (int)p->n[r - 1];
        a.is = is_ax[r - 1];
        a.os = os_ax[r - 1];
        for (int j = 0; j < r - 1; ++j) a.batch.push_back(Dim{p->n[j], is_ax[j], os_ax[j], j});
        a.batch.push_back(Dim{p->batch, p->idist, p->odist, 10});
        a.in_buf = B_IN;
        a.out_buf = B_OUT;
        if ((st = program_add(prog, p->dtype, a)) != FFTB_SUCCESS) return st;
        for (int ax = r - 2; ax >= 0; --ax) {
            AxisPass c;
            c.kind = K_C2C_FWD;
            c.n = (int)p->n[ax];
            c.is = c.os = os_ax[ax];
            for (int j = 0; j < r; ++j)
                if (j != ax) c.batch.push_back(Dim{count_of(j, true), os_ax[j], os_ax[j], j});
            c.batch.push_back(Dim{p->batch, p->odist, p->odist, 10});
            c.in_buf = c.out_buf = B_OUT;
            if ((st = program_add(prog, p->dtype, c)) != FFTB_SUCCESS) return st;
        }
    } else if (dir == FFTB_C2R) {
        for (int ax = 0; ax <= r - 2; ++ax) {
            AxisPass c;
            c.kind = K_C2C_INV;
            c.n = (int)p->n[ax];
            c.is = c.os = is_ax[ax];
            for (int j = 0; j < r; ++j)
                if (j != ax) c.batch.push_back(Dim{count_of(j, true), is_ax[j], is_ax[j], j});
            c.batch.push_back(Dim{p->batch, p->idist, p->idist, 10});
            c.in_buf = c.out_buf = B_IN;
            if ((st = program_add(prog, p->dtype, c)) != FFTB_SUCCESS) return st;
        }
        AxisPass a;
        a.kind = K_C2R;
        a.n = (int)p->n[r - 1];
        a.is = is_ax[r - 1];
        a.os = os_ax[r - 1];
        for (int j = 0; j < r - 1; ++j) a.batch.push_back(Dim{p->n[j], is_ax[j], os_ax[j], j});
        a.batch.push_back(Dim{p->batch, p->idist, p->odist, 10});
        a.in_buf = B_IN;
        a.out_buf = B_OUT;
        if ((st = program_add(prog, p->dtype, a)) != FFTB_SUCCESS) return st;
    } else {
        const int kind = dir == FFTB_C2CF ? K_C2C_FWD : K_C2C_INV;
        for (int ax = r - 1; ax >= 0; --ax) {
            AxisPass c;
            c.kind = kind;
            c.n = (int)p->n[ax];
            const bool first = (ax == r - 1);
            c.is = first ? is_ax[ax] : os_ax[ax];
            c.os = os_ax[ax];
            for (int j = 0; j < r; ++j)
                if (j != ax) c.batch.push_back(Dim{p->n[j], first ? is_ax[j] : os_ax[j], os_ax[j], j});
            c.batch.push_back(Dim{p->batch, first ? p->idist : p->odist, p->odist, 10});
            c.in_buf = first ? B_IN : B_OUT;
            c.out_buf = B_OUT;
            if ((st = program_add(prog, p->dtype, c)) != FFTB_SUCCESS) return st;
        }
    }
    return FFTB_SUCCESS;
}

} // namespace

extern "C" {

const char *fftb_version(void) { return "0.1.0"; }

const char *fftb_status_string(int s)
{
    switch (s) {
    case FFTB_SUCCESS: return "success";
    case FFTB_ERROR_INVALID_VALUE: return "invalid value";
    case FFTB_ERROR_UNSUPPORTED_SIZE: return "unsupported transform size";
    case FFTB_ERROR_CUDA: return "CUDA error";
    case FFTB_ERROR_ALLOC: return "device allocation failed";
    case FFTB_ERROR_INVALID_HANDLE: return "invalid handle";
    case FFTB_ERROR_NOT_INITIALIZED: return "ffts: call init() before using the transform.";
    case FFTB_ERROR_WRONG_DIMENSION: return "ffts: used with the wrong dimension";
    case FFTB_ERROR_ALREADY_INITIALIZED: return "ffts::init can only be called once per instance.";
    case FFTB_ERROR_MISALIGNED: return "misaligned pointer";
    case FFTB_ERROR_NO_WORK_AREA: return "work area required";
    case FFTB_ERROR_CACHE_IO: return "autotune cache cannot be read, parsed or written";
    case FFTB_ERROR_CACHE_MISMATCH: return "autotune cache does not match this problem or hardware";
    case FFTB_ERROR_CACHE_MISSING: return "autotune cache file does not exist";
    case FFTB_ERROR_TUNE_FAILED: return "no autotune candidate passed its round-trip check";
    default: return "unknown status";
    }
}

const char *fftb_last_error_message(void) { return last_error(); }

int fftb_plan_create(int direction, int dtype, int rank, const long long *n, const long long *inembed,
                     long long istride, long long idist, const long long *onembed, long long ostride,
                     long long odist, long long batch, fftb_plan *plan, size_t *work_bytes)
{
    if (!plan) return FFTB_ERROR_INVALID_VALUE;
    *plan = nullptr;
    if (direction < FFTB_R2C || direction > FFTB_C2CB || !valid_dtype(dtype) || rank < 1 || rank > 3 || !n ||
        batch < 1)
        return FFTB_ERROR_INVALID_VALUE;
    for (int j = 0; j < rank; ++j)
        if (n[j] < 1 || n[j] > (1LL << 30)) return FFTB_ERROR_INVALID_VALUE;
    if ((inembed == nullptr) != (onembed == nullptr)) return FFTB_ERROR_INVALID_VALUE;
    fftb_plan_s *p = new (std::nothrow) fftb_plan_s();
    if (!p) return FFTB_ERROR_ALLOC;
    p->dir = direction;
    p->dtype = dtype;
    p->rank = rank;
    for (int j = 0; j < rank; ++j) p->n[j] = n[j];
    const long long nh = n[rank - 1] / 2 + 1;
    long long in_dims[3], out_dims[3];
    for (int j = 0; j < rank; ++j) {
        in_dims[j] = (direction == FFTB_C2R && j == rank - 1) ? nh : n[j];
        out_dims[j] = (direction == FFTB_R2C && j == rank - 1) ? nh : n[j];
    }
    if (!inembed) {
        p->default_layout = true;
        long long id = 1, od = 1;
        for (int j = 0; j < rank; ++j) {
            p->ie[j] = in_dims[j];
            p->oe[j] = out_dims[j];
            id *= in_dims[j];
            od *= out_dims[j];
        }
        p->istride = p->ostride = 1;
        p->idist = id;
        p->odist = od;
    } else {
        for (int j = 0; j < rank; ++j) {
            p->ie[j] = inembed[j];
            p->oe[j] = onembed[j];
            if (j > 0 && (inembed[j] < in_dims[j] || onembed[j] < out_dims[j])) {
                delete p;
                return FFTB_ERROR_INVALID_VALUE;
            }
        }
        p->istride = istride;
        p->idist = idist;
        p->ostride = ostride;
        p->odist = odist;
        if (istride < 1 || ostride < 1 || (batch > 1 && (idist < 1 || odist < 1))) {
            delete p;
            return FFTB_ERROR_INVALID_VALUE;
        }
    }
    p->batch = batch;
    int st = build_plan_program(p, direction, p->prog);
    if (st == FFTB_SUCCESS && (direction == FFTB_C2CF || direction == FFTB_C2CB))
        st = build_plan_program(p, direction == FFTB_C2CF ? FFTB_C2CB : FFTB_C2CF, p->prog_alt);
    if (st != FFTB_SUCCESS) {
        delete p;
        return st;
    }
    if (work_bytes) *work_bytes = 0;
    *plan = p;
    return FFTB_SUCCESS;
}

int fftb_plan_get_work_size(fftb_plan plan, size_t *work_bytes)
{
    if (!plan || !work_bytes) return FFTB_ERROR_INVALID_HANDLE;
    *work_bytes = 0;
    return FFTB_SUCCESS;
}

int fftb_plan_set_work_area(fftb_plan plan, void *work)
{
    if (!plan) return FFTB_ERROR_INVALID_HANDLE;
    plan->work = work;
    return FFTB_SUCCESS;
}

int fftb_plan_set_stream(fftb_plan plan, void *stream)
{
    if (!plan) return FFTB_ERROR_INVALID_HANDLE;
    plan->stream = (cudaStream_t)stream;
    return FFTB_SUCCESS;
}

int fftb_exec(fftb_plan plan, void *in, void *out)
{
    if (!plan) return FFTB_ERROR_INVALID_HANDLE;
    if (!in || !out) return FFTB_ERROR_INVALID_VALUE;
    return program_exec(plan->prog, in, out, plan->work, plan->stream);
}

int fftb_exec_direction(fftb_plan plan, int direction, void *in, void *out)
{
    if (!plan) return FFTB_ERROR_INVALID_HANDLE;
    if (!in || !out) return FFTB_ERROR_INVALID_VALUE;
    if (direction == plan->dir) return program_exec(plan->prog, in, out, plan->work, plan->stream);
    if ((plan->dir == FFTB_C2CF || plan->dir == FFTB_C2CB) && (direction == FFTB_C2CF || direction == FFTB_C2CB))
        return program_exec(plan->prog_alt, in, out, plan->work, plan->stream);
    return FFTB_ERROR_INVALID_VALUE;
}

int fftb_plan_describe(fftb_plan plan, int *direction, int *dtype, int *rank, long long *n, long long *inembed,
                       long long *istride, long long *idist, long long *onembed, long long *ostride,
                       long long *odist, long long *batch)
{
    if (!plan) return FFTB_ERROR_INVALID_HANDLE;
    if (direction) *direction = plan->dir;
    if (dtype) *dtype = plan->dtype;
    if (rank) *rank = plan->rank;
    for (int j = 0; j < 3; ++j) {
        if (n) n[j] = j < plan->rank ? plan->n[j] : 0;
        if (inembed) inembed[j] = j < plan->rank ? plan->ie[j] : 0;
        if (onembed) onembed[j] = j < plan->rank ? plan->oe[j] : 0;
    }
    if (istride) *istride = plan->istride;
    if (idist) *idist = plan->idist;
    if (ostride) *ostride = plan->ostride;
    if (odist) *odist = plan->odist;
    if (batch) *batch = plan->batch;
    return FFTB_SUCCESS;
}

int fftb_plan_num_launches(fftb_plan plan, int *launches)
{
    if (!plan || !launches) return FFTB_ERROR_INVALID_HANDLE;
    *launches = (int)plan->prog.launches.size();
    return FFTB_SUCCESS;
}

int fftb_plan_destroy(fftb_plan plan)
{
    if (!plan) return FFTB_ERROR_INVALID_HANDLE;
    delete plan;
    return FFTB_SUCCESS;
}

} // extern "C"
