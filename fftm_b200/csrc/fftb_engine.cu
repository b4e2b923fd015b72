// fftb_engine.cu -- kernel registry, twiddle tables, program builder / executor.
#include "fftb_engine.h"
#include "fftb_bluestein.h"
#include "fftb_longline.h"

#include <algorithm>
#include <cstring>
#include <cstdio>
#include <map>
#include <mutex>
#include <set>
#include <tuple>

#include "../../include/fftb.h"
#include "fftb_device.cuh"

#ifndef FFTB_NPARTS
#define FFTB_NPARTS 8
#endif

// Kernel tables exported by the fftb_pass_inst.cu objects.
#define FFTB_DECL_PART(R, k) extern "C" int fftb_pass_table_##R##_part##k(fftb::PassKernelInfo *, int);
#define FFTB_DECL_PARTS(R)                                                                                            \
    FFTB_DECL_PART(R, 0) FFTB_DECL_PART(R, 1) FFTB_DECL_PART(R, 2) FFTB_DECL_PART(R, 3) FFTB_DECL_PART(R, 4)          \
    FFTB_DECL_PART(R, 5) FFTB_DECL_PART(R, 6) FFTB_DECL_PART(R, 7)
FFTB_DECL_PARTS(float)
FFTB_DECL_PARTS(double)

namespace fftb {

namespace {

thread_local std::string g_last_error;

struct Registry {
    std::map<int, PassKernelInfo> tab[2];
    std::set<std::pair<int, const void *>> smem_configured;  // (device, kernel): the limit is per device
    std::map<std::tuple<int, int, int>, void *> roots;  // (device, dtype, ntw) -> device table
    std::mutex mu;

    Registry()
    {
        typedef int (*part_fn)(PassKernelInfo *, int);
        const part_fn f32[] = {fftb_pass_table_float_part0, fftb_pass_table_float_part1,
                               fftb_pass_table_float_part2, fftb_pass_table_float_part3,
                               fftb_pass_table_float_part4, fftb_pass_table_float_part5,
                               fftb_pass_table_float_part6, fftb_pass_table_float_part7};
        const part_fn f64[] = {fftb_pass_table_double_part0, fftb_pass_table_double_part1,
                               fftb_pass_table_double_part2, fftb_pass_table_double_part3,
                               fftb_pass_table_double_part4, fftb_pass_table_double_part5,
                               fftb_pass_table_double_part6, fftb_pass_table_double_part7};
        PassKernelInfo buf[256];
        for (int d = 0; d < 2; ++d)
            for (int p = 0; p < 8; ++p) {
                const int n = (d == 0 ? f32[p] : f64[p])(buf, 256);
                for (int i = 0; i < n && i < 256; ++i) tab[d][buf[i].nf] = buf[i];
            }
    }
};

Registry &reg()
{
    static Registry r;
    return r;
}

template <typename R> __global__ void make_roots_kernel(cpx<R> *w, int n)
{
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m < n) {
        double s, c;
        // exp(-2 pi i m / n) evaluated in FP64, then rounded to R
        sincospi(-2.0 * (double)m / (double)n, &s, &c);
        w[m] = mk<R>((R)c, (R)s);
    }
}

int get_roots(int dtype, int ntw, void **out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return set_status_from_cuda(e);
    Registry &r = reg();
    std::lock_guard<std::mutex> lk(r.mu);
    auto key = std::make_tuple(dev, dtype, ntw);
    auto it = r.roots.find(key);
    if (it != r.roots.end()) {
        *out = it->second;
        return FFTB_SUCCESS;
    }
    void *p = nullptr;
    e = cudaMalloc(&p, complex_bytes(dtype) * (size_t)ntw);
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_last_error("cudaMalloc of a twiddle table failed");
        return FFTB_ERROR_ALLOC;
    }
    const int bs = 256, gs = (ntw + bs - 1) / bs;
    if (dtype == FFTB_F32) make_roots_kernel<float><<<gs, bs>>>((float2 *)p, ntw);
    else make_roots_kernel<double><<<gs, bs>>>((double2 *)p, ntw);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        cudaFree(p);
        return set_status_from_cuda(e);
    }
    r.roots[key] = p;
    *out = p;
    return FFTB_SUCCESS;
}

long long labs_ll(long long v) { return v < 0 ? -v : v; }

int floor_pow2(int v)
{
    int p = 1;
    while (p * 2 <= v) p *= 2;
    return p;
}

} // namespace

void set_last_error(const std::string &msg) { g_last_error = msg; }
const char *last_error() { return g_last_error.c_str(); }

int set_status_from_cuda(cudaError_t e)
{
    if (e == cudaSuccess) return FFTB_SUCCESS;
    set_last_error(std::string("CUDA: ") + cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? FFTB_ERROR_ALLOC : FFTB_ERROR_CUDA;
}

bool has_kernel(int dtype, int nf)
{
    Registry &r = reg();
    return r.tab[dtype].count(nf) != 0;
}

int engine_roots(int dtype, int ntw, void **out) { return get_roots(dtype, ntw, out); }

bool lookup_kernel(int dtype, int nf, PassKernelInfo *out)
{
    Registry &r = reg();
    auto it = r.tab[dtype].find(nf);
    if (it == r.tab[dtype].end()) return false;
    *out = it->second;
    return true;
}

int program_add(Program &prog, int dtype, const AxisPass &p)
{
    if (p.n < 1) return FFTB_ERROR_INVALID_VALUE;
    Launch L;
    memset(&L.args, 0, sizeof(L.args));
    PassArgs &a = L.args;
    const bool realk = (p.kind == K_R2C || p.kind == K_C2R);
    bool half = realk && (p.n % 2 == 0);
    int nf = half ? p.n / 2 : p.n;
    Registry &r = reg();
    auto it = r.tab[dtype].find(nf);
    if (it == r.tab[dtype].end() && half) {
        // no half-length kernel: the real line as a full complex line
        half = false;
        nf = p.n;
        it = r.tab[dtype].find(nf);
    }
    bool chirpz = false;
    if (it != r.tab[dtype].end()) {
        L.k = it->second;
    } else if (bluestein_kernel(dtype, p.n, &L.k)) {
        chirpz = true;   // L.k.nf is the convolution length
        const void *ch = nullptr, *bh = nullptr;
        int st = bluestein_tables(dtype, p.n, &ch, &bh);
        if (st != FFTB_SUCCESS) return st;
        a.bs_n = p.n;
        a.bs_chirp = ch;
        a.bs_bhat = bh;
    } else {
        // longer than one pass kernel holds: a long-line step (four-step or chirp-z)
        if (p.in_blk || p.out_blk) {
            set_last_error("blocked point indices need a C2C pass kernel (line length up to 4096)");
            return FFTB_ERROR_UNSUPPORTED_SIZE;
        }
        std::shared_ptr<LongLine> ll;
        int st = longline_create(dtype, p, ll);
        if (st != FFTB_SUCCESS) return st;
        Launch S;
        memset(&S.args, 0, sizeof(S.args));
        S.in_buf = p.in_buf;
        S.out_buf = p.out_buf;
        S.in_off_bytes = S.out_off_bytes = 0;
        S.pair_candidate = 0;
        S.real_align = 0;
        S.real_side = 0;
        S.block = 0;
        S.smem = 0;
        S.ep_dynamic = p.ep_dynamic;
        S.alg_bytes = longline_alg_bytes(*ll);
        static const char *kn[] = {"c2c_fwd", "c2c_inv", "r2c", "c2r", "sandwich"};
        S.name = std::string("fftb_long_line<") + (dtype == 0 ? "f32" : "f64") + ">/" + kn[p.kind] + "/n" +
                 std::to_string(p.n);
        S.longline = ll;
        prog.dtype = dtype;
        prog.launches.push_back(S);
        return FFTB_SUCCESS;
    }
    const int ntw = chirpz ? L.k.nf : (half ? 2 * nf : nf);
    void *roots = nullptr;
    int st = get_roots(dtype, ntw, &roots);
    if (st != FFTB_SUCCESS) return st;

    // batch dims: drop trivial ones, sort by input stride so dim 0 is the most contiguous
    std::vector<Dim> b;
    for (const Dim &d : p.batch)
        if (d.count > 1) b.push_back(d);
    std::stable_sort(b.begin(), b.end(), [](const Dim &x, const Dim &y) { return labs_ll(x.is) < labs_ll(y.is); });
    if (b.size() > 3) {
        set_last_error("more than three batch dimensions");
        return FFTB_ERROR_INVALID_VALUE;
    }
    while (b.size() < 3) b.push_back(Dim{1, 0, 0, -1});
    long long nlines = b[0].count * b[1].count * b[2].count;

    a.kind = p.kind;
    a.half = half ? 1 : 0;
    a.is = p.is;
    a.os = p.os;
    a.nlines = nlines;
    a.c0 = b[0].count;
    a.c1 = b[1].count;
    a.ib0 = b[0].is; a.ib1 = b[1].is; a.ib2 = b[2].is;
    a.ob0 = b[0].os; a.ob1 = b[1].os; a.ob2 = b[2].os;
    a.in_pts_fast = (labs_ll(p.is) == 1) || (b[0].count == 1) ||
                    (labs_ll(b[0].is) != 1 && labs_ll(p.is) < labs_ll(b[0].is));
    a.out_pts_fast = (labs_ll(p.os) == 1) || (b[0].count == 1) ||
                     (labs_ll(b[0].os) != 1 && labs_ll(p.os) < labs_ll(b[0].os));
    a.tw = roots;
    a.ntw = ntw;
    a.ep_tw = p.ep_tw;
    if ((p.in_blk || p.out_blk) && (chirpz || (p.kind != K_C2C_FWD && p.kind != K_C2C_INV) ||
                                    (p.out_blk && p.n / p.out_blk > 8))) {
        set_last_error("blocked point indices need a C2C pass kernel and at most 8 blocks");
        return FFTB_ERROR_UNSUPPORTED_SIZE;
    }
    a.in_blk = p.in_blk;
    a.in_hi = p.in_hi;
    a.out_blk = p.out_blk;
    a.out_hi = p.out_hi;
    const size_t cb = complex_bytes(dtype);
    a.tw_smem = ((size_t)ntw * cb <= 16384) ? 1 : 0;

    // epilogue
    a.ep_mode = p.ep_mode;
    a.ep_scale = p.ep_scale;
    a.ep_sign = p.ep_sign;
    a.ep_gauss = p.ep_gauss;
    a.ep_hw = p.ep_hw;
    a.ep_naxes = (int)p.ep_axes.size();
    if (a.ep_naxes > 4) return FFTB_ERROR_INVALID_VALUE;
    for (int i = 0; i < a.ep_naxes; ++i) {
        const EpAxis &e = p.ep_axes[i];
        int src = 0;
        if (!e.from_point) {
            src = -1;
            for (int j = 0; j < 3; ++j)
                if (b[j].id == e.dim_id && b[j].count > 1) src = j + 1;
            if (src < 0) {
                // a dimension of count 1 contributes index 0; use the point slot of an
                // axis that is always zero by pointing at an unused batch slot
                for (int j = 2; j >= 0; --j)
                    if (b[j].count == 1) { src = j + 1; break; }
            }
            if (src < 0) return FFTB_ERROR_INVALID_VALUE;
        }
        a.ep_src[i] = src;
        a.ep_n[i] = e.n;
        a.ep_half[i] = e.half;
        a.ep_kscale[i] = 1.0;
    }
    L.ep_dynamic = p.ep_dynamic;

    // real side pairing: contiguous real line with even batch strides
    L.real_side = (p.kind == K_R2C) ? 1 : (p.kind == K_C2R ? 2 : 0);
    L.pair_candidate = 0;
    if (half) {
        if (p.kind == K_R2C)
            L.pair_candidate = (p.is == 1) && b[0].is % 2 == 0 && b[1].is % 2 == 0 && b[2].is % 2 == 0 &&
                               p.in_base % 2 == 0;
        else
            L.pair_candidate = (p.os == 1) && b[0].os % 2 == 0 && b[1].os % 2 == 0 && b[2].os % 2 == 0 &&
                               p.out_base % 2 == 0;
    }
    L.real_align = 2 * real_bytes(dtype);

    // lines per CTA
    const int T = L.k.threads_per_line;
    int G = std::max(1, 256 / T);
    if (!a.in_pts_fast || !a.out_pts_fast) G = std::max(G, 16);
    G = std::min(G, std::max(1, 512 / T));
    G = floor_pow2(G);
    const long long lines_pow2 = nlines;
    while (G > 1 && G / 2 >= lines_pow2) G /= 2;
    auto smem_of = [&](int g) -> size_t {
        return (a.tw_smem ? (size_t)ntw * cb : 0) + (size_t)g * 32 + (size_t)g * (size_t)L.k.line_pitch * cb;
    };
    while (G > 1 && smem_of(G) > 160 * 1024) G /= 2;
    if (smem_of(G) > 227 * 1024) {
        set_last_error("line too long for shared memory");
        return FFTB_ERROR_UNSUPPORTED_SIZE;
    }
    a.G = G;
    int gs = 0;
    while ((1 << gs) < G) ++gs;
    a.gshift = gs;
    L.block = G * T;
    L.smem = smem_of(G);
    const long long ncta = (nlines + G - 1) / G;
    if (ncta > 0x7fffffffLL) return FFTB_ERROR_INVALID_VALUE;
    L.grid = dim3((unsigned)ncta, 1, 1);
    {
        std::lock_guard<std::mutex> lk(r.mu);
        if (L.smem > 48 * 1024) {
            int dev = 0;
            cudaError_t e = cudaGetDevice(&dev);
            if (e != cudaSuccess) return set_status_from_cuda(e);
            if (!r.smem_configured.count({dev, L.k.fn})) {
                e = cudaFuncSetAttribute(L.k.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
                if (e != cudaSuccess) return set_status_from_cuda(e);
                r.smem_configured.insert({dev, L.k.fn});
            }
        }
    }
    L.in_buf = p.in_buf;
    L.out_buf = p.out_buf;
    const size_t in_el = (p.kind == K_R2C) ? real_bytes(dtype) : cb;
    const size_t out_el = (p.kind == K_C2R) ? real_bytes(dtype) : cb;
    L.in_off_bytes = (size_t)p.in_base * in_el;
    L.out_off_bytes = (size_t)p.out_base * out_el;
    {
        static const char *kn[] = {"c2c_fwd", "c2c_inv", "r2c", "c2r", "sandwich"};
        const long long pin = (p.kind == K_C2R) ? (long long)(p.n / 2 + 1) : (long long)p.n;
        const long long pout = (p.kind == K_R2C) ? (long long)(p.n / 2 + 1) : (long long)p.n;
        L.alg_bytes = (double)nlines * ((double)pin * (double)in_el + (double)pout * (double)out_el);
        L.name = std::string(chirpz ? "fftb_bluestein_kernel<" : "fftb_pass_kernel<") + (dtype == 0 ? "f32" : "f64") +
                 "," + std::to_string(chirpz ? L.k.nf : nf) + ">/" + kn[p.kind] + "/n" + std::to_string(p.n);
    }
    prog.dtype = dtype;
    prog.launches.push_back(L);
    return FFTB_SUCCESS;
}

int LaunchTimer::reserve(size_t n)
{
    release();
    ev.resize(n, nullptr);
    for (size_t i = 0; i < n; ++i) {
        cudaError_t e = cudaEventCreate(&ev[i]);
        if (e != cudaSuccess) {
            ev.resize(i);
            return set_status_from_cuda(e);
        }
    }
    owner.assign(n, -1);
    names.assign(n, std::string());
    bytes.assign(n, 0.0);
    used = 0;
    return FFTB_SUCCESS;
}

void LaunchTimer::release()
{
    for (cudaEvent_t e : ev)
        if (e) cudaEventDestroy(e);
    ev.clear();
    owner.clear();
    names.clear();
    bytes.clear();
    used = 0;
}

int timer_mark(LaunchTimer *t, cudaStream_t s, const std::string &name, double b)
{
    if (!t || t->used >= t->ev.size()) return FFTB_SUCCESS;
    const size_t i = t->used++;
    t->owner[i] = 1;
    t->names[i] = name;
    t->bytes[i] = b;
    return set_status_from_cuda(cudaEventRecord(t->ev[i], s));
}

int timer_end(LaunchTimer *t, cudaStream_t s)
{
    if (!t || t->used >= t->ev.size()) return FFTB_SUCCESS;
    const size_t i = t->used++;
    t->owner[i] = -1;
    return set_status_from_cuda(cudaEventRecord(t->ev[i], s));
}

int program_exec(const Program &prog, void *in, void *out, void *work, cudaStream_t stream, const EpValues *ep,
                 LaunchTimer *timer)
{
    void *bufs[3] = {in, out, work};
    for (const Launch &L : prog.launches) {
        if (timer) {
            int ts = timer_mark(timer, stream, L.name, L.alg_bytes);
            if (ts != FFTB_SUCCESS) return ts;
        }
        if (L.longline) {
            int st = longline_exec(*L.longline, bufs, stream, ep && L.ep_dynamic ? ep : nullptr);
            if (st != FFTB_SUCCESS) return st;
            continue;
        }
        PassArgs a = L.args;
        char *ib = (char *)bufs[L.in_buf];
        char *ob = (char *)bufs[L.out_buf];
        if (!ib || !ob) {
            set_last_error("missing buffer");
            return L.in_buf == B_WORK || L.out_buf == B_WORK ? FFTB_ERROR_NO_WORK_AREA : FFTB_ERROR_INVALID_VALUE;
        }
        a.in = ib + L.in_off_bytes;
        a.out = ob + L.out_off_bytes;
        a.pair_io = 0;
        if (L.pair_candidate) {
            const void *rp = L.real_side == 1 ? a.in : a.out;
            a.pair_io = ((uintptr_t)rp % L.real_align) == 0;
        }
        if (ep && L.ep_dynamic) {
            a.ep_scale = ep->scale;
            a.ep_sign = ep->sign;
            a.ep_gauss = ep->gauss;
            if (ep->mode >= 0) a.ep_mode = ep->mode;
        }
        void *args[] = {&a};
        cudaError_t e = cudaLaunchKernel(L.k.fn, L.grid, dim3(L.block), args, L.smem, stream);
        if (e != cudaSuccess) return set_status_from_cuda(e);
    }
    if (timer) return timer_end(timer, stream);
    return FFTB_SUCCESS;
}

} // namespace fftb
