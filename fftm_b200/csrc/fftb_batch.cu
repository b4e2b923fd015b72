// fftb_batch.cu -- many 3D transforms of uneven sizes in one persistent launch or in
// one launch per (stage, line length) group.
//
// Every transform of the batch is compiled into its pass program (the same passes
// as a single ffts object).  The passes of all transforms are flattened into one
// work list of (pass, tile) items ordered stage by stage: first every tile of the
// first pass of every transform, then every tile of the second passes, and so on.
// A persistent kernel (one or more CTAs per SM) takes items from the head of that
// list with an atomic counter; before working on a tile of pass p it waits until
// every tile of the previous pass of the same transform has been counted done.
// Because items are taken in list order, every item a CTA waits for has already
// been taken by a running CTA that waits only on items earlier still, so the wait
// always ends; it is nevertheless bounded (kSpinLimit polls unless the caller set another
// limit), after which the kernel raises an error flag that fftb_batch_status reports and
// every CTA returns.
// The launch (counter reset + kernel) is captured once into a CUDA graph per buffer
// binding and replayed.
//
// The grouped form runs the same items as one plain launch per (stage, line length)
// group, each a kernel specialised for its length, in stream order (no waits), and
// can be replayed from a CUDA graph the same way.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <new>
#include <string>
#include <vector>

#include "../../include/fftb.h"
#include "fftb_coltile.cuh"
#include "fftb_engine.h"
#include "fftb_fused3d.h"
#include "fftb_pass.cuh"

namespace fftb {
namespace {

constexpr int kBatchThreads = 256;
constexpr long long kSpinLimit = 1LL << 22;  // ~0.5 s of polling at most

struct BatchItem {
    int pass;
    int tile;
};

// buffer binding of one pass: 0 in, 1 out, 2 work
struct PassBind {
    int in_buf, out_buf;
    long long in_off, out_off;  // bytes
    int nf;
    // the tile form of a pass on the fused path's kernels (f32): 0 the pass kernel's tile;
    // 1 a column tile (ckind 0-2 x forward / inverse / sandwich, 3-4 y forward / inverse) of
    // n-point lines; 2 a row-pair tile of n-point z rows (ckind 0 R2C, 1 C2R)
    int fast, ckind, n;
    int lines, ny, nz;      // column: lines of the spectrum, its ny and nz; row: rows
    float scale, sign;      // row C2R scale; column sandwich scale and Poisson sign
    int ep_mode;            // column sandwich multiply
    const float2 *roots;    // n-point root table
};

__device__ __forceinline__ int ld_acquire(const int *p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

#define FFTB_BATCH_NF_LIST(X) X(8) X(12) X(16) X(20) X(24) X(32) X(40) X(48) X(64) X(80) X(96) X(128) X(160) X(192) X(256)

// Column and row-pair tiles of the persistent launch, one non-inlined function per kind and
// length (their own register allocation, as the pass tiles have).
template <int N, int KIND> __device__ __noinline__ void batch_col_tile(const PassBind *b, void *data, int tile)
{
    if constexpr (KIND <= 2) {
        XColEp ep = {};
        ep.mode = b->ep_mode;
        ep.scale_f = b->scale;
        ep.sign_f = b->sign;
        ep.scale = b->scale;
        ep.sign = b->sign;
        ep.ny = b->ny;
        ep.nz = b->nz;
        ep.nzh = b->nz / 2 + 1;
        ep.hn = b->nz;
        ep.hw_f = 1.f;
        ep.hw = 1.0;
        xcol_tile<float, N, KIND, false>(reinterpret_cast<float2 *>(data), b->lines, b->lines, 0, nullptr, b->roots, ep,
                                         tile, 0);
    } else {
        const XGroupItem it{0, b->lines, tile, b->ny, b->nz};
        ycol_tile<N, KIND - 3>(it, reinterpret_cast<float2 *>(data), b->roots);
    }
}
template <int N, int DIR>
__device__ __noinline__ void batch_row_tile(const PassBind *b, const void *in, void *out, int tile)
{
    const RowGroupItem it{0, 0, b->lines, tile, b->scale};
    row_tile<N, DIR>(it, in, out, b->roots);
}

#define FFTB_BATCH_COL_LIST(X) X(32) X(48) X(64) X(96) X(128) X(256)
#define FFTB_BATCH_ROW_LIST(X) X(64) X(128) X(256)

// One tile of a pass of line length NF; not inlined, so every length keeps its own
// register allocation instead of the union of all of them.  The tile stages its lines
// with cp.async: thread 0's acquire load of the producer counters followed by the
// CTA barrier orders these loads after the producers' fenced stores (PTX memory model).
template <int NF>
__device__ __noinline__ void batch_tile(const PassArgs *a, const void *in, void *out, long long line0,
                                        unsigned char *smem)
{
    pass_body<float, NF, false, false>(*a, in, out, line0, smem);
}

// ctl[0]: queue head, ctl[1]: error flag, ctl[2 + p]: finished tiles of pass p
__global__ void __launch_bounds__(kBatchThreads)
    batch_persistent_kernel(const BatchItem *__restrict__ items, int nitems, const PassArgs *__restrict__ passes,
                            const PassBind *__restrict__ binds, const int *__restrict__ deps,
                            const int *__restrict__ ntiles, int *ctl, const void *in, void *out, void *work,
                            long long spin_limit)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int s_item, s_ok;
    // thread 0 takes the next item from the queue one item ahead, so the atomic's round trip
    // overlaps the current item.  No deadlock: the unfinished item with the smallest index
    // has all its producers finished (they come earlier in the stage order), and the CTA
    // holding it either runs it or first finishes a current item with a smaller index.
    int nxt = 0;
    if (threadIdx.x == 0) nxt = atomicAdd(&ctl[0], 1);
    for (;;) {
        if (threadIdx.x == 0) {
            const int it = nxt;
            if (it < nitems) nxt = atomicAdd(&ctl[0], 1);
            int ok = 1;
            if (it < nitems) {
                const int dp = deps[items[it].pass];
                if (dp >= 0) {
                    const int need = ntiles[dp];
                    long long k = 0;
                    while (ld_acquire(&ctl[2 + dp]) < need) {
                        if (ld_acquire(&ctl[1]) != 0) { ok = 0; break; }
                        if (++k > spin_limit) {
                            atomicExch(&ctl[1], 1);
                            ok = 0;
                            break;
                        }
                        __nanosleep(128);
                    }
                }
            }
            s_item = it;
            s_ok = ok;
        }
        __syncthreads();
        const int it = s_item;
        const int ok = s_ok;
        __syncthreads();
        if (it >= nitems || !ok) break;
        const BatchItem bi = items[it];
        const PassArgs *a = passes + bi.pass;
        const PassBind b = binds[bi.pass];
        const void *bufs[3] = {in, out, work};
        const void *pin = (const char *)bufs[b.in_buf] + b.in_off;
        void *pout = (char *)const_cast<void *>(bufs[b.out_buf]) + b.out_off;
        const long long line0 = (long long)bi.tile * a->G;
        if (b.fast == 1) {
            void *data = const_cast<void *>(pin);
            switch (b.n * 8 + b.ckind) {
#define FFTB_CCASE(n)                                                                                                 \
    case n * 8 + 0: batch_col_tile<n, 0>(&binds[bi.pass], data, bi.tile); break;                                     \
    case n * 8 + 1: batch_col_tile<n, 1>(&binds[bi.pass], data, bi.tile); break;                                     \
    case n * 8 + 2: batch_col_tile<n, 2>(&binds[bi.pass], data, bi.tile); break;                                     \
    case n * 8 + 3: batch_col_tile<n, 3>(&binds[bi.pass], data, bi.tile); break;                                     \
    case n * 8 + 4: batch_col_tile<n, 4>(&binds[bi.pass], data, bi.tile); break;
                FFTB_BATCH_COL_LIST(FFTB_CCASE)
#undef FFTB_CCASE
            default:
                break;
            }
        } else if (b.fast == 2) {
            switch (b.n * 2 + b.ckind) {
#define FFTB_RCASE(n)                                                                                                 \
    case n * 2 + 0: batch_row_tile<n, 0>(&binds[bi.pass], pin, pout, bi.tile); break;                                 \
    case n * 2 + 1: batch_row_tile<n, 1>(&binds[bi.pass], pin, pout, bi.tile); break;
                FFTB_BATCH_ROW_LIST(FFTB_RCASE)
#undef FFTB_RCASE
            default:
                break;
            }
        } else {
            switch (b.nf) {
#define FFTB_CASE(n)                                                                                                  \
    case n:                                                                                                           \
        batch_tile<n>(a, pin, pout, line0, smem_raw);                                                                 \
        break;
                FFTB_BATCH_NF_LIST(FFTB_CASE)
#undef FFTB_CASE
            default:
                break;
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            atomicAdd(&ctl[2 + bi.pass], 1);
        }
    }
}

// Grouped form: one plain launch per (stage, line length) over the tiles of every
// transform in that group, each CTA one (pass, tile) item.  Every launch is specialised
// for its line length, so there is no register union and no dependency wait: stream
// order separates the stages.
__device__ __forceinline__ const void *batch_buf(int k, const void *in, void *out, void *work)
{
    return k == 0 ? in : (k == 1 ? (const void *)out : (const void *)work);
}

template <int NF>
__global__ void __launch_bounds__(kBatchThreads)
    batch_group_kernel(const BatchItem *__restrict__ items, const PassArgs *__restrict__ passes,
                       const PassBind *__restrict__ binds, const void *in, void *out, void *work)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const BatchItem bi = items[blockIdx.x];
    const PassArgs &a = passes[bi.pass];
    const PassBind b = binds[bi.pass];
    const void *pin = (const char *)batch_buf(b.in_buf, in, out, work) + b.in_off;
    void *pout = (char *)const_cast<void *>(batch_buf(b.out_buf, in, out, work)) + b.out_off;
    pass_body<float, NF, false, false>(a, pin, pout, (long long)bi.tile * a.G, smem_raw);
}

const void *batch_group_fn(int nf)
{
    switch (nf) {
#define FFTB_CASE(n)                                                                                                  \
    case n:                                                                                                           \
        return (const void *)&batch_group_kernel<n>;
        FFTB_BATCH_NF_LIST(FFTB_CASE)
#undef FFTB_CASE
    default:
        return nullptr;
    }
}

bool batch_nf_supported(int nf)
{
    switch (nf) {
#define FFTB_CASE(n) case n:
        FFTB_BATCH_NF_LIST(FFTB_CASE)
#undef FFTB_CASE
        return true;
    default:
        return false;
    }
}

// Raises a kernel's dynamic shared-memory limit to the most the device allows beside its
// static shared memory.  The limit belongs to the kernel, not to one plan: setting it to
// one plan's need could lower it under the launches of another plan.
cudaError_t raise_smem_limit(const void *fn)
{
    int dev = 0, optin = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaFuncAttributes fa;
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, fn);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
    return e;
}

int floor_pow2(int v)
{
    int p = 1;
    while (p * 2 <= v) p *= 2;
    return p;
}

enum BatchOp { OP_FORWARD = 0, OP_BACKWARD = 1, OP_ROUNDTRIP = 2, OP_POISSON = 3, OP_COUNT = 4 };

struct OpPlan {
    bool built = false;
    double sign = 0.0;               // Poisson sign the plan was built for
    Program seq;                     // every pass of every transform, in transform order
    int npasses = 0, nitems = 0, nstages = 0;
    size_t smem = 0;
    void *blob = nullptr;            // device: items, passes, binds, deps, ntiles
    BatchItem *d_items = nullptr;
    PassArgs *d_passes = nullptr;
    PassBind *d_binds = nullptr;
    int *d_deps = nullptr, *d_ntiles = nullptr;
    int *d_ctl = nullptr;
    int grid = 0;
    // grouped form: the items ordered by (stage, line length), one launch per group
    struct Group {
        int offset, count, nf;
        size_t smem;
        // x and y stages of lengths with a column kernel: one grouped column-kernel launch
        // over count tiles (XGroupItem offset ..) instead of the pass items
        bool xcol = false;
        bool zrow = false;    // z stage as one grouped row-pair launch (RowGroupItem offset ..)
        int in_buf = B_IN, out_buf = B_OUT;
        int ckind = 0;        // col_group kind: 0/1/2 x forward / inverse / sandwich, 3/4 y
        int buf = B_WORK;     // the buffer holding the spectra (in place)
        void *roots = nullptr;
        int ep_mode = 0;      // the sandwich's multiply (the pass epilogue)
        double ep_scale = 1.0, ep_sign = -1.0;
    };
    std::vector<Group> groups;
    BatchItem *d_gitems = nullptr;
    XGroupItem *d_xitems = nullptr;
    RowGroupItem *d_ritems = nullptr;
    // CUDA graph of the persistent launch (mode 2) or of the grouped launches (mode 4)
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    int g_mode = 0;
    const void *g_in = nullptr;
    void *g_out = nullptr, *g_work = nullptr;
    bool persistent_ok = false;
};

} // namespace
} // namespace fftb

using namespace fftb;

struct fftb_batch_s {
    int dtype = 0, count = 0;
    std::vector<long long> dims;              // nx, ny, nz per transform
    std::vector<long long> roff, soff;        // element offsets into the packed real / spectrum arrays
    long long rtotal = 0, stotal = 0;
    OpPlan ops[OP_COUNT];
    void *work = nullptr;
    bool own_work = false;
    cudaStream_t stream = 0;
    int tiles_scale = 1;                      // autotune knob: tiles of G/tiles_scale lines
    int ctas_per_sm = 0;                      // autotune knob: 0 = occupancy limit
    long long wait_limit = kSpinLimit;        // polls of a dependency wait before the error flag
};

namespace {

// The pass list of transform i for op, with buffers: in/out are the packed user
// arrays, work holds the packed spectrum for the round trip and the Poisson solve.
int transform_passes(fftb_batch_s *b, int i, int op, double sign, std::vector<AxisPass> &out)
{
    const long long nx = b->dims[3 * i], ny = b->dims[3 * i + 1], nz = b->dims[3 * i + 2];
    const long long nzh = nz / 2 + 1, C3 = ny * nzh;
    const long long ro = b->roff[i], so = b->soff[i];
    auto mk = [](int kind, long long n, long long is, long long os, std::vector<Dim> batch, int ib, int ob,
                 long long ibase, long long obase) {
        AxisPass p;
        p.kind = kind;
        p.n = (int)n;
        p.is = is;
        p.os = os;
        p.batch = std::move(batch);
        p.in_buf = ib;
        p.out_buf = ob;
        p.in_base = ibase;
        p.out_base = obase;
        return p;
    };
    const double invN = 1.0 / (double)(nx * ny * nz);
    if (op == OP_FORWARD) {
        out.push_back(mk(K_R2C, nz, 1, 1, {Dim{ny, nz, nzh, 1}, Dim{nx, ny * nz, C3, 0}}, B_IN, B_OUT, ro, so));
        out.push_back(mk(K_C2C_FWD, ny, nzh, nzh, {Dim{nzh, 1, 1, 2}, Dim{nx, C3, C3, 0}}, B_OUT, B_OUT, so, so));
        out.push_back(mk(K_C2C_FWD, nx, C3, C3, {Dim{nzh, 1, 1, 2}, Dim{ny, nzh, nzh, 1}}, B_OUT, B_OUT, so, so));
    } else if (op == OP_BACKWARD) {
        out.push_back(mk(K_C2C_INV, nx, C3, C3, {Dim{nzh, 1, 1, 2}, Dim{ny, nzh, nzh, 1}}, B_IN, B_IN, so, so));
        out.push_back(mk(K_C2C_INV, ny, nzh, nzh, {Dim{nzh, 1, 1, 2}, Dim{nx, C3, C3, 0}}, B_IN, B_IN, so, so));
        AxisPass c = mk(K_C2R, nz, 1, 1, {Dim{ny, nzh, nz, 1}, Dim{nx, C3, ny * nz, 0}}, B_IN, B_OUT, so, ro);
        c.ep_mode = EP_SCALE;
        c.ep_scale = invN;
        out.push_back(c);
    } else {
        out.push_back(mk(K_R2C, nz, 1, 1, {Dim{ny, nz, nzh, 1}, Dim{nx, ny * nz, C3, 0}}, B_IN, B_WORK, ro, so));
        out.push_back(mk(K_C2C_FWD, ny, nzh, nzh, {Dim{nzh, 1, 1, 2}, Dim{nx, C3, C3, 0}}, B_WORK, B_WORK, so, so));
        AxisPass s = mk(K_SANDWICH, nx, C3, C3, {Dim{nzh, 1, 1, 2}, Dim{ny, nzh, nzh, 1}}, B_WORK, B_WORK, so, so);
        s.ep_mode = EP_SCALE | (op == OP_POISSON ? EP_POISSON : 0);
        s.ep_scale = 1.0;
        s.ep_sign = sign;
        s.ep_axes = {EpAxis{1, -1, (int)nx, 0}, EpAxis{0, 1, (int)ny, 0}, EpAxis{0, 2, (int)nz, 1}};
        out.push_back(s);
        out.push_back(mk(K_C2C_INV, ny, nzh, nzh, {Dim{nzh, 1, 1, 2}, Dim{nx, C3, C3, 0}}, B_WORK, B_WORK, so, so));
        AxisPass c = mk(K_C2R, nz, 1, 1, {Dim{ny, nzh, nz, 1}, Dim{nx, C3, ny * nz, 0}}, B_WORK, B_OUT, so, ro);
        c.ep_mode = EP_SCALE;
        c.ep_scale = invN;
        out.push_back(c);
    }
    return FFTB_SUCCESS;
}

void free_plan(OpPlan &p)
{
    if (p.gexec) cudaGraphExecDestroy(p.gexec);
    if (p.graph) cudaGraphDestroy(p.graph);
    if (p.blob) cudaFree(p.blob);
    p = OpPlan();
}

int build_plan(fftb_batch_s *b, int op, double sign)
{
    OpPlan &P = b->ops[op];
    if (P.built && (op != OP_POISSON || P.sign == sign)) return FFTB_SUCCESS;
    free_plan(P);
    P.sign = sign;
    // per-transform programs (the sequential mode runs them as they are)
    std::vector<std::vector<int>> tpass(b->count);
    for (int i = 0; i < b->count; ++i) {
        std::vector<AxisPass> ps;
        int st = transform_passes(b, i, op, sign, ps);
        if (st != FFTB_SUCCESS) return st;
        for (const AxisPass &p : ps) {
            tpass[i].push_back((int)P.seq.launches.size());
            if ((st = program_add(P.seq, b->dtype, p)) != FFTB_SUCCESS) return st;
        }
    }
    P.nstages = (int)tpass[0].size();
    P.npasses = (int)P.seq.launches.size();
    // persistent form: the same passes with G capped to kBatchThreads threads per tile
    P.persistent_ok = (b->dtype == FFTB_F32);
    std::vector<PassArgs> args(P.npasses);
    std::vector<PassBind> binds(P.npasses);
    std::vector<int> deps(P.npasses, -1), ntiles(P.npasses, 0);
    size_t smem = 0;
    std::vector<size_t> pass_smem(P.npasses, 0);
    // per stage: the column kind (x passes step C3 = ny * nzh between points, y passes nzh) or
    // the z direction (R2C of contiguous real rows, scaled C2R back to them) of the stages the
    // fused path's tiles can run (f32, in place for the column stages); the same for every
    // transform, taken from the first
    std::vector<int> st_ckind(P.nstages, -1), st_zdir(P.nstages, -1);
    for (int s = 0; s < P.nstages; ++s) {
        const Launch &L0 = P.seq.launches[tpass[0][s]];
        const PassArgs &a0 = L0.args;
        if (b->dtype != FFTB_F32 || L0.longline != nullptr || a0.bs_n != 0) continue;
        const long long ny0 = b->dims[1], nzh0 = b->dims[2] / 2 + 1;
        const bool inplace = L0.in_buf == L0.out_buf && L0.in_off_bytes == L0.out_off_bytes;
        if (inplace && ny0 > 1) {
            if (a0.kind == K_SANDWICH && a0.is == ny0 * nzh0) st_ckind[s] = 2;
            else if ((a0.kind == K_C2C_FWD || a0.kind == K_C2C_INV) && a0.ep_mode == 0)
                st_ckind[s] = a0.is == ny0 * nzh0 ? (a0.kind == K_C2C_FWD ? 0 : 1)
                                                  : (a0.is == nzh0 ? (a0.kind == K_C2C_FWD ? 3 : 4) : -1);
        }
        if (a0.half && a0.is == 1 && a0.os == 1) {
            if (a0.kind == K_R2C && a0.ep_mode == 0) st_zdir[s] = 0;
            else if (a0.kind == K_C2R && (a0.ep_mode & ~EP_SCALE) == 0) st_zdir[s] = 1;
        }
    }
    std::vector<int> stage_of(P.npasses, 0), trans_of(P.npasses, 0);
    std::map<int, void *> roots_of;
    for (int i = 0; i < b->count; ++i)
        for (int s = 0; s < P.nstages; ++s) {
            stage_of[tpass[i][s]] = s;
            trans_of[tpass[i][s]] = i;
        }
    for (int p = 0; p < P.npasses; ++p) {
        const Launch &L = P.seq.launches[p];
        PassArgs a = L.args;
        const int T = L.k.threads_per_line;
        if (!batch_nf_supported(L.k.nf) || a.bs_n != 0) P.persistent_ok = false;  // chirp-z lines: sequential
        int G = std::min(a.G, floor_pow2(std::max(1, kBatchThreads / T)));
        G = std::max(1, G / b->tiles_scale);
        a.G = G;
        int gs = 0;
        while ((1 << gs) < G) ++gs;
        a.gshift = gs;
        a.pair_io = L.pair_candidate ? 1 : 0;  // buffers are 16-byte aligned (checked at execution)
        const size_t cb = complex_bytes(b->dtype);
        const size_t sm = (a.tw_smem ? (size_t)a.ntw * cb : 0) + (size_t)G * 32 + (size_t)G * L.k.line_pitch * cb;
        smem = std::max(smem, sm);
        pass_smem[p] = sm;
        args[p] = a;
        PassBind pb = {};
        pb.in_buf = L.in_buf;
        pb.out_buf = L.out_buf;
        pb.in_off = (long long)L.in_off_bytes;
        pb.out_off = (long long)L.out_off_bytes;
        pb.nf = L.k.nf;
        ntiles[p] = (int)((a.nlines + G - 1) / G);
        // the fused path's tile for this pass, where the stage has one for this length
        const int st = stage_of[p], ti = trans_of[p];
        const long long nx = b->dims[3 * ti], ny = b->dims[3 * ti + 1], nz = b->dims[3 * ti + 2];
        const int FZ = st_zdir[st] >= 0 ? row_group_tile_pairs(b->dtype, 2 * L.k.nf) : 0;
        const int W = FZ == 0 && st_ckind[st] >= 0 ? col_group_tile_lines(b->dtype, L.k.nf) : 0;
        void *roots = nullptr;
        // the kernels' set-up (shared-memory limit, root table) once per kind and length
        auto prepared = [&](int key, auto prepare) -> int {
            auto it = roots_of.find(key);
            if (it != roots_of.end()) {
                roots = it->second;
                return FFTB_SUCCESS;
            }
            int rs = prepare();
            if (rs == FFTB_SUCCESS) roots_of[key] = roots;
            return rs;
        };
        if (FZ > 0) {
            int rs = prepared(100000 + st_zdir[st] * 1000 + 2 * L.k.nf,
                              [&] { return row_group_prepare(b->dtype, st_zdir[st], 2 * L.k.nf, &roots); });
            if (rs != FFTB_SUCCESS) return rs;
            pb.fast = 2;
            pb.ckind = st_zdir[st];
            pb.n = 2 * L.k.nf;
            pb.lines = (int)(nx * ny);
            pb.scale = st_zdir[st] == 1 && (a.ep_mode & EP_SCALE) ? (float)a.ep_scale : 1.0f;
            pb.roots = (const float2 *)roots;
            ntiles[p] = (int)(((nx * ny + 1) / 2 + FZ - 1) / FZ);
            smem = std::max(smem, row_group_smem(pb.n));
        } else if (W > 0) {
            int rs = prepared(st_ckind[st] * 1000 + L.k.nf,
                              [&] { return col_group_prepare(b->dtype, st_ckind[st], L.k.nf, &roots); });
            if (rs != FFTB_SUCCESS) return rs;
            pb.fast = 1;
            pb.ckind = st_ckind[st];
            pb.n = L.k.nf;
            pb.lines = (int)((st_ckind[st] <= 2 ? ny : nx) * (nz / 2 + 1));
            pb.ny = (int)ny;
            pb.nz = (int)nz;
            pb.scale = (float)a.ep_scale;
            pb.sign = (float)a.ep_sign;
            pb.ep_mode = a.ep_mode;
            pb.roots = (const float2 *)roots;
            ntiles[p] = (pb.lines + W - 1) / W;
            smem = std::max(smem, col_group_smem(pb.n));
        }
        binds[p] = pb;
    }
    for (int i = 0; i < b->count; ++i)
        for (int s = 1; s < P.nstages; ++s) deps[tpass[i][s]] = tpass[i][s - 1];
    std::vector<BatchItem> items;
    for (int s = 0; s < P.nstages; ++s)
        for (int i = 0; i < b->count; ++i) {
            const int p = tpass[i][s];
            for (int t = 0; t < ntiles[p]; ++t) items.push_back(BatchItem{p, t});
        }
    P.nitems = (int)items.size();
    P.smem = smem;
    // grouped order: within each stage, the items of each line length together; the x and y
    // stages of lengths that have a column kernel run as one grouped column-kernel launch
    // each (the fused 3D path's register-resident column FFT, tiles of W lines)
    std::vector<BatchItem> gitems;
    std::vector<XGroupItem> xitems;
    std::vector<RowGroupItem> ritems;
    gitems.reserve(items.size());
    for (int s = 0; s < P.nstages; ++s) {
        std::vector<int> nfs;
        for (int i = 0; i < b->count; ++i) nfs.push_back(binds[tpass[i][s]].nf);
        std::sort(nfs.begin(), nfs.end());
        nfs.erase(std::unique(nfs.begin(), nfs.end()), nfs.end());
        const int ckind = st_ckind[s], zdir = st_zdir[s];
        for (int nf : nfs) {
            // nf is the half length for the z stages: the row length is 2 nf
            const int FZ = zdir >= 0 ? row_group_tile_pairs(b->dtype, 2 * nf) : 0;
            if (FZ > 0) {
                OpPlan::Group g{(int)ritems.size(), 0, nf, 0};
                g.zrow = true;
                const Launch &L0 = P.seq.launches[tpass[0][s]];
                g.in_buf = L0.in_buf;
                g.out_buf = L0.out_buf;
                g.ckind = zdir;
                int st = row_group_prepare(b->dtype, zdir, 2 * nf, &g.roots);
                if (st != FFTB_SUCCESS) return st;
                for (int i = 0; i < b->count; ++i) {
                    const long long nx = b->dims[3 * i], ny = b->dims[3 * i + 1], nz = b->dims[3 * i + 2];
                    if (nz != 2 * nf) continue;
                    const Launch &L = P.seq.launches[tpass[i][s]];
                    const long long roff = (long long)((zdir == 0 ? L.in_off_bytes : L.out_off_bytes) / real_bytes(b->dtype));
                    const long long soff =
                        (long long)((zdir == 0 ? L.out_off_bytes : L.in_off_bytes) / complex_bytes(b->dtype));
                    const long long rows = nx * ny, pairs = (rows + 1) / 2;
                    const float sc = zdir == 1 && (L.args.ep_mode & EP_SCALE) ? (float)L.args.ep_scale : 1.0f;
                    for (long long t = 0; t < (pairs + FZ - 1) / FZ; ++t)
                        ritems.push_back(RowGroupItem{roff, soff, (int)rows, (int)t, sc});
                }
                g.count = (int)ritems.size() - g.offset;
                if (g.count > 0) P.groups.push_back(g);
                continue;
            }
            const int W = ckind >= 0 ? col_group_tile_lines(b->dtype, nf) : 0;
            if (W > 0) {
                OpPlan::Group g{(int)xitems.size(), 0, nf, 0};
                g.xcol = true;
                g.ckind = ckind;
                const Launch &L0 = P.seq.launches[tpass[0][s]];
                g.buf = L0.in_buf;
                g.ep_mode = L0.args.ep_mode;
                g.ep_scale = L0.args.ep_scale;
                g.ep_sign = L0.args.ep_sign;
                int st = col_group_prepare(b->dtype, ckind, nf, &g.roots);
                if (st != FFTB_SUCCESS) return st;
                for (int i = 0; i < b->count; ++i) {
                    const long long nx = b->dims[3 * i], ny = b->dims[3 * i + 1], nz = b->dims[3 * i + 2];
                    if ((ckind <= 2 ? nx : ny) != nf) continue;
                    const Launch &L = P.seq.launches[tpass[i][s]];
                    const long long lines = (ckind <= 2 ? ny : nx) * (nz / 2 + 1);
                    for (long long t = 0; t < (lines + W - 1) / W; ++t)
                        xitems.push_back(XGroupItem{(long long)(L.in_off_bytes / complex_bytes(b->dtype)),
                                                    (int)lines, (int)t, (int)ny, (int)nz});
                }
                g.count = (int)xitems.size() - g.offset;
                if (g.count > 0) P.groups.push_back(g);
                continue;
            }
            OpPlan::Group g{(int)gitems.size(), 0, nf, 0};
            for (int i = 0; i < b->count; ++i) {
                const int p = tpass[i][s];
                if (binds[p].nf != nf) continue;
                g.smem = std::max(g.smem, pass_smem[p]);
                for (int t = 0; t < ntiles[p]; ++t) gitems.push_back(BatchItem{p, t});
            }
            g.count = (int)gitems.size() - g.offset;
            if (g.count > 0) P.groups.push_back(g);
        }
    }
    if (P.persistent_ok) {
        auto al = [](size_t v) { return (v + 255) & ~(size_t)255; };
        const size_t s_items = al(items.size() * sizeof(BatchItem)), s_args = al(args.size() * sizeof(PassArgs)),
                     s_binds = al(binds.size() * sizeof(PassBind)), s_deps = al(deps.size() * sizeof(int)),
                     s_nt = al(ntiles.size() * sizeof(int)), s_ctl = al((2 + P.npasses) * sizeof(int));
        const size_t s_gitems = al(gitems.size() * sizeof(BatchItem));
        const size_t s_xitems = al(xitems.size() * sizeof(XGroupItem));
        const size_t s_ritems = al(ritems.size() * sizeof(RowGroupItem));
        const size_t tot = s_items + s_args + s_binds + s_deps + s_nt + s_ctl + s_gitems + s_xitems + s_ritems;
        cudaError_t e = cudaMalloc(&P.blob, tot);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return FFTB_ERROR_ALLOC;
        }
        char *q = (char *)P.blob;
        P.d_items = (BatchItem *)q; q += s_items;
        P.d_passes = (PassArgs *)q; q += s_args;
        P.d_binds = (PassBind *)q; q += s_binds;
        P.d_deps = (int *)q; q += s_deps;
        P.d_ntiles = (int *)q; q += s_nt;
        P.d_ctl = (int *)q; q += s_ctl;
        P.d_gitems = (BatchItem *)q; q += s_gitems;
        P.d_xitems = (XGroupItem *)q; q += s_xitems;
        P.d_ritems = (RowGroupItem *)q;
        e = cudaMemcpy(P.d_items, items.data(), items.size() * sizeof(BatchItem), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(P.d_passes, args.data(), args.size() * sizeof(PassArgs), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(P.d_binds, binds.data(), binds.size() * sizeof(PassBind), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(P.d_deps, deps.data(), deps.size() * sizeof(int), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(P.d_ntiles, ntiles.data(), ntiles.size() * sizeof(int), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemset(P.d_ctl, 0, (2 + P.npasses) * sizeof(int));
        if (e == cudaSuccess)
            e = cudaMemcpy(P.d_gitems, gitems.data(), gitems.size() * sizeof(BatchItem), cudaMemcpyHostToDevice);
        if (e == cudaSuccess && !xitems.empty())
            e = cudaMemcpy(P.d_xitems, xitems.data(), xitems.size() * sizeof(XGroupItem), cudaMemcpyHostToDevice);
        if (e == cudaSuccess && !ritems.empty())
            e = cudaMemcpy(P.d_ritems, ritems.data(), ritems.size() * sizeof(RowGroupItem), cudaMemcpyHostToDevice);
        // the limit is per kernel, not per plan: raise it to the maximum once, so a later
        // plan with a smaller need cannot lower it under an earlier plan's launches
        for (const OpPlan::Group &g : P.groups)
            if (e == cudaSuccess && !g.xcol && !g.zrow && g.smem > 48 * 1024)
                e = raise_smem_limit(batch_group_fn(g.nf));
        if (e != cudaSuccess) return set_status_from_cuda(e);
        if (smem > 48 * 1024) {
            e = raise_smem_limit((const void *)batch_persistent_kernel);
            if (e != cudaSuccess) return set_status_from_cuda(e);
        }
        int dev = 0, sms = 0, occ = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, (const void *)batch_persistent_kernel, kBatchThreads,
                                                          smem);
        if (e != cudaSuccess) return set_status_from_cuda(e);
        if (occ < 1) return FFTB_ERROR_UNSUPPORTED_SIZE;
        const int per = b->ctas_per_sm > 0 ? std::min(b->ctas_per_sm, occ) : occ;
        P.grid = std::max(1, std::min(sms * per, P.nitems));
    }
    P.built = true;
    return FFTB_SUCCESS;
}

int launch_persistent(OpPlan &P, const void *in, void *out, void *work, cudaStream_t s, long long wait_limit)
{
    cudaError_t e = cudaMemsetAsync(P.d_ctl, 0, (2 + P.npasses) * sizeof(int), s);
    if (e != cudaSuccess) return set_status_from_cuda(e);
    batch_persistent_kernel<<<P.grid, kBatchThreads, P.smem, s>>>(P.d_items, P.nitems, P.d_passes, P.d_binds,
                                                                 P.d_deps, P.d_ntiles, P.d_ctl, in, out, work,
                                                                 wait_limit);
    return set_status_from_cuda(cudaGetLastError());
}

int launch_groups(OpPlan &P, const void *in, void *out, void *work, cudaStream_t s)
{
    const void *bufs[3] = {in, out, work};
    for (const OpPlan::Group &g : P.groups) {
        if (g.zrow) {
            int st = launch_row_group(g.ckind, 2 * g.nf, P.d_ritems + g.offset, g.count, bufs[g.in_buf],
                                      const_cast<void *>(bufs[g.out_buf]), g.roots, s);
            if (st != FFTB_SUCCESS) return st;
            continue;
        }
        if (g.xcol) {
            void *data = g.buf == B_IN ? const_cast<void *>(in) : (g.buf == B_OUT ? out : work);
            int st = launch_col_group(g.ckind, g.nf, P.d_xitems + g.offset, g.count, data, g.roots, g.ep_mode,
                                      g.ep_scale, g.ep_sign, s);
            if (st != FFTB_SUCCESS) return st;
            continue;
        }
        const BatchItem *items = P.d_gitems + g.offset;
        const PassArgs *passes = P.d_passes;
        const PassBind *binds = P.d_binds;
        void *args[] = {&items, &passes, &binds, &in, &out, &work};
        cudaError_t e = cudaLaunchKernel(batch_group_fn(g.nf), dim3((unsigned)g.count), dim3(kBatchThreads), args,
                                         g.smem, s);
        if (e != cudaSuccess) return set_status_from_cuda(e);
    }
    return FFTB_SUCCESS;
}

int ensure_work(fftb_batch_s *b)
{
    if (b->work) return FFTB_SUCCESS;
    void *p = nullptr;
    cudaError_t e = cudaMalloc(&p, (size_t)b->stotal * complex_bytes(b->dtype));
    if (e != cudaSuccess) {
        cudaGetLastError();
        return FFTB_ERROR_ALLOC;
    }
    b->work = p;
    b->own_work = true;
    return FFTB_SUCCESS;
}

} // namespace

namespace fftb {
int batch_identity(const fftb_batch_s *b, int *dtype, int *count, const long long **dims, int *tiles_scale,
                   int *ctas_per_sm, void **stream)
{
    if (!b) return FFTB_ERROR_INVALID_HANDLE;
    *stream = (void *)b->stream;
    *dtype = b->dtype;
    *count = b->count;
    *dims = b->dims.data();
    *tiles_scale = b->tiles_scale;
    *ctas_per_sm = b->ctas_per_sm;
    return FFTB_SUCCESS;
}
} // namespace fftb

extern "C" {

int fftb_batch_create(int dtype, int count, const long long *dims, fftb_batch *out)
{
    if (!out) return FFTB_ERROR_INVALID_VALUE;
    *out = nullptr;
    if ((dtype != FFTB_F32 && dtype != FFTB_F64) || count < 1 || !dims) return FFTB_ERROR_INVALID_VALUE;
    for (int i = 0; i < 3 * count; ++i)
        if (dims[i] < 2 || dims[i] > 4096) return FFTB_ERROR_INVALID_VALUE;
    fftb_batch_s *b = new (std::nothrow) fftb_batch_s();
    if (!b) return FFTB_ERROR_ALLOC;
    b->dtype = dtype;
    b->count = count;
    b->dims.assign(dims, dims + 3 * count);
    for (int i = 0; i < count; ++i) {
        const long long nx = dims[3 * i], ny = dims[3 * i + 1], nz = dims[3 * i + 2];
        b->roff.push_back(b->rtotal);
        b->soff.push_back(b->stotal);
        // keep every transform's arrays 16-byte aligned
        b->rtotal += (nx * ny * nz + 3) & ~3LL;
        b->stotal += (nx * ny * (nz / 2 + 1) + 1) & ~1LL;
    }
    *out = b;
    return FFTB_SUCCESS;
}

int fftb_batch_destroy(fftb_batch b)
{
    if (!b) return FFTB_ERROR_INVALID_HANDLE;
    for (OpPlan &p : b->ops) free_plan(p);
    if (b->own_work && b->work) cudaFree(b->work);
    delete b;
    return FFTB_SUCCESS;
}

int fftb_batch_layout(fftb_batch b, long long *real_offsets, long long *spectrum_offsets, long long *real_total,
                      long long *spectrum_total)
{
    if (!b) return FFTB_ERROR_INVALID_HANDLE;
    for (int i = 0; i < b->count; ++i) {
        if (real_offsets) real_offsets[i] = b->roff[i];
        if (spectrum_offsets) spectrum_offsets[i] = b->soff[i];
    }
    if (real_total) *real_total = b->rtotal;
    if (spectrum_total) *spectrum_total = b->stotal;
    return FFTB_SUCCESS;
}

int fftb_batch_work_size(fftb_batch b, size_t *bytes)
{
    if (!b || !bytes) return FFTB_ERROR_INVALID_HANDLE;
    *bytes = (size_t)b->stotal * complex_bytes(b->dtype);
    return FFTB_SUCCESS;
}

int fftb_batch_set_work_area(fftb_batch b, void *work)
{
    if (!b) return FFTB_ERROR_INVALID_HANDLE;
    if ((uintptr_t)work % 256) return FFTB_ERROR_MISALIGNED;
    if (b->own_work && b->work) cudaFree(b->work);
    b->own_work = false;
    b->work = work;
    for (OpPlan &p : b->ops) p.g_work = nullptr;  // graphs bound to the old area are recaptured
    return FFTB_SUCCESS;
}

int fftb_batch_set_stream(fftb_batch b, void *stream)
{
    if (!b) return FFTB_ERROR_INVALID_HANDLE;
    b->stream = (cudaStream_t)stream;
    return FFTB_SUCCESS;
}

int fftb_batch_set_tuning(fftb_batch b, int tiles_scale, int ctas_per_sm)
{
    if (!b || tiles_scale < 1 || ctas_per_sm < 0) return FFTB_ERROR_INVALID_VALUE;
    b->tiles_scale = tiles_scale;
    b->ctas_per_sm = ctas_per_sm;
    for (OpPlan &p : b->ops) free_plan(p);
    return FFTB_SUCCESS;
}

int fftb_batch_set_wait_limit(fftb_batch b, long long polls)
{
    if (!b || polls < 0) return FFTB_ERROR_INVALID_VALUE;
    b->wait_limit = polls == 0 ? kSpinLimit : polls;
    for (OpPlan &p : b->ops) free_plan(p);  // captured graphs hold the old limit
    return FFTB_SUCCESS;
}

// The persistent kernel on a one-item work list whose producer pass has no items: its
// dependency wait can only end by running out of polls, which must raise the error flag and
// return.  Checks the bounded-wait path without faulting or hanging anything.
int fftb_batch_wait_selftest(long long polls, int *error_flag)
{
    if (!error_flag || polls < 1) return FFTB_ERROR_INVALID_VALUE;
    *error_flag = 0;
    const BatchItem item = {1, 0};
    const int deps[2] = {-1, 0}, ntiles[2] = {1, 1};
    const size_t off_args = 256, off_binds = off_args + 2 * sizeof(PassArgs), off_deps = off_binds + 2 * sizeof(PassBind);
    const size_t off_nt = off_deps + 64, off_ctl = off_nt + 64, total = off_ctl + 64;
    char *blob = nullptr;
    cudaError_t e = cudaMalloc(&blob, total);
    if (e != cudaSuccess) return set_status_from_cuda(e);
    if (e == cudaSuccess) e = cudaMemset(blob, 0, total);
    if (e == cudaSuccess) e = cudaMemcpy(blob, &item, sizeof(item), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(blob + off_deps, deps, sizeof(deps), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(blob + off_nt, ntiles, sizeof(ntiles), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        int *ctl = (int *)(blob + off_ctl);
        batch_persistent_kernel<<<1, kBatchThreads, 0>>>((const BatchItem *)blob, 1, (const PassArgs *)(blob + off_args),
                                                         (const PassBind *)(blob + off_binds),
                                                         (const int *)(blob + off_deps), (const int *)(blob + off_nt),
                                                         ctl, nullptr, nullptr, nullptr, polls);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        if (e == cudaSuccess) e = cudaMemcpy(error_flag, ctl + 1, sizeof(int), cudaMemcpyDeviceToHost);
    }
    cudaFree(blob);
    return set_status_from_cuda(e);
}

int fftb_batch_exec(fftb_batch b, int op, const void *in, void *out, double sign, int mode)
{
    if (!b) return FFTB_ERROR_INVALID_HANDLE;
    if (op < 0 || op >= OP_COUNT || !in || !out || mode < 0 || mode > 4) return FFTB_ERROR_INVALID_VALUE;
    int st = build_plan(b, op, sign);
    if (st != FFTB_SUCCESS) return st;
    OpPlan &P = b->ops[op];
    void *work = nullptr;
    if (op == OP_ROUNDTRIP || op == OP_POISSON) {
        if ((st = ensure_work(b)) != FFTB_SUCCESS) return st;
        work = b->work;
    }
    if (mode == 0 || !P.persistent_ok) {
        // one transform after another, each with its own pass launches
        return program_exec(P.seq, const_cast<void *>(in), out, work, b->stream);
    }
    if ((uintptr_t)in % 16 || (uintptr_t)out % 16 || (uintptr_t)work % 16) return FFTB_ERROR_MISALIGNED;
    if (mode == 1) return launch_persistent(P, in, out, work, b->stream, b->wait_limit);
    if (mode == 3) return launch_groups(P, in, out, work, b->stream);
    // modes 2 and 4: replay the captured graph (captured on first use of this binding)
    if (!P.gexec || P.g_mode != mode || P.g_in != in || P.g_out != out || P.g_work != work) {
        if (P.gexec) cudaGraphExecDestroy(P.gexec);
        if (P.graph) cudaGraphDestroy(P.graph);
        P.gexec = nullptr;
        P.graph = nullptr;
        cudaStream_t cap;
        cudaError_t e = cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking);
        if (e != cudaSuccess) return set_status_from_cuda(e);
        e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            st = mode == 2 ? launch_persistent(P, in, out, work, cap, b->wait_limit) : launch_groups(P, in, out, work, cap);
            cudaGraph_t g = nullptr;
            e = cudaStreamEndCapture(cap, &g);
            if (st == FFTB_SUCCESS && e == cudaSuccess) {
                P.graph = g;
                e = cudaGraphInstantiate(&P.gexec, g, 0);
            } else if (g) {
                cudaGraphDestroy(g);
            }
        }
        cudaStreamDestroy(cap);
        if (st != FFTB_SUCCESS) return st;
        if (e != cudaSuccess) return set_status_from_cuda(e);
        P.g_mode = mode;
        P.g_in = in;
        P.g_out = out;
        P.g_work = work;
    }
    return set_status_from_cuda(cudaGraphLaunch(P.gexec, b->stream));
}

int fftb_batch_status(fftb_batch b, int op, int *error_flag)
{
    if (!b || !error_flag || op < 0 || op >= OP_COUNT) return FFTB_ERROR_INVALID_HANDLE;
    *error_flag = 0;
    OpPlan &P = b->ops[op];
    if (!P.built || !P.persistent_ok) return FFTB_SUCCESS;
    int v = 0;
    cudaError_t e = cudaMemcpy(&v, P.d_ctl + 1, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return set_status_from_cuda(e);
    *error_flag = v;
    return FFTB_SUCCESS;
}

int fftb_batch_describe(fftb_batch b, int op, double sign, int *passes, int *items, int *grid, int *persistent)
{
    if (!b || op < 0 || op >= OP_COUNT) return FFTB_ERROR_INVALID_HANDLE;
    int st = build_plan(b, op, sign);
    if (st != FFTB_SUCCESS) return st;
    const OpPlan &P = b->ops[op];
    if (passes) *passes = P.npasses;
    if (items) *items = P.nitems;
    if (grid) *grid = P.grid;
    if (persistent) *persistent = P.persistent_ok ? 1 : 0;
    return FFTB_SUCCESS;
}

} // extern "C"
