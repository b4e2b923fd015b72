// fftb_fused3d.cu -- specialised 3D kernels for power-of-two sizes.
//
// A 3D R2C + C2R round trip (and the Poisson solve between them) runs as three
// kernels instead of the reference's cuFFT 3D plan plus separate multiply and
// scale kernels:
//
//   plane_fwd  per x-plane: R2C of every z row, then the FFT of every kz column
//              over y; writes the plane [ky][kz] of the spectrum.
//   xcol       per tile of W spectrum columns (ky,kz): the x FFT (forward,
//              inverse, or forward -> spectral multiply -> inverse).
//   plane_inv  per x-plane: inverse FFT over y, then C2R of every row, times a
//              scale (1/N for the normalised inverse and the Poisson solve).
//
// All FFTs are register resident (fftb_regfft.cuh); shared memory holds the
// plane between the z and y stages.  A plane too large for one CTA (a 256x256
// plane is 133 KB of spectrum) is split over a cluster of 2, 4 or 8 CTAs: each CTA
// transforms a block of rows along z and owns a block of kz columns for the y
// stage, and the data that changes owner in between is pushed into the owner's
// shared memory with distributed-shared-memory stores, so no plane round-trips
// through global memory between the z and y stages.
#include <cooperative_groups.h>
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <mutex>
#include <string>

#include "../../include/fftb.h"
#include "fftb_coltile.cuh"
#include "fftb_fused3d.h"
#include "fftb_regfft.cuh"
#include "fftb_tc.cuh"

namespace cg = cooperative_groups;

namespace fftb {

// Cluster barrier split into its two halves: every CTA arrives at kernel entry and waits
// before its first distributed-shared-memory store, which guarantees that every CTA of the
// cluster has started (its shared memory exists) before any peer writes into it, while the
// stage-table build overlaps the barrier.
__device__ __forceinline__ void cluster_arrive_relaxed() { asm volatile("barrier.cluster.arrive.relaxed.aligned;\n" ::: "memory"); }
__device__ __forceinline__ void cluster_wait() { asm volatile("barrier.cluster.wait.aligned;\n" ::: "memory"); }

constexpr int kRingWaitLimit = 1 << 22;  // polls of a bounded bulk-copy wait (seconds)
__device__ int g_ring_wait_error;        // set when a bounded wait gave up (a copy never completed)

// 1D bulk copy global -> this CTA's shared memory (16-byte aligned addresses, size a
// multiple of 16), completing on `bar`
__device__ __forceinline__ void bulk_load(void *dst, const void *src, unsigned bytes, unsigned long long *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// 1D bulk copy this CTA's shared memory -> global (16-byte aligned addresses, size a multiple
// of 16) in the thread's bulk group; bulk_store_wait() waits for the thread's stores to finish
__device__ __forceinline__ void bulk_store(void *dst, const void *src, unsigned bytes)
{
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;\n" ::"l"(dst), "r"(smem_u32(src)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_store_commit() { asm volatile("cp.async.bulk.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void bulk_store_wait() { asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory"); }

// ------------------------------------------------------------------ plane kernels
// Work split (CL CTAs per plane, CL in {1, 2, 4, 8}):
//   rows   : CTA c owns rows [c*M, (c+1)*M) for the z stage            (M = NY / CL)
//   columns: CTA c owns column slots [c*S, (c+1)*S) for the y stage     (S = NZ / (2 CL))
// Slot s < NZ/2 is spectrum column kz = s, except slot 0, which packs the two
// real-per-row columns kz = 0 and kz = NZ/2 as one complex column (kz=0 in the
// real part, kz=NZ/2 in the imaginary part); their y FFTs are separated by
// Hermitian symmetry (forward), or the two columns are made Hermitian in ky before
// one packed inverse FFT (inverse, where the C2R keeps only the real parts of the
// kz = 0 and NZ/2 results).  Data that changes owner
// between the stages is pushed with distributed-shared-memory stores, so no CTA
// ever reads another CTA's shared memory.
template <int NY, int NZ, int CL, int NT_> struct PlaneShapeT {
    static constexpr int NT = NT_;                           // threads per CTA

    static constexpr int M = NY / CL;                        // rows per CTA (z stage)
    static constexpr int S = NZ / (2 * CL);                  // column slots per CTA (y stage)
    static constexpr int NS = NZ / 2;                        // slots of the plane
    static constexpr int TZ = RegFFTShape<NZ>::T;
    static constexpr int TY = RegFFTShape<NY>::T;
    static constexpr int FZ = NT / TZ, FY = NT / TY;         // concurrent FFTs per stage
    static constexpr int NMAX = NY > NZ ? NY : NZ;
    // forward: y-stage plane [NY][PF], PF = 16/TY (mod 16) -> conflict-free column reads
    static constexpr int PMOD = 16 / TY;
    static constexpr int PF = S + ((PMOD - S % 16) % 16 + 16) % 16;
    static constexpr int SCR_Z = FZ * RegFFTShape<NZ>::REGION;
    static constexpr int SCR_Y = FY * RegFFTShape<NY>::REGION;
    static constexpr int SCRF = SCR_Z > SCR_Y ? SCR_Z : SCR_Y;
    // inverse: z-stage rows [M][PR] (PR odd -> conflict-free column pushes) and a
    // column-major staging area of FY columns of PC entries (PC odd, >= REGION) that
    // also serves as the FFT exchange regions
    static constexpr int PR = NS + 1;
    static constexpr int REGY = RegFFTShape<NY>::REGION > NY ? RegFFTShape<NY>::REGION : NY;
    static constexpr int PC = REGY | 1;
    static constexpr int STG = FY * PC > SCR_Z ? FY * PC : SCR_Z;
    template <typename R> static constexpr size_t smem_fwd()
    {
        return sizeof(cpx<R>) * ((size_t)NY * PF + SCRF);
    }
    template <typename R> static constexpr size_t smem_inv()
    {
        return sizeof(cpx<R>) * ((size_t)M * PR + STG + NY);  // + the staged kz = NZ/2 column
    }
    // CTAs per SM the register budget is sized for: 8-CTA clusters keep a CTA's shared
    // memory under a third of the SM's, so three CTAs (24 warps) fit when registers are
    // capped to match; smaller planes get up to 16 warps per SM as their shared memory allows
    static constexpr int minb(size_t smem)
    {
        return CL >= 8 ? 3 : ((512 / NT) * smem <= 227 * 1024 ? 512 / NT : (2 * smem <= 227 * 1024 ? 2 : 1));
    }
    static constexpr int MINB_FWD = minb(smem_fwd<float>());
    static constexpr int MINB_INV = minb(smem_inv<float>());
};

// Threads per CTA: 256, or fewer where the plane has fewer row pairs (z stage) or
// column slots (y stage) than 256 threads have FFT groups, so no group idles
template <int NY, int NZ, int CL> constexpr int plane_threads()
{
    constexpr int tz = RegFFTShape<NZ>::T * (NY / CL / 2), ty = RegFFTShape<NY>::T * (NZ / (2 * CL));
    constexpr int t = tz < ty ? tz : ty;
    return t < 256 ? (t < 32 ? 32 : t) : 256;
}
template <int NY, int NZ, int CL> using PlaneShape = PlaneShapeT<NY, NZ, CL, plane_threads<NY, NZ, CL>()>;

template <typename R, int NY, int NZ, int CL>
__global__ void __launch_bounds__(PlaneShape<NY, NZ, CL>::NT, PlaneShape<NY, NZ, CL>::MINB_FWD)
    plane_fwd_kernel(const R *__restrict__ in, cpx<R> *__restrict__ out, const cpx<R> *__restrict__ roots)
{
    using C = cpx<R>;
    using S = PlaneShape<NY, NZ, CL>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *plane = reinterpret_cast<C *>(smem_raw);   // [NY][PF]: this CTA's column slots
    C *scr = plane + NY * S::PF;
    // Row `row` starts at row * PF + skew(row).  With four threads per z FFT, the eight row
    // pairs a warp pushes at once sit 2 PF apart, which is 8 words mod 16 when PF = 4 mod 16
    // (what the y stage's column reads need), so they would share half the bank pairs; the
    // skew (4 entries on every other row pair, inside the row padding) spreads them over all
    // 16.  It is constant across the rows t + TY r one column read touches, so the column
    // reads keep their spread.
    constexpr int SKEW = (S::TZ == 4 && (2 * S::PF) % 16 == 8 && S::PF - S::S >= 4) ? 4 : 0;
    auto row_at = [&](int row) { return row * S::PF + SKEW * ((row >> 2) & 1); };
    if constexpr (CL > 1) cluster_arrive_relaxed();
    const int tid = threadIdx.x;
    const int c = (CL > 1) ? (int)cg::this_cluster().block_rank() : 0;
    const int x = (int)(blockIdx.x / CL);
    C *dst[CL];
#pragma unroll
    for (int q = 0; q < CL; ++q) dst[q] = plane;
    if constexpr (CL > 1) {
#pragma unroll
        for (int q = 0; q < CL; ++q) dst[q] = cg::this_cluster().map_shared_rank(plane, (unsigned)q);
    }
    if constexpr (CL > 1) cluster_wait();  // every peer's shared memory exists from here on

    // ---- stage z: R2C of this CTA's rows (two rows per complex FFT), pushed to the slot owners
    {
        constexpr int TZ = S::TZ, FZ = S::FZ;
        const int f = tid / TZ, t = tid - (tid / TZ) * TZ;
        C twz[16];
        load_stage_twiddles<R, NZ>(twz, roots, S::NMAX, t);
        C *reg = scr + f * RegFFTShape<NZ>::REGION;
        const R *rows = in + ((size_t)x * NY + (size_t)c * S::M) * NZ;
        // the rows of the next round are loaded into registers before this round's FFT,
        // so their memory latency overlaps the arithmetic (not with the register-capped
        // 8-CTA clusters)
        constexpr bool PREFETCH = CL < 8;
        auto load_rows = [&](int p0, C (&w)[16]) {
            const int p = p0 + f;
            const int pp = p < S::M / 2 ? p : 0;
            const R *ra = rows + (size_t)(2 * pp) * NZ;
            const R *rb = ra + NZ;
#pragma unroll
            for (int r = 0; r < 16; ++r) {
                w[r].x = ra[t + TZ * r];
                w[r].y = rb[t + TZ * r];
            }
        };
        // One CTA per plane whose rows fit one round: the CTA's rows come in as row bulk copies
        // (one per row, 16-byte aligned, pitch NZ + 4 floats so a warp's eight row pairs
        // spread over the banks) into the plane buffer, which the pushes only fill after
        // every row is read; the groups then read their row pairs from shared memory
        constexpr int ZP = NZ + 4;
        constexpr bool BULKZ = CL == 1 && sizeof(R) == 4 && S::M / 2 <= FZ && (NZ * sizeof(R)) % 16 == 0 &&
                               (size_t)S::M * ZP * sizeof(R) <= (size_t)NY * S::PF * sizeof(C);
        const bool bulkz = BULKZ && (reinterpret_cast<uintptr_t>(in) & 15) == 0;
        if (BULKZ && bulkz) {
            __shared__ __align__(8) unsigned long long zbar;
            __shared__ int zok;
            R *zst = reinterpret_cast<R *>(plane);
            if (tid == 0) {
                mbar_init(&zbar, 1);
                mbar_init_fence();
                mbar_arrive_expect_tx(&zbar, (unsigned)(S::M * NZ * sizeof(R)));
            }
            __syncthreads();  // the barrier exists before any copy completes on it
            for (int row = tid; row < S::M; row += S::NT)
                bulk_load(zst + row * ZP, rows + (size_t)row * NZ, (unsigned)(NZ * sizeof(R)), &zbar);
            if (tid == 0) zok = mbar_wait(&zbar, 0, kRingWaitLimit) ? 1 : 0;
            __syncthreads();
            if (!zok) {  // a copy never completed: flag it and leave
                if (tid == 0) atomicExch(&g_ring_wait_error, 4);
                return;
            }
        }
        C nxt[16];
        if (PREFETCH && !bulkz) load_rows(0, nxt);
#pragma unroll 1
        for (int p0 = 0; p0 < S::M / 2; p0 += FZ) {
            const int p = p0 + f;
            const bool ok = p < S::M / 2;
            const int pp = ok ? p : 0;
            C v[16];
            if (BULKZ && bulkz) {
                const R *zst = reinterpret_cast<const R *>(plane);
                const R *ra = zst + (2 * pp) * ZP, *rb = ra + ZP;
#pragma unroll
                for (int r = 0; r < 16; ++r) v[r] = mk<R>(ra[t + TZ * r], rb[t + TZ * r]);
                __syncthreads();  // every staged row is read before the pushes overwrite it
            } else if (PREFETCH) {
#pragma unroll
                for (int r = 0; r < 16; ++r) v[r] = nxt[r];
                if (p0 + FZ < S::M / 2) load_rows(p0 + FZ, nxt);
            } else {
                load_rows(p0, v);
            }
            regfft_warp_rt<R, NZ, -1>(v, reg, twz, t);
            // separate the two real rows with Z[-k] fetched from the partner lane:
            // Z[t + TZ j] sits in lane t, register j; Z[NZ - (t + TZ j)] in lane (TZ - t) mod TZ,
            // register 15 - j (t > 0) or in this lane, register (16 - j) mod 16 (t = 0)
            const int lane = threadIdx.x & 31;
            const int src = (lane - t) + ((TZ - t) & (TZ - 1));
            // every lane runs the shuffles (groups of one warp may differ in `ok`)
            const int ya = c * S::M + 2 * pp;  // row index within the plane
            const C zn = mk<R>(__shfl_sync(0xffffffffu, v[8].x, lane - t),
                               __shfl_sync(0xffffffffu, v[8].y, lane - t));  // Z[NZ/2]: lane t=0, j=8
#pragma unroll
            for (int j = 0; j < NZ / (2 * TZ); ++j) {
                const int k = t + TZ * j;      // k < NZ/2
                const C zk = v[j];
                C zp;
                zp.x = __shfl_sync(0xffffffffu, v[15 - j].x, src);
                zp.y = __shfl_sync(0xffffffffu, v[15 - j].y, src);
                if (t == 0) zp = v[(16 - j) & 15];
                const C zm = cconj(zp);
                C A = cscale(cadd(zk, zm), R(0.5));
                C B = cscale(mul_si<-1>(csub(zk, zm)), R(0.5));
                if (k == 0) {
                    // pack kz = 0 (real) and kz = NZ/2 (real) into slot 0
                    A = mk<R>(zk.x, zn.x);
                    B = mk<R>(zk.y, zn.y);
                }
                if (ok) {
                    const int owner = k / S::S, ls = k - owner * S::S;
                    C *d = dst[owner];
                    d[row_at(ya) + ls] = A;
                    d[row_at(ya + 1) + ls] = B;
                }
            }
            __syncwarp();
        }
    }
    if constexpr (CL > 1) cg::this_cluster().sync();
    else __syncthreads();

    // ---- stage y: FFT over the NY rows of every owned slot, in place
    {
        constexpr int TY = S::TY, FY = S::FY;
        const int f = tid / TY, t = tid - (tid / TY) * TY;
        C twy[16];
        load_stage_twiddles<R, NY>(twy, roots, S::NMAX, t);
        C *reg = scr + f * RegFFTShape<NY>::REGION;
        C *oplane = out + (size_t)x * NY * (NZ / 2 + 1);
#pragma unroll 1
        for (int s0 = 0; s0 < S::S; s0 += FY) {
            const int sl = s0 + f;
            const bool ok = sl < S::S;
            const int slc = ok ? sl : 0;
            C v[16];
#pragma unroll
            for (int r = 0; r < 16; ++r) v[r] = plane[row_at(t + TY * r) + slc];
            regfft_warp_rt<R, NY, -1>(v, reg, twy, t);
            // the packed slot (slot 0 of CTA 0, first round, warp 0):
            // X0[ky] = (W[ky] + conj W[-ky]) / 2, XN[ky] = (W[ky] - conj W[-ky]) / 2i
            if (c == 0 && s0 == 0 && (tid >> 5) == 0) {
                __syncwarp();
#pragma unroll
                for (int j = 0; j < 16; ++j) reg[t + TY * j] = v[j];
                __syncwarp();
                if (sl == 0) {
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        const int ky = t + TY * j;
                        const C wk = v[j];
                        const C wm = cconj(reg[(NY - ky) & (NY - 1)]);
                        v[j] = cscale(cadd(wk, wm), R(0.5));
                        oplane[(size_t)ky * (NZ / 2 + 1) + NZ / 2] = cscale(mul_si<-1>(csub(wk, wm)), R(0.5));
                    }
                }
                __syncwarp();
            }
            if (ok) {
#pragma unroll
                for (int j = 0; j < 16; ++j) plane[row_at(t + TY * j) + slc] = v[j];
            }
            // coalesced row-segment stores of this round's slots, out[x][ky][c*S + s]; they
            // drain while the next round computes
            __syncthreads();
            // block width: a compile-time constant when the slots split into whole blocks
            const int ns = S::S % FY == 0 ? FY : ((S::S - s0) < FY ? (S::S - s0) : FY);
            C *orow = oplane + c * S::S + s0;
#pragma unroll 4
            for (int e = tid; e < NY * ns; e += S::NT) {
                const int row = e / ns, q = e - (e / ns) * ns;
                orow[(size_t)row * (NZ / 2 + 1) + q] = plane[row_at(row) + s0 + q];
            }
        }
    }
}

template <typename R, int NY, int NZ, int CL>
__global__ void __launch_bounds__(PlaneShape<NY, NZ, CL>::NT, PlaneShape<NY, NZ, CL>::MINB_INV)
    plane_inv_kernel(const cpx<R> *__restrict__ in, R *__restrict__ out, const cpx<R> *__restrict__ roots, R scale)
{
    using C = cpx<R>;
    using S = PlaneShape<NY, NZ, CL>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *rowsm = reinterpret_cast<C *>(smem_raw);   // [M][PR]: this CTA's rows, every slot
    C *stg = rowsm + S::M * S::PR;                // column staging / FFT exchange regions
    C *nyq = stg + S::STG;                        // the kz = NZ/2 column (CTA 0 of a cluster)
    if constexpr (CL > 1) cluster_arrive_relaxed();
    const int tid = threadIdx.x;
    const int c = (CL > 1) ? (int)cg::this_cluster().block_rank() : 0;
    const int x = (int)(blockIdx.x / CL);
    C *dst[CL];
#pragma unroll
    for (int q = 0; q < CL; ++q) dst[q] = rowsm;
    if constexpr (CL > 1) {
#pragma unroll
        for (int q = 0; q < CL; ++q) dst[q] = cg::this_cluster().map_shared_rank(rowsm, (unsigned)q);
    }
    const C *iplane = in + (size_t)x * NY * (NZ / 2 + 1);
    if constexpr (CL > 1) cluster_wait();  // every peer's shared memory exists from here on

    // ---- stage y, one CTA per plane: the plane's spectrum rows [NY][NZ/2+1] are contiguous in
    // global memory with the pitch of rowsm, so one bulk copy brings the whole plane in (no
    // per-element transposing copies); each group reads its column into registers, and the
    // inverse y FFT results go back to the same places (a spectrum that is not 16-byte
    // aligned takes the staged path below)
    bool bulk = false;
    if constexpr (CL == 1) bulk = (reinterpret_cast<uintptr_t>(in) & 15) == 0;
    if (bulk) {
      if constexpr (CL == 1) {
        constexpr int TY = S::TY, FY = S::FY;
        constexpr unsigned BYTES = NY * (NZ / 2 + 1) * sizeof(C);
        constexpr unsigned CHUNK = 16384;
        static_assert(BYTES % 16 == 0 && S::PR == NZ / 2 + 1 && S::M == NY, "one plane per CTA");
        __shared__ __align__(8) unsigned long long bar;
        __shared__ int ok_s;
        const int f = tid / TY, t = tid - (tid / TY) * TY;
        if (tid == 0) {
            mbar_init(&bar, 1);
            mbar_init_fence();
            mbar_arrive_expect_tx(&bar, BYTES);
            for (unsigned o = 0; o < BYTES; o += CHUNK)
                bulk_load(reinterpret_cast<char *>(rowsm) + o, reinterpret_cast<const char *>(iplane) + o,
                          BYTES - o < CHUNK ? BYTES - o : CHUNK, &bar);
        }
        C twy[16];
        load_stage_twiddles<R, NY>(twy, roots, S::NMAX, t);
        C *reg = stg + f * RegFFTShape<NY>::REGION;
        if (tid == 0) ok_s = mbar_wait(&bar, 0, kRingWaitLimit) ? 1 : 0;
        __syncthreads();
        if (!ok_s) {  // the copy never completed: flag it and leave
            if (tid == 0) atomicExch(&g_ring_wait_error, 3);
            return;
        }
        // slot of this group within a block of FY slots: the G = 32 / TY groups of a warp take
        // slots TY apart, so the warp's 32 column reads (rows t + TY r, row pitch NZ/2 + 1,
        // one mod 16 in 8-byte words) cover the 16 bank pairs twice each, the minimum for 256
        // bytes; consecutive slots would hit 11 bank pairs, up to 4 lanes each
        constexpr int G = 32 / TY, W = S::NT / 32;
        const int g = f % G, w = f / G;
        const int perm = W >= TY ? g * TY + w % TY + (w / TY) * 32 : w + W * g;
#pragma unroll 1
        for (int s0 = 0; s0 < S::S; s0 += FY) {
            const int sl = s0 + perm;
            const bool ok = sl < S::S;
            const int slc = ok ? sl : 0;
            C v[16];
#pragma unroll
            for (int r = 0; r < 16; ++r) v[r] = rowsm[(t + TY * r) * S::PR + slc];
            if (ok && sl == 0) {
                // the packed slot (see the cluster path below), partners read from the plane
#pragma unroll
                for (int r = 0; r < 16; ++r) {
                    const int ky = t + TY * r, km = (NY - ky) & (NY - 1);
                    const C x0m = rowsm[km * S::PR];
                    const C xnk = rowsm[ky * S::PR + S::NS];
                    const C xnm = rowsm[km * S::PR + S::NS];
                    const C h0 = cscale(cadd(v[r], cconj(x0m)), R(0.5));
                    const C hn = cscale(cadd(xnk, cconj(xnm)), R(0.5));
                    v[r] = mk<R>(h0.x - hn.y, h0.y + hn.x);
                }
            }
            // no barrier: each group writes back only its own slot column, and the packed
            // slot's partners (column 0, its own, and the kz = NZ/2 column) are never written
            regfft_warp_rt<R, NY, +1>(v, reg, twy, t);
            if (ok) {
#pragma unroll
                for (int j = 0; j < 16; ++j) rowsm[(t + TY * j) * S::PR + sl] = v[j];
            }
        }
      }
    } else {
    // ---- stage y: inverse FFT of the owned slots, rows pushed to their owners
    {
        constexpr int TY = S::TY, FY = S::FY;
        const int f = tid / TY, t = tid - (tid / TY) * TY;
        C twy[16];
        load_stage_twiddles<R, NY>(twy, roots, S::NMAX, t);
        // stage the ns columns of block s0 (all NY rows) with coalesced asynchronous copies
        auto stage = [&](int s0, C *buf) {
            const int ns = S::S % FY == 0 ? FY : ((S::S - s0) < FY ? (S::S - s0) : FY);
            for (int e = tid; e < NY * ns; e += S::NT) {
                const int row = e / ns, sl = e - (e / ns) * ns;
                cp_async<sizeof(C)>(&buf[sl * S::PC + row],
                                    iplane + (size_t)row * (NZ / 2 + 1) + c * S::S + s0 + sl, true);
            }
            if (c == 0 && s0 == 0)  // the packed slot's partner column, read by the first block
                for (int row = tid; row < NY; row += S::NT)
                    cp_async<sizeof(C)>(&nyq[row], iplane + (size_t)row * (NZ / 2 + 1) + NZ / 2, true);
            cp_async_commit();
        };
        stage(0, stg);
#pragma unroll 1
        for (int s0 = 0; s0 < S::S; s0 += FY) {
            const int ns = S::S % FY == 0 ? FY : ((S::S - s0) < FY ? (S::S - s0) : FY);
            C *cur = stg;
            cp_async_wait_group<0>();
            __syncthreads();
            const int sl = s0 + f;
            const bool ok = f < ns;
            C *col = cur + f * S::PC;  // every group owns a column slot (idle ones compute on stale data)
            C v[16];
#pragma unroll
            for (int r = 0; r < 16; ++r) v[r] = col[t + TY * r];
            if (ok && c == 0 && sl == 0) {
                // packed slot: W = H0 + i HN with H(ky) = (X(ky) + conj X(-ky)) / 2 for the columns
                // kz = 0 (X0, staged in col) and kz = NZ/2 (XN, read here).  The inverse y FFT of
                // H is the real part of that of X, which is all the C2R keeps of these two
                // columns; so the pair packs exactly, Hermitian-consistent input or not.
#pragma unroll
                for (int r = 0; r < 16; ++r) {
                    const int ky = t + TY * r, km = (NY - ky) & (NY - 1);
                    const C x0m = col[km];
                    const C xnk = nyq[ky];
                    const C xnm = nyq[km];
                    const C h0 = cscale(cadd(v[r], cconj(x0m)), R(0.5));
                    const C hn = cscale(cadd(xnk, cconj(xnm)), R(0.5));
                    v[r] = mk<R>(h0.x - hn.y, h0.y + hn.x);
                }
            }
            regfft_warp_rt<R, NY, +1>(v, col, twy, t);
            if constexpr (CL == 1) {
                // one CTA per plane: straight from the registers into the rows (row
                // t + TY j), no staging round trip and one barrier per block
                if (ok) {
#pragma unroll
                    for (int j = 0; j < 16; ++j) rowsm[(t + TY * j) * S::PR + sl] = v[j];
                }
            } else {
                // back into the staging column, then push whole row segments to the row
                // owners: contiguous slots per row keep the distributed-shared-memory stores
                // coalesced (pushing every register straight to its owner scatters them one
                // row per lane, measured 7% slower at 256x256 with 2-CTA clusters)
                __syncwarp();
#pragma unroll
                for (int j = 0; j < 16; ++j) col[t + TY * j] = v[j];
                __syncthreads();
                for (int e = tid; e < NY * ns; e += S::NT) {
                    const int m = e / ns, q = e - (e / ns) * ns;
                    const int owner = m / S::M;
                    dst[owner][(m - owner * S::M) * S::PR + c * S::S + s0 + q] = cur[q * S::PC + m];
                }
            }
            __syncthreads();  // the staging area is refilled for the next block
            if (s0 + FY < S::S) stage(s0 + FY, stg);
        }
    }
    }
    if constexpr (CL > 1) cg::this_cluster().sync();
    else __syncthreads();

    // ---- stage z: C2R of two rows per complex FFT
    {
        constexpr int TZ = S::TZ, FZ = S::FZ;
        const int f = tid / TZ, t = tid - (tid / TZ) * TZ;
        C twz[16];
        load_stage_twiddles<R, NZ>(twz, roots, S::NMAX, t);
        C *reg = stg + f * RegFFTShape<NZ>::REGION;
        R *rows = out + ((size_t)x * NY + (size_t)c * S::M) * NZ;
        // one CTA per plane, rows in one round: the real rows are collected in the staging
        // area (pitch NZ + 4 floats) and leave as one bulk copy per row
        constexpr int ZP = NZ + 4;
        constexpr bool BULKS = CL == 1 && sizeof(R) == 4 && S::M / 2 <= FZ && (NZ * sizeof(R)) % 16 == 0 &&
                               (size_t)S::M * ZP * sizeof(R) <= (size_t)S::STG * sizeof(C);
        const bool bulks = BULKS && (reinterpret_cast<uintptr_t>(out) & 15) == 0;
#pragma unroll 1
        for (int p0 = 0; p0 < S::M / 2; p0 += FZ) {
            const int p = p0 + f;
            const bool ok = p < S::M / 2;
            const int pp = ok ? p : 0;
            const C *ha_row = rowsm + (2 * pp) * S::PR;
            const C *hb_row = ha_row + S::PR;
            C v[16];
            // n = t + TZ r with t < TZ and NZ = 16 TZ: registers r < 8 hold n < NZ/2 (k = n),
            // r > 8 hold n > NZ/2 (k = NZ - n, conjugated); only lane t = 0 of registers 0 and 8
            // meets the real kz = 0 / NZ/2 pair packed in slot 0
#pragma unroll
            for (int r = 0; r < 16; ++r) {
                C ha, hb;
                if (r < 8) {
                    const int k = t + TZ * r;
                    ha = ha_row[k];
                    hb = hb_row[k];
                } else {
                    const int k = TZ * (16 - r) - t;
                    ha = cconj(ha_row[k]);
                    hb = cconj(hb_row[k]);
                }
                if ((r == 0 || r == 8) && t == 0) {
                    // slot 0 holds kz = 0 in .x and kz = NZ/2 in .y (both real)
                    const C pa = ha_row[0], pb = hb_row[0];
                    ha = mk<R>(r == 0 ? pa.x : pa.y, R(0));
                    hb = mk<R>(r == 0 ? pb.x : pb.y, R(0));
                }
                v[r] = mk<R>(ha.x - hb.y, ha.y + hb.x);  // Ha + i Hb
            }
            regfft_warp_rt<R, NZ, +1>(v, reg, twz, t);
            if (BULKS && bulks) {
                R *zst = reinterpret_cast<R *>(stg);
                __syncthreads();  // every group's FFT exchange in the staging area is done
                if (ok) {
                    R *ra = zst + (2 * pp) * ZP;
                    R *rb = ra + ZP;
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        ra[t + TZ * j] = v[j].x * scale;
                        rb[t + TZ * j] = v[j].y * scale;
                    }
                }
                fence_proxy_async_smem();  // the rows are visible to the bulk copies
                __syncthreads();
                for (int row = tid; row < S::M; row += S::NT)
                    bulk_store(rows + (size_t)row * NZ, zst + row * ZP, (unsigned)(NZ * sizeof(R)));
                bulk_store_commit();
                bulk_store_wait();  // the staging area stays valid until the copies have read it
            } else if (ok) {
                R *ra = rows + (size_t)(2 * pp) * NZ;
                R *rb = ra + NZ;
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    ra[t + TZ * j] = v[j].x * scale;
                    rb[t + TZ * j] = v[j].y * scale;
                }
            }
            __syncwarp();
        }
    }
}

template <typename R, int NX, int MODE, bool TC>
__global__ void __launch_bounds__(256, 3) xcol_kernel(cpx<R> *__restrict__ data, long long stride, int ncols,
                                                   long long bstride, cpx<R> *__restrict__ tdata,
                                                   const cpx<R> *__restrict__ roots, XColEp ep)
{
    xcol_tile<R, NX, MODE, TC>(data, stride, ncols, bstride, tdata, roots, ep, (int)blockIdx.x, (int)blockIdx.y);
}

// One launch over the column tiles of many 3D spectra of one x length (the batched
// transforms' x stage; MODE 0 forward, 1 inverse, 2 sandwich): item i is tile items[i].tile of
// the spectrum at data + items[i].off with ny * (nz/2 + 1) columns; the spectral multiply
// takes that spectrum's ny and nz.
template <int NX, int MODE>
__global__ void __launch_bounds__(256, 2) xcol_group_kernel(const XGroupItem *__restrict__ items,
                                                         float2 *__restrict__ data,
                                                         const float2 *__restrict__ roots, XColEp ep)
{
    const XGroupItem it = items[blockIdx.x];
    ep.ny = it.ny;
    ep.nz = it.nz;
    ep.nzh = it.nz / 2 + 1;
    ep.hn = it.nz;
    xcol_tile<float, NX, MODE, false>(data + it.off, it.ncols, it.ncols, 0, nullptr, roots, ep, it.tile, 0);
}

// The y FFT (MODE 0 forward, 1 inverse) of many 3D spectra [nx][ny][nzh] of one y length in
// one launch: the lines (x, kz) of a spectrum, kz fastest, in tiles of W lines, so a warp
// reads 32 consecutive lines of a y row (contiguous within each x); the FFT is the column
// kernel's register-resident one.  items[i].ncols holds nx * nzh (the lines), .tile the
// tile, .ny / .nz the spectrum's sizes.
template <int NY, int MODE>
__global__ void __launch_bounds__(256, 2) ycol_group_kernel(const XGroupItem *__restrict__ items,
                                                         float2 *__restrict__ data,
                                                         const float2 *__restrict__ roots)
{
    ycol_tile<NY, MODE>(items[blockIdx.x], data, roots);
}
// ------------------------------------------------------------------ x column kernel, TMA ring
// Persistent form of xcol_kernel (MODE 0, 1, 2) for 16-byte aligned spectra: each CTA walks
// the tiles (W columns x NX rows; blockIdx.x, + gridDim.x, ...) with NSTAGE tiles in flight,
// brought into shared memory by tensor copies that one thread issues while the CTA
// transforms the oldest tile.  A tile's shared memory doubles as the exchange area of its
// FFTs, so the ring is the only shared memory the kernel needs; each thread keeps its
// stage twiddles w_NX^(t k1) in registers for every tile it transforms.
constexpr int kRingStages = 3;

template <typename R, int NX>
__device__ __forceinline__ void xcol_fft_regtw(cpx<R> (&v)[16], cpx<R> *scr, const cpx<R> (&tw)[16], int t, int col,
                                               bool inverse)
{
    using C = cpx<R>;
    constexpr int T = XColShape<NX>::T, W = XColShape<NX>::W;
    if (inverse) dft16<+1, C, R>(v);
    else dft16<-1, C, R>(v);
#pragma unroll
    for (int k1 = 1; k1 < 16; ++k1) v[k1] = inverse ? cmulc(v[k1], tw[k1]) : cmul(v[k1], tw[k1]);
    __syncthreads();
#pragma unroll
    for (int k1 = 0; k1 < 16; ++k1) scr[(k1 * T + t) * W + col] = v[k1];
    __syncthreads();
    constexpr int A = 16 / T;
#pragma unroll
    for (int a = 0; a < A; ++a) {
        C u[T];
#pragma unroll
        for (int q = 0; q < T; ++q) u[q] = scr[((t + T * a) * T + q) * W + col];
        if (inverse) dft_small<+1, T, C, R>(u);
        else dft_small<-1, T, C, R>(u);
#pragma unroll
        for (int k2 = 0; k2 < T; ++k2) v[a + A * k2] = u[k2];
    }
}

// tmap: float32 view [nbatch][NX][2 * ncols] of the spectrum (row pitch `stride`, batch pitch
// `bstride` complex entries), box {2W, NX, 1}.  Tile k = (batch k / tpb, column block k % tpb).
template <typename R, int NX, int MODE>
__global__ void __launch_bounds__(256, 2)
    xcol_ring_kernel(const __grid_constant__ CUtensorMap tmap, cpx<R> *__restrict__ data, long long stride,
                     int ncols, int tpb, int ntiles, long long bstride, cpx<R> *__restrict__ tdata,
                     const cpx<R> *__restrict__ roots, XColEp ep)
{
    using C = cpx<R>;
    constexpr int T = XColShape<NX>::T, W = XColShape<NX>::W;
    constexpr int TILE = NX * W;
    constexpr unsigned TILE_BYTES = TILE * sizeof(C);
    static_assert(16 * T * W <= TILE, "a tile holds its exchange area");
    // dynamic shared memory: [pad to 128 B][kRingStages tiles][kRingStages mbarriers][flag]; the
    // tensor copies need 128-byte aligned destinations, so the ring is aligned by hand
    extern __shared__ __align__(128) unsigned char ring_smem_raw[];
    const unsigned pad = (128u - (smem_u32(ring_smem_raw) & 127u)) & 127u;
    C *ring = reinterpret_cast<C *>(ring_smem_raw + pad);
    unsigned long long *full = reinterpret_cast<unsigned long long *>(ring_smem_raw + pad + kRingStages * TILE_BYTES);
    int &ok_s = *reinterpret_cast<int *>(full + kRingStages);
    const int tid = threadIdx.x;
    const int t = tid / W, col = tid - (tid / W) * W;
    if ((smem_u32(ring) & 127u) != 0u) {  // never issue a copy to a misaligned destination
        if (tid == 0) atomicExch(&g_ring_wait_error, 2);
        return;
    }
    auto issue = [&](int stage, int k) {
        const int b = k / tpb, tx = k - (k / tpb) * tpb;
        mbar_arrive_expect_tx(&full[stage], TILE_BYTES);
        tma_load_3d(ring + stage * TILE, &tmap, &full[stage], 2 * W * tx, 0, b);
    };
    if (tid == 0) {
        for (int q = 0; q < kRingStages; ++q) mbar_init(&full[q], 1);
        mbar_init_fence();
    }
    __syncthreads();
    if (tid == 0)
        for (int q = 0; q < kRingStages; ++q)
            if (blockIdx.x + q * gridDim.x < (unsigned)ntiles) issue(q, blockIdx.x + q * gridDim.x);
    C tw[16];
    tw[0] = mk<R>(R(1), R(0));
#pragma unroll
    for (int k1 = 1; k1 < 16; ++k1) tw[k1] = roots[t * k1];
    int it = 0;
#pragma unroll 1
    for (int k = blockIdx.x; k < ntiles; k += gridDim.x, ++it) {
        const int stage = it % kRingStages;
        if (tid == 0) ok_s = mbar_wait(&full[stage], (unsigned)(it / kRingStages) & 1u, kRingWaitLimit) ? 1 : 0;
        __syncthreads();
        if (!ok_s) {
            // a copy never completed: wait (bounded) for the other copies in flight into this
            // CTA's shared memory, flag the error and leave
            if (tid == 0) {
                for (int q = 1; q < kRingStages; ++q) {
                    const int kk = k + q * (int)gridDim.x;
                    if (kk < ntiles) mbar_wait(&full[(it + q) % kRingStages], (unsigned)((it + q) / kRingStages) & 1u,
                                               kRingWaitLimit);
                }
                atomicExch(&g_ring_wait_error, 1);
            }
            return;
        }
        C *buf = ring + stage * TILE;
        const int b = k / tpb, tx = k - (k / tpb) * tpb;
        const int cg0 = tx * W + col;
        C v[16];
#pragma unroll
        for (int r = 0; r < 16; ++r) v[r] = buf[(t + T * r) * W + col];
        xcol_fft_regtw<R, NX>(v, buf, tw, t, col, MODE == 1);
        if (MODE == 2) {
            xcol_multiply<R, NX>(v, t, cg0, ep);
            xcol_fft_regtw<R, NX>(v, buf, tw, t, col, true);
        }
        if (MODE != 2 && (ep.mode & EP_HALFW)) xcol_halfw<R>(v, cg0, ep);
        if (cg0 < ncols) {
            C *q = ((MODE == 2 && tdata) ? tdata : data) + (size_t)b * bstride + cg0;
#pragma unroll
            for (int j = 0; j < 16; ++j) q[(size_t)(t + T * j) * stride] = v[j];
        }
        __syncthreads();  // every thread is done with this tile's shared memory
        const int kn = k + kRingStages * (int)gridDim.x;
        if (tid == 0 && kn < ntiles) {
            fence_proxy_async_smem();
            issue(stage, kn);
        }
    }
}

// ------------------------------------------------------------------ host side
namespace {

struct PlaneEntry {
    int dtype, ny, nz, cl, nt;
    const void *fwd, *inv;
    size_t smem_fwd, smem_inv;
};

template <typename R, int NY, int NZ, int CL> PlaneEntry plane_entry(int dtype)
{
    using S = PlaneShape<NY, NZ, CL>;
    return PlaneEntry{dtype, NY, NZ, CL, S::NT, (const void *)&plane_fwd_kernel<R, NY, NZ, CL>,
                      (const void *)&plane_inv_kernel<R, NY, NZ, CL>, S::template smem_fwd<R>(),
                      S::template smem_inv<R>()};
}

#define FFTB_PLANE3(R, D, NY, NZ)                                                                                   \
    plane_entry<R, NY, NZ, 1>(D), plane_entry<R, NY, NZ, 2>(D), plane_entry<R, NY, NZ, 4>(D)
#define FFTB_PLANE4(R, D, NY, NZ) FFTB_PLANE3(R, D, NY, NZ), plane_entry<R, NY, NZ, 8>(D)
#define FFTB_PLANES(R, D)                                                                                          \
    FFTB_PLANE3(R, D, 64, 64), FFTB_PLANE3(R, D, 64, 128), FFTB_PLANE3(R, D, 64, 256), FFTB_PLANE3(R, D, 128, 64), \
        FFTB_PLANE4(R, D, 128, 128), FFTB_PLANE4(R, D, 128, 256), FFTB_PLANE3(R, D, 256, 64),                     \
        FFTB_PLANE4(R, D, 256, 128), FFTB_PLANE4(R, D, 256, 256)

const PlaneEntry *find_plane(int dtype, int ny, int nz, int cl)
{
    static const PlaneEntry tab[] = {FFTB_PLANES(float, FFTB_F32)};
    for (const PlaneEntry &e : tab)
        if (e.dtype == dtype && e.ny == ny && e.nz == nz && e.cl == cl) return &e;
    return nullptr;
}

// ------------------------------------------------------------------ grouped z rows (batches)
// The R2C (DIR 0) or C2R (DIR 1) of the contiguous z rows of many 3D transforms of one even z
// length NZ in one launch, two real rows per complex NZ-point FFT (the plane kernels' z stage
// without the plane): a group of TZ = NZ / 16 threads holds the row pair in registers, so the
// rows go from HBM to registers and back with one exchange through shared memory for the
// FFT.  R2C: z = a + i b, X_a[k] = (Z[k] + conj Z[-k]) / 2, X_b[k] = (Z[k] - conj Z[-k]) / 2i,
// DC and Nyquist real.  C2R: Z = X_a + i X_b over the Hermitian extension (the imaginary
// parts of DC and Nyquist ignored, as the C2R pass does), a = Re IFFT(Z), b = Im IFFT(Z),
// times the item's scale.  Item i: pair tile items[i].tile of the nrows rows at real
// offset roff and spectrum offset soff.
template <int NZ, int DIR>
__global__ void __launch_bounds__(256) row_group_kernel(const RowGroupItem *__restrict__ items,
                                                        const void *__restrict__ in, void *__restrict__ out,
                                                        const float2 *__restrict__ roots)
{
    row_tile<NZ, DIR>(items[blockIdx.x], in, out, roots);
}

struct XColEntry {
    int dtype, nx;
    const void *fn[5];
    size_t smem;
    const void *fn_tc[5];  // first radix-16 stage on the tensor cores
    size_t smem_tc;
    const void *fn_ring[3];  // persistent TMA-ring form of modes 0, 1, 2
    size_t smem_ring;
};

template <typename R, int NX> XColEntry xcol_entry(int dtype)
{
    constexpr int T = XColShape<NX>::T, W = XColShape<NX>::W;
    constexpr size_t scr = (size_t)16 * T * W > (size_t)W * (NX + 1) ? (size_t)16 * T * W : (size_t)W * (NX + 1);
    constexpr size_t smem = sizeof(cpx<R>) * (scr + NX);
    return XColEntry{dtype,
                     NX,
                     {(const void *)&xcol_kernel<R, NX, 0, false>, (const void *)&xcol_kernel<R, NX, 1, false>,
                      (const void *)&xcol_kernel<R, NX, 2, false>, (const void *)&xcol_kernel<R, NX, 3, false>,
                      (const void *)&xcol_kernel<R, NX, 4, false>},
                     smem,
                     {(const void *)&xcol_kernel<R, NX, 0, true>, (const void *)&xcol_kernel<R, NX, 1, true>,
                      (const void *)&xcol_kernel<R, NX, 2, true>, (const void *)&xcol_kernel<R, NX, 3, true>,
                      (const void *)&xcol_kernel<R, NX, 4, true>},
                     smem + (size_t)(256 / 32) * kTcWarpBytes,
                     {(const void *)&xcol_ring_kernel<R, NX, 0>, (const void *)&xcol_ring_kernel<R, NX, 1>,
                      (const void *)&xcol_ring_kernel<R, NX, 2>},
                     (size_t)kRingStages * NX * W * sizeof(cpx<R>) + 128 + 64};
}

const XColEntry *find_xcol(int dtype, int nx)
{
    static const XColEntry tab[] = {xcol_entry<float, 32>(FFTB_F32), xcol_entry<float, 64>(FFTB_F32),
                                    xcol_entry<float, 128>(FFTB_F32), xcol_entry<float, 256>(FFTB_F32)};
    for (const XColEntry &e : tab)
        if (e.dtype == dtype && e.nx == nx) return &e;
    return nullptr;
}

// Raises the kernel's dynamic shared-memory limit to what the device allows beside its
// static shared memory (once for all uses: a per-use value could lower it under another
// object's launches of the same kernel).
int configure(const void *fn, size_t smem)
{
    if (smem <= 48 * 1024) return FFTB_SUCCESS;
    int dev = 0, optin = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaFuncAttributes fa;
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, fn);
    if (e == cudaSuccess && smem + fa.sharedSizeBytes > (size_t)optin) return FFTB_ERROR_UNSUPPORTED_SIZE;
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
    return set_status_from_cuda(e);
}

// One launch of a plane kernel over `nplanes` planes.
int launch_plane_n(const PlaneEntry *e, long long nplanes, bool inverse, const void *in, void *out, void *roots,
                   double scale, cudaStream_t s, LaunchTimer *tm)
{
    float sc = (float)scale;
    const void *fn = inverse ? e->inv : e->fwd;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(nplanes * e->cl));
    cfg.blockDim = dim3(e->nt);
    cfg.dynamicSmemBytes = inverse ? e->smem_inv : e->smem_fwd;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    cfg.attrs = attr;
    cfg.numAttrs = 0;
    if (e->cl > 1) {
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = e->cl;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.numAttrs = 1;
    }
    const double bytes = (double)nplanes * e->ny * (4.0 * e->nz + 8.0 * (e->nz / 2 + 1));
    if (tm) {
        int st = timer_mark(tm, s,
                            std::string(inverse ? "plane_inv_kernel" : "plane_fwd_kernel") + "<f32," +
                                std::to_string(e->ny) + "," + std::to_string(e->nz) + ",cl" + std::to_string(e->cl) +
                                ">",
                            bytes);
        if (st != FFTB_SUCCESS) return st;
    }
    cudaError_t err;
    if (inverse) {
        const float2 *a0 = (const float2 *)in;
        float *a1 = (float *)out;
        const float2 *a2 = (const float2 *)roots;
        void *args[] = {&a0, &a1, &a2, &sc};
        err = cudaLaunchKernelExC(&cfg, fn, args);
    } else {
        const float *a0 = (const float *)in;
        float2 *a1 = (float2 *)out;
        const float2 *a2 = (const float2 *)roots;
        void *args[] = {&a0, &a1, &a2};
        err = cudaLaunchKernelExC(&cfg, fn, args);
    }
    return set_status_from_cuda(err);
}

int launch_plane(const Fused3D &f, bool inverse, const void *in, void *out, double scale, cudaStream_t s,
                 LaunchTimer *tm)
{
    return launch_plane_n((const PlaneEntry *)(inverse ? f.plane_inv : f.plane), f.nx, inverse, in, out,
                          f.roots_plane, scale, s, tm);
}

XColEp make_ep(const EpValues *ep)
{
    XColEp x = {};
    x.mode = ep ? (ep->mode < 0 ? 0 : ep->mode) : 0;
    x.scale = ep ? ep->scale : 1.0;
    x.sign = ep ? ep->sign : -1.0;
    x.gauss = ep ? ep->gauss : 0.0;
    x.scale_f = (float)x.scale;
    x.sign_f = (float)x.sign;
    x.gauss_f = (float)x.gauss;
    x.hw = ep ? ep->hw : 1.0;
    x.hw_f = (float)x.hw;
    return x;
}

int device_sms()
{
    static int sms[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (!sms[dev] && cudaDeviceGetAttribute(&sms[dev], cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        sms[dev] = 148;
    return sms[dev];
}

// The persistent TMA-ring column kernel takes modes 0-2 of a 16-byte aligned spectrum whose
// row and batch pitches are multiples of 16 bytes (the tensor map's stride rule).
bool ring_eligible(int mode, const void *data, long long stride, long long nbatch, long long bstride,
                   const void *tdata, const XColEp &x)
{
    if (mode > 2 || x.tc || getenv("FFTB_DISABLE_RING")) return false;
    if ((uintptr_t)data % 16 || (tdata && (uintptr_t)tdata % 16)) return false;
    if ((stride * 8) % 16 || (nbatch > 1 && (bstride * 8) % 16)) return false;
    return true;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point, so the library has no
// link-time dependency on the driver library (it loads on machines without a GPU)
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    });
    return fn;
}

int launch_xcol_ring(const XColEntry *e, int mode, void *data, long long stride, long long ncols, long long nbatch,
                     long long bstride, void *tdata, void *roots, XColEp x, cudaStream_t s)
{
    const int W = 256 / (e->nx / 16);
    PFN_cuTensorMapEncodeTiled_v12000 encode = tensor_map_encoder();
    if (!encode) {
        set_last_error("cuTensorMapEncodeTiled is not available from the CUDA driver");
        return FFTB_ERROR_CUDA;
    }
    CUtensorMap map;
    const cuuint64_t dims[3] = {(cuuint64_t)(2 * ncols), (cuuint64_t)e->nx, (cuuint64_t)nbatch};
    const cuuint64_t strides[2] = {(cuuint64_t)(stride * 8),
                                   (cuuint64_t)((nbatch > 1 ? bstride : stride * e->nx) * 8)};
    const cuuint32_t box[3] = {(cuuint32_t)(2 * W), (cuuint32_t)e->nx, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = encode(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, data, dims, strides, box, estr,
                                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_last_error("cuTensorMapEncodeTiled failed for the column kernel's tensor map");
        return FFTB_ERROR_CUDA;
    }
    const long long tpb = (ncols + W - 1) / W, ntiles = tpb * nbatch;
    const long long ctas = std::min<long long>(ntiles, 2LL * device_sms());
    float2 *d = (float2 *)data;
    float2 *td = (float2 *)tdata;
    int nc = (int)ncols, tp = (int)tpb, nt = (int)ntiles;
    const float2 *rt = (const float2 *)roots;
    void *args[] = {&map, &d, &stride, &nc, &tp, &nt, &bstride, &td, &rt, &x};
    return set_status_from_cuda(
        cudaLaunchKernel(e->fn_ring[mode], dim3((unsigned)ctas), dim3(256), args, e->smem_ring, s));
}

// One launch of a column kernel: ncols columns `stride` apart per batch, nbatch batches.
int launch_xcol_n(const XColEntry *e, int mode, void *data, long long stride, long long ncols, long long nbatch,
                  long long bstride, void *tdata, void *roots, XColEp x, cudaStream_t s, LaunchTimer *tm)
{
    const int W = 256 / (e->nx / 16);
    const bool ring = ring_eligible(mode, data, stride, nbatch, bstride, tdata, x);
    if (tm) {
        static const char *mn[] = {"fwd", "inv", "sandwich", "fwd_t", "inv_t"};
        int st = timer_mark(tm, s,
                            std::string(ring ? "xcol_ring_kernel<f32," : "xcol_kernel<f32,") + std::to_string(e->nx) +
                                "," + mn[mode] + ">",
                            (double)e->nx * ncols * nbatch * 16.0);
        if (st != FFTB_SUCCESS) return st;
    }
    if (ring) return launch_xcol_ring(e, mode, data, stride, ncols, nbatch, bstride, tdata, roots, x, s);
    float2 *d = (float2 *)data;
    float2 *td = (float2 *)tdata;
    int nc = (int)ncols;
    const float2 *rt = (const float2 *)roots;
    void *args[] = {&d, &stride, &nc, &bstride, &td, &rt, &x};
    const dim3 grid((unsigned)((ncols + W - 1) / W), (unsigned)nbatch);
    return set_status_from_cuda(cudaLaunchKernel(x.tc ? e->fn_tc[mode] : e->fn[mode], grid, dim3(256), args,
                                                 x.tc ? e->smem_tc : e->smem, s));
}

int launch_xcol(const Fused3D &f, int mode, void *data, const EpValues *ep, cudaStream_t s, LaunchTimer *tm)
{
    const long long nzh = f.nz / 2 + 1;
    const long long ncols = f.ny * nzh;
    XColEp x = make_ep(ep);
    x.nzh = (int)nzh;
    x.ny = (int)f.ny;
    x.nz = (int)f.nz;
    x.hn = (int)f.nz;
    x.tc = f.tc ? 1 : 0;
    return launch_xcol_n((const XColEntry *)f.xcol, mode, data, ncols, ncols, 1, 0, nullptr, f.roots_x, x, s, tm);
}

} // namespace

namespace {
// kind: 0 x forward, 1 x inverse, 2 x sandwich, 3 y forward, 4 y inverse
const void *col_group_fn(int kind, int n)
{
#define FFTB_COLG(N)                                                                                                   \
    case N:                                                                                                            \
        return kind == 0   ? (const void *)&xcol_group_kernel<N, 0>                                                    \
               : kind == 1 ? (const void *)&xcol_group_kernel<N, 1>                                                    \
               : kind == 2 ? (const void *)&xcol_group_kernel<N, 2>                                                    \
               : kind == 3 ? (const void *)&ycol_group_kernel<N, 0>                                                    \
                           : (const void *)&ycol_group_kernel<N, 1>;
    if (kind < 0 || kind > 4) return nullptr;
    switch (n) {
        FFTB_COLG(32)
        FFTB_COLG(48)
        FFTB_COLG(64)
        FFTB_COLG(96)
        FFTB_COLG(128)
        FFTB_COLG(256)
    default:
        return nullptr;
    }
#undef FFTB_COLG
}

} // namespace

// dynamic shared memory of a column tile: the exchange / transposing area and the root table
size_t col_group_smem(int n)
{
    const int T = n / 16, W = 256 / T;
    const size_t scr = (size_t)16 * T * W > (size_t)W * (n + 1) ? (size_t)16 * T * W : (size_t)W * (n + 1);
    return sizeof(float2) * (scr + (size_t)n);
}

namespace {
const void *row_group_fn(int dir, int nz)
{
    switch (nz) {
    case 32: return dir ? (const void *)&row_group_kernel<32, 1> : (const void *)&row_group_kernel<32, 0>;
    case 64: return dir ? (const void *)&row_group_kernel<64, 1> : (const void *)&row_group_kernel<64, 0>;
    case 128: return dir ? (const void *)&row_group_kernel<128, 1> : (const void *)&row_group_kernel<128, 0>;
    case 256: return dir ? (const void *)&row_group_kernel<256, 1> : (const void *)&row_group_kernel<256, 0>;
    default: return nullptr;
    }
}
} // namespace

// one exchange region (RegFFTShape<nz>::REGION) per row-pair group
size_t row_group_smem(int nz)
{
    const int T = nz / 16;
    const int region = T == 1 ? 16 : 16 * (T + 1) + (T == 16 ? 0 : T);
    return sizeof(float2) * (size_t)(256 / T) * region;
}

// Rows of 32 points are left to the pass kernel: two threads per FFT read and write 8 bytes
// per row at a time, a quarter of a sector, and measured slower than its staged loads
// (67 / 88 us against 58 / 61 us for the R2C / C2R of the 512-shape batch's 32-point rows).
int row_group_tile_pairs(int dtype, int nz)
{
    return dtype == FFTB_F32 && nz >= 64 && row_group_fn(0, nz) ? 256 / (nz / 16) : 0;
}

int row_group_prepare(int dtype, int dir, int nz, void **roots)
{
    if (dtype != FFTB_F32 || !row_group_fn(dir, nz)) return FFTB_ERROR_UNSUPPORTED_SIZE;
    int st = configure(row_group_fn(dir, nz), row_group_smem(nz));
    if (st != FFTB_SUCCESS) return st;
    return engine_roots(dtype, nz, roots);
}

int launch_row_group(int dir, int nz, const RowGroupItem *items, int nitems, const void *in, void *out,
                     const void *roots, cudaStream_t s)
{
    const void *fn = row_group_fn(dir, nz);
    if (!fn || nitems <= 0) return FFTB_ERROR_INVALID_VALUE;
    const float2 *rt = (const float2 *)roots;
    void *args[] = {&items, &in, &out, &rt};
    return set_status_from_cuda(cudaLaunchKernel(fn, dim3((unsigned)nitems), dim3(256), args, row_group_smem(nz), s));
}

int col_group_tile_lines(int dtype, int n)
{
    return dtype == FFTB_F32 && col_group_fn(0, n) ? 256 / (n / 16) : 0;
}

int col_group_prepare(int dtype, int kind, int n, void **roots)
{
    if (dtype != FFTB_F32 || !col_group_fn(kind, n)) return FFTB_ERROR_UNSUPPORTED_SIZE;
    int st = configure(col_group_fn(kind, n), col_group_smem(n));
    if (st != FFTB_SUCCESS) return st;
    return engine_roots(dtype, n, roots);
}

int launch_col_group(int kind, int n, const XGroupItem *items, int nitems, void *data, const void *roots,
                     int ep_mode, double scale, double sign, cudaStream_t s)
{
    const void *fn = col_group_fn(kind, n);
    if (!fn || nitems <= 0) return FFTB_ERROR_INVALID_VALUE;
    const size_t smem = col_group_smem(n);
    float2 *d = (float2 *)data;
    const float2 *rt = (const float2 *)roots;
    if (kind >= 3) {
        void *args[] = {&items, &d, &rt};
        return set_status_from_cuda(cudaLaunchKernel(fn, dim3((unsigned)nitems), dim3(256), args, smem, s));
    }
    EpValues ev;
    ev.mode = ep_mode;
    ev.scale = scale;
    ev.sign = sign;
    XColEp x = make_ep(&ev);
    void *args[] = {&items, &d, &rt, &x};
    return set_status_from_cuda(cudaLaunchKernel(fn, dim3((unsigned)nitems), dim3(256), args, smem, s));
}

int fused3d_clusters(int dtype, long long nx, long long ny, long long nz, int *clusters, int cap)
{
    int n = 0;
    if (dtype != FFTB_F32 || !find_xcol(dtype, (int)nx)) return 0;
    for (int cl = 1; cl <= 8; cl *= 2) {
        const PlaneEntry *e = find_plane(dtype, (int)ny, (int)nz, cl);
        if (e && e->smem_fwd <= 227 * 1024 && e->smem_inv <= 227 * 1024 && n < cap) clusters[n++] = cl;
    }
    return n;
}

int fused3d_init(Fused3D &f, int dtype, long long nx, long long ny, long long nz, int force_cluster)
{
    f.enabled = false;
    f.dtype = dtype;
    f.nx = nx;
    f.ny = ny;
    f.nz = nz;
    f.cluster = 0;
    if (dtype != FFTB_F32) return FFTB_SUCCESS;
    if (getenv("FFTB_DISABLE_FUSED3D")) return FFTB_SUCCESS;
    // the smallest cluster whose plane fits the shared memory of its CTAs: measured on B200,
    // fewer CTAs per plane wins over more resident warps (64^3, 128^3 and 256x128x256 run
    // fastest with one CTA per plane, 256^3 with two), because every extra CTA moves a
    // larger share of the plane through distributed shared memory and cluster barriers
    const PlaneEntry *pe = nullptr;
    for (int cl = force_cluster > 0 ? force_cluster : 1; cl <= 8 && !pe; cl *= 2) {
        const PlaneEntry *e = find_plane(dtype, (int)ny, (int)nz, cl);
        if (e && e->smem_fwd <= 227 * 1024 && e->smem_inv <= 227 * 1024) pe = e;
        if (force_cluster > 0) break;
    }
    const XColEntry *xe = find_xcol(dtype, (int)nx);
    if (!pe || !xe) return FFTB_SUCCESS;
    // The inverse plane kernel is a launch of its own, so it may use another cluster size:
    // unless one was forced, the smallest cluster (up to 4) whose inverse CTAs fit two per SM,
    // when the forward's cluster leaves one per SM.  Measured on B200 at 256x256 planes: the
    // inverse runs 67 us with 4-CTA clusters (two quarter planes per SM) against 71 us with
    // 2-CTA clusters, while the forward is fastest with 2 (56 against 60 us).
    const PlaneEntry *pi = pe;
    if (force_cluster <= 0 && 2 * pe->smem_inv > 227 * 1024)
        for (int cl = pe->cl * 2; cl <= 4; cl *= 2) {
            const PlaneEntry *e = find_plane(dtype, (int)ny, (int)nz, cl);
            if (e && 2 * e->smem_inv <= 227 * 1024) {
                pi = e;
                break;
            }
        }
    int st;
    if ((st = configure(pe->fwd, pe->smem_fwd)) != FFTB_SUCCESS) return st;
    if ((st = configure(pi->inv, pi->smem_inv)) != FFTB_SUCCESS) return st;
    for (int m = 0; m < 5; ++m)
        if ((st = configure(xe->fn[m], xe->smem)) != FFTB_SUCCESS ||
            (st = configure(xe->fn_tc[m], xe->smem_tc)) != FFTB_SUCCESS ||
            (m < 3 && (st = configure(xe->fn_ring[m], xe->smem_ring)) != FFTB_SUCCESS))
            return st;
    const int nmax = (int)(ny > nz ? ny : nz);
    if ((st = engine_roots(dtype, nmax, &f.roots_plane)) != FFTB_SUCCESS) return st;
    if ((st = engine_roots(dtype, (int)nx, &f.roots_x)) != FFTB_SUCCESS) return st;
    f.plane = pe;
    f.plane_inv = pi;
    f.xcol = xe;
    f.cluster = pe->cl;
    f.cluster_inv = pi->cl;
    f.enabled = true;
    return FFTB_SUCCESS;
}

int fused3d_forward(const Fused3D &f, const void *in, void *out, cudaStream_t s, LaunchTimer *t)
{
    int st = launch_plane(f, false, in, out, 1.0, s, t);
    if (st == FFTB_SUCCESS) st = launch_xcol(f, 0, out, nullptr, s, t);
    if (st == FFTB_SUCCESS && t) st = timer_end(t, s);
    return st;
}

int fused3d_backward(const Fused3D &f, void *in, void *out, double scale, cudaStream_t s, LaunchTimer *t)
{
    int st = launch_xcol(f, 1, in, nullptr, s, t);
    if (st == FFTB_SUCCESS) st = launch_plane(f, true, in, out, scale, s, t);
    if (st == FFTB_SUCCESS && t) st = timer_end(t, s);
    return st;
}

int fused3d_spectral(const Fused3D &f, const void *in, void *out, void *work, const EpValues &ep, cudaStream_t s,
                     LaunchTimer *t)
{
    if (!work) return FFTB_ERROR_NO_WORK_AREA;
    int st = launch_plane(f, false, in, work, 1.0, s, t);
    if (st == FFTB_SUCCESS) st = launch_xcol(f, 2, work, &ep, s, t);
    if (st == FFTB_SUCCESS)
        st = launch_plane(f, true, work, out, 1.0 / (double)(f.nx * f.ny * f.nz), s, t);
    if (st == FFTB_SUCCESS && t) st = timer_end(t, s);
    return st;
}

// du/d(axis): plane R2C into spec, the x column sandwich (forward, i k, inverse) in place,
// the inverse planes with 1/N
int fused3d_derivative(const Fused3D &f, const void *in, void *spec, void *out, int axis, cudaStream_t s,
                       LaunchTimer *t)
{
    const long long nzh = f.nz / 2 + 1;
    int st = launch_plane(f, false, in, spec, 1.0, s, t);
    if (st == FFTB_SUCCESS) {
        XColEp x = make_ep(nullptr);
        x.mode = EP_DERIV;
        x.daxis = axis;
        x.dscale = 1.0;
        x.dscale_f = 1.f;
        x.nzh = (int)nzh;
        x.ny = (int)f.ny;
        x.nz = (int)f.nz;
        x.hn = (int)f.nz;
        x.tc = f.tc ? 1 : 0;
        st = launch_xcol_n((const XColEntry *)f.xcol, 2, spec, f.ny * nzh, f.ny * nzh, 1, 0, nullptr, f.roots_x, x, s,
                           t);
    }
    if (st == FFTB_SUCCESS) st = launch_plane(f, true, spec, out, 1.0 / (double)(f.nx * f.ny * f.nz), s, t);
    if (st == FFTB_SUCCESS && t) st = timer_end(t, s);
    return st;
}

// every first derivative: the planes' R2C once into spec; per axis the column sandwich
// with the i k multiply from spec into spec2 and the inverse planes into outs[axis]
int fused3d_gradient(const Fused3D &f, const void *in, void *spec, void *spec2, void *const *outs, cudaStream_t s,
                     LaunchTimer *t)
{
    const long long nzh = f.nz / 2 + 1;
    int st = launch_plane(f, false, in, spec, 1.0, s, t);
    for (int a = 0; a < 3 && st == FFTB_SUCCESS; ++a) {
        XColEp x = make_ep(nullptr);
        x.mode = EP_DERIV;
        x.daxis = a;
        x.dscale = 1.0;
        x.dscale_f = 1.f;
        x.nzh = (int)nzh;
        x.ny = (int)f.ny;
        x.nz = (int)f.nz;
        x.hn = (int)f.nz;
        x.tc = f.tc ? 1 : 0;
        st = launch_xcol_n((const XColEntry *)f.xcol, 2, spec, f.ny * nzh, f.ny * nzh, 1, 0, spec2, f.roots_x, x, s,
                           t);
        if (st == FFTB_SUCCESS)
            st = launch_plane(f, true, spec2, outs[a], 1.0 / (double)(f.nx * f.ny * f.nz), s, t);
    }
    if (st == FFTB_SUCCESS && t) st = timer_end(t, s);
    return st;
}

// adjoint of the forward R2C: C2R of the gradient with interior kz bins weighted 1/2
int fused3d_forward_adjoint(const Fused3D &f, void *gspec, void *greal, cudaStream_t s, LaunchTimer *t)
{
    EpValues ep;
    ep.mode = EP_HALFW;
    ep.hw = 0.5;
    int st = launch_xcol(f, 1, gspec, &ep, s, t);
    if (st == FFTB_SUCCESS) st = launch_plane(f, true, gspec, greal, 1.0, s, t);
    if (st == FFTB_SUCCESS && t) st = timer_end(t, s);
    return st;
}

// adjoint of the (unnormalised) C2R: R2C of the gradient with interior kz bins doubled
int fused3d_backward_adjoint(const Fused3D &f, const void *greal, void *gspec, cudaStream_t s, LaunchTimer *t)
{
    EpValues ep;
    ep.mode = EP_HALFW;
    ep.hw = 2.0;
    int st = launch_plane(f, false, greal, gspec, 1.0, s, t);
    if (st == FFTB_SUCCESS) st = launch_xcol(f, 0, gspec, &ep, s, t);
    if (st == FFTB_SUCCESS && t) st = timer_end(t, s);
    return st;
}

int fused3d_num_launches(const Fused3D &f, int which)
{
    (void)f;
    return which <= 1 ? 2 : 3;
}

// ------------------------------------------------------------------ 4D slab / native_xzwy
// real [x][y][z][w]; work / slab spectrum [x][y][kz][kw<nw/2+1]; native spectrum
// [ky][kz][kw][kx].  Stages: the (z,w) plane R2C over the nx*ny planes (the 3D plane
// kernels), the y FFT (column kernel batched over x), the x FFT (column kernel; for
// native_xzwy written transposed so kx becomes the contiguous axis).
int fused4d_init(Fused4D &f, int dtype, int layout, long long nx, long long ny, long long nz, long long nw)
{
    f.enabled = false;
    f.dtype = dtype;
    f.layout = layout;
    f.nx = nx; f.ny = ny; f.nz = nz; f.nw = nw;
    if (dtype != FFTB_F32 || (layout != FFTB_4D_SLAB && layout != FFTB_4D_NATIVE_XZWY)) return FFTB_SUCCESS;
    if (getenv("FFTB_DISABLE_FUSED3D")) return FFTB_SUCCESS;
    const PlaneEntry *pe = find_plane(dtype, (int)nz, (int)nw, 1);
    const XColEntry *xe = find_xcol(dtype, (int)nx);
    const XColEntry *ye = find_xcol(dtype, (int)ny);
    if (!pe || !xe || !ye || pe->smem_fwd > 113 * 1024 || pe->smem_inv > 113 * 1024) return FFTB_SUCCESS;
    int st;
    if ((st = configure(pe->fwd, pe->smem_fwd)) != FFTB_SUCCESS) return st;
    if ((st = configure(pe->inv, pe->smem_inv)) != FFTB_SUCCESS) return st;
    for (const XColEntry *e : {xe, ye})
        for (int m = 0; m < 5; ++m)
            if ((st = configure(e->fn[m], e->smem)) != FFTB_SUCCESS ||
                (st = configure(e->fn_tc[m], e->smem_tc)) != FFTB_SUCCESS ||
                (m < 3 && (st = configure(e->fn_ring[m], e->smem_ring)) != FFTB_SUCCESS))
                return st;
    const int nmax = (int)(nz > nw ? nz : nw);
    if ((st = engine_roots(dtype, nmax, &f.roots_plane)) != FFTB_SUCCESS) return st;
    if ((st = engine_roots(dtype, (int)nx, &f.roots_x)) != FFTB_SUCCESS) return st;
    if ((st = engine_roots(dtype, (int)ny, &f.roots_y)) != FFTB_SUCCESS) return st;
    f.plane = pe;
    f.xcol = xe;
    f.ycol = ye;
    f.enabled = true;
    return FFTB_SUCCESS;
}

namespace {
XColEp ep4(const Fused4D &f, const EpValues *ep)
{
    XColEp x = make_ep(ep);
    x.nd4 = 1;
    x.ny = (int)f.ny;
    x.nz = (int)f.nz;
    x.nwh = (int)(f.nw / 2 + 1);
    x.nzh = 1;
    x.hn = (int)f.nw;
    x.tc = f.tc ? 1 : 0;
    return x;
}
} // namespace

// out: the spectrum in the object's layout; work: slab-layout scratch (native only)
int fused4d_forward(const Fused4D &f, const void *in, void *out, void *work, cudaStream_t s, LaunchTimer *t)
{
    const long long C = f.nz * (f.nw / 2 + 1), YC = f.ny * C;
    const bool native = f.layout == FFTB_4D_NATIVE_XZWY;
    void *slab = native ? work : out;
    if (native && !work) return FFTB_ERROR_NO_WORK_AREA;
    const PlaneEntry *pe = (const PlaneEntry *)f.plane;
    int st = launch_plane_n(pe, f.nx * f.ny, false, in, slab, f.roots_plane, 1.0, s, t);
    if (st == FFTB_SUCCESS)
        st = launch_xcol_n((const XColEntry *)f.ycol, 0, slab, C, C, f.nx, YC, nullptr, f.roots_y, ep4(f, nullptr), s, t);
    if (st == FFTB_SUCCESS)
        st = launch_xcol_n((const XColEntry *)f.xcol, native ? 3 : 0, slab, YC, YC, 1, 0, out, f.roots_x,
                           ep4(f, nullptr), s, t);
    if (st == FFTB_SUCCESS && t) st = timer_end(t, s);
    return st;
}

int fused4d_backward(const Fused4D &f, void *in, void *out, void *work, double scale, cudaStream_t s, LaunchTimer *t)
{
    const long long C = f.nz * (f.nw / 2 + 1), YC = f.ny * C;
    const bool native = f.layout == FFTB_4D_NATIVE_XZWY;
    void *slab = native ? work : in;
    if (native && !work) return FFTB_ERROR_NO_WORK_AREA;
    const PlaneEntry *pe = (const PlaneEntry *)f.plane;
    int st = launch_xcol_n((const XColEntry *)f.xcol, native ? 4 : 1, slab, YC, YC, 1, 0, in, f.roots_x,
                           ep4(f, nullptr), s, t);
    if (st == FFTB_SUCCESS)
        st = launch_xcol_n((const XColEntry *)f.ycol, 1, slab, C, C, f.nx, YC, nullptr, f.roots_y, ep4(f, nullptr), s, t);
    if (st == FFTB_SUCCESS) st = launch_plane_n(pe, f.nx * f.ny, true, slab, out, f.roots_plane, scale, s, t);
    if (st == FFTB_SUCCESS && t) st = timer_end(t, s);
    return st;
}

int fused4d_spectral(const Fused4D &f, const void *in, void *out, void *work, const EpValues &ep, cudaStream_t s,
                     LaunchTimer *t)
{
    if (!work) return FFTB_ERROR_NO_WORK_AREA;
    const long long C = f.nz * (f.nw / 2 + 1), YC = f.ny * C;
    const PlaneEntry *pe = (const PlaneEntry *)f.plane;
    int st = launch_plane_n(pe, f.nx * f.ny, false, in, work, f.roots_plane, 1.0, s, t);
    if (st == FFTB_SUCCESS)
        st = launch_xcol_n((const XColEntry *)f.ycol, 0, work, C, C, f.nx, YC, nullptr, f.roots_y, ep4(f, nullptr), s, t);
    if (st == FFTB_SUCCESS)
        st = launch_xcol_n((const XColEntry *)f.xcol, 2, work, YC, YC, 1, 0, nullptr, f.roots_x, ep4(f, &ep), s, t);
    if (st == FFTB_SUCCESS)
        st = launch_xcol_n((const XColEntry *)f.ycol, 1, work, C, C, f.nx, YC, nullptr, f.roots_y, ep4(f, nullptr), s, t);
    if (st == FFTB_SUCCESS)
        st = launch_plane_n(pe, f.nx * f.ny, true, work, out, f.roots_plane,
                            1.0 / (double)(f.nx * f.ny * f.nz * f.nw), s, t);
    if (st == FFTB_SUCCESS && t) st = timer_end(t, s);
    return st;
}

int fused4d_forward_adjoint(const Fused4D &f, void *gspec, void *greal, void *work, cudaStream_t s, LaunchTimer *t)
{
    const long long C = f.nz * (f.nw / 2 + 1), YC = f.ny * C;
    const bool native = f.layout == FFTB_4D_NATIVE_XZWY;
    void *slab = native ? work : gspec;
    if (native && !work) return FFTB_ERROR_NO_WORK_AREA;
    EpValues ev;
    ev.mode = EP_HALFW;
    ev.hw = 0.5;
    int st = launch_xcol_n((const XColEntry *)f.xcol, native ? 4 : 1, slab, YC, YC, 1, 0, gspec, f.roots_x,
                           ep4(f, &ev), s, t);
    if (st == FFTB_SUCCESS)
        st = launch_xcol_n((const XColEntry *)f.ycol, 1, slab, C, C, f.nx, YC, nullptr, f.roots_y, ep4(f, nullptr), s, t);
    if (st == FFTB_SUCCESS)
        st = launch_plane_n((const PlaneEntry *)f.plane, f.nx * f.ny, true, slab, greal, f.roots_plane, 1.0, s, t);
    if (st == FFTB_SUCCESS && t) st = timer_end(t, s);
    return st;
}

int fused4d_backward_adjoint(const Fused4D &f, const void *greal, void *gspec, void *work, cudaStream_t s,
                             LaunchTimer *t)
{
    const long long C = f.nz * (f.nw / 2 + 1), YC = f.ny * C;
    const bool native = f.layout == FFTB_4D_NATIVE_XZWY;
    void *slab = native ? work : gspec;
    if (native && !work) return FFTB_ERROR_NO_WORK_AREA;
    EpValues ev;
    ev.mode = EP_HALFW;
    ev.hw = 2.0;
    int st = launch_plane_n((const PlaneEntry *)f.plane, f.nx * f.ny, false, greal, slab, f.roots_plane, 1.0, s, t);
    if (st == FFTB_SUCCESS)
        st = launch_xcol_n((const XColEntry *)f.ycol, 0, slab, C, C, f.nx, YC, nullptr, f.roots_y, ep4(f, nullptr), s, t);
    if (st == FFTB_SUCCESS)
        st = launch_xcol_n((const XColEntry *)f.xcol, native ? 3 : 0, slab, YC, YC, 1, 0, gspec, f.roots_x,
                           ep4(f, &ev), s, t);
    if (st == FFTB_SUCCESS && t) st = timer_end(t, s);
    return st;
}

int fused4d_num_launches(const Fused4D &f, int which)
{
    (void)f;
    return which <= 1 ? 3 : 5;
}

} // namespace fftb
