/*
 * fft_oracle.c -- FP64 CPU oracle for the single-GPU transform path of fftm.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: tests, the smoke entry
 * and the CPU-baseline leg of the benchmark may call it.  The product library
 * (fftm_b200) never links or calls it.
 *
 * What it restates:
 *   - The transform semantics that fftm's `ffts` frontend obtains from cuFFT
 *     (cuFFT 11.x as shipped with CUDA 12.9; pinned in the reference only through
 *     its base image, Docker_config/poisson/Dockerfile.cuda:2).  cuFFT is closed,
 *     so its *published* contract is restated: unnormalised DFT with forward
 *     sign -1 and inverse sign +1 (source/external_wrap/cufft_wrap.h:356,386),
 *     "advanced data layout" addressing for cufftMakePlanMany64
 *     (source/external_wrap/cufft_wrap.h:1237-1259), half spectrum on the last
 *     axis for R2C / C2R, and C2R ignoring the imaginary parts of the DC and
 *     Nyquist bins of the last axis after the leading axes were inverted.
 *   - The plan parameters and stage order of `ffts` for 3D (source/ffts.hpp:677-695)
 *     and 4D pencil / slab (source/ffts.hpp:697-776, 809-867), the fftm 4D
 *     native_xzwy (y,x) plan (source/fftm.hpp:2941-2961), the 4D permutations
 *     (source/detail/direct_transpose_4d.h:17-32, 42-120) and the array
 *     arrangers (source/detail/array_arrangers.h:11-58: the first listed index is
 *     the fastest-varying one).
 *   - The Poisson multiply (examples/poisson/source/poisson_periodic_3d_autotuned.cpp:74-103,
 *     examples/poisson/source/poisson_periodic_4d_autotuned.cpp:252-286,
 *     source/tests/detail/versioned_ffts_3d_test_driver.h:128-154) and the 1/N
 *     scale (source/tests/detail/fft_benchmark_common.h:271-281).
 *   - The splitmix64 hash generator of the reference's tests
 *     (source/tests/detail/fft_benchmark_common.h:201-257).
 *
 * The 1D kernel is a recursive mixed-radix decimation-in-time DFT (any length;
 * prime lengths fall back to the O(n^2) definition).  Twiddles are exp(-2*pi*i*m/n)
 * evaluated in double precision.  OpenMP parallelises over independent lines.
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double _Complex cplx;

enum { ORC_R2C = 1, ORC_C2R = 2, ORC_C2CF = 3, ORC_C2CB = 4 }; /* source/fft_direction.h:9-15 */

static int g_threads = 1;

void orc_set_threads(int n) { g_threads = n < 1 ? 1 : n; }
int orc_get_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------ generator */
/* source/tests/detail/fft_benchmark_common.h:201-217 */
uint64_t orc_splitmix64(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

static double unit_from_state(uint64_t state)
{
    const uint64_t bits = orc_splitmix64(state);
    return (double)(bits >> 11) * (1.0 / 9007199254740992.0);
}

/* 3D fill by logical index (x,y,z) (fft_benchmark_common.h:219-237); element goes to
 * out[x*sx + y*sy + z*sz].  single != 0 reproduces unit_random_from_state<float>. */
void orc_fill_random_3d(double *out, long nx, long ny, long nz, long sx, long sy, long sz, uint64_t seed,
                        int single)
{
    for (long x = 0; x < nx; ++x)
        for (long y = 0; y < ny; ++y)
            for (long z = 0; z < nz; ++z) {
                const uint64_t st = seed ^ ((uint64_t)x * 0xD6E8FEB86659FD93ull) ^
                                    ((uint64_t)y * 0xA5A3564E27F886A5ull) ^ ((uint64_t)z * 0x9E3779B97F4A7C15ull);
                const double u = unit_from_state(st);
                double v;
                if (single) {
                    const float uf = (float)u;
                    v = (double)(2.0f * uf - 1.0f);
                } else {
                    v = 2.0 * u - 1.0;
                }
                out[x * sx + y * sy + z * sz] = v;
            }
}

/* 4D fill by logical index (x,y,z,w) (fft_benchmark_common.h:239-257). */
void orc_fill_random_4d(double *out, long nx, long ny, long nz, long nw, long sx, long sy, long sz, long sw,
                        uint64_t seed, int single)
{
    for (long x = 0; x < nx; ++x)
        for (long y = 0; y < ny; ++y)
            for (long z = 0; z < nz; ++z)
                for (long w = 0; w < nw; ++w) {
                    const uint64_t st = seed ^ ((uint64_t)x * 0xD6E8FEB86659FD93ull) ^
                                        ((uint64_t)y * 0xA5A3564E27F886A5ull) ^
                                        ((uint64_t)z * 0x9E3779B97F4A7C15ull) ^ ((uint64_t)w * 0x94D049BB133111EBull);
                    const double u = unit_from_state(st);
                    double v;
                    if (single) {
                        const float uf = (float)u;
                        v = (double)(2.0f * uf - 1.0f);
                    } else {
                        v = 2.0 * u - 1.0;
                    }
                    out[x * sx + y * sy + z * sz + w * sw] = v;
                }
}

/* ------------------------------------------------------------------ 1D DFT */
typedef struct {
    long n;
    cplx *w; /* w[m] = exp(-2*pi*i*m/n), m in [0,n) */
} twiddles;

static void twiddles_init(twiddles *t, long n)
{
    t->n = n;
    t->w = (cplx *)malloc(sizeof(cplx) * (size_t)(n > 0 ? n : 1));
    for (long m = 0; m < n; ++m) {
        const double a = -2.0 * M_PI * (double)m / (double)n;
        t->w[m] = cos(a) + I * sin(a);
    }
}

static void twiddles_free(twiddles *t) { free(t->w); }

static long smallest_factor(long n)
{
    if (n % 4 == 0) return 4;
    if (n % 2 == 0) return 2;
    for (long p = 3; p * p <= n; p += 2)
        if (n % p == 0) return p;
    return n;
}

/* out[k] = sum_j in[j*is] * W^(j*k) for k in [0,n), W = exp(sign*2*pi*i/n).
 * tw is the table of the top-level length N0; a root of this level is tw[step]. */
static void dft_rec(const cplx *in, long is, cplx *out, long n, const twiddles *tw, long step, int sign)
{
    if (n == 1) {
        out[0] = in[0];
        return;
    }
    const long N0 = tw->n;
#define ROOT(e) (sign < 0 ? tw->w[((e) % n) * step] : conj(tw->w[((e) % n) * step]))
    long p = smallest_factor(n);
    if (p == n) {
        for (long k = 0; k < n; ++k) {
            cplx acc = 0;
            for (long j = 0; j < n; ++j) acc += in[j * is] * ROOT(j * k);
            out[k] = acc;
        }
        return;
    }
    const long m = n / p;
    for (long q = 0; q < p; ++q) dft_rec(in + q * is, is * p, out + q * m, m, tw, step * p, sign);
    cplx tloc[64];
    cplx *t = p <= 64 ? tloc : (cplx *)malloc(sizeof(cplx) * (size_t)p);
    cplx sloc[64];
    cplx *s = p <= 64 ? sloc : (cplx *)malloc(sizeof(cplx) * (size_t)p);
    for (long k = 0; k < m; ++k) {
        for (long q = 0; q < p; ++q) t[q] = out[q * m + k] * ROOT(q * k);
        for (long r = 0; r < p; ++r) {
            cplx acc = 0;
            for (long q = 0; q < p; ++q) acc += t[q] * ROOT(q * r * m);
            s[r] = acc;
        }
        for (long r = 0; r < p; ++r) out[k + m * r] = s[r];
    }
    if (t != tloc) free(t);
    if (s != sloc) free(s);
    (void)N0;
#undef ROOT
}

/* In-place 1D complex DFT of a contiguous line (buf is scratch of n entries). */
static void dft_line(cplx *line, cplx *buf, long n, const twiddles *tw, int sign)
{
    memcpy(buf, line, sizeof(cplx) * (size_t)n);
    dft_rec(buf, 1, line, n, tw, 1, sign);
}

/* Complex row-major array with dims d[0..r-1]; DFT along axis a for all lines. */
static void dft_axis(cplx *a, int r, const long *d, int axis, int sign)
{
    long n = d[axis];
    long inner = 1, outer = 1;
    for (int j = axis + 1; j < r; ++j) inner *= d[j];
    for (int j = 0; j < axis; ++j) outer *= d[j];
    const long lines = inner * outer;
    twiddles tw;
    twiddles_init(&tw, n);
#pragma omp parallel num_threads(g_threads)
    {
        cplx *line = (cplx *)malloc(sizeof(cplx) * (size_t)n);
        cplx *buf = (cplx *)malloc(sizeof(cplx) * (size_t)n);
#pragma omp for schedule(static)
        for (long l = 0; l < lines; ++l) {
            const long o = l / inner, i = l % inner;
            cplx *base = a + o * n * inner + i;
            for (long j = 0; j < n; ++j) line[j] = base[j * inner];
            dft_line(line, buf, n, &tw, sign);
            for (long j = 0; j < n; ++j) base[j * inner] = line[j];
        }
        free(line);
        free(buf);
    }
    twiddles_free(&tw);
}

/* 1D C2R of one Hermitian half line h[0..n/2] into real out (length n), unnormalised. */
static void c2r_line(const cplx *h, double *out, long n, cplx *full, cplx *buf, const twiddles *tw)
{
    const long nh = n / 2 + 1;
    for (long k = 0; k < nh; ++k) full[k] = h[k];
    full[0] = creal(full[0]);
    if (n % 2 == 0) full[n / 2] = creal(full[n / 2]);
    for (long k = nh; k < n; ++k) full[k] = conj(full[n - k]);
    dft_line(full, buf, n, tw, +1);
    for (long j = 0; j < n; ++j) out[j] = creal(full[j]);
}

/* ------------------------------------------------------------------ plan exec */
/* Offset of a multi-index in the "advanced layout" (cuFFT docs; used by
 * cufftMakePlanMany64 in source/external_wrap/cufft_wrap.h:1237-1259). */
static long adv_offset(int r, const long *idx, const long *embed, long stride)
{
    long off = 0;
    for (int j = 0; j < r; ++j) off = off * (j == 0 ? 1 : embed[j]) + idx[j];
    return off * stride;
}

static void unravel(long lin, int r, const long *d, long *idx)
{
    for (int j = r - 1; j >= 0; --j) {
        idx[j] = lin % d[j];
        lin /= d[j];
    }
}

/*
 * Executes one plan with fftm's BaseFFT semantics: add_plan_{1D,2D,3D}<dir>
 * (source/external_wrap/fft_wrap_many.h:137-186) followed by exec(name, in, out)
 * (:375-383).  Real arrays are double, complex arrays are interleaved double pairs.
 * inembed/onembed may be NULL for the default (tight) layout.  Returns 0 on success.
 */
int orc_exec(int dir, int rank, const long *n, const long *inembed, long istride, long idist, const long *onembed,
             long ostride, long odist, long batch, const double *in, double *out)
{
    if (rank < 1 || rank > 3) return -1;
    long nn[3], ie[3], oe[3];
    long nh_last = n[rank - 1] / 2 + 1;
    for (int j = 0; j < rank; ++j) nn[j] = n[j];
    long total = 1;
    for (int j = 0; j < rank; ++j) total *= nn[j];
    long cdims[3];
    for (int j = 0; j < rank; ++j) cdims[j] = nn[j];
    cdims[rank - 1] = nh_last;
    long ctotal = 1;
    for (int j = 0; j < rank; ++j) ctotal *= cdims[j];

    /* default layouts (embed == NULL): tight */
    const long *in_dims = (dir == ORC_C2R) ? cdims : nn;
    const long *out_dims = (dir == ORC_R2C) ? cdims : nn;
    long def_is = 1, def_os = 1, def_id, def_od;
    def_id = 1;
    def_od = 1;
    for (int j = 0; j < rank; ++j) {
        def_id *= in_dims[j];
        def_od *= out_dims[j];
    }
    for (int j = 0; j < rank; ++j) {
        ie[j] = inembed ? inembed[j] : in_dims[j];
        oe[j] = onembed ? onembed[j] : out_dims[j];
    }
    if (!inembed) {
        istride = def_is;
        idist = def_id;
    }
    if (!onembed) {
        ostride = def_os;
        odist = def_od;
    }

    const int cin = (dir != ORC_R2C);
    const int cout = (dir != ORC_C2R);
    const cplx *cinp = (const cplx *)in;
    cplx *coutp = (cplx *)out;
    long idx[3];

    for (long b = 0; b < batch; ++b) {
        if (dir == ORC_C2CF || dir == ORC_C2CB || dir == ORC_R2C) {
            cplx *a = (cplx *)malloc(sizeof(cplx) * (size_t)total);
            for (long l = 0; l < total; ++l) {
                unravel(l, rank, nn, idx);
                const long off = b * idist + adv_offset(rank, idx, ie, istride);
                a[l] = cin ? cinp[off] : (cplx)in[off];
            }
            const int sign = (dir == ORC_C2CB) ? +1 : -1;
            for (int ax = rank - 1; ax >= 0; --ax) dft_axis(a, rank, nn, ax, sign);
            const long *od = cout && dir == ORC_R2C ? cdims : nn;
            long otot = 1;
            for (int j = 0; j < rank; ++j) otot *= od[j];
            for (long l = 0; l < otot; ++l) {
                unravel(l, rank, od, idx);
                long lin = 0;
                for (int j = 0; j < rank; ++j) lin = lin * nn[j] + idx[j];
                coutp[b * odist + adv_offset(rank, idx, oe, ostride)] = a[lin];
            }
            free(a);
        } else { /* C2R: invert the leading axes, then C2R on the last axis */
            cplx *a = (cplx *)malloc(sizeof(cplx) * (size_t)ctotal);
            for (long l = 0; l < ctotal; ++l) {
                unravel(l, rank, cdims, idx);
                a[l] = cinp[b * idist + adv_offset(rank, idx, ie, istride)];
            }
            for (int ax = rank - 2; ax >= 0; --ax) dft_axis(a, rank, cdims, ax, +1);
            const long nl = nn[rank - 1];
            const long lines = ctotal / nh_last;
            twiddles tw;
            twiddles_init(&tw, nl);
#pragma omp parallel num_threads(g_threads)
            {
                cplx *full = (cplx *)malloc(sizeof(cplx) * (size_t)nl);
                cplx *buf = (cplx *)malloc(sizeof(cplx) * (size_t)nl);
                double *row = (double *)malloc(sizeof(double) * (size_t)nl);
                long lidx[3];
#pragma omp for schedule(static)
                for (long l = 0; l < lines; ++l) {
                    c2r_line(a + l * nh_last, row, nl, full, buf, &tw);
                    unravel(l * nn[rank - 1], rank, nn, lidx);
                    for (long j = 0; j < nl; ++j) {
                        lidx[rank - 1] = j;
                        out[b * odist + adv_offset(rank, lidx, oe, ostride)] = row[j];
                    }
                }
                free(full);
                free(buf);
                free(row);
            }
            twiddles_free(&tw);
            free(a);
        }
    }
    return 0;
}

/* ------------------------------------------------------------------ ffts 3D */
/* forward_3d plan: source/ffts.hpp:680-686.  real [x][y][z] -> complex [kx][ky][kz<nz/2+1] */
int orc_ffts3d_forward(long nx, long ny, long nz, const double *in, double *out)
{
    const long n[3] = {nx, ny, nz}, ie[3] = {nx, ny, nz}, oe[3] = {nx, ny, nz / 2 + 1};
    return orc_exec(ORC_R2C, 3, n, ie, 1, nx * ny * nz, oe, 1, nx * ny * (nz / 2 + 1), 1, in, out);
}

/* inverse_3d plan: source/ffts.hpp:688-694 (unnormalised) */
int orc_ffts3d_backward(long nx, long ny, long nz, const double *in, double *out)
{
    const long n[3] = {nx, ny, nz}, ie[3] = {nx, ny, nz / 2 + 1}, oe[3] = {nx, ny, nz};
    return orc_exec(ORC_C2R, 3, n, ie, 1, nx * ny * (nz / 2 + 1), oe, 1, nx * ny * nz, 1, in, out);
}

/* 2D: source/ffts.hpp:659-675 */
int orc_ffts2d_forward(long nx, long ny, const double *in, double *out)
{
    const long n[2] = {nx, ny}, ie[2] = {nx, ny}, oe[2] = {nx, ny / 2 + 1};
    return orc_exec(ORC_R2C, 2, n, ie, 1, nx * ny, oe, 1, nx * (ny / 2 + 1), 1, in, out);
}

int orc_ffts2d_backward(long nx, long ny, const double *in, double *out)
{
    const long n[2] = {nx, ny}, ie[2] = {nx, ny / 2 + 1}, oe[2] = {nx, ny};
    return orc_exec(ORC_C2R, 2, n, ie, 1, nx * (ny / 2 + 1), oe, 1, nx * ny, 1, in, out);
}

/* ------------------------------------------------------------------ ffts 4D */
/* Physical offset of logical index idx[0..3] with logical dims d[0..3] under a
 * custom_index_fast_arranger<order...> (order lists logical axes fastest first). */
static long arr_off(const long *idx, const long *d, const int *order)
{
    long off = 0, mult = 1;
    for (int j = 0; j < 4; ++j) {
        off += idx[order[j]] * mult;
        mult *= d[order[j]];
    }
    return off;
}

/* direct_transpose_4d_functor (source/detail/direct_transpose_4d.h:17-32):
 * out(c[D0],c[D1],c[D2],c[D3]) = in(c) over the source logical range. */
static void permute4(const cplx *src, const long *sd, const int *sord, cplx *dst, const long *dd, const int *dord,
                     const int *D)
{
    long c[4], o[4];
    for (c[0] = 0; c[0] < sd[0]; ++c[0])
        for (c[1] = 0; c[1] < sd[1]; ++c[1])
            for (c[2] = 0; c[2] < sd[2]; ++c[2])
                for (c[3] = 0; c[3] < sd[3]; ++c[3]) {
                    for (int j = 0; j < 4; ++j) o[j] = c[D[j]];
                    dst[arr_off(o, dd, dord)] = src[arr_off(c, sd, sord)];
                }
}

enum { ORC_4D_PENCIL = 0, ORC_4D_SLAB = 1, ORC_4D_NATIVE_XZWY = 2 };

static const int A0123[4] = {0, 1, 2, 3}, A0213[4] = {0, 2, 1, 3}, A3210[4] = {3, 2, 1, 0},
                 A1032[4] = {1, 0, 3, 2}, A2103[4] = {2, 1, 0, 3};

/* 4D forward.  layout: 0 = ffts pencil (source/ffts.hpp:809-825),
 * 1 = ffts slab (:827-837), 2 = fftm slab with native_xzwy spectrum
 * (source/fftm.hpp:2941-2961; 2D R2C (z,w) then (y,x) C2C). */
int orc_ffts4d_forward(int layout, long nx, long ny, long nz, long nw, const double *in, double *out)
{
    const long nwh = nw / 2 + 1;
    const long vol = nx * ny * nz * nwh;
    cplx *s0 = (cplx *)malloc(sizeof(cplx) * (size_t)vol);
    cplx *s1 = (cplx *)malloc(sizeof(cplx) * (size_t)vol);
    cplx *o = (cplx *)out;
    int rc = 0;
    if (layout == ORC_4D_PENCIL) {
        const long rb = nx * ny * nz, zb = nx * ny * nwh, yb = nx * nz * nwh, xb = ny * nz * nwh;
        const long ws = nx * ny * nz, zs = nx * ny * nwh, ys = nx * nz * nwh;
        long n1;
        long e1 = 1;
        n1 = nw;
        rc |= orc_exec(ORC_R2C, 1, &n1, &e1, ws, 1, &e1, ws, 1, rb, in, (double *)s0); /* forward_w */
        {
            const long sd[4] = {nx, ny, nz, nwh}, dd[4] = {nx, ny, nwh, nz};
            const int D[4] = {0, 1, 3, 2};
            permute4(s0, sd, A0123, s1, dd, A0123, D); /* xyzw_to_xywz */
        }
        n1 = nz;
        rc |= orc_exec(ORC_C2CF, 1, &n1, &e1, zs, 1, &e1, zs, 1, zb, (double *)s1, (double *)s1); /* forward_z */
        {
            const long sd[4] = {nx, ny, nwh, nz}, dd[4] = {nx, nz, nwh, ny};
            const int D[4] = {0, 3, 2, 1};
            permute4(s1, sd, A0123, s0, dd, A0213, D); /* xywz_to_xzwy */
        }
        n1 = ny;
        rc |= orc_exec(ORC_C2CF, 1, &n1, &e1, ys, 1, &e1, ys, 1, yb, (double *)s0, (double *)s0); /* forward_y */
        {
            const long sd[4] = {nx, nz, nwh, ny}, dd[4] = {ny, nz, nwh, nx};
            const int D[4] = {3, 1, 2, 0};
            permute4(s0, sd, A0213, o, dd, A3210, D); /* xzwy_to_yzwx */
        }
        n1 = nx;
        long ex = nx;
        rc |= orc_exec(ORC_C2CF, 1, &n1, &ex, 1, nx, &ex, 1, nx, xb, out, out); /* forward_x */
    } else if (layout == ORC_4D_SLAB) {
        const long n2[2] = {nz, nw}, ie[2] = {nz, nw}, oe[2] = {nz, nwh};
        rc |= orc_exec(ORC_R2C, 2, n2, ie, 1, nz * nw, oe, 1, nz * nwh, nx * ny, in, (double *)s0); /* forward_zw */
        {
            const long sd[4] = {nx, ny, nz, nwh}, dd[4] = {nz, nwh, nx, ny};
            const int D[4] = {2, 3, 0, 1};
            permute4(s0, sd, A3210, s1, dd, A1032, D); /* xyzw_to_zwxy */
        }
        const long nxy[2] = {nx, ny};
        rc |= orc_exec(ORC_C2CF, 2, nxy, nxy, nz * nwh, 1, nxy, nz * nwh, 1, nz * nwh, (double *)s1,
                       (double *)s1); /* forward_xy */
        {
            const long sd[4] = {nz, nwh, nx, ny}, dd[4] = {ny, nz, nwh, nx};
            const int D[4] = {3, 0, 1, 2};
            permute4(s1, sd, A1032, o, dd, A2103, D); /* zwxy_to_yzwx */
        }
    } else if (layout == ORC_4D_NATIVE_XZWY) {
        const long n2[2] = {nz, nw}, ie[2] = {nz, nw}, oe[2] = {nz, nwh};
        rc |= orc_exec(ORC_R2C, 2, n2, ie, 1, nz * nw, oe, 1, nz * nwh, nx * ny, in, (double *)s0);
        /* local permute of the slab spectrum [x][y][kz][kw] to stage2 (x,z,w,y) under
         * arranger_0213 = physical [y][kz][kw][x] (source/fftm.hpp:201-228) */
        {
            const long sd[4] = {nx, ny, nz, nwh}, dd[4] = {nx, nz, nwh, ny};
            const int D[4] = {0, 2, 3, 1};
            permute4(s0, sd, A3210, o, dd, A0213, D);
        }
        /* forward_xy_xzwy_native: 2D C2C n=(ny,nx), inembed=(ny, nx*nz*nwh), istride 1,
         * idist nx, batch nz*nwh (source/fftm.hpp:2941-2961) */
        const long n2b[2] = {ny, nx}, e2b[2] = {ny, nx * nz * nwh};
        rc |= orc_exec(ORC_C2CF, 2, n2b, e2b, 1, nx, e2b, 1, nx, nz * nwh, out, out);
    } else {
        rc = -1;
    }
    free(s0);
    free(s1);
    return rc;
}

/* 4D inverse (unnormalised).  Destroys `in` like ffts::backward (source/ffts.hpp:377-383). */
int orc_ffts4d_backward(int layout, long nx, long ny, long nz, long nw, double *in, double *out)
{
    const long nwh = nw / 2 + 1;
    const long vol = nx * ny * nz * nwh;
    cplx *s0 = (cplx *)malloc(sizeof(cplx) * (size_t)vol);
    cplx *s1 = (cplx *)malloc(sizeof(cplx) * (size_t)vol);
    cplx *ci = (cplx *)in;
    int rc = 0;
    if (layout == ORC_4D_PENCIL) { /* source/ffts.hpp:839-855 */
        const long rb = nx * ny * nz, zb = nx * ny * nwh, yb = nx * nz * nwh, xb = ny * nz * nwh;
        const long ws = nx * ny * nz, zs = nx * ny * nwh, ys = nx * nz * nwh;
        long n1 = nx, ex = nx, e1 = 1;
        rc |= orc_exec(ORC_C2CB, 1, &n1, &ex, 1, nx, &ex, 1, nx, xb, in, in); /* inverse_x */
        {
            const long sd[4] = {ny, nz, nwh, nx}, dd[4] = {nx, nz, nwh, ny};
            const int D[4] = {3, 1, 2, 0};
            permute4(ci, sd, A3210, s0, dd, A0213, D); /* yzwx_to_xzwy */
        }
        n1 = ny;
        rc |= orc_exec(ORC_C2CB, 1, &n1, &e1, ys, 1, &e1, ys, 1, yb, (double *)s0, (double *)s0);
        {
            const long sd[4] = {nx, nz, nwh, ny}, dd[4] = {nx, ny, nwh, nz};
            const int D[4] = {0, 3, 2, 1};
            permute4(s0, sd, A0213, s1, dd, A0123, D); /* xzwy_to_xywz */
        }
        n1 = nz;
        rc |= orc_exec(ORC_C2CB, 1, &n1, &e1, zs, 1, &e1, zs, 1, zb, (double *)s1, (double *)s1);
        {
            const long sd[4] = {nx, ny, nwh, nz}, dd[4] = {nx, ny, nz, nwh};
            const int D[4] = {0, 1, 3, 2};
            permute4(s1, sd, A0123, s0, dd, A0123, D); /* xywz_to_xyzw */
        }
        n1 = nw;
        rc |= orc_exec(ORC_C2R, 1, &n1, &e1, ws, 1, &e1, ws, 1, rb, (double *)s0, out); /* inverse_w */
    } else if (layout == ORC_4D_SLAB) { /* source/ffts.hpp:857-867 */
        {
            const long sd[4] = {ny, nz, nwh, nx}, dd[4] = {nz, nwh, nx, ny};
            const int D[4] = {1, 2, 3, 0};
            permute4(ci, sd, A2103, s1, dd, A1032, D); /* yzwx_to_zwxy */
        }
        const long nxy[2] = {nx, ny};
        rc |= orc_exec(ORC_C2CB, 2, nxy, nxy, nz * nwh, 1, nxy, nz * nwh, 1, nz * nwh, (double *)s1,
                       (double *)s1);
        {
            const long sd[4] = {nz, nwh, nx, ny}, dd[4] = {nx, ny, nz, nwh};
            const int D[4] = {2, 3, 0, 1};
            permute4(s1, sd, A1032, s0, dd, A3210, D); /* zwxy_to_xyzw */
        }
        const long n2[2] = {nz, nw}, ie[2] = {nz, nwh}, oe[2] = {nz, nw};
        rc |= orc_exec(ORC_C2R, 2, n2, ie, 1, nz * nwh, oe, 1, nz * nw, nx * ny, (double *)s0, out);
    } else if (layout == ORC_4D_NATIVE_XZWY) {
        const long n2b[2] = {ny, nx}, e2b[2] = {ny, nx * nz * nwh};
        rc |= orc_exec(ORC_C2CB, 2, n2b, e2b, 1, nx, e2b, 1, nx, nz * nwh, in, in);
        {
            const long sd[4] = {nx, nz, nwh, ny}, dd[4] = {nx, ny, nz, nwh};
            const int D[4] = {0, 3, 1, 2};
            permute4(ci, sd, A0213, s0, dd, A3210, D);
        }
        const long n2[2] = {nz, nw}, ie[2] = {nz, nwh}, oe[2] = {nz, nw};
        rc |= orc_exec(ORC_C2R, 2, n2, ie, 1, nz * nwh, oe, 1, nz * nw, nx * ny, (double *)s0, out);
    } else {
        rc = -1;
    }
    free(s0);
    free(s1);
    return rc;
}

/* ------------------------------------------------------------------ spectral ops */
static long wavenumber(long i, long n, int halved) { return halved ? i : (i <= n / 2 ? i : i - n); }

/* Poisson multiply on a 3D [kx][ky][kz<nz/2+1] spectrum: u_hat = sign * f_hat / |k|^2,
 * k = 0 -> 0 (source/tests/detail/versioned_ffts_3d_test_driver.h:128-154 with
 * sign = -1; examples/poisson/source/poisson_periodic_3d_autotuned.cpp:74-103 with sign = +1). */
void orc_poisson3d(long nx, long ny, long nz, double sign, double *spec)
{
    const long nzh = nz / 2 + 1;
    cplx *s = (cplx *)spec;
    for (long x = 0; x < nx; ++x)
        for (long y = 0; y < ny; ++y)
            for (long z = 0; z < nzh; ++z) {
                const long kx = wavenumber(x, nx, 0), ky = wavenumber(y, ny, 0), kz = z;
                const double k2 = (double)(kx * kx + ky * ky + kz * kz);
                cplx *v = &s[(x * ny + y) * nzh + z];
                *v = (k2 == 0.0) ? 0.0 : *v * (sign / k2);
            }
}

/* 4D Poisson multiply on each supported spectrum layout
 * (examples/poisson/source/poisson_periodic_4d_autotuned.cpp:252-286). */
void orc_poisson4d(int layout, long nx, long ny, long nz, long nw, double sign, double *spec)
{
    const long nwh = nw / 2 + 1;
    cplx *s = (cplx *)spec;
    for (long x = 0; x < nx; ++x)
        for (long y = 0; y < ny; ++y)
            for (long z = 0; z < nz; ++z)
                for (long w = 0; w < nwh; ++w) {
                    const long kx = wavenumber(x, nx, 0), ky = wavenumber(y, ny, 0), kz = wavenumber(z, nz, 0);
                    const double k2 = (double)(kx * kx + ky * ky + kz * kz + w * w);
                    long off;
                    if (layout == ORC_4D_SLAB)
                        off = ((x * ny + y) * nz + z) * nwh + w; /* [kx][ky][kz][kw] */
                    else
                        off = ((y * nz + z) * nwh + w) * nx + x; /* [ky][kz][kw][kx] */
                    s[off] = (k2 == 0.0) ? 0.0 : s[off] * (sign / k2);
                }
}

void orc_scale(double *a, long n, double s)
{
    for (long i = 0; i < n; ++i) a[i] *= s;
}
