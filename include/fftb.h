/*
 * fftb.h -- C ABI of the B200-native (sm_100a) replacement for fftm's
 * single-GPU transform path.
 *
 * Two layers are exported, both with plain pointers, sizes and int status codes
 * (0 = success, negative = error; no exceptions cross the ABI):
 *
 *  1. Plan objects that stand in for one `cufft::fft<T, D>` plan of the
 *     reference's backend (reference source/external_wrap/cufft_wrap.h:456-480,
 *     483-1282).  Parameters have cuFFT "advanced layout" meaning with 64-bit
 *     sizes, exactly as fft_wrap_many::add_plan_{1D,2D,3D} passes them
 *     (source/external_wrap/fft_wrap_many.h:137-186).  Work areas are external
 *     and optional; streams are per plan.
 *
 *  2. `ffts` transform objects that stand in for fftm::ffts<...>
 *     (source/ffts.hpp:159-383): 2D/3D and 4D R2C forward / C2R inverse with
 *     the reference's physical array layouts, plus the fused periodic Poisson
 *     solve of examples/poisson and source/tests/test_{3D,4D}_poisson.cu.
 *
 * All execution calls are asynchronous on the object's stream.  Device pointers
 * only.  One host thread per object (the reference has no internal locking
 * either, source/ffts.hpp:159).
 */
#ifndef FFTB_H
#define FFTB_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status codes */
#define FFTB_SUCCESS 0
#define FFTB_ERROR_INVALID_VALUE (-1)     /* bad size, stride, direction, dtype, layout */
#define FFTB_ERROR_UNSUPPORTED_SIZE (-2)  /* a line length the kernels do not cover */
#define FFTB_ERROR_CUDA (-3)              /* a CUDA runtime call or launch failed */
#define FFTB_ERROR_ALLOC (-4)             /* device allocation failed */
#define FFTB_ERROR_INVALID_HANDLE (-5)
#define FFTB_ERROR_NOT_INITIALIZED (-6)   /* ffts object used before init (source/ffts.hpp:639-645) */
#define FFTB_ERROR_WRONG_DIMENSION (-7)   /* 3D object used as 4D etc. (source/ffts.hpp:647-657) */
#define FFTB_ERROR_ALREADY_INITIALIZED (-8) /* init twice (source/ffts.hpp:631-637) */
#define FFTB_ERROR_MISALIGNED (-9)        /* pointer not aligned to its element type */
#define FFTB_ERROR_NO_WORK_AREA (-10)     /* work area required but missing */
#define FFTB_ERROR_CACHE_IO (-11)         /* autotune cache unreadable, not KEY=VALUE, or not writable */
#define FFTB_ERROR_CACHE_MISMATCH (-12)   /* autotune cache for another problem, schema or hardware */
#define FFTB_ERROR_CACHE_MISSING (-13)    /* autotune cache absent and creation not requested */
#define FFTB_ERROR_TUNE_FAILED (-14)      /* every autotune candidate failed */

/* direction values equal fftm::direction (source/fft_direction.h:9-15) */
#define FFTB_R2C 1
#define FFTB_C2R 2
#define FFTB_C2CF 3
#define FFTB_C2CB 4

#define FFTB_F32 0
#define FFTB_F64 1

/* 4D layouts:
 *  PENCIL      ffts<..., strategy_4d_pencil_pencil>: real [w][z][y][x] -> spectrum [ky][kz][kw<nw/2+1][kx]
 *              (source/ffts.hpp:126-134, 809-825)
 *  SLAB        ffts<..., strategy_4d_slab_slab>:     real [x][y][z][w] -> spectrum [kx][ky][kz][kw<nw/2+1]
 *              (source/ffts.hpp:144-150, 827-837)
 *  NATIVE_XZWY fftm slab with fftm_4d_spectral_layout::native_xzwy: real [x][y][z][w] -> spectrum
 *              [ky][kz][kw<nw/2+1][kx] (source/fftm_options.hpp:48-52, source/fftm.hpp:2941-2961) */
#define FFTB_4D_PENCIL 0
#define FFTB_4D_SLAB 1
#define FFTB_4D_NATIVE_XZWY 2

const char *fftb_status_string(int status);
/* detail message of the last failing call on this host thread ("" if none) */
const char *fftb_last_error_message(void);
/* library version "major.minor.patch" */
const char *fftb_version(void);

/* ------------------------------------------------------------------ plans */
typedef struct fftb_plan_s *fftb_plan;

/* Replaces cufft::fft<T,D>::fft(n, inembed, istride, idist, onembed, ostride, odist,
 * batch) -> create_plan -> cufftMakePlanMany64 (source/external_wrap/cufft_wrap.h:533-566,
 * :1237-1259).  inembed/onembed may be NULL for the default tight layout
 * (cufft_wrap.h:568-587).  *work_bytes receives the work-area size (may be 0).
 * Line lengths: any length up to 4096 runs one pass kernel per axis (radix passes, or
 * chirp-z for a large prime factor); longer lines (up to 2^24 points, or 2^21 when a
 * prime factor above 4096 needs chirp-z) run a long-line step -- four-step through two
 * pass kernels, or chirp-z over a power-of-two four-step convolution -- that keeps two
 * work lines of its own (lines x length complex values each) for the plan's lifetime. */
int fftb_plan_create(int direction, int dtype, int rank, const long long *n, const long long *inembed,
                     long long istride, long long idist, const long long *onembed, long long ostride,
                     long long odist, long long batch, fftb_plan *plan, size_t *work_bytes);
/* Replaces fft_base::get_work_size (cufft_wrap.h:599-602) */
int fftb_plan_get_work_size(fftb_plan plan, size_t *work_bytes);
/* Replaces fft_base::set_work_area (cufft_wrap.h:605-609) */
int fftb_plan_set_work_area(fftb_plan plan, void *work_area);
/* Replaces fft_base::set_stream (cufft_wrap.h:611-615); stream is a cudaStream_t */
int fftb_plan_set_stream(fftb_plan plan, void *stream);
/* Replaces fft_base::exec / exec_no_sync (cufft_wrap.h:649-662): asynchronous.
 * Multi-dimensional C2R plans overwrite `in`, as cuFFT's do. */
int fftb_exec(fftb_plan plan, void *in, void *out);
/* Replaces fft_base::exec_direction (cufft_wrap.h:664-700): a C2C plan may run
 * either sign; R2C/C2R plans only their own direction. */
int fftb_exec_direction(fftb_plan plan, int direction, void *in, void *out);
/* Replaces fft_base::get_direction / descriptor (cufft_wrap.h:470-472,
 * source/external_wrap/fft_plan_descriptor.h:15-32).  Arrays have 3 entries. */
int fftb_plan_describe(fftb_plan plan, int *direction, int *dtype, int *rank, long long *n, long long *inembed,
                       long long *istride, long long *idist, long long *onembed, long long *ostride,
                       long long *odist, long long *batch);
/* number of kernel launches one exec issues */
int fftb_plan_num_launches(fftb_plan plan, int *launches);
/* Replaces ~fft (cufft_wrap.h:589-595) */
int fftb_plan_destroy(fftb_plan plan);

/* ------------------------------------------------------------------ ffts transforms */
typedef struct fftb_ffts_s *fftb_ffts;

/* Profiling options of an ffts object: the reference's ffts_init_options
 * (source/ffts.hpp:64-72).  A key that is NULL or empty turns that profiler off.  The
 * profiler records, per API call scope ("ffts::forward<3>" ...), calls, host milliseconds and
 * device milliseconds (events on the object's stream; skipped while it is being captured);
 * the memory profiler records the object's own device allocations (work area, derivative
 * spectra) with their peaks.  The print flags print the reports to stdout when the object is
 * destroyed (source/ffts.hpp:199-208). */
typedef struct fftb_init_options {
    const char *profiling_key;
    const char *memory_profiling_key;
    int print_profile_summary_on_destroy;
    int print_profile_totals_on_destroy;
    int print_memory_profile_on_destroy;
    int print_memory_totals_on_destroy;
} fftb_init_options;

/* The reference's defaults: keys "ffts_prof" / "ffts_mem", every print on. */
void fftb_init_options_default(fftb_init_options *options);

/* ffts() + ffts::init(nx, ny[, nz[, nw]]) (source/ffts.hpp:192-285).  layout4d is
 * one of FFTB_4D_* and ignored for 2D/3D.  nz = nw = 0 selects 2D; nw = 0 3D. */
int fftb_ffts_create(int dtype, long long nx, long long ny, long long nz, long long nw, int layout4d,
                     fftb_ffts *obj);
/* fftb_ffts_create with profiling options (NULL: fftb_init_options_default); fftb_ffts_create
 * itself has both profilers off. */
int fftb_ffts_create_ex(int dtype, long long nx, long long ny, long long nz, long long nw, int layout4d,
                        const fftb_init_options *options, fftb_ffts *obj);
int fftb_ffts_destroy(fftb_ffts obj);
/* One report of the object's profilers as text (which: 0 profile summary, 1 profile totals,
 * 2 memory profile, 3 memory totals; empty when that profiler is off).  *needed receives the
 * size with the terminating zero; text is truncated to capacity. */
int fftb_ffts_profile_report(fftb_ffts obj, int which, char *text, size_t capacity, size_t *needed);
/* ffts::dimension (source/ffts.hpp:330-334) */
int fftb_ffts_dimension(fftb_ffts obj, int *dim);
/* Work bytes the object needs for forward/backward/poisson (the reference's shared
 * work buffer plus 4D stage scratch, source/ffts.hpp:439-447, 778-796). */
int fftb_ffts_work_size(fftb_ffts obj, size_t *work_bytes);
/* Supplies the work area (caller-owned, >= work_size bytes, 256-byte aligned).  If
 * never called, the first execution that needs scratch allocates it. */
int fftb_ffts_set_work_area(fftb_ffts obj, void *work);
int fftb_ffts_set_stream(fftb_ffts obj, void *stream);
/* ffts::forward (source/ffts.hpp:338-375): unnormalised R2C, e^{-i theta}. */
int fftb_ffts_forward(fftb_ffts obj, const void *real_in, void *complex_out);
/* ffts::backward (source/ffts.hpp:344-383): unnormalised C2R, e^{+i theta}.
 * `complex_in` may be overwritten (the reference's 3D/4D backward is destructive). */
int fftb_ffts_backward(fftb_ffts obj, void *complex_in, void *real_out);
/* backward followed by the 1/N scale of the reference drivers
 * (source/tests/detail/fft_benchmark_common.h:271-281), fused into the last pass. */
int fftb_ffts_backward_normalized(fftb_ffts obj, void *complex_in, void *real_out);
/* Periodic spectral Poisson solve on [0, 2pi)^d with integer wavenumbers:
 * u = C2R( sign * R2C(f) / |k|^2 ) / N, k = 0 mode set to 0.  sign = -1 solves
 * lap u = f (source/tests/test_3D_poisson.cu:82-111), sign = +1 solves -lap u = f
 * (examples/poisson/source/poisson_periodic_3d_autotuned.cpp:74-103).  The
 * multiply is fused into the FFT passes; the spectrum lives in the work area.
 * rhs and solution may alias. */
int fftb_ffts_poisson(fftb_ffts obj, const void *rhs, void *solution, double sign);
/* Spectral filter round trip: u = C2R( G(k) * R2C(f) ) / N with the Gaussian
 * G(k) = exp(-|k|^2 / (2 sigma^2)); optionally followed in the same fused pass by
 * the Poisson multiply (poisson_sign = 0 disables it). */
int fftb_ffts_filter(fftb_ffts obj, const void *in, void *out, double sigma, double poisson_sign);
/* Adjoint kernels for reverse-mode differentiation (no counterpart in the reference).
 * Treat the half spectrum Y as independent complex variables with gradient
 * G = dL/dRe(Y) + i dL/dIm(Y).
 * fftb_ffts_forward_adjoint: the transpose of fftb_ffts_forward, dL/dx = C2R(W G), W = 1/2
 *   on interior bins of the half axis (1 on its DC and Nyquist bins), unnormalised;
 *   grad_spectrum may be overwritten.
 * fftb_ffts_backward_adjoint: the transpose of fftb_ffts_backward (unnormalised C2R),
 *   G = W2 R2C(dL/dx), W2 = 2 on interior half-axis bins, 1 on DC / Nyquist.
 * The spectral multiplies and the Poisson / filter round trips are real diagonal in k and
 * therefore self-adjoint: their adjoint is the same call. */
int fftb_ffts_forward_adjoint(fftb_ffts obj, void *grad_spectrum, void *grad_real);
int fftb_ffts_backward_adjoint(fftb_ffts obj, const void *grad_real, void *grad_spectrum);
/* In-place spectral multiplies on a spectrum in this object's layout (the
 * reference's standalone functors): Poisson sign/|k|^2 (k=0 -> 0) with an extra
 * scale, examples/poisson/source/poisson_periodic_{3d,4d}_autotuned.cpp. */
int fftb_ffts_spectrum_poisson(fftb_ffts obj, void *spectrum, double sign, double scale);
/* Spectral derivative along a logical axis (0 = x, 1 = y, 2 = z, 3 = w) on a spectrum in
 * this object's layout: spec_out = i k_axis spec_in * scale (the reference's
 * derivative_spectra_functor, source/tests/test_3D_poisson.cu:113-145: k = index on the
 * half axis, index or index - n on the full axes, Nyquist bins kept).  In place allowed. */
int fftb_ffts_spectrum_derivative(fftb_ffts obj, const void *spec_in, void *spec_out, int axis, double scale);
/* Spectral truncation in place (the turbulence example's filters,
 * examples/turbulence/source/taylor_green_kernels.h:41-44, 186-200): TWO_THIRDS keeps
 * |k_a| <= n_a / 3 on every axis (dealiasing), BOX keeps |k_a| <= cutoff (cutoff <= 0
 * keeps all); every other mode is set to 0.  k as in fftb_ffts_spectrum_derivative. */
#define FFTB_TRUNCATE_TWO_THIRDS 0
#define FFTB_TRUNCATE_BOX 1
int fftb_ffts_spectrum_truncate(fftb_ffts obj, void *spectrum, int rule, int cutoff);
/* du/d(axis) of a periodic field on [0, 2 pi)^d: C2R(i k_axis R2C(u)) / N, through a
 * spectrum buffer the object allocates on first use.  in and out may alias. */
int fftb_ffts_derivative(fftb_ffts obj, const void *in, void *out, int axis);
/* Every first derivative of u from one forward transform (the reference test's dx, dy,
 * dz spectra, source/tests/test_3D_poisson.cu:113-145): outs[a] = du/d(axis a) for the
 * object's dim axes (x, y, z[, w]); each output is a real array of the input's shape. */
int fftb_ffts_gradient(fftb_ffts obj, const void *in, void *const *outs);
/* number of kernel launches of forward (which=0) / backward (1) / poisson (2) / filter (3) */
int fftb_ffts_num_launches(fftb_ffts obj, int which, int *launches);
/* Profiling hook (the role of the reference's ffts profiler, source/ffts.hpp:64-72,
 * 449-629, but timed on the device): with max_launches > 0, every later execution
 * records a CUDA event on the object's stream before each kernel launch and after
 * the last, for up to max_launches launches; 0 disables and frees the events. */
int fftb_ffts_timing_enable(fftb_ffts obj, int max_launches);
/* Waits for the recorded events and returns, per recorded launch in issue order, its
 * device time in ms, its algorithmic bytes (one read of its input and one write of
 * its output) and its kernel name (NUL-terminated, name_stride bytes per entry).
 * Clears the record. */
int fftb_ffts_timing_read(fftb_ffts obj, float *ms, double *bytes, char *names, int name_stride, int cap,
                          int *count);

/* Execution strategy of an ffts object (the knob the autotuner below measures; the
 * role of fftm's FFTM_AUTOTUNE_STRATEGY_3D/_4D choice, source/fftm_autotune.hpp:31-70).
 *  AUTO    the default: fused multi-axis kernels where the size has them, with the plane
 *          cluster size picked by occupancy; per-axis pass programs otherwise
 *  FUSED   fused kernels (FFTB_ERROR_UNSUPPORTED_SIZE when the size has none); for 3D,
 *          plane_cluster 1, 2, 4 or 8 picks the CTAs per (y, z) plane (0: by occupancy)
 *  STAGED  one pass kernel per axis (the generic pass programs)
 *  FUSED_TC  FUSED with the column kernels (3D: x; 4D: y and x) running their first
 *          radix-16 stage as a 16x16 complex contraction on the tensor cores in split
 *          FP16 (head + tail operands, FP32 accumulation); float32 only */
#define FFTB_STRATEGY_AUTO 0
#define FFTB_STRATEGY_FUSED 1
#define FFTB_STRATEGY_STAGED 2
#define FFTB_STRATEGY_FUSED_TC 3
int fftb_ffts_set_strategy(fftb_ffts obj, int strategy, int plane_cluster);
/* the strategy in effect (FUSED, FUSED_TC or STAGED) and its plane cluster size (0 when STAGED) */
int fftb_ffts_get_strategy(fftb_ffts obj, int *strategy, int *plane_cluster);

/* ------------------------------------------------------------------ batched uneven 3D transforms */
/* Many independent 3D R2C / C2R transforms of different sizes (no counterpart in the
 * reference, whose ffts holds one size).  Transform i has real shape dims[3i..3i+2] =
 * (nx, ny, nz) in the ffts layouts; the user's arrays pack the transforms back to back
 * at the element offsets fftb_batch_layout returns (16-byte aligned).  The passes of
 * all transforms run either one transform after another (mode 0, plain launches) or
 * in ONE persistent launch that takes (pass, tile) items from a stage-ordered work
 * list with per-pass completion counters (mode 1), replayed from a CUDA graph captured
 * per buffer binding (mode 2), or as one launch per (stage, line length) group (modes 3,
 * 4).  Modes 1-4 are float32; float64 batches run mode 0. */
typedef struct fftb_batch_s *fftb_batch;
#define FFTB_BATCH_FORWARD 0   /* in: packed real, out: packed spectrum */
#define FFTB_BATCH_BACKWARD 1  /* in: packed spectrum (overwritten), out: packed real, 1/N scaled */
#define FFTB_BATCH_ROUNDTRIP 2 /* in, out: packed real; C2R(R2C(x)) / N, spectrum in the work area */
#define FFTB_BATCH_POISSON 3   /* in: packed right-hand sides, out: solutions (sign as in fftb_ffts_poisson) */
int fftb_batch_create(int dtype, int count, const long long *dims, fftb_batch *batch);
int fftb_batch_destroy(fftb_batch batch);
/* per-transform element offsets (count entries each; may be NULL) and the packed totals */
int fftb_batch_layout(fftb_batch batch, long long *real_offsets, long long *spectrum_offsets,
                      long long *real_total, long long *spectrum_total);
int fftb_batch_work_size(fftb_batch batch, size_t *bytes);
int fftb_batch_set_work_area(fftb_batch batch, void *work);
int fftb_batch_set_stream(fftb_batch batch, void *stream);
/* Tuning knobs chosen by the autotuner: tiles of (default lines)/tiles_scale lines and
 * at most ctas_per_sm persistent CTAs per SM (0: the occupancy limit). */
int fftb_batch_set_tuning(fftb_batch batch, int tiles_scale, int ctas_per_sm);
/* op: FFTB_BATCH_*; sign: Poisson sign (ignored otherwise); mode: 0 sequential plain
 * launches, 1 one persistent launch, 2 persistent launch replayed from a CUDA graph,
 * 3 grouped launches (one plain launch per stage and line length over the tiles of all
 * transforms in it, each kernel specialised for its line length), 4 the grouped launches
 * replayed from a CUDA graph.  Modes 1-4 need float32. */
int fftb_batch_exec(fftb_batch batch, int op, const void *in, void *out, double sign, int mode);
/* error flag of the last persistent launch of op: 1 if a dependency wait ran out its
 * bounded number of polls (the launch then returned early); synchronises the device. */
int fftb_batch_status(fftb_batch batch, int op, int *error_flag);
/* Polls a dependency wait of the persistent launch makes before it raises the error flag and
 * every CTA returns (0 restores the default, 2^22 polls, about half a second).  Cached CUDA
 * graphs of the batch are rebuilt. */
int fftb_batch_set_wait_limit(fftb_batch batch, long long polls);
/* Self-test of that bounded wait: the persistent kernel on a one-item work list whose
 * producer has no items waits `polls` polls, raises the flag and returns; *error_flag
 * receives it (1 when the path works).  Faults and hangs nothing; the context stays usable. */
int fftb_batch_wait_selftest(long long polls, int *error_flag);
int fftb_batch_describe(fftb_batch batch, int op, double sign, int *passes, int *items, int *grid,
                        int *persistent);

/* ------------------------------------------------------------------ autotuner */
/* The replacement of fftm's autotune surface (source/fftm_autotune.hpp:31-169, 452-477,
 * 660-676; source/fftm_autotune_measure.hpp:21-55, 432-520, 798-854;
 * source/detail/fftm_autotune_hardware.inc:285-425) for the single-GPU transforms:
 * measured candidates, the least median of timed forward+backward pairs (each pair timed
 * with CUDA events on a private stream after `warmup` untimed pairs; every candidate must
 * pass a round-trip check at 64 sampled points, tolerance 1000 eps max(1, log2 N)), and
 * a KEY=VALUE cache file written to <path>.tmp and renamed into place.  The cache carries
 * fftm's schema-2 identity keys (FFTM_AUTOTUNE_SCHEMA=2, _POLICY_VERSION, _LIBRARY=fftb,
 * _DIM, _NUM_GPUS=1, _SIZE_2D/_3D/_4D, _SPECTRAL_LAYOUT_4D, _SOURCE), a "v2:" hardware
 * signature (64-bit FNV-1a of the device class; _STRICT adds UUID and PCI bus id) with
 * the device metadata keys, and the tuned FFTB_AUTOTUNE_* keys. */
#define FFTB_TUNE_CREATE_IF_MISSING 1      /* autotune_options::create_if_missing */
#define FFTB_TUNE_OVERWRITE_ON_MISMATCH 2  /* cache_mismatch_policy::overwrite (else error) */
#define FFTB_TUNE_NO_HARDWARE_CHECK 4      /* validate_hardware = false */
#define FFTB_TUNE_STRICT_DEVICE 8          /* strict_device_identity */
#define FFTB_TUNE_FORCE_MEASURE 16         /* measure and rewrite even if the cache matches */
/* Reads and parses a cache file; returns its canonical text (sorted KEY=VALUE lines).
 * *needed receives the bytes the text takes including its NUL; text may be NULL with
 * capacity 0 to query it.  FFTB_ERROR_CACHE_IO on an unreadable file, an empty file or
 * a line that is not KEY=VALUE. */
int fftb_autotune_load_file(const char *path, char *text, size_t capacity, size_t *needed);
/* Parses KEY=VALUE text and writes it to path through <path>.tmp and rename. */
int fftb_autotune_save_file(const char *path, const char *text);
/* Checks a cache against expected identity and hardware keys (the keys present in
 * expected_text are compared; the cache must also be a measured fftb cache).  Returns
 * FFTB_ERROR_CACHE_MISMATCH with a message naming the first differing key. */
int fftb_autotune_validate(const char *cache_text, const char *expected_text, int flags);
/* "v2:" + 64-bit FNV-1a (16 hex digits) of a canonical hardware description: the hash the
 * reference's hardware signatures use (source/detail/fftm_autotune_hardware.inc:87-97). */
int fftb_autotune_signature(const char *canonical, char *text, size_t capacity, size_t *needed);
/* The hardware keys (signatures and device metadata) of a CUDA device. */
int fftb_autotune_hardware(int device, char *text, size_t capacity, size_t *needed);
/* load_or_measure for an ffts problem (dims and layout4d as fftb_ffts_create) on the
 * current device: use the cache when it matches; measure when it is missing (with
 * CREATE_IF_MISSING, else FFTB_ERROR_CACHE_MISSING) or mismatches (with
 * OVERWRITE_ON_MISMATCH, else FFTB_ERROR_CACHE_MISMATCH).  Returns the config text and
 * *from_cache = 1 when it came from the file.  Candidates: fused kernels with each
 * available plane cluster size, and the staged per-axis passes. */
int fftb_autotune_ffts(int dtype, long long nx, long long ny, long long nz, long long nw, int layout4d,
                       const char *cache_file, int flags, int warmup, int iterations, char *text, size_t capacity,
                       size_t *needed, int *from_cache);
/* Applies the FFTB_AUTOTUNE_STRATEGY / _PLANE_CLUSTER of a config to an ffts object. */
int fftb_ffts_apply_config(fftb_ffts obj, const char *text);
/* load_or_measure for a batch and one op: candidates are sequential launches, the
 * graph-replayed persistent launch with tiles_scale {1, 2} x ctas_per_sm {0, 1, 2}, and
 * the graph-replayed grouped launches with tiles_scale {1, 2}.  The winner's knobs are
 * applied to the batch and its mode returned in *mode. */
int fftb_autotune_batch(fftb_batch batch, int op, double sign, const char *cache_file, int flags, int warmup,
                        int iterations, char *text, size_t capacity, size_t *needed, int *from_cache, int *mode);
/* Applies FFTB_AUTOTUNE_TILES_SCALE / _CTAS_PER_SM of a config; *mode = FFTB_AUTOTUNE_BATCH_MODE. */
int fftb_batch_apply_config(fftb_batch batch, const char *text, int *mode);

/* ------------------------------------------------------------------ slab-distributed transforms */
/* The rank-local part of a 3D (x slabs, the reference's slab path with its same_x
 * redistribution, source/detail/mpi_transpose_3d_same_x.h) or 4D (slab-slab with the
 * same_xw redistribution, source/detail/mpi_transpose_4d_same_xw.h:437-497) R2C / C2R
 * distributed over nranks processes, one GPU each.  The pack of the reference's exchange is
 * the store of the last FFT pass before it and the unpack the load of the first pass after
 * it, so the exchange is one contiguous block per destination (an all-to-all the caller
 * runs: NCCL between GPUs), or nothing when the pack pass stores straight into the peers'
 * receive buffers (fftb_slab_set_peers).
 *   3D: real slab [nx/P][ny][nz] -> spectrum slab [kx][ny/P][nz/2+1] (rank r: ky block r);
 *   4D: real slab [nx/P][ny][nz][nw] -> spectrum [kx][ky][nz/P][nw/2+1] (FFTB_4D_SLAB) or
 *       fftm's native [ky][nz/P][nw/2+1][kx] (FFTB_4D_NATIVE_XZWY), kz block r.
 * Forward: fftb_slab_forward_local(in -> send) ; exchange send -> recv ;
 *          fftb_slab_forward_finish(recv -> spectrum: in place on recv, or into out for
 *          the 4D native layout).  Backward (unnormalised): fftb_slab_backward_local
 *          (spectrum -> send: in place for 3D) ; exchange ; fftb_slab_backward_finish
 *          (recv -> real slab).  Exchange blocks are exchange_elems / nranks complex values,
 *          block q going to rank q and block q of recv coming from rank q.  With one rank,
 *          send and recv may be the same buffer. */
typedef struct fftb_slab_s *fftb_slab;
int fftb_slab_create(int dtype, long long nx, long long ny, long long nz, long long nw, int layout4d, int nranks,
                     int rank, fftb_slab *obj);
int fftb_slab_destroy(fftb_slab obj);
/* elements of the real slab, the spectrum slab, the send / receive buffers (complex) and the
 * work buffer (complex) */
int fftb_slab_sizes(fftb_slab obj, long long *real_elems, long long *spectrum_elems, long long *exchange_elems,
                    long long *work_elems);
int fftb_slab_set_stream(fftb_slab obj, void *stream);
/* receive_blocks[q]: where this rank's block lands in rank q's receive buffer, as an address
 * this GPU can store to (a peer mapping); the forward pack pass then writes there directly
 * and the caller only synchronises the ranks before forward_finish.  NULL: the pack pass
 * writes the send buffer. */
int fftb_slab_set_peers(fftb_slab obj, void *const *receive_blocks);
int fftb_slab_forward_local(fftb_slab obj, const void *in, void *send, void *work);
int fftb_slab_forward_finish(fftb_slab obj, void *recv, void *out);
int fftb_slab_backward_local(fftb_slab obj, void *spectrum, void *send);
int fftb_slab_backward_finish(fftb_slab obj, void *recv, void *out, void *work);

/* SHA-256 (hex) of the sources the library was compiled from (fftm_b200/csrc and include/),
 * so a caller can check that the library it loaded matches a source tree.  No counterpart in
 * the reference (a header-only library, compiled into its caller). */
const char *fftb_build_digest(void);

/* ------------------------------------------------------------------ allocation-free entry point */
/* Bytes of the spectrum scratch that fftb_poisson3d_f32_noalloc keeps in static
 * device memory (nx * ny * (nz/2+1) * 8 must not exceed it). */
#define FFTB_NOALLOC_MAX_SPECTRUM_BYTES (16u * 1024u * 1024u)

/* 3D periodic Poisson solve in float32 that allocates no device memory, for
 * callers that cannot call cudaMalloc: a framework or serving process whose
 * memory pool owns the device, or a job that must not allocate (and so must not
 * risk the implicit synchronisation of cudaMalloc/cudaFree) between steps.  No
 * counterpart in the reference, whose ffts allocates its work buffer
 * (source/ffts.hpp:439-447).
 *
 * Same result as fftb_ffts_poisson on a float32 [x][y][z] field: u = C2R(sign *
 * R2C(f) / |k|^2) / N with k = 0 set to 0.  rhs and solution are caller-owned
 * device arrays of nx*ny*nz floats (they may alias); stream is a cudaStream_t
 * (NULL: the legacy default stream).  2 <= nx, ny, nz <= 4096 and the spectrum at
 * most FFTB_NOALLOC_MAX_SPECTRUM_BYTES (e.g. 128^3); larger sizes return
 * FFTB_ERROR_INVALID_VALUE.  Every line length must have a direct pass kernel (the
 * lengths 2^a * {1, 3, 5, 7, 9, 15, 21, 25, 27}, 11 and 13 times a power of two up to
 * 832, and the odd products listed with the pass kernels; for nz, nz or nz/2): lengths
 * that the regular path runs through chirp-z passes (a large prime factor) need a padded
 * work line and return FFTB_ERROR_UNSUPPORTED_SIZE here.
 *
 * The scratch (twiddle tables and spectrum) is one static __device__ array that
 * every GPU loading the library holds until the process exits.  The first call on
 * a device looks up its address (cudaGetSymbolAddress) for that device; make that
 * first call before any stream capture.  All calls share the array and it keeps
 * the last call's contents (each call rewrites what it reads), so calls whose
 * executions overlap on the GPU -- on different streams, or from different host
 * threads -- race on it and must be serialised by the caller. */
int fftb_poisson3d_f32_noalloc(const float *rhs, float *solution, long long nx, long long ny, long long nz,
                               double sign, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* FFTB_H */
