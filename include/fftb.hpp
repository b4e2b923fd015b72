/* fftb.hpp -- header-only C++ host layer over the fftb C ABI (fftb.h).
 *
 * Mirrors the reference's C++ interfaces for the single-GPU transform path so that C++
 * callers keep their call sites:
 *
 *   fftb::fft<T, D>            cufft::fft<T, D> / fft_base<T>
 *                              (source/external_wrap/cufft_wrap.h:456-480, :483-1282)
 *   fftb::fft_wrap_many<T>     the BaseFFT plan registry of fftm::ffts
 *                              (source/external_wrap/fft_wrap_many.h:25-447)
 *   fftb::ffts<T, S>           fftm::ffts<BaseFFT, Backend, Strategy4D> (source/ffts.hpp:159-383)
 *                              with the fused Poisson solve of examples/poisson
 *   fftb::autotune_options,    fftm_autotune's options, selected_3d_config and
 *   fftb::load_or_measure_config  load_or_measure_3d_config
 *                              (source/fftm_autotune.hpp:46-70, source/fftm_autotune_measure.hpp:432-520)
 *   fftb::batch<T>             many uneven 3D transforms in one graph-replayed launch
 *   fftb::poisson3d_noalloc    the allocation-free float32 3D Poisson solve
 *
 * Error behaviour is the reference's: API misuse throws std::logic_error (init twice, not
 * initialised, wrong dimension, plans added after activation -- source/ffts.hpp:631-657,
 * fft_wrap_many.h:127-130), unknown plan names std::out_of_range (std::map::at), and
 * library failures fftb::error, a std::runtime_error carrying the status code (the
 * reference's CUFFT_SAFE_CALL, source/external_wrap/cufft_wrap.h:31-40).
 *
 * Every exec is asynchronous on the object's stream (the default stream unless
 * set_stream was called); arrays are device pointers, or any array object with a
 * raw_ptr() member (the reference's SCFD arrays).  Link with -lfftb_b200 -lcudart. */
#ifndef FFTB_HPP
#define FFTB_HPP

#include <cuda_runtime.h>

#include <array>
#include <cstddef>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "fftb.h"

namespace fftb {

/* fftm::direction (source/fft_direction.h:9-15) */
enum class direction : int { R2C = FFTB_R2C, C2R = FFTB_C2R, C2CF = FFTB_C2CF, C2CB = FFTB_C2CB };

/* the 4D strategies of ffts and fftm's native_xzwy spectrum (source/fftm_options.hpp:48-52) */
enum class strategy_4d : int {
    pencil_pencil = FFTB_4D_PENCIL,
    slab_slab = FFTB_4D_SLAB,
    native_xzwy = FFTB_4D_NATIVE_XZWY
};

/* ffts_init_options (source/ffts.hpp:64-72): both profilers on and every report printed
 * when the object is destroyed, unless a key is emptied or a flag cleared. */
struct ffts_init_options {
    std::string profiling_key = "ffts_prof";
    std::string memory_profiling_key = "ffts_mem";
    bool print_profile_summary_on_destroy = true;
    bool print_profile_totals_on_destroy = true;
    bool print_memory_profile_on_destroy = true;
    bool print_memory_totals_on_destroy = true;
};

/* fftm_reporting_options (source/fftm_options.hpp:220-229) and the profiling preset
 * (:231-242); on one GPU the fftm frontend's path is this ffts, so they map onto
 * ffts_init_options. */
struct fftm_reporting_options {
    std::string profiling_key;
    std::string memory_profiling_key;
    bool verbose = false;
    bool print_profile_summary_on_destroy = false;
    bool print_profile_totals_on_destroy = false;
    bool print_memory_profile_on_destroy = false;
    bool print_memory_totals_on_destroy = false;
};
inline fftm_reporting_options profiling_reporting_options()
{
    fftm_reporting_options o;
    o.profiling_key = "fftm_prof";
    o.memory_profiling_key = "fftm_mem";
    o.print_profile_summary_on_destroy = true;
    o.print_profile_totals_on_destroy = true;
    o.print_memory_profile_on_destroy = true;
    o.print_memory_totals_on_destroy = true;
    return o;
}
inline ffts_init_options to_ffts_init_options(const fftm_reporting_options &r)
{
    ffts_init_options o;
    o.profiling_key = r.profiling_key;
    o.memory_profiling_key = r.memory_profiling_key;
    o.print_profile_summary_on_destroy = r.print_profile_summary_on_destroy;
    o.print_profile_totals_on_destroy = r.print_profile_totals_on_destroy;
    o.print_memory_profile_on_destroy = r.print_memory_profile_on_destroy;
    o.print_memory_totals_on_destroy = r.print_memory_totals_on_destroy;
    return o;
}

/* fftm_4d_spectral_layout (source/fftm_options.hpp:48-52) and the single-GPU part of
 * fftm_init_options (:347-357): public_yzwx is the ffts pencil spectrum [ky][kz][kw][kx]
 * (byte-identical), native_xzwy fftm's slab path with the same spectrum order. */
enum class fftm_4d_spectral_layout { public_yzwx, native_xzwy };
struct fftm_init_options {
    bool use_optimized = true;
    fftm_4d_spectral_layout spectral_layout_4d = fftm_4d_spectral_layout::public_yzwx;
    fftm_reporting_options reporting;
};
inline strategy_4d strategy_for(fftm_4d_spectral_layout l)
{
    return l == fftm_4d_spectral_layout::native_xzwy ? strategy_4d::native_xzwy : strategy_4d::pencil_pencil;
}

/* A named byte counter with peaks: the memory profiler fft_wrap_many::set_memory_profiler
 * reports into (the role of the reference's memory_profiler_t). */
class memory_profiler {
public:
    using bytes_type = long long;
    struct entry {
        bytes_type current_bytes = 0, peak_bytes = 0;
    };
    void set_bytes(const std::string &name, bytes_type b)
    {
        entry &e = entries_[name];
        e.current_bytes = b;
        if (b > e.peak_bytes) e.peak_bytes = b;
    }
    const std::map<std::string, entry> &entries() const { return entries_; }
    bytes_type total_current() const
    {
        bytes_type t = 0;
        for (const auto &kv : entries_) t += kv.second.current_bytes;
        return t;
    }

private:
    std::map<std::string, entry> entries_;
};

/* A library failure: the status code and the library's message. */
class error : public std::runtime_error {
public:
    error(int status, const std::string &what) : std::runtime_error(what), status_(status) {}
    int status() const noexcept { return status_; }

private:
    int status_;
};

inline void check(int status, const char *where)
{
    if (status == FFTB_SUCCESS) return;
    std::string msg = std::string(where) + ": " + fftb_status_string(status);
    const char *detail = fftb_last_error_message();
    if (detail && *detail) msg += std::string(" (") + detail + ")";
    if (status == FFTB_ERROR_NOT_INITIALIZED || status == FFTB_ERROR_WRONG_DIMENSION ||
        status == FFTB_ERROR_ALREADY_INITIALIZED)
        throw std::logic_error(msg);
    throw error(status, msg);
}

namespace detail {
template <typename T> struct dtype_code;
template <> struct dtype_code<float> { static constexpr int value = FFTB_F32; };
template <> struct dtype_code<double> { static constexpr int value = FFTB_F64; };

template <typename A, typename = void> struct has_raw_ptr : std::false_type {};
template <typename A>
struct has_raw_ptr<A, std::void_t<decltype(std::declval<const A &>().raw_ptr())>> : std::true_type {};

/* a device pointer, or the raw_ptr() of an array object */
template <typename A> void *raw(const A &a)
{
    if constexpr (std::is_pointer<A>::value)
        return const_cast<void *>(static_cast<const void *>(a));
    else if constexpr (std::is_same<A, std::nullptr_t>::value)
        return nullptr;
    else {
        static_assert(has_raw_ptr<A>::value, "pass a device pointer or an array with raw_ptr()");
        return const_cast<void *>(static_cast<const void *>(a.raw_ptr()));
    }
}

/* a C ABI call that fills a text buffer: one call into 64 KiB (a measuring call must
 * not run twice), again only if the text needs more */
template <typename F> std::string fetch_text(F &&call, const char *where)
{
    std::string s(65536, '\0');
    size_t need = 0;
    int st = call(&s[0], s.size(), &need);
    if (st != FFTB_SUCCESS && need > s.size()) {
        s.assign(need, '\0');
        st = call(&s[0], s.size(), &need);
    }
    check(st, where);
    s.resize(s.find('\0') == std::string::npos ? s.size() : s.find('\0'));
    return s;
}
}  // namespace detail

/* ====================================================================== plans */

/* fft_plan_descriptor (source/external_wrap/fft_plan_descriptor.h:15-50) */
struct plan_descriptor {
    direction dir = direction::R2C;
    int rank = 0;
    std::array<long long, 3> n{}, inembed{}, onembed{};
    long long istride = 0, idist = 0, ostride = 0, odist = 0, batch = 0;
};

/* The per-plan object behind a name of fft_wrap_many: fft_base<T>
 * (source/external_wrap/cufft_wrap.h:456-480). */
template <typename T> class fft_base {
public:
    using real = T;
    fft_base(const fft_base &) = delete;
    fft_base &operator=(const fft_base &) = delete;
    virtual ~fft_base()
    {
        if (plan_) fftb_plan_destroy(plan_);
    }

    void exec(void *in, void *out) { check(fftb_exec(plan_, in, out), "fft::exec"); }
    void exec_no_sync(void *in, void *out) { check(fftb_exec(plan_, in, out), "fft::exec_no_sync"); }
    /* a C2C plan runs either sign; R2C / C2R only their own (else std::logic_error, as
     * cufft_wrap.h:664-700) */
    void exec_direction(direction d, void *in, void *out)
    {
        if (d != dir_ && !(is_c2c(dir_) && is_c2c(d)))
            throw std::logic_error("fft::exec_direction: incompatible execution direction");
        check(fftb_exec_direction(plan_, static_cast<int>(d), in, out), "fft::exec_direction");
    }
    void exec_direction_no_sync(direction d, void *in, void *out) { exec_direction(d, in, out); }
    direction get_direction() const { return dir_; }
    plan_descriptor descriptor() const
    {
        plan_descriptor p;
        int d = 0, dt = 0;
        check(fftb_plan_describe(plan_, &d, &dt, &p.rank, p.n.data(), p.inembed.data(), &p.istride, &p.idist,
                                 p.onembed.data(), &p.ostride, &p.odist, &p.batch),
              "fft::descriptor");
        p.dir = static_cast<direction>(d);
        return p;
    }
    std::size_t get_work_size() const { return work_; }
    void set_work_area(void *w) { check(fftb_plan_set_work_area(plan_, w), "fft::set_work_area"); }
    void set_stream(cudaStream_t s) { check(fftb_plan_set_stream(plan_, (void *)s), "fft::set_stream"); }
    /* the plans hold no stream- or work-bound state, so nothing is rebuilt */
    void recreate_with_stream_and_work_area(cudaStream_t s, void *w)
    {
        set_stream(s);
        set_work_area(w);
    }
    int num_launches() const
    {
        int l = 0;
        check(fftb_plan_num_launches(plan_, &l), "fft::num_launches");
        return l;
    }
    fftb_plan handle() const { return plan_; }

protected:
    fft_base(direction d, int rank, const long long *n, const long long *inembed, long long istride, long long idist,
             const long long *onembed, long long ostride, long long odist, long long batch)
        : dir_(d)
    {
        check(fftb_plan_create(static_cast<int>(d), detail::dtype_code<T>::value, rank, n, inembed, istride, idist,
                               onembed, ostride, odist, batch, &plan_, &work_),
              "fft::create_plan");
    }

private:
    static bool is_c2c(direction d) { return d == direction::C2CF || d == direction::C2CB; }
    direction dir_;
    fftb_plan plan_ = nullptr;
    std::size_t work_ = 0;
};

/* cufft::fft<T, D>: one plan with cuFFT advanced-layout parameters. */
template <typename T, direction D> class fft : public fft_base<T> {
public:
    template <std::size_t Rank>
    fft(const std::array<long long, Rank> &n, const std::array<long long, Rank> &inembed, long long istride,
        long long idist, const std::array<long long, Rank> &onembed, long long ostride, long long odist,
        long long batch)
        : fft_base<T>(D, int(Rank), n.data(), inembed.data(), istride, idist, onembed.data(), ostride, odist, batch)
    {
    }
    /* the tight default layout (cufft_wrap.h:568-587) */
    template <std::size_t Rank>
    fft(const std::array<long long, Rank> &n, long long batch)
        : fft_base<T>(D, int(Rank), n.data(), nullptr, 1, 0, nullptr, 1, 0, batch)
    {
    }
};

/* ====================================================================== fft_wrap_many */

/* The named plan registry (the BaseFFT contract of ffts). */
template <typename T> class fft_wrap_many {
public:
    using real = T;
    using wrap_t = fft_base<T>;

    fft_wrap_many() = default;
    fft_wrap_many(const fft_wrap_many &) = delete;
    fft_wrap_many &operator=(const fft_wrap_many &) = delete;
    ~fft_wrap_many() { release_noexcept(); }

    template <direction D, std::size_t Rank>
    void add_plan(const std::string &name, const std::array<long long, Rank> &n,
                  const std::array<long long, Rank> &inembed, long long istride, long long idist,
                  const std::array<long long, Rank> &onembed, long long ostride, long long odist, long long batch)
    {
        if (activated_) throw std::logic_error("fft_wrap_many::add_plan: cannot add new plans after activation.");
        container_.emplace(name, std::unique_ptr<wrap_t>(
                                     new fft<T, D>(n, inembed, istride, idist, onembed, ostride, odist, batch)));
    }
    template <direction D>
    void add_plan_1D(const std::string &name, long long n, long long inembed, long long istride, long long idist,
                     long long onembed, long long ostride, long long odist, long long batch)
    {
        add_plan<D, 1>(name, {n}, {inembed}, istride, idist, {onembed}, ostride, odist, batch);
    }
    template <direction D> void add_plan_1D_default(const std::string &name, long long n, long long batch)
    {
        if (activated_)
            throw std::logic_error("fft_wrap_many::add_plan_1D_default: cannot add new plans after activation.");
        container_.emplace(name, std::unique_ptr<wrap_t>(new fft<T, D>(std::array<long long, 1>{n}, batch)));
    }
    template <direction D>
    void add_plan_2D(const std::string &name, long long n0, long long n1, long long inembed0, long long inembed1,
                     long long istride, long long idist, long long onembed0, long long onembed1, long long ostride,
                     long long odist, long long batch)
    {
        add_plan<D, 2>(name, {n0, n1}, {inembed0, inembed1}, istride, idist, {onembed0, onembed1}, ostride, odist,
                       batch);
    }
    template <direction D>
    void add_plan_3D(const std::string &name, long long n0, long long n1, long long n2, long long inembed0,
                     long long inembed1, long long inembed2, long long istride, long long idist, long long onembed0,
                     long long onembed1, long long onembed2, long long ostride, long long odist, long long batch)
    {
        add_plan<D, 3>(name, {n0, n1, n2}, {inembed0, inembed1, inembed2}, istride, idist,
                       {onembed0, onembed1, onembed2}, ostride, odist, batch);
    }

    std::size_t activate_work_size()
    {
        for (const auto &el : container_) work_area_size_ = std::max(work_area_size_, el.second->get_work_size());
        return work_area_size_;
    }
    /* allocates the shared work area (if any plan needs one) and binds it to every plan */
    void activate()
    {
        if (activated_) throw std::logic_error("fft_wrap_many::activate: cannot activate again.");
        activate_work_size();
        if (work_area_size_ > 0) {
            if (cudaMalloc(&work_area_, work_area_size_) != cudaSuccess) {
                work_area_ = nullptr;
                throw error(FFTB_ERROR_ALLOC, "fft_wrap_many::activate: cudaMalloc of the work area failed");
            }
            for (auto &el : container_) el.second->set_work_area(work_area_);
        }
        activated_ = true;
        update_memory_profile_();
    }
    void set_external_work_area(void *w)
    {
        if (activated_)
            throw std::logic_error("fft_wrap_many::set_external_work_area: cannot set external work_area with "
                                   "activated local work_area.");
        for (auto &el : container_) el.second->set_work_area(w);
        external_activated_ = true;
        update_memory_profile_();
    }
    std::size_t get_work_size() const { return work_area_size_; }
    /* reports "<prefix>/work_area" (the bytes this object allocated; 0 with an external work
     * area) to `profiler`, now and whenever it changes (source/external_wrap/fft_wrap_many.h:298-303) */
    void set_memory_profiler(memory_profiler *profiler, const std::string &prefix)
    {
        memory_profiler_ = profiler;
        memory_profile_prefix_ = prefix;
        update_memory_profile_();
    }
    void set_stream(cudaStream_t s)
    {
        for (auto &el : container_) el.second->set_stream(s);
    }

    template <class ArrayIn, class ArrayOut> void exec(const std::string &name, const ArrayIn &in, ArrayOut &out)
    {
        container_.at(name)->exec(detail::raw(in), detail::raw(out));
    }
    template <class ArrayIn, class ArrayOut>
    void exec_named_no_sync(const std::string &name, const ArrayIn &in, ArrayOut &out)
    {
        container_.at(name)->exec_no_sync(detail::raw(in), detail::raw(out));
    }
    void exec_raw(const std::string &name, void *in, void *out) { container_.at(name)->exec(in, out); }
    void exec_raw_direction(const std::string &name, direction d, void *in, void *out)
    {
        container_.at(name)->exec_direction(d, in, out);
    }
    wrap_t &plan(const std::string &name) { return *container_.at(name); }
    bool has_plan(const std::string &name) const { return container_.count(name) != 0; }

    void release() { release_noexcept(); }

private:
    void release_noexcept() noexcept
    {
        container_.clear();  // plans go before the work area they point to
        if (work_area_) cudaFree(work_area_);
        work_area_ = nullptr;
        work_area_size_ = 0;
        activated_ = false;
        try {
            update_memory_profile_();
        } catch (...) {
        }
    }
    void update_memory_profile_()
    {
        if (!memory_profiler_ || memory_profile_prefix_.empty()) return;
        memory_profiler_->set_bytes(memory_profile_prefix_ + "/work_area",
                                    external_activated_ ? 0 : (memory_profiler::bytes_type)work_area_size_);
    }
    std::map<std::string, std::unique_ptr<wrap_t>> container_;
    std::size_t work_area_size_ = 0;
    void *work_area_ = nullptr;
    bool activated_ = false;
    bool external_activated_ = false;
    memory_profiler *memory_profiler_ = nullptr;
    std::string memory_profile_prefix_;
};

/* ====================================================================== autotune */

enum class cache_mismatch_policy { error, overwrite };

/* fftm_autotune's autotune_options (source/fftm_autotune.hpp:46-56) */
struct autotune_options {
    std::string cache_file;
    bool create_if_missing = true;
    cache_mismatch_policy mismatch_policy = cache_mismatch_policy::error;
    bool validate_hardware = true;
    bool strict_device_identity = false;
    bool force_measure = false;

    int flags() const
    {
        int f = 0;
        if (create_if_missing) f |= FFTB_TUNE_CREATE_IF_MISSING;
        if (mismatch_policy == cache_mismatch_policy::overwrite) f |= FFTB_TUNE_OVERWRITE_ON_MISMATCH;
        if (!validate_hardware) f |= FFTB_TUNE_NO_HARDWARE_CHECK;
        if (strict_device_identity) f |= FFTB_TUNE_STRICT_DEVICE;
        if (force_measure) f |= FFTB_TUNE_FORCE_MEASURE;
        return f;
    }
};

/* measured_options (source/fftm_autotune_measure.hpp:21-40) */
struct measured_options {
    int warmup = 2;
    int iterations = 5;
};

using config_map = std::map<std::string, std::string>;

/* KEY=VALUE lines, '#' comments (source/fftm_autotune.hpp:126-169) */
inline config_map parse_key_value_text(const std::string &text)
{
    config_map m;
    std::istringstream in(text);
    std::string line;
    while (std::getline(in, line)) {
        const auto a = line.find_first_not_of(" \t\r");
        if (a == std::string::npos || line[a] == '#') continue;
        const auto eq = line.find('=');
        if (eq == std::string::npos) throw error(FFTB_ERROR_CACHE_IO, "autotune: line is not KEY=VALUE: " + line);
        auto trim = [](std::string s) {
            const auto b = s.find_first_not_of(" \t\r"), e = s.find_last_not_of(" \t\r");
            return b == std::string::npos ? std::string() : s.substr(b, e - b + 1);
        };
        m[trim(line.substr(0, eq))] = trim(line.substr(eq + 1));
    }
    return m;
}

inline std::string to_key_value_text(const config_map &m)
{
    std::string s;
    for (const auto &kv : m) s += kv.first + "=" + kv.second + "\n";
    return s;
}

inline config_map load_key_value_file(const std::string &path)
{
    return parse_key_value_text(detail::fetch_text(
        [&](char *t, size_t c, size_t *n) { return fftb_autotune_load_file(path.c_str(), t, c, n); },
        "load_key_value_file"));
}

/* written to <path>.tmp and renamed into place */
inline void save_key_value_file(const std::string &path, const config_map &m)
{
    check(fftb_autotune_save_file(path.c_str(), to_key_value_text(m).c_str()), "save_key_value_file");
}

/* selected_3d_config (source/fftm_autotune.hpp:58-70) */
struct selected_config {
    config_map config;
    std::string source;  // "cache" or "measured"

    std::string strategy() const { return value("FFTB_AUTOTUNE_STRATEGY"); }
    int plane_cluster() const
    {
        const std::string v = value("FFTB_AUTOTUNE_PLANE_CLUSTER");
        return v.empty() ? 0 : std::stoi(v);
    }
    std::string text() const { return to_key_value_text(config); }
    std::string value(const std::string &k) const
    {
        const auto it = config.find(k);
        return it == config.end() ? std::string() : it->second;
    }
};

/* load_or_measure_3d_config (source/fftm_autotune_measure.hpp:432-520) for a 2D, 3D or
 * 4D ffts problem on the current device: the cache when it matches, else a measurement
 * (per the options), the winner written back to the cache file. */
template <typename T>
selected_config load_or_measure_config(const std::vector<long long> &dims, const autotune_options &options,
                                       const measured_options &measured = measured_options(),
                                       strategy_4d layout = strategy_4d::pencil_pencil)
{
    if (dims.size() < 2 || dims.size() > 4) throw std::invalid_argument("load_or_measure_config: 2 to 4 sizes");
    const long long nz = dims.size() > 2 ? dims[2] : 0, nw = dims.size() > 3 ? dims[3] : 0;
    int from_cache = 0;
    const std::string text = detail::fetch_text(
        [&](char *t, size_t c, size_t *n) {
            return fftb_autotune_ffts(detail::dtype_code<T>::value, dims[0], dims[1], nz, nw, static_cast<int>(layout),
                                      options.cache_file.c_str(), options.flags(), measured.warmup,
                                      measured.iterations, t, c, n, &from_cache);
        },
        "load_or_measure_config");
    return selected_config{parse_key_value_text(text), from_cache ? "cache" : "measured"};
}

/* ====================================================================== ffts */

/* fftm::ffts: 2D / 3D / 4D R2C forward and C2R backward in the reference's layouts, with
 * the fused spectral operators.  S selects the 4D layout (pencil real [w][z][y][x] with
 * spectrum [ky][kz][kw][kx]; slab real [x][y][z][w] with spectrum [kx][ky][kz][kw];
 * native_xzwy real [x][y][z][w] with spectrum [ky][kz][kw][kx]). */
template <typename T, strategy_4d S = strategy_4d::pencil_pencil> class ffts {
public:
    using real = T;
    ffts() = default;
    ffts(const ffts &) = delete;
    ffts &operator=(const ffts &) = delete;
    ~ffts()
    {
        if (h_) fftb_ffts_destroy(h_);
    }

    /* init with the reference's overloads (source/ffts.hpp:227-285): the default options turn
     * both profilers on and print their reports when the object is destroyed */
    void init(long long nx, long long ny, const ffts_init_options &o = ffts_init_options()) { init_(nx, ny, 0, 0, o); }
    void init(long long nx, long long ny, long long nz, const ffts_init_options &o = ffts_init_options())
    {
        init_(nx, ny, nz, 0, o);
    }
    void init(long long nx, long long ny, long long nz, long long nw, const ffts_init_options &o = ffts_init_options())
    {
        init_(nx, ny, nz, nw, o);
    }
    template <std::size_t Dim>
    void init(const std::array<std::size_t, Dim> &grid, const ffts_init_options &o = ffts_init_options())
    {
        static_assert(Dim >= 2 && Dim <= 4, "ffts: 2D, 3D or 4D");
        init_((long long)grid[0], (long long)grid[1], Dim > 2 ? (long long)grid[Dim > 2 ? 2 : 0] : 0,
              Dim > 3 ? (long long)grid[Dim > 3 ? 3 : 0] : 0, o);
    }
    /* one report of the profilers as text: 0 profile summary, 1 totals, 2 memory, 3 memory totals */
    std::string profile_report(int which = 0) const
    {
        ensure_initialized_();
        size_t need = 0;
        check(fftb_ffts_profile_report(h_, which, nullptr, 0, &need), "ffts::profile_report");
        std::string t(need, '\0');
        check(fftb_ffts_profile_report(h_, which, &t[0], t.size(), &need), "ffts::profile_report");
        t.resize(need ? need - 1 : 0);
        return t;
    }

    bool is_initialized() const { return h_ != nullptr; }
    std::size_t dimension() const
    {
        ensure_initialized_();
        return dim_;
    }
    const std::array<long long, 4> &sizes() const { return n_; }
    /* real points and complex (half-spectrum) elements of one field */
    long long real_size() const
    {
        ensure_initialized_();
        long long p = 1;
        for (std::size_t a = 0; a < dim_; ++a) p *= n_[a];
        return p;
    }
    long long spectrum_size() const
    {
        const long long last = n_[half_axis_()];
        return real_size() / last * (last / 2 + 1);
    }

    std::size_t work_size() const
    {
        ensure_initialized_();
        size_t w = 0;
        check(fftb_ffts_work_size(h_, &w), "ffts::work_size");
        return w;
    }
    void set_work_area(void *w)
    {
        ensure_initialized_();
        check(fftb_ffts_set_work_area(h_, w), "ffts::set_work_area");
    }
    void set_stream(cudaStream_t s)
    {
        ensure_initialized_();
        check(fftb_ffts_set_stream(h_, (void *)s), "ffts::set_stream");
    }

    /* a dimension check for callers that know their arrays' rank (source/ffts.hpp:647-657) */
    void ensure_dimension(std::size_t expected) const
    {
        ensure_initialized_();
        if (dim_ != expected)
            throw std::logic_error("ffts: initialized for " + std::to_string(dim_) + "D but used as " +
                                   std::to_string(expected) + "D.");
    }

    template <class In, class Out> void forward(const In &in, Out &out)
    {
        ensure_initialized_();
        check(fftb_ffts_forward(h_, detail::raw(in), detail::raw(out)), "ffts::forward");
    }
    /* unnormalised; `in` is overwritten, as the reference's 3D/4D backward */
    template <class In, class Out> void backward(In &in, Out &out)
    {
        ensure_initialized_();
        check(fftb_ffts_backward(h_, detail::raw(in), detail::raw(out)), "ffts::backward");
    }
    template <class In, class Out> void backward_normalized(In &in, Out &out)
    {
        ensure_initialized_();
        check(fftb_ffts_backward_normalized(h_, detail::raw(in), detail::raw(out)), "ffts::backward_normalized");
    }
    /* u = C2R(sign R2C(f) / |k|^2) / N; sign -1 solves lap u = f, +1 solves -lap u = f */
    template <class In, class Out> void poisson(const In &rhs, Out &u, double sign = -1.0)
    {
        ensure_initialized_();
        check(fftb_ffts_poisson(h_, detail::raw(rhs), detail::raw(u), sign), "ffts::poisson");
    }
    template <class In, class Out> void filter(const In &in, Out &out, double sigma, double poisson_sign = 0.0)
    {
        ensure_initialized_();
        check(fftb_ffts_filter(h_, detail::raw(in), detail::raw(out), sigma, poisson_sign), "ffts::filter");
    }
    template <class Spec> void spectrum_poisson(Spec &spec, double sign = -1.0, double scale = 1.0)
    {
        ensure_initialized_();
        check(fftb_ffts_spectrum_poisson(h_, detail::raw(spec), sign, scale), "ffts::spectrum_poisson");
    }
    template <class In, class Out> void spectrum_derivative(const In &in, Out &out, int axis, double scale = 1.0)
    {
        ensure_initialized_();
        check(fftb_ffts_spectrum_derivative(h_, detail::raw(in), detail::raw(out), axis, scale),
              "ffts::spectrum_derivative");
    }
    template <class Spec> void spectrum_truncate(Spec &spec, int rule = FFTB_TRUNCATE_TWO_THIRDS, int cutoff = 0)
    {
        ensure_initialized_();
        check(fftb_ffts_spectrum_truncate(h_, detail::raw(spec), rule, cutoff), "ffts::spectrum_truncate");
    }
    template <class In, class Out> void derivative(const In &u, Out &du, int axis)
    {
        ensure_initialized_();
        check(fftb_ffts_derivative(h_, detail::raw(u), detail::raw(du), axis), "ffts::derivative");
    }
    /* every first derivative; outs holds dimension() device pointers */
    template <class In> void gradient(const In &u, const std::vector<void *> &outs)
    {
        ensure_dimension(outs.size());
        check(fftb_ffts_gradient(h_, detail::raw(u), outs.data()), "ffts::gradient");
    }
    /* the adjoints of forward and backward (hand-written kernels) */
    template <class G, class R> void forward_adjoint(G &grad_spectrum, R &grad_real)
    {
        ensure_initialized_();
        check(fftb_ffts_forward_adjoint(h_, detail::raw(grad_spectrum), detail::raw(grad_real)),
              "ffts::forward_adjoint");
    }
    template <class R, class G> void backward_adjoint(const R &grad_real, G &grad_spectrum)
    {
        ensure_initialized_();
        check(fftb_ffts_backward_adjoint(h_, detail::raw(grad_real), detail::raw(grad_spectrum)),
              "ffts::backward_adjoint");
    }

    int num_launches(int which = 0) const
    {
        ensure_initialized_();
        int l = 0;
        check(fftb_ffts_num_launches(h_, which, &l), "ffts::num_launches");
        return l;
    }
    void set_strategy(int strategy, int plane_cluster = 0)
    {
        ensure_initialized_();
        check(fftb_ffts_set_strategy(h_, strategy, plane_cluster), "ffts::set_strategy");
    }
    std::pair<int, int> strategy() const
    {
        ensure_initialized_();
        int s = 0, c = 0;
        check(fftb_ffts_get_strategy(h_, &s, &c), "ffts::strategy");
        return {s, c};
    }
    void apply_config(const selected_config &c)
    {
        ensure_initialized_();
        check(fftb_ffts_apply_config(h_, c.text().c_str()), "ffts::apply_config");
    }
    /* load_or_measure for this object's problem, then the winner applied */
    selected_config autotune(const autotune_options &options, const measured_options &measured = measured_options())
    {
        ensure_initialized_();
        std::vector<long long> dims(n_.begin(), n_.begin() + dim_);
        selected_config c = load_or_measure_config<T>(dims, options, measured, S);
        apply_config(c);
        return c;
    }
    fftb_ffts handle() const { return h_; }

private:
    void init_(long long nx, long long ny, long long nz, long long nw, const ffts_init_options &o)
    {
        if (h_) throw std::logic_error("ffts::init can only be called once per instance.");
        fftb_init_options c;
        c.profiling_key = o.profiling_key.c_str();
        c.memory_profiling_key = o.memory_profiling_key.c_str();
        c.print_profile_summary_on_destroy = o.print_profile_summary_on_destroy ? 1 : 0;
        c.print_profile_totals_on_destroy = o.print_profile_totals_on_destroy ? 1 : 0;
        c.print_memory_profile_on_destroy = o.print_memory_profile_on_destroy ? 1 : 0;
        c.print_memory_totals_on_destroy = o.print_memory_totals_on_destroy ? 1 : 0;
        check(fftb_ffts_create_ex(detail::dtype_code<T>::value, nx, ny, nz, nw, static_cast<int>(S), &c, &h_),
              "ffts::init");
        n_ = {nx, ny, nz, nw};
        dim_ = nw ? 4 : (nz ? 3 : 2);
    }
    void ensure_initialized_() const
    {
        if (!h_) throw std::logic_error("ffts: call init() before using the transform.");
    }
    /* the R2C (half) axis is the last size given to init -- y, z or w -- in every layout */
    std::size_t half_axis_() const { return dim_ - 1; }

    fftb_ffts h_ = nullptr;
    std::array<long long, 4> n_{};
    std::size_t dim_ = 0;
};

/* The rank-local part of the slab-distributed 3D / 4D transforms (fftb_slab_*): the pack
 * pass writes send blocks (or the peers' receive buffers, set_peers), the caller exchanges
 * block q to rank q (an NCCL all-to-all), the finish passes read the received blocks. */
template <typename T> class slab {
public:
    slab(long long nx, long long ny, long long nz, long long nw, int nranks, int rank,
         strategy_4d layout = strategy_4d::native_xzwy)
    {
        check(fftb_slab_create(detail::dtype_code<T>::value, nx, ny, nz, nw, static_cast<int>(layout), nranks, rank,
                               &h_),
              "slab::slab");
        check(fftb_slab_sizes(h_, &real_, &spec_, &exch_, &work_), "slab::sizes");
    }
    slab(const slab &) = delete;
    slab &operator=(const slab &) = delete;
    ~slab()
    {
        if (h_) fftb_slab_destroy(h_);
    }
    long long real_elems() const { return real_; }
    long long spectrum_elems() const { return spec_; }
    long long exchange_elems() const { return exch_; }   // complex values of send / receive
    long long work_elems() const { return work_; }       // complex values of the work buffer
    void set_stream(cudaStream_t s) { check(fftb_slab_set_stream(h_, (void *)s), "slab::set_stream"); }
    void set_peers(const std::vector<void *> &receive_blocks)
    {
        check(fftb_slab_set_peers(h_, receive_blocks.empty() ? nullptr : receive_blocks.data()), "slab::set_peers");
    }
    void forward_local(const void *in, void *send, void *work)
    {
        check(fftb_slab_forward_local(h_, in, send, work), "slab::forward_local");
    }
    void forward_finish(void *recv, void *out = nullptr)
    {
        check(fftb_slab_forward_finish(h_, recv, out), "slab::forward_finish");
    }
    void backward_local(void *spectrum, void *send = nullptr)
    {
        check(fftb_slab_backward_local(h_, spectrum, send), "slab::backward_local");
    }
    void backward_finish(void *recv, void *out, void *work)
    {
        check(fftb_slab_backward_finish(h_, recv, out, work), "slab::backward_finish");
    }

private:
    fftb_slab h_ = nullptr;
    long long real_ = 0, spec_ = 0, exch_ = 0, work_ = 0;
};

/* The allocation-free 3D float32 Poisson solve (fftb_poisson3d_f32_noalloc): static
 * device scratch, spectra up to FFTB_NOALLOC_MAX_SPECTRUM_BYTES, overlapping calls
 * serialised by the caller. */
template <class In, class Out>
void poisson3d_noalloc(const In &rhs, Out &u, long long nx, long long ny, long long nz, double sign = -1.0,
                       cudaStream_t stream = nullptr)
{
    check(fftb_poisson3d_f32_noalloc(static_cast<const float *>(detail::raw(rhs)), static_cast<float *>(detail::raw(u)),
                                     nx, ny, nz, sign, (void *)stream),
          "poisson3d_noalloc");
}

/* ====================================================================== batches */

/* Many 3D R2C / C2R transforms of uneven sizes over packed buffers, in one persistent
 * (or grouped) launch replayed from a CUDA graph. */
template <typename T> class batch {
public:
    enum op_t { forward = FFTB_BATCH_FORWARD, backward = FFTB_BATCH_BACKWARD, roundtrip = FFTB_BATCH_ROUNDTRIP,
                poisson = FFTB_BATCH_POISSON };

    explicit batch(const std::vector<std::array<long long, 3>> &shapes) : count_((int)shapes.size())
    {
        std::vector<long long> d;
        for (const auto &s : shapes) d.insert(d.end(), s.begin(), s.end());
        check(fftb_batch_create(detail::dtype_code<T>::value, count_, d.data(), &h_), "batch::create");
        real_off_.resize(count_);
        spec_off_.resize(count_);
        check(fftb_batch_layout(h_, real_off_.data(), spec_off_.data(), &real_total_, &spec_total_),
              "batch::layout");
    }
    batch(const batch &) = delete;
    batch &operator=(const batch &) = delete;
    ~batch()
    {
        if (h_) fftb_batch_destroy(h_);
    }

    long long real_total() const { return real_total_; }
    long long spectrum_total() const { return spec_total_; }
    long long real_offset(int i) const { return real_off_.at(i); }
    long long spectrum_offset(int i) const { return spec_off_.at(i); }
    std::size_t work_size() const
    {
        size_t b = 0;
        check(fftb_batch_work_size(h_, &b), "batch::work_size");
        return b;
    }
    void set_work_area(void *w) { check(fftb_batch_set_work_area(h_, w), "batch::set_work_area"); }
    void set_stream(cudaStream_t s) { check(fftb_batch_set_stream(h_, (void *)s), "batch::set_stream"); }
    /* mode: 0-4 as fftb_batch_exec; -1 = the tuned mode, else 4 (grouped launches
     * replayed from a CUDA graph) for float and 0 for double */
    void exec(op_t op, const void *in, void *out, double sign = -1.0, int mode = -1)
    {
        check(fftb_batch_exec(h_, op, in, out, sign, mode < 0 ? mode_ : mode), "batch::exec");
    }
    int error_flag(op_t op) const
    {
        int f = 0;
        check(fftb_batch_status(h_, op, &f), "batch::status");
        return f;
    }
    selected_config autotune(op_t op, const autotune_options &options,
                             const measured_options &measured = measured_options(), double sign = -1.0)
    {
        int from_cache = 0, mode = 0;
        const std::string text = detail::fetch_text(
            [&](char *t, size_t c, size_t *n) {
                return fftb_autotune_batch(h_, op, sign, options.cache_file.c_str(), options.flags(),
                                           measured.warmup, measured.iterations, t, c, n, &from_cache, &mode);
            },
            "batch::autotune");
        mode_ = mode;
        return selected_config{parse_key_value_text(text), from_cache ? "cache" : "measured"};
    }
    fftb_batch handle() const { return h_; }

private:
    int count_;
    fftb_batch h_ = nullptr;
    std::vector<long long> real_off_, spec_off_;
    long long real_total_ = 0, spec_total_ = 0;
    int mode_ = std::is_same<T, float>::value ? 4 : 0;
};

}  // namespace fftb

#endif  // FFTB_HPP
