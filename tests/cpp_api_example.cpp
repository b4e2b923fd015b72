// A C++ caller of the header-only host layer include/fftb.hpp, written the way the
// reference's own C++ tests and examples use fftm (source/tests/test_fft_3D.cu:30-57 for
// the plan registry, examples/poisson for ffts + Poisson, fftm_autotune for the cache):
//   1. fft_wrap_many<double>: named 3D R2C / C2R plans over arrays with raw_ptr(),
//      a single-mode known answer and a round trip;
//   2. the reference's error behaviour: logic_error / out_of_range / runtime_error;
//   3. ffts<float> 3D: Poisson (and the allocation-free solve) and a derivative against
//      closed-form solutions;
//   4. ffts<double, native_xzwy> 4D round trip;
//   5. load_or_measure_config: measured once, then read back from the cache;
//   6. batch<float>: uneven 3D round trips in one graph-replayed launch;
//   7. the profiling options (ffts_init_options, fftm_reporting_options) and reports.
// Prints one line per check and "ok" last; exit status 0 when every check passes.
// argv[1]: a writable directory for the autotune cache, or "--host-only" to run just the
// checks that need no GPU (status -> exception mapping, KEY=VALUE text, option flags).
#include <cmath>
#include <complex>
#include <cstdio>
#include <string>
#include <vector>

#include "fftb.hpp"

namespace {

int failures = 0;

void expect(bool ok, const std::string &what)
{
    std::printf("%s %s\n", ok ? "pass" : "FAIL", what.c_str());
    if (!ok) ++failures;
}

// a device array with the raw_ptr() accessor of the reference's SCFD arrays
template <typename E> struct device_array {
    explicit device_array(std::size_t n) : n(n)
    {
        if (cudaMalloc(&p, n * sizeof(E)) != cudaSuccess) throw std::runtime_error("cudaMalloc");
    }
    ~device_array() { cudaFree(p); }
    device_array(const device_array &) = delete;
    E *raw_ptr() const { return p; }
    void put(const std::vector<E> &h) { cudaMemcpy(p, h.data(), n * sizeof(E), cudaMemcpyHostToDevice); }
    std::vector<E> get() const
    {
        std::vector<E> h(n);
        cudaMemcpy(h.data(), p, n * sizeof(E), cudaMemcpyDeviceToHost);
        return h;
    }
    E *p = nullptr;
    std::size_t n;
};

template <typename E> double rel_l2(const std::vector<E> &a, const std::vector<double> &b)
{
    double num = 0, den = 0;
    for (std::size_t i = 0; i < b.size(); ++i) {
        num += (double(a[i]) - b[i]) * (double(a[i]) - b[i]);
        den += b[i] * b[i];
    }
    return std::sqrt(num / den);
}

template <typename F> bool throws_logic(F &&f)
{
    try {
        f();
    } catch (const std::logic_error &) {
        return true;
    } catch (...) {
    }
    return false;
}

const double pi = 3.14159265358979323846;

void host_only()
{
    fftb::ffts<float> f;
    expect(throws_logic([&] { f.dimension(); }), "ffts used before init -> std::logic_error");
    expect(throws_logic([] { fftb::check(FFTB_ERROR_ALREADY_INITIALIZED, "x"); }), "status -8 -> std::logic_error");
    expect(throws_logic([] { fftb::check(FFTB_ERROR_WRONG_DIMENSION, "x"); }), "status -7 -> std::logic_error");
    int status = 0;
    try {
        fftb::check(FFTB_ERROR_UNSUPPORTED_SIZE, "x");
    } catch (const fftb::error &e) {
        status = e.status();
    }
    expect(status == FFTB_ERROR_UNSUPPORTED_SIZE, "status -2 -> fftb::error with its code");
    const fftb::config_map m = fftb::parse_key_value_text("# comment\nFFTM_AUTOTUNE_SCHEMA = 2\n\nA=b c\n");
    expect(m.size() == 2 && m.at("FFTM_AUTOTUNE_SCHEMA") == "2" && m.at("A") == "b c", "KEY=VALUE parse");
    expect(fftb::parse_key_value_text(fftb::to_key_value_text(m)) == m, "KEY=VALUE text round trip");
    bool bad_line = false;
    try {
        fftb::parse_key_value_text("no equals sign\n");
    } catch (const fftb::error &e) {
        bad_line = e.status() == FFTB_ERROR_CACHE_IO;
    }
    expect(bad_line, "a line without '=' -> FFTB_ERROR_CACHE_IO");
    fftb::autotune_options o;
    o.mismatch_policy = fftb::cache_mismatch_policy::overwrite;
    o.validate_hardware = false;
    expect(o.flags() == (FFTB_TUNE_CREATE_IF_MISSING | FFTB_TUNE_OVERWRITE_ON_MISMATCH | FFTB_TUNE_NO_HARDWARE_CHECK),
           "autotune_options flags");
    // the reference's option structs and presets (source/ffts.hpp:64-72, source/fftm_options.hpp:220-242)
    const fftb::ffts_init_options io;
    expect(io.profiling_key == "ffts_prof" && io.memory_profiling_key == "ffts_mem" &&
               io.print_profile_summary_on_destroy && io.print_memory_totals_on_destroy,
           "ffts_init_options defaults");
    const fftb::fftm_reporting_options quiet;
    const fftb::ffts_init_options qo = fftb::to_ffts_init_options(quiet);
    expect(qo.profiling_key.empty() && !qo.print_profile_summary_on_destroy, "fftm_reporting_options defaults off");
    const fftb::ffts_init_options po = fftb::to_ffts_init_options(fftb::profiling_reporting_options());
    expect(po.profiling_key == "fftm_prof" && po.memory_profiling_key == "fftm_mem" && po.print_memory_profile_on_destroy,
           "profiling_reporting_options preset");
    expect(fftb::strategy_for(fftb::fftm_4d_spectral_layout::native_xzwy) == fftb::strategy_4d::native_xzwy &&
               fftb::strategy_for(fftb::fftm_4d_spectral_layout::public_yzwx) == fftb::strategy_4d::pencil_pencil,
           "fftm spectral layout -> ffts strategy");
    // memory profiler attached to a plan registry (source/external_wrap/fft_wrap_many.h:298-303)
    fftb::memory_profiler mp;
    mp.set_bytes("a", 100);
    mp.set_bytes("a", 40);
    expect(mp.entries().at("a").current_bytes == 40 && mp.entries().at("a").peak_bytes == 100, "memory profiler peaks");
    fftb::fft_wrap_many<float> reg;
    reg.set_memory_profiler(&mp, "ffts/base_fft");
    reg.activate();
    expect(mp.entries().count("ffts/base_fft/work_area") == 1 &&
               mp.entries().at("ffts/base_fft/work_area").current_bytes == 0,
           "fft_wrap_many reports its work area to the memory profiler");
}

void plan_registry()
{
    using C = std::complex<double>;
    const long long nx = 12, ny = 10, nz = 8, nzc = nz / 2 + 1, n = nx * ny * nz;
    fftb::fft_wrap_many<double> fft;
    fft.add_plan_3D<fftb::direction::R2C>("3D_r2c", nx, ny, nz, nx, ny, nz, 1, n, nx, ny, nzc, 1, nx * ny * nzc, 1);
    fft.add_plan_3D<fftb::direction::C2R>("3D_c2r", nx, ny, nz, nx, ny, nzc, 1, nx * ny * nzc, nx, ny, nz, 1, n, 1);
    fft.activate();
    std::printf("work_size: %zu bytes\n", fft.get_work_size());
    device_array<double> x(n), y(n);
    device_array<C> s(nx * ny * nzc);
    // x = cos(2 pi (2 i / nx + 3 k / nz)): the spectrum is n / 2 at (kx, ky, kz) = (2, 0, 3), 0 elsewhere
    std::vector<double> h(n);
    for (long long i = 0; i < nx; ++i)
        for (long long j = 0; j < ny; ++j)
            for (long long k = 0; k < nz; ++k) h[(i * ny + j) * nz + k] = std::cos(2 * pi * (2.0 * i / nx + 3.0 * k / nz));
    x.put(h);
    fft.exec("3D_r2c", x, s);
    const std::vector<C> hs = s.get();
    double off = 0;
    for (long long i = 0; i < nx * ny * nzc; ++i)
        if (i != (2 * ny + 0) * nzc + 3) off = std::max(off, std::abs(hs[i]));
    const C peak = hs[(2 * ny + 0) * nzc + 3];
    expect(std::abs(peak - C(n / 2.0, 0)) < 1e-9 * n && off < 1e-9 * n, "fft_wrap_many R2C single-mode spectrum");
    fft.exec("3D_c2r", s, y);
    std::vector<double> back = y.get();
    for (auto &v : back) v /= double(n);
    expect(rel_l2(back, h) < 1e-13, "fft_wrap_many C2R round trip");
    expect(fft.plan("3D_r2c").descriptor().n[2] == nz, "plan descriptor");

    expect(throws_logic([&] { fft.add_plan_1D_default<fftb::direction::C2CF>("late", 16, 1); }),
           "add_plan after activate -> std::logic_error");
    bool oor = false;
    try {
        fft.exec_raw("no_such_plan", x.p, s.p);
    } catch (const std::out_of_range &) {
        oor = true;
    }
    expect(oor, "unknown plan name -> std::out_of_range");
    expect(throws_logic([&] { fft.exec_raw_direction("3D_r2c", fftb::direction::C2R, x.p, s.p); }),
           "incompatible exec direction -> std::logic_error");
    int status = 0;
    try {
        // every length up to 2^24 points has a kernel (radix, chirp-z or the long-line step)
        fftb::fft<float, fftb::direction::C2CF> big(std::array<long long, 1>{(1LL << 24) + 2}, 1);
    } catch (const fftb::error &e) {
        status = e.status();
    }
    expect(status == FFTB_ERROR_UNSUPPORTED_SIZE, "unsupported length -> fftb::error (runtime_error)");
}

void ffts_3d()
{
    const int N = 32;
    const long long n = (long long)N * N * N;
    fftb::ffts<float> f;
    expect(throws_logic([&] { f.dimension(); }), "ffts used before init -> std::logic_error");
    f.init(N, N, N);
    expect(throws_logic([&] { f.init(N, N, N); }), "ffts::init twice -> std::logic_error");
    expect(throws_logic([&] { f.ensure_dimension(4); }), "3D ffts used as 4D -> std::logic_error");
    expect(f.dimension() == 3 && f.spectrum_size() == (long long)N * N * (N / 2 + 1), "ffts sizes");
    {
        // profilers with their reports read back instead of printed
        fftb::ffts_init_options po;
        po.profiling_key = "p3";
        po.memory_profiling_key = "m3";
        po.print_profile_summary_on_destroy = po.print_profile_totals_on_destroy = false;
        po.print_memory_profile_on_destroy = po.print_memory_totals_on_destroy = false;
        fftb::ffts<float> g;
        g.init(std::array<std::size_t, 3>{(std::size_t)N, (std::size_t)N, (std::size_t)N}, po);
        device_array<float> a(n), b(n);
        cudaMemset(a.raw_ptr(), 0, n * sizeof(float));
        g.poisson(a, b, -1.0);
        g.poisson(a, b, -1.0);
        cudaDeviceSynchronize();
        const std::string rep = g.profile_report(0), mem = g.profile_report(2);
        expect(rep.find("Profile p3:") != std::string::npos && rep.find("ffts::poisson<3>: calls=2") != std::string::npos &&
                   rep.find("ffts::init<3>: calls=1") != std::string::npos,
               "ffts profile report (scopes and calls)");
        expect(mem.find("ffts/shared_work_buffer: current(sum/max/avg)=" + std::to_string(g.work_size())) !=
                   std::string::npos,
               "ffts memory profile (the work area it allocated)");
    }
    std::vector<float> rhs(n);
    std::vector<double> u_exact(n), uy_exact(n);
    for (int x = 0; x < N; ++x)
        for (int y = 0; y < N; ++y)
            for (int z = 0; z < N; ++z) {
                const double gx = 2 * pi * x / N, gy = 2 * pi * y / N, gz = 2 * pi * z / N;
                const std::size_t i = ((std::size_t)x * N + y) * N + z;
                u_exact[i] = std::sin(gx) * std::sin(2 * gy) * std::cos(3 * gz);
                uy_exact[i] = 2 * std::sin(gx) * std::cos(2 * gy) * std::cos(3 * gz);
                rhs[i] = float(-14.0 * u_exact[i]);
            }
    device_array<float> d_rhs(n), d_u(n);
    d_rhs.put(rhs);
    f.poisson(d_rhs, d_u, -1.0);  // lap u = f
    expect(rel_l2(d_u.get(), u_exact) < 1e-5, "ffts<float>::poisson vs the exact solution");
    device_array<float> u_in(n), du(n);
    std::vector<float> uf(u_exact.begin(), u_exact.end());
    u_in.put(uf);
    f.derivative(u_in, du, 1);
    expect(rel_l2(du.get(), uy_exact) < 1e-5, "ffts<float>::derivative (y) vs the exact derivative");
    device_array<float> u_na(n);
    fftb::poisson3d_noalloc(d_rhs, u_na, N, N, N, -1.0);
    expect(rel_l2(u_na.get(), u_exact) < 1e-5, "poisson3d_noalloc vs the exact solution");
}

void slab_one_rank()
{
    // one rank: the exchange is nothing (send and receive one buffer); the spectrum slab is
    // then the whole spectrum, equal to ffts' forward
    const long long nx = 16, ny = 12, nz = 10, n = nx * ny * nz, nc = nx * ny * (nz / 2 + 1);
    fftb::slab<float> s(nx, ny, nz, 0, 1, 0);
    expect(s.real_elems() == n && s.spectrum_elems() == nc && s.exchange_elems() == nc, "slab sizes");
    std::vector<float> h(n);
    for (long long i = 0; i < n; ++i) h[i] = std::sin(0.37 * (double)i) + 0.01 * (double)(i % 7);
    device_array<float> x(n);
    x.put(h);
    device_array<std::complex<float>> buf(nc), work(s.work_elems()), ref(nc);
    s.forward_local(x.raw_ptr(), buf.raw_ptr(), work.raw_ptr());
    s.forward_finish(buf.raw_ptr());
    fftb::ffts<float> f;
    fftb::ffts_init_options quiet;
    quiet.profiling_key.clear();
    quiet.memory_profiling_key.clear();
    f.init(nx, ny, nz, quiet);
    f.forward(x, ref);
    cudaDeviceSynchronize();
    const std::vector<std::complex<float>> a = buf.get(), b = ref.get();
    double num = 0, den = 0;
    for (long long i = 0; i < nc; ++i) {
        num += std::norm(std::complex<double>(a[i]) - std::complex<double>(b[i]));
        den += std::norm(std::complex<double>(b[i]));
    }
    expect(std::sqrt(num / den) < 2e-6, "slab<float> one rank equals ffts forward");
}

void ffts_4d_native()
{
    const long long nx = 8, ny = 6, nz = 10, nw = 12, n = nx * ny * nz * nw;
    fftb::ffts<double, fftb::strategy_4d::native_xzwy> f;
    f.init(nx, ny, nz, nw);
    std::vector<double> h(n);
    for (long long i = 0; i < n; ++i) h[i] = std::sin(0.37 * i) + 0.25 * std::cos(1.3 * i * i);
    device_array<double> x(n), y(n);
    device_array<std::complex<double>> s(f.spectrum_size());
    x.put(h);
    f.forward(x, s);
    f.backward_normalized(s, y);
    expect(rel_l2(y.get(), h) < 1e-13, "ffts<double, native_xzwy> 4D round trip");
}

void autotune(const std::string &dir)
{
    fftb::autotune_options o;
    o.cache_file = dir + "/fftb_cpp_autotune_64.env";
    o.create_if_missing = true;
    o.force_measure = true;
    fftb::measured_options m;
    m.warmup = 1;
    m.iterations = 3;
    const fftb::selected_config first = fftb::load_or_measure_config<float>({64, 64, 64}, o, m);
    expect(first.source == "measured" && !first.strategy().empty(), "load_or_measure_config measures");
    o.force_measure = false;
    fftb::ffts<float> f;
    f.init(64, 64, 64);
    const fftb::selected_config again = f.autotune(o, m);
    expect(again.source == "cache" && again.strategy() == first.strategy(), "autotune cache read back");
    const fftb::config_map file = fftb::load_key_value_file(o.cache_file);
    expect(file.count("FFTM_AUTOTUNE_SCHEMA") == 1, "cache file carries the schema key");
}

void batches()
{
    fftb::batch<float> b({{32, 48, 64}, {64, 64, 32}, {48, 32, 96}});
    const long long n = b.real_total();
    std::vector<float> h(n);
    for (long long i = 0; i < n; ++i) h[i] = float(std::sin(0.11 * i) * std::cos(0.007 * i));
    device_array<float> x(n), y(n);
    x.put(h);
    b.exec(fftb::batch<float>::roundtrip, x.p, y.p);
    std::vector<double> hd(h.begin(), h.end());
    expect(rel_l2(y.get(), hd) < 2e-6 && b.error_flag(fftb::batch<float>::roundtrip) == 0,
           "batch<float> uneven round trips");
}

}  // namespace

int main(int argc, char **argv)
{
    const std::string dir = argc > 1 ? argv[1] : ".";
    try {
        host_only();
        if (dir == "--host-only") {
            std::printf(failures ? "FAILED\n" : "ok\n");
            return failures ? 1 : 0;
        }
        plan_registry();
        ffts_3d();
        ffts_4d_native();
        slab_one_rank();
        autotune(dir);
        batches();
    } catch (const std::exception &e) {
        std::printf("FAIL unexpected exception: %s\n", e.what());
        ++failures;
    }
    std::printf(failures ? "FAILED\n" : "ok\n");
    return failures ? 1 : 0;
}
