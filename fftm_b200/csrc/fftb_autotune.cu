// fftb_autotune.cu -- measured autotuner with a KEY=VALUE cache file, the replacement of
// fftm's autotune surface for the single-GPU transforms of this library:
//   cache IO        source/fftm_autotune.hpp:126-169   (KEY=VALUE, '#' comments, written
//                                                       to <path>.tmp then renamed)
//   identity keys   source/fftm_autotune.hpp:660-676   (FFTM_AUTOTUNE_SCHEMA=2, _LIBRARY,
//                                                       _DIM, _NUM_GPUS, _SIZE_3D, ...)
//   policy version  source/fftm_autotune.hpp:452-477
//   load_or_measure source/fftm_autotune_measure.hpp:432-520 (use the cache when it
//                   matches; measure when it is missing and creation is asked for, or
//                   when it mismatches and the policy is overwrite; else an error)
//   measurement     source/fftm_autotune_measure.hpp:798-854 (warm-up forward+backward
//                   pairs, then timed pairs; the winner is the least median; every
//                   candidate must pass a round-trip check at sampled points with the
//                   tolerance 1000 eps max(1, log2 N))
//   hardware        source/detail/fftm_autotune_hardware.inc:285-425 ("v2:" + 64-bit
//                   FNV-1a of a canonical device description, compatible and strict)
// The pairs are timed with CUDA events on a private stream rather than wall clock.
// The knobs measured here are the ffts execution strategy (fused multi-axis kernels with
// 1, 2, 4 or 8 CTAs per plane, the same with tensor-core column kernels, or one pass
// kernel per axis) and, for batches, the execution mode, tile height and persistent CTAs
// per SM.
#include <cuda_runtime.h>

#include <cctype>

#include <sys/stat.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/fftb.h"
#include "fftb_engine.h"
#include "fftb_fused3d.h"

namespace fftb {
int batch_identity(const fftb_batch_s *b, int *dtype, int *count, const long long **dims, int *tiles_scale,
                   int *ctas_per_sm, void **stream);
}

using namespace fftb;

namespace {

using Config = std::map<std::string, std::string>;

const char *kPolicyVersion = "fftb-1";
const char *kMeasuredSource = "fftb-measured-v1";

std::string trim(const std::string &s)
{
    const char *ws = " \t\r\n";
    const size_t a = s.find_first_not_of(ws);
    if (a == std::string::npos) return "";
    const size_t b = s.find_last_not_of(ws);
    return s.substr(a, b - a + 1);
}

std::string get(const Config &c, const std::string &k)
{
    auto it = c.find(k);
    return it == c.end() ? std::string() : it->second;
}

int parse_text(const std::string &text, const std::string &origin, Config &out)
{
    out.clear();
    std::istringstream in(text);
    std::string line;
    size_t line_no = 0;
    while (std::getline(in, line)) {
        ++line_no;
        line = trim(line);
        if (line.empty() || line[0] == '#') continue;
        const size_t eq = line.find('=');
        if (eq == std::string::npos || trim(line.substr(0, eq)).empty()) {
            set_last_error("autotune config " + origin + ":" + std::to_string(line_no) + " is not KEY=VALUE");
            return FFTB_ERROR_CACHE_IO;
        }
        out[trim(line.substr(0, eq))] = trim(line.substr(eq + 1));
    }
    if (out.empty()) {
        set_last_error("autotune config is empty: " + origin);
        return FFTB_ERROR_CACHE_IO;
    }
    return FFTB_SUCCESS;
}

std::string to_text(const Config &c)
{
    std::string t = "# fftb autotune cache\n";
    for (const auto &kv : c) t += kv.first + "=" + kv.second + "\n";
    return t;
}

bool file_exists(const std::string &path)
{
    struct stat st;
    return stat(path.c_str(), &st) == 0;
}

int load_file(const std::string &path, Config &out)
{
    FILE *f = fopen(path.c_str(), "rb");
    if (!f) {
        set_last_error("autotune config cannot be opened: " + path);
        return FFTB_ERROR_CACHE_IO;
    }
    std::string text;
    char buf[4096];
    size_t n;
    while ((n = fread(buf, 1, sizeof(buf), f)) > 0) text.append(buf, n);
    const bool bad = ferror(f) != 0;
    fclose(f);
    if (bad) {
        set_last_error("autotune config cannot be read: " + path);
        return FFTB_ERROR_CACHE_IO;
    }
    return parse_text(text, path, out);
}

int save_file(const std::string &path, const Config &c)
{
    const std::string tmp = path + ".tmp";
    FILE *f = fopen(tmp.c_str(), "wb");
    if (!f) {
        set_last_error("autotune config cannot be written: " + tmp);
        return FFTB_ERROR_CACHE_IO;
    }
    const std::string text = to_text(c);
    const bool ok = fwrite(text.data(), 1, text.size(), f) == text.size();
    const bool closed = fclose(f) == 0;
    if (!ok || !closed || std::rename(tmp.c_str(), path.c_str()) != 0) {
        std::remove(tmp.c_str());
        set_last_error("autotune config cannot be moved into place: " + path);
        return FFTB_ERROR_CACHE_IO;
    }
    return FFTB_SUCCESS;
}

int put_text(const std::string &text, char *out, size_t capacity, size_t *needed)
{
    if (needed) *needed = text.size() + 1;
    if (!out) return capacity == 0 ? FFTB_SUCCESS : FFTB_ERROR_INVALID_VALUE;
    if (capacity < text.size() + 1) {
        set_last_error("text buffer holds " + std::to_string(capacity) + " bytes, " + std::to_string(text.size() + 1) +
                       " needed");
        return FFTB_ERROR_INVALID_VALUE;
    }
    memcpy(out, text.c_str(), text.size() + 1);
    return FFTB_SUCCESS;
}

// 64-bit FNV-1a (Fowler, Noll, Vo): offset basis 14695981039346656037, prime 1099511628211.
std::string fnv1a_hex(const std::string &s)
{
    uint64_t h = 14695981039346656037ULL;
    for (unsigned char c : s) {
        h ^= (uint64_t)c;
        h *= 1099511628211ULL;
    }
    char buf[17];
    snprintf(buf, sizeof(buf), "%016llx", (unsigned long long)h);
    return buf;
}

// --------------------------------------------------------------------------- hardware
// The hardware signature is the reference's, for one rank, so that a cache fftm wrote on
// this machine validates here and the other way round
// (source/detail/fftm_autotune_hardware.inc:28-97 token rules, :101-124 device class and
// transport environment, :285-310 canonical strings, :312-343 metadata keys): the
// compatibility string names the rank count, node layout, MPI library ("unavailable"
// without MPI), device class (backend, model, compute capability, memory, runtime and
// driver versions), transport ("local") and transport environment; the strict string adds
// device UUIDs, PCI bus ids and node names ("local").  Each is hashed with 64-bit FNV-1a.

// separators (NUL, white space, ';', '=', ',', '|') become one '_', none at the ends
std::string hw_token(const std::string &v)
{
    std::string r;
    bool prev = false;
    for (unsigned char ch : v) {
        const bool sep = ch == '\0' || std::isspace(ch) || ch == ';' || ch == '=' || ch == ',' || ch == '|';
        if (sep) {
            if (!r.empty() && !prev) r.push_back('_');
            prev = true;
            continue;
        }
        r.push_back((char)ch);
        prev = false;
    }
    while (!r.empty() && r.back() == '_') r.pop_back();
    return r.empty() ? "unknown" : r;
}

std::string hw_env(const char *name)
{
    const char *v = getenv(name);
    return hw_token(v ? v : "default");
}

int hardware_config(int device, Config &c)
{
    cudaDeviceProp p;
    cudaError_t e = cudaGetDeviceProperties(&p, device);
    if (e != cudaSuccess) return set_status_from_cuda(e);
    int rt = 0, drv = 0;
    cudaRuntimeGetVersion(&rt);
    cudaDriverGetVersion(&drv);
    char uuid[40];
    for (int i = 0; i < 16; ++i) snprintf(uuid + 2 * i, 3, "%02x", (unsigned char)p.uuid.bytes[i]);
    char pci[32] = {};
    if (cudaDeviceGetPCIBusId(pci, (int)sizeof(pci), device) != cudaSuccess) {
        cudaGetLastError();
        snprintf(pci, sizeof(pci), "unavailable");
    }
    const std::string arch = std::to_string(p.major) + "." + std::to_string(p.minor);
    const std::string cls = "backend=cuda:model=" + hw_token(p.name) + ":arch=" + hw_token(arch) +
                            ":memory=" + std::to_string((unsigned long long)p.totalGlobalMem) +
                            ":runtime=" + std::to_string(rt) + ":driver=" + std::to_string(drv);
    const std::string env = "affinity=" + hw_env("FFTM_MPI_RANK_AFFINITY_MODE") + ":ucx_tls=" + hw_env("UCX_TLS") +
                            ":ucx_net_devices=" + hw_env("UCX_NET_DEVICES") + ":mpi_pml=" + hw_env("OMPI_MCA_pml") +
                            ":mpi_btl=" + hw_env("OMPI_MCA_btl");
    const std::string compat = "version=2;mpi_ranks=1;node_count=1;ranks_per_node=1;devices_per_node=1"
                               ";mpi_library=unavailable;device_classes=" + hw_token(cls) +
                               ";transport=local;transport_env=" + hw_token(env);
    const std::string strict = compat + ";device_uuids=" + hw_token(uuid) + ";pci_bus_ids=" + hw_token(pci) +
                               ";nodes=local";
    c["FFTM_AUTOTUNE_HARDWARE_SIGNATURE_VERSION"] = "2";
    c["FFTM_AUTOTUNE_HARDWARE_SIGNATURE"] = "v2:" + fnv1a_hex(compat);
    c["FFTM_AUTOTUNE_HARDWARE_SIGNATURE_STRICT"] = "v2:" + fnv1a_hex(strict);
    c["FFTM_AUTOTUNE_HARDWARE_BACKENDS"] = "cuda";
    c["FFTM_AUTOTUNE_GPU_MODELS"] = hw_token(p.name);
    c["FFTM_AUTOTUNE_GPU_ARCHITECTURES"] = hw_token(arch);
    c["FFTM_AUTOTUNE_DEVICE_UUIDS"] = hw_token(uuid);
    c["FFTM_AUTOTUNE_DEVICE_PCI_BUS_IDS"] = hw_token(pci);
    c["FFTM_AUTOTUNE_DEVICE_TOTAL_BYTES"] = std::to_string((unsigned long long)p.totalGlobalMem);
    c["FFTM_AUTOTUNE_RUNTIME_VERSIONS"] = std::to_string(rt);
    c["FFTM_AUTOTUNE_DRIVER_VERSIONS"] = std::to_string(drv);
    c["FFTM_AUTOTUNE_MPI_LIBRARY"] = "unavailable";
    c["FFTM_AUTOTUNE_NODE_COUNT"] = "1";
    c["FFTM_AUTOTUNE_RANKS_PER_NODE"] = "1";
    c["FFTM_AUTOTUNE_DEVICES_PER_NODE"] = "1";
    c["FFTM_AUTOTUNE_NODE_NAMES"] = "local";
    c["FFTM_AUTOTUNE_TRANSPORT"] = "local";
    c["FFTM_AUTOTUNE_TRANSPORT_ENVIRONMENT"] = hw_token(env);
    c["FFTB_AUTOTUNE_CANONICAL_COMPATIBILITY"] = compat;
    return FFTB_SUCCESS;
}

// --------------------------------------------------------------------------- validation
// Keys that name the problem; a cache matches only if each one present in `expect`
// has the same value in the cache (source/fftm_autotune.hpp validate_match).
const char *kIdentityKeys[] = {
    "FFTM_AUTOTUNE_SCHEMA", "FFTM_AUTOTUNE_POLICY_VERSION", "FFTM_AUTOTUNE_LIBRARY", "FFTM_AUTOTUNE_DIM",
    "FFTM_AUTOTUNE_NUM_GPUS", "FFTM_AUTOTUNE_SIZE_2D", "FFTM_AUTOTUNE_SIZE_3D", "FFTM_AUTOTUNE_SIZE_4D",
    "FFTM_AUTOTUNE_SPECTRAL_LAYOUT_4D", "FFTB_AUTOTUNE_DTYPE", "FFTB_AUTOTUNE_BATCH_COUNT",
    "FFTB_AUTOTUNE_BATCH_SHAPES", "FFTB_AUTOTUNE_BATCH_OP",
};

int validate_hardware(const Config &cache, const Config &expect, int flags);

// A cache the reference wrote for one GPU (FFTM_AUTOTUNE_LIBRARY=fftm: its policy or measured
// cache, source/fftm_autotune.hpp:660-676): schema 2, the same dimension, sizes and one rank,
// and the same hardware.  Its strategy keys name MPI decompositions (slab-pencil,
// pencil-slab, pencil-pencil in 3D; slab-slab, pencil-pencil in 4D) that all reduce to the
// one single-GPU transform, so they map onto this library's own default execution.
int validate_reference(const Config &cache, const Config &expect, int flags)
{
    const char *keys[] = {"FFTM_AUTOTUNE_SCHEMA", "FFTM_AUTOTUNE_DIM", "FFTM_AUTOTUNE_NUM_GPUS",
                          "FFTM_AUTOTUNE_SIZE_2D", "FFTM_AUTOTUNE_SIZE_3D", "FFTM_AUTOTUNE_SIZE_4D"};
    for (const char *k : keys) {
        auto it = expect.find(k);
        if (it == expect.end()) continue;
        if (get(cache, k) != it->second) {
            set_last_error(std::string("fftm autotune cache ") + k + "='" + get(cache, k) + "' does not match '" +
                           it->second + "'");
            return FFTB_ERROR_CACHE_MISMATCH;
        }
    }
    if (expect.count("FFTB_AUTOTUNE_BATCH_COUNT")) {
        set_last_error("an fftm autotune cache has no batched form");
        return FFTB_ERROR_CACHE_MISMATCH;
    }
    return validate_hardware(cache, expect, flags);
}

// The fftb config that a validated reference cache stands for: the problem and hardware
// keys of `expect`, the default execution, and the reference's choice kept for the record.
Config translate_reference(const Config &cache, const Config &expect)
{
    Config c = expect;
    c["FFTM_AUTOTUNE_SOURCE"] = "fftm-cache:" + get(cache, "FFTM_AUTOTUNE_SOURCE");
    c["FFTB_AUTOTUNE_STRATEGY"] = "auto";
    c["FFTB_AUTOTUNE_PLANE_CLUSTER"] = "0";
    const std::string s3 = get(cache, "FFTM_AUTOTUNE_STRATEGY_3D"), s4 = get(cache, "FFTM_AUTOTUNE_STRATEGY_4D");
    if (!s3.empty()) c["FFTB_AUTOTUNE_REFERENCE_STRATEGY_3D"] = s3;
    if (!s4.empty()) c["FFTB_AUTOTUNE_REFERENCE_STRATEGY_4D"] = s4;
    return c;
}

int validate(const Config &cache, const Config &expect, int flags)
{
    if (get(cache, "FFTM_AUTOTUNE_LIBRARY") == "fftm") return validate_reference(cache, expect, flags);
    for (const char *k : kIdentityKeys) {
        auto it = expect.find(k);
        if (it == expect.end()) continue;
        const std::string have = get(cache, k);
        if (have != it->second) {
            set_last_error(std::string("autotune cache ") + k + "='" + have + "' does not match '" + it->second + "'");
            return FFTB_ERROR_CACHE_MISMATCH;
        }
    }
    if (get(cache, "FFTM_AUTOTUNE_SOURCE").rfind("fftb-measured", 0) != 0) {
        set_last_error("autotune cache is not a measured fftb cache (FFTM_AUTOTUNE_SOURCE='" +
                       get(cache, "FFTM_AUTOTUNE_SOURCE") + "')");
        return FFTB_ERROR_CACHE_MISMATCH;
    }
    return validate_hardware(cache, expect, flags);
}

int validate_hardware(const Config &cache, const Config &expect, int flags)
{
    if (!(flags & FFTB_TUNE_NO_HARDWARE_CHECK)) {
        const std::string sig = get(cache, "FFTM_AUTOTUNE_HARDWARE_SIGNATURE");
        if (sig.rfind("v2:", 0) != 0) {
            set_last_error("autotune cache has no versioned hardware signature");
            return FFTB_ERROR_CACHE_MISMATCH;
        }
        if (sig != get(expect, "FFTM_AUTOTUNE_HARDWARE_SIGNATURE")) {
            set_last_error("autotune cache hardware signature '" + sig + "' does not match current hardware '" +
                           get(expect, "FFTM_AUTOTUNE_HARDWARE_SIGNATURE") + "'");
            return FFTB_ERROR_CACHE_MISMATCH;
        }
        if ((flags & FFTB_TUNE_STRICT_DEVICE) &&
            get(cache, "FFTM_AUTOTUNE_HARDWARE_SIGNATURE_STRICT") !=
                get(expect, "FFTM_AUTOTUNE_HARDWARE_SIGNATURE_STRICT")) {
            set_last_error("autotune cache strict device signature does not match the current device");
            return FFTB_ERROR_CACHE_MISMATCH;
        }
    }
    return FFTB_SUCCESS;
}

// --------------------------------------------------------------------------- measurement
struct Candidate {
    std::string name;
    int a = 0, b = 0, c = 0;   // ffts: strategy, cluster; batch: mode, tiles_scale, ctas_per_sm
    bool valid = false;
    double median_ms = std::numeric_limits<double>::infinity();
    std::string error;
};

double median(std::vector<double> v)
{
    std::sort(v.begin(), v.end());
    const size_t m = v.size() / 2;
    return v.size() % 2 == 0 ? 0.5 * (v[m - 1] + v[m]) : v[m];
}

// deterministic input values in [-1, 1) (64-bit LCG, Knuth's MMIX constants)
void fill_host(std::vector<double> &h)
{
    uint64_t s = 0x2545F4914F6CDD1DULL;
    for (double &v : h) {
        s = s * 6364136223846793005ULL + 1442695040888963407ULL;
        v = (double)(s >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
    }
}

struct DevBuf {
    void *p = nullptr;
    ~DevBuf()
    {
        if (p) cudaFree(p);
    }
    int alloc(size_t bytes)
    {
        if (cudaMalloc(&p, bytes) != cudaSuccess) {
            cudaGetLastError();
            p = nullptr;
            set_last_error("autotune buffer allocation of " + std::to_string(bytes) + " bytes failed");
            return FFTB_ERROR_ALLOC;
        }
        return FFTB_SUCCESS;
    }
};

struct Events {
    cudaEvent_t a = nullptr, b = nullptr;
    cudaStream_t s = nullptr;
    ~Events()
    {
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
        if (s) cudaStreamDestroy(s);
    }
    int init()
    {
        cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreate(&a);
        if (e == cudaSuccess) e = cudaEventCreate(&b);
        return set_status_from_cuda(e);
    }
};

int upload(void *dst, const std::vector<double> &h, int dtype)
{
    cudaError_t e;
    if (dtype == FFTB_F32) {
        std::vector<float> f(h.begin(), h.end());
        e = cudaMemcpy(dst, f.data(), f.size() * 4, cudaMemcpyHostToDevice);
    } else {
        e = cudaMemcpy(dst, h.data(), h.size() * 8, cudaMemcpyHostToDevice);
    }
    return set_status_from_cuda(e);
}

// the values at n_samples evenly spread offsets
int sample(const void *dev, size_t n, int dtype, std::vector<double> &out)
{
    const size_t ns = std::min<size_t>(64, n);
    out.assign(ns, 0.0);
    for (size_t i = 0; i < ns; ++i) {
        const size_t off = (i * (n - 1)) / (ns > 1 ? ns - 1 : 1);
        cudaError_t e;
        if (dtype == FFTB_F32) {
            float v;
            e = cudaMemcpy(&v, (const float *)dev + off, 4, cudaMemcpyDeviceToHost);
            out[i] = v;
        } else {
            e = cudaMemcpy(&out[i], (const double *)dev + off, 8, cudaMemcpyDeviceToHost);
        }
        if (e != cudaSuccess) return set_status_from_cuda(e);
    }
    return FFTB_SUCCESS;
}

std::string fmt(double v)
{
    char b[64];
    snprintf(b, sizeof(b), "%.6g", v);
    return b;
}

std::string dtype_name(int dtype) { return dtype == FFTB_F32 ? "float32" : "float64"; }

const char *layout_name(int layout)
{
    return layout == FFTB_4D_SLAB ? "slab" : layout == FFTB_4D_NATIVE_XZWY ? "native_xzwy" : "pencil";
}

Config ffts_identity(int dtype, long long nx, long long ny, long long nz, long long nw, int layout)
{
    Config c;
    const int dim = nz == 0 ? 2 : (nw == 0 ? 3 : 4);
    c["FFTM_AUTOTUNE_SCHEMA"] = "2";
    c["FFTM_AUTOTUNE_POLICY_VERSION"] = kPolicyVersion;
    c["FFTM_AUTOTUNE_LIBRARY"] = "fftb";
    c["FFTM_AUTOTUNE_DIM"] = std::to_string(dim);
    c["FFTM_AUTOTUNE_NUM_GPUS"] = "1";
    c["FFTB_AUTOTUNE_DTYPE"] = dtype_name(dtype);
    const std::string s2 = std::to_string(nx) + "x" + std::to_string(ny);
    if (dim == 2) c["FFTM_AUTOTUNE_SIZE_2D"] = s2;
    if (dim == 3) c["FFTM_AUTOTUNE_SIZE_3D"] = s2 + "x" + std::to_string(nz);
    if (dim == 4) {
        c["FFTM_AUTOTUNE_SIZE_4D"] = s2 + "x" + std::to_string(nz) + "x" + std::to_string(nw);
        c["FFTM_AUTOTUNE_SPECTRAL_LAYOUT_4D"] = layout_name(layout);
    }
    return c;
}

// Times `warmup` + `iters` forward+backward pairs of one strategy of ffts object o.
void measure_ffts_candidate(fftb_ffts o, Candidate &cand, int dtype, size_t nreal, double nnorm, void *x, void *x0,
                            void *spec, Events &ev, int warmup, int iters, const std::vector<double> &ref)
{
    int st = fftb_ffts_set_strategy(o, cand.a, cand.b);
    if (st != FFTB_SUCCESS) {
        cand.error = std::string(fftb_status_string(st)) + ": " + last_error();
        return;
    }
    const size_t bytes = nreal * real_bytes(dtype);
    std::vector<double> times;
    for (int it = 0; it < warmup + iters && st == FFTB_SUCCESS; ++it) {
        cudaError_t e = cudaMemcpyAsync(x, x0, bytes, cudaMemcpyDeviceToDevice, ev.s);
        if (e == cudaSuccess) e = cudaEventRecord(ev.a, ev.s);
        if (e != cudaSuccess) {
            st = set_status_from_cuda(e);
            break;
        }
        st = fftb_ffts_forward(o, x, spec);
        if (st == FFTB_SUCCESS) st = fftb_ffts_backward(o, spec, x);
        if (st != FFTB_SUCCESS) break;
        e = cudaEventRecord(ev.b, ev.s);
        if (e == cudaSuccess) e = cudaEventSynchronize(ev.b);
        float ms = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, ev.a, ev.b);
        if (e != cudaSuccess) {
            st = set_status_from_cuda(e);
            break;
        }
        if (it >= warmup) times.push_back(ms);
    }
    if (st != FFTB_SUCCESS) {
        cand.error = std::string(fftb_status_string(st)) + ": " + last_error();
        return;
    }
    std::vector<double> got;
    if ((st = sample(x, nreal, dtype, got)) != FFTB_SUCCESS) {
        cand.error = "sample read failed";
        return;
    }
    double err = 0.0;
    for (size_t i = 0; i < got.size(); ++i) {
        const double expect = ref[i] * nnorm;
        err = std::max(err, std::fabs(got[i] - expect) / std::max(std::fabs(expect), 1.0));
    }
    const double eps = dtype == FFTB_F32 ? (double)std::numeric_limits<float>::epsilon()
                                         : std::numeric_limits<double>::epsilon();
    const double tol = 1000.0 * eps * std::max(1.0, std::log2(nnorm));
    if (!std::isfinite(err) || err > tol) {
        cand.error = "round-trip check failed: relative error " + fmt(err) + " > " + fmt(tol);
        return;
    }
    cand.valid = true;
    cand.median_ms = median(times);
}

int measure_ffts(int dtype, long long nx, long long ny, long long nz, long long nw, int layout, int warmup, int iters,
                 Config &out)
{
    fftb_ffts o = nullptr;
    int st = fftb_ffts_create(dtype, nx, ny, nz, nw, layout, &o);
    if (st != FFTB_SUCCESS) return st;
    struct Guard {
        fftb_ffts o;
        ~Guard() { fftb_ffts_destroy(o); }
    } guard{o};
    const int dim = nz == 0 ? 2 : (nw == 0 ? 3 : 4);
    std::vector<Candidate> cands;
    if (dim == 3) {
        int cl[4];
        const int n = fused3d_clusters(dtype, nx, ny, nz, cl, 4);
        if (n > 0) {
            // the library's own choice: the smallest cluster that fits for the forward planes,
            // and for the inverse planes a larger one when that doubles their CTAs per SM
            // (a pair no forced cluster size gives)
            Candidate c;
            c.name = "fused";
            c.a = FFTB_STRATEGY_FUSED;
            c.b = 0;
            cands.push_back(c);
        }
        for (int i = 0; i < n; ++i) {
            Candidate c;
            c.name = "fused-cl" + std::to_string(cl[i]);
            c.a = FFTB_STRATEGY_FUSED;
            c.b = cl[i];
            cands.push_back(c);
        }
        if (n > 0) {
            Candidate c;
            c.name = "fused-tc";
            c.a = FFTB_STRATEGY_FUSED_TC;
            c.b = 0;
            cands.push_back(c);
        }
    } else if (dim == 4) {
        Fused4D f;
        if (fused4d_init(f, dtype, layout, nx, ny, nz, nw) == FFTB_SUCCESS && f.enabled) {
            Candidate c;
            c.name = "fused";
            c.a = FFTB_STRATEGY_FUSED;
            c.b = 0;
            cands.push_back(c);
            c.name = "fused-tc";
            c.a = FFTB_STRATEGY_FUSED_TC;
            cands.push_back(c);
        }
    }
    {
        Candidate c;
        c.name = "staged";
        c.a = FFTB_STRATEGY_STAGED;
        cands.push_back(c);
    }
    const size_t nreal = (size_t)nx * ny * (nz ? nz : 1) * (nw ? nw : 1);
    const long long last = dim == 2 ? ny : (dim == 3 ? nz : nw);
    const size_t nspec = nreal / last * (last / 2 + 1);
    size_t work = 0;
    if ((st = fftb_ffts_work_size(o, &work)) != FFTB_SUCCESS) return st;
    DevBuf x, x0, spec, wk;
    if ((st = x.alloc(nreal * real_bytes(dtype))) != FFTB_SUCCESS) return st;
    if ((st = x0.alloc(nreal * real_bytes(dtype))) != FFTB_SUCCESS) return st;
    if ((st = spec.alloc(nspec * complex_bytes(dtype))) != FFTB_SUCCESS) return st;
    if (work && (st = wk.alloc(work)) != FFTB_SUCCESS) return st;
    if (work && (st = fftb_ffts_set_work_area(o, wk.p)) != FFTB_SUCCESS) return st;
    Events ev;
    if ((st = ev.init()) != FFTB_SUCCESS) return st;
    if ((st = fftb_ffts_set_stream(o, ev.s)) != FFTB_SUCCESS) return st;
    std::vector<double> h(nreal);
    fill_host(h);
    if ((st = upload(x0.p, h, dtype)) != FFTB_SUCCESS) return st;
    std::vector<double> ref;
    if ((st = sample(x0.p, nreal, dtype, ref)) != FFTB_SUCCESS) return st;
    const Candidate *best = nullptr;
    std::string list;
    for (Candidate &c : cands) {
        measure_ffts_candidate(o, c, dtype, nreal, (double)nreal, x.p, x0.p, spec.p, ev, warmup, iters, ref);
        list += (list.empty() ? "" : ",") + c.name;
        if (c.valid) {
            out["FFTB_AUTOTUNE_MEDIAN_MS_" + c.name] = fmt(c.median_ms);
            if (!best || c.median_ms < best->median_ms) best = &c;
        } else {
            out["FFTB_AUTOTUNE_FAILED_" + c.name] = c.error;
        }
    }
    out["FFTB_AUTOTUNE_CANDIDATES"] = list;
    if (!best) {
        set_last_error("no autotune candidate passed: " + cands.back().error);
        return FFTB_ERROR_TUNE_FAILED;
    }
    out["FFTB_AUTOTUNE_STRATEGY"] =
        best->a == FFTB_STRATEGY_FUSED ? "fused" : (best->a == FFTB_STRATEGY_FUSED_TC ? "fused_tc" : "staged");
    out["FFTB_AUTOTUNE_PLANE_CLUSTER"] = std::to_string(best->b);
    out[dim == 4 ? "FFTM_AUTOTUNE_STRATEGY_4D" : "FFTM_AUTOTUNE_STRATEGY_3D"] = best->name;
    out["FFTB_AUTOTUNE_MEDIAN_MS"] = fmt(best->median_ms);
    out["FFTB_AUTOTUNE_WARMUP"] = std::to_string(warmup);
    out["FFTB_AUTOTUNE_ITERATIONS"] = std::to_string(iters);
    return FFTB_SUCCESS;
}

// ---- batch
Config batch_identity_config(fftb_batch b, int op)
{
    int dtype = 0, count = 0, ts = 0, cps = 0;
    const long long *dims = nullptr;
    void *stream = nullptr;
    batch_identity(b, &dtype, &count, &dims, &ts, &cps, &stream);
    std::string shapes;
    for (int i = 0; i < 3 * count; ++i) shapes += std::to_string(dims[i]) + (i % 3 == 2 ? ";" : "x");
    Config c;
    c["FFTM_AUTOTUNE_SCHEMA"] = "2";
    c["FFTM_AUTOTUNE_POLICY_VERSION"] = kPolicyVersion;
    c["FFTM_AUTOTUNE_LIBRARY"] = "fftb";
    c["FFTM_AUTOTUNE_DIM"] = "3";
    c["FFTM_AUTOTUNE_NUM_GPUS"] = "1";
    c["FFTB_AUTOTUNE_DTYPE"] = dtype_name(dtype);
    c["FFTB_AUTOTUNE_BATCH_COUNT"] = std::to_string(count);
    c["FFTB_AUTOTUNE_BATCH_SHAPES"] = "fnv1a:" + fnv1a_hex(shapes);
    c["FFTB_AUTOTUNE_BATCH_OP"] = std::to_string(op);
    return c;
}

int measure_batch(fftb_batch b, int op, double sign, int warmup, int iters, Config &out)
{
    int dtype = 0, count = 0, ts0 = 1, cps0 = 0;
    const long long *dims = nullptr;
    void *stream0 = nullptr;
    batch_identity(b, &dtype, &count, &dims, &ts0, &cps0, &stream0);
    // the batch runs on the private timing stream while it is measured
    struct StreamBack {
        fftb_batch b;
        void *s;
        ~StreamBack() { fftb_batch_set_stream(b, s); }
    } stream_back{b, stream0};
    long long rtot = 0, stot = 0;
    int st = fftb_batch_layout(b, nullptr, nullptr, &rtot, &stot);
    if (st != FFTB_SUCCESS) return st;
    std::vector<Candidate> cands;
    {
        Candidate c;
        c.name = "sequential";
        c.a = 0;
        c.b = 1;
        cands.push_back(c);
    }
    if (dtype == FFTB_F32) {
        for (int ts : {1, 2})
            for (int cps : {0, 1, 2}) {
                Candidate c;
                c.name = "graph-t" + std::to_string(ts) + "-c" + std::to_string(cps);
                c.a = 2;
                c.b = ts;
                c.c = cps;
                cands.push_back(c);
            }
        for (int ts : {1, 2}) {
            Candidate c;
            c.name = "grouped-graph-t" + std::to_string(ts);
            c.a = 4;
            c.b = ts;
            c.c = 0;
            cands.push_back(c);
        }
    }
    const bool in_spec = op == FFTB_BATCH_BACKWARD, out_spec = op == FFTB_BATCH_FORWARD;
    const size_t nin = in_spec ? (size_t)stot * 2 : (size_t)rtot;     // reals
    const size_t nout = out_spec ? (size_t)stot * 2 : (size_t)rtot;
    DevBuf in, in0, outb;
    if ((st = in.alloc(nin * real_bytes(dtype))) != FFTB_SUCCESS) return st;
    if ((st = in0.alloc(nin * real_bytes(dtype))) != FFTB_SUCCESS) return st;
    if ((st = outb.alloc(nout * real_bytes(dtype))) != FFTB_SUCCESS) return st;
    Events ev;
    if ((st = ev.init()) != FFTB_SUCCESS) return st;
    if ((st = fftb_batch_set_stream(b, ev.s)) != FFTB_SUCCESS) return st;
    std::vector<double> h(nin);
    fill_host(h);
    if ((st = upload(in0.p, h, dtype)) != FFTB_SUCCESS) return st;
    // the round trip reproduces its input; the other ops are checked for finite output
    std::vector<double> ref;
    if ((st = sample(in0.p, nin, dtype, ref)) != FFTB_SUCCESS) return st;
    const Candidate *best = nullptr;
    std::string list;
    for (Candidate &c : cands) {
        list += (list.empty() ? "" : ",") + c.name;
        st = fftb_batch_set_tuning(b, c.a == 0 ? ts0 : c.b, c.a == 0 ? cps0 : c.c);
        std::vector<double> times;
        for (int it = 0; it < warmup + iters && st == FFTB_SUCCESS; ++it) {
            cudaError_t e = cudaMemcpyAsync(in.p, in0.p, nin * real_bytes(dtype), cudaMemcpyDeviceToDevice, ev.s);
            if (e == cudaSuccess) e = cudaEventRecord(ev.a, ev.s);
            if (e != cudaSuccess) {
                st = set_status_from_cuda(e);
                break;
            }
            st = fftb_batch_exec(b, op, in.p, outb.p, sign, c.a);
            if (st != FFTB_SUCCESS) break;
            e = cudaEventRecord(ev.b, ev.s);
            if (e == cudaSuccess) e = cudaEventSynchronize(ev.b);
            float ms = 0.f;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, ev.a, ev.b);
            if (e != cudaSuccess) {
                st = set_status_from_cuda(e);
                break;
            }
            if (it >= warmup) times.push_back(ms);
        }
        int flag = 0;
        if (st == FFTB_SUCCESS && (c.a == 1 || c.a == 2)) st = fftb_batch_status(b, op, &flag);
        std::vector<double> got;
        if (st == FFTB_SUCCESS) st = sample(outb.p, nout, dtype, got);
        if (st != FFTB_SUCCESS) {
            c.error = std::string(fftb_status_string(st)) + ": " + last_error();
        } else if (flag != 0) {
            c.error = "persistent launch reported an expired dependency wait";
        } else {
            double err = 0.0;
            for (size_t i = 0; i < got.size(); ++i) {
                if (!std::isfinite(got[i])) err = std::numeric_limits<double>::infinity();
                else if (op == FFTB_BATCH_ROUNDTRIP)
                    err = std::max(err, std::fabs(got[i] - ref[i]) / std::max(std::fabs(ref[i]), 1.0));
            }
            const double eps = dtype == FFTB_F32 ? (double)std::numeric_limits<float>::epsilon()
                                                 : std::numeric_limits<double>::epsilon();
            const double tol = 1000.0 * eps * std::log2(4096.0 * 4096.0 * 4096.0);
            if (!std::isfinite(err) || err > tol) c.error = "round-trip check failed: relative error " + fmt(err);
            else {
                c.valid = true;
                c.median_ms = median(times);
            }
        }
        if (c.valid) {
            out["FFTB_AUTOTUNE_MEDIAN_MS_" + c.name] = fmt(c.median_ms);
            if (!best || c.median_ms < best->median_ms) best = &c;
        } else {
            out["FFTB_AUTOTUNE_FAILED_" + c.name] = c.error;
        }
    }
    out["FFTB_AUTOTUNE_CANDIDATES"] = list;
    if (!best) {
        fftb_batch_set_tuning(b, ts0, cps0);
        set_last_error("no batch autotune candidate passed: " + cands.back().error);
        return FFTB_ERROR_TUNE_FAILED;
    }
    out["FFTB_AUTOTUNE_BATCH_MODE"] = std::to_string(best->a);
    out["FFTB_AUTOTUNE_TILES_SCALE"] = std::to_string(best->a == 0 ? ts0 : best->b);
    out["FFTB_AUTOTUNE_CTAS_PER_SM"] = std::to_string(best->a == 0 ? cps0 : best->c);
    out["FFTM_AUTOTUNE_STRATEGY_3D"] = best->name;
    out["FFTB_AUTOTUNE_MEDIAN_MS"] = fmt(best->median_ms);
    out["FFTB_AUTOTUNE_WARMUP"] = std::to_string(warmup);
    out["FFTB_AUTOTUNE_ITERATIONS"] = std::to_string(iters);
    return FFTB_SUCCESS;
}

int to_int(const std::string &s, int *v)
{
    if (s.empty()) return FFTB_ERROR_INVALID_VALUE;
    char *end = nullptr;
    const long r = strtol(s.c_str(), &end, 10);
    if (*end != '\0' || r < -1000000 || r > 1000000) return FFTB_ERROR_INVALID_VALUE;
    *v = (int)r;
    return FFTB_SUCCESS;
}

// The shared load-or-measure flow; `identity` holds the problem keys, `measure` fills
// the tuned keys of a fresh config.
template <typename Measure>
int load_or_measure(const char *cache_file, int flags, int device, const Config &identity, Measure measure,
                    Config &result, int *from_cache)
{
    if (!cache_file || !*cache_file) {
        set_last_error("autotune cache_file must not be empty");
        return FFTB_ERROR_INVALID_VALUE;
    }
    Config expect = identity;
    int st = hardware_config(device, expect);
    if (st != FFTB_SUCCESS) return st;
    const std::string path = cache_file;
    bool need = (flags & FFTB_TUNE_FORCE_MEASURE) != 0;
    if (!need) {
        if (!file_exists(path)) {
            if (!(flags & FFTB_TUNE_CREATE_IF_MISSING)) {
                set_last_error("autotune cache file does not exist: " + path);
                return FFTB_ERROR_CACHE_MISSING;
            }
            need = true;
        } else {
            Config cached;
            st = load_file(path, cached);
            if (st == FFTB_SUCCESS) st = validate(cached, expect, flags);
            if (st == FFTB_SUCCESS) {
                result = get(cached, "FFTM_AUTOTUNE_LIBRARY") == "fftm" ? translate_reference(cached, expect) : cached;
                if (from_cache) *from_cache = 1;
                return FFTB_SUCCESS;
            }
            if (!(flags & FFTB_TUNE_OVERWRITE_ON_MISMATCH)) return st;
            need = true;
        }
    }
    Config fresh = expect;
    fresh["FFTM_AUTOTUNE_SOURCE"] = kMeasuredSource;
    if ((st = measure(fresh)) != FFTB_SUCCESS) return st;
    if ((st = save_file(path, fresh)) != FFTB_SUCCESS) return st;
    result = fresh;
    if (from_cache) *from_cache = 0;
    return FFTB_SUCCESS;
}

} // namespace

extern "C" {

int fftb_autotune_load_file(const char *path, char *text, size_t capacity, size_t *needed)
{
    if (!path) return FFTB_ERROR_INVALID_VALUE;
    Config c;
    int st = load_file(path, c);
    if (st != FFTB_SUCCESS) return st;
    return put_text(to_text(c), text, capacity, needed);
}

int fftb_autotune_save_file(const char *path, const char *text)
{
    if (!path || !text) return FFTB_ERROR_INVALID_VALUE;
    Config c;
    int st = parse_text(text, "<text>", c);
    if (st != FFTB_SUCCESS) return st;
    return save_file(path, c);
}

int fftb_autotune_validate(const char *cache_text, const char *expected_text, int flags)
{
    if (!cache_text || !expected_text) return FFTB_ERROR_INVALID_VALUE;
    Config cache, expect;
    int st = parse_text(cache_text, "<cache>", cache);
    if (st == FFTB_SUCCESS) st = parse_text(expected_text, "<expected>", expect);
    if (st == FFTB_SUCCESS) st = validate(cache, expect, flags);
    return st;
}

int fftb_autotune_signature(const char *canonical, char *text, size_t capacity, size_t *needed)
{
    if (!canonical) return FFTB_ERROR_INVALID_VALUE;
    return put_text("v2:" + fnv1a_hex(canonical), text, capacity, needed);
}

int fftb_autotune_hardware(int device, char *text, size_t capacity, size_t *needed)
{
    Config c;
    int st = hardware_config(device, c);
    if (st != FFTB_SUCCESS) return st;
    return put_text(to_text(c), text, capacity, needed);
}

int fftb_autotune_ffts(int dtype, long long nx, long long ny, long long nz, long long nw, int layout4d,
                       const char *cache_file, int flags, int warmup, int iterations, char *text, size_t capacity,
                       size_t *needed, int *from_cache)
{
    if ((dtype != FFTB_F32 && dtype != FFTB_F64) || nx < 1 || ny < 1 || nz < 0 || nw < 0 || (nz == 0 && nw > 0) ||
        warmup < 0 || iterations < 1)
        return FFTB_ERROR_INVALID_VALUE;
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return set_status_from_cuda(e);
    Config result;
    int st = load_or_measure(
        cache_file, flags, device, ffts_identity(dtype, nx, ny, nz, nw, layout4d),
        [&](Config &c) { return measure_ffts(dtype, nx, ny, nz, nw, layout4d, warmup, iterations, c); }, result,
        from_cache);
    if (st != FFTB_SUCCESS) return st;
    return put_text(to_text(result), text, capacity, needed);
}

int fftb_ffts_apply_config(fftb_ffts obj, const char *text)
{
    if (!obj) return FFTB_ERROR_INVALID_HANDLE;
    if (!text) return FFTB_ERROR_INVALID_VALUE;
    Config c;
    int st = parse_text(text, "<config>", c);
    if (st != FFTB_SUCCESS) return st;
    const std::string strat = get(c, "FFTB_AUTOTUNE_STRATEGY");
    int cl = 0;
    if ((strat != "fused" && strat != "fused_tc" && strat != "staged" && strat != "auto") ||
        to_int(get(c, "FFTB_AUTOTUNE_PLANE_CLUSTER"), &cl) != FFTB_SUCCESS) {
        set_last_error("autotune config has no valid FFTB_AUTOTUNE_STRATEGY / FFTB_AUTOTUNE_PLANE_CLUSTER");
        return FFTB_ERROR_CACHE_MISMATCH;
    }
    const int code = strat == "fused"      ? FFTB_STRATEGY_FUSED
                     : strat == "fused_tc" ? FFTB_STRATEGY_FUSED_TC
                     : strat == "auto"     ? FFTB_STRATEGY_AUTO
                                           : FFTB_STRATEGY_STAGED;
    return fftb_ffts_set_strategy(obj, code, cl);
}

int fftb_autotune_batch(fftb_batch batch, int op, double sign, const char *cache_file, int flags, int warmup,
                        int iterations, char *text, size_t capacity, size_t *needed, int *from_cache, int *mode)
{
    if (!batch) return FFTB_ERROR_INVALID_HANDLE;
    if (op < FFTB_BATCH_FORWARD || op > FFTB_BATCH_POISSON || warmup < 0 || iterations < 1)
        return FFTB_ERROR_INVALID_VALUE;
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return set_status_from_cuda(e);
    Config result;
    int st = load_or_measure(
        cache_file, flags, device, batch_identity_config(batch, op),
        [&](Config &c) { return measure_batch(batch, op, sign, warmup, iterations, c); }, result, from_cache);
    if (st != FFTB_SUCCESS) return st;
    const std::string t = to_text(result);
    if ((st = fftb_batch_apply_config(batch, t.c_str(), mode)) != FFTB_SUCCESS) return st;
    return put_text(t, text, capacity, needed);
}

int fftb_batch_apply_config(fftb_batch batch, const char *text, int *mode)
{
    if (!batch) return FFTB_ERROR_INVALID_HANDLE;
    if (!text) return FFTB_ERROR_INVALID_VALUE;
    Config c;
    int st = parse_text(text, "<config>", c);
    if (st != FFTB_SUCCESS) return st;
    int m = 0, ts = 0, cps = 0;
    if (to_int(get(c, "FFTB_AUTOTUNE_BATCH_MODE"), &m) != FFTB_SUCCESS ||
        to_int(get(c, "FFTB_AUTOTUNE_TILES_SCALE"), &ts) != FFTB_SUCCESS ||
        to_int(get(c, "FFTB_AUTOTUNE_CTAS_PER_SM"), &cps) != FFTB_SUCCESS || m < 0 || m > 4) {
        set_last_error("autotune config has no valid FFTB_AUTOTUNE_BATCH_MODE / _TILES_SCALE / _CTAS_PER_SM");
        return FFTB_ERROR_CACHE_MISMATCH;
    }
    if ((st = fftb_batch_set_tuning(batch, ts, cps)) != FFTB_SUCCESS) return st;
    if (mode) *mode = m;
    return FFTB_SUCCESS;
}

} // extern "C"
