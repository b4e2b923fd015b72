// fftb_profile.h -- the profiling and memory-profiling hooks of an ffts object (the role
// of the reference's profiler and memory profiler behind ffts_init_options,
// source/ffts.hpp:64-72, :449-629).
//
// Profiler: one entry per named scope (ffts::init<3>, ffts::forward<3>, ...): calls, host
// milliseconds of the calls, and device milliseconds between two events recorded on the
// object's stream around the call (skipped while the stream is being captured into a
// graph).  Device times are resolved when a report is made.
// Memory profiler: named byte counts (the object's own allocations) with their peaks,
// reported in the reference's "current(sum/max/avg) ... peak(sum/max/avg)" form; one
// process, so sum, max and average are the same number.
#pragma once

#include <cuda_runtime.h>

#include <chrono>
#include <cstdio>
#include <map>
#include <string>
#include <vector>

namespace fftb {

struct Profiler {
    bool enabled = false;
    std::string key;
    struct Entry {
        long long calls = 0;
        double host_ms = 0.0, device_ms = 0.0;
        long long device_samples = 0;
    };
    std::map<std::string, Entry> entries;
    struct Pending {
        std::string name;
        cudaEvent_t a = nullptr, b = nullptr;
    };
    std::vector<Pending> pending;

    void resolve()
    {
        for (Pending &p : pending) {
            float ms = 0.f;
            if (cudaEventSynchronize(p.b) == cudaSuccess && cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
                Entry &e = entries[p.name];
                e.device_ms += ms;
                e.device_samples += 1;
            }
            cudaEventDestroy(p.a);
            cudaEventDestroy(p.b);
        }
        pending.clear();
    }
    void clear_events()
    {
        for (Pending &p : pending) {
            cudaEventDestroy(p.a);
            cudaEventDestroy(p.b);
        }
        pending.clear();
    }
    std::string summary()
    {
        resolve();
        std::string s = "Profile " + key + ":";
        char buf[512];
        for (const auto &kv : entries) {
            const Entry &e = kv.second;
            std::snprintf(buf, sizeof(buf),
                          "\n  %s: calls=%lld host_ms(total/avg)=%.4f/%.4f device_ms(total/avg)=%.4f/%.4f",
                          kv.first.c_str(), e.calls, e.host_ms, e.calls ? e.host_ms / e.calls : 0.0, e.device_ms,
                          e.device_samples ? e.device_ms / e.device_samples : 0.0);
            s += buf;
        }
        return s + "\n";
    }
    std::string totals()
    {
        resolve();
        long long calls = 0;
        double h = 0.0, d = 0.0;
        for (const auto &kv : entries) {
            calls += kv.second.calls;
            h += kv.second.host_ms;
            d += kv.second.device_ms;
        }
        char buf[256];
        std::snprintf(buf, sizeof(buf), "Profile totals %s: scopes=%zu calls=%lld host_ms=%.4f device_ms=%.4f\n",
                      key.c_str(), entries.size(), calls, h, d);
        return buf;
    }
};

// RAII scope: host time always; device time when the stream is not capturing.
struct ProfScope {
    Profiler *p;
    std::string name;
    cudaStream_t stream;
    std::chrono::steady_clock::time_point t0;
    cudaEvent_t a = nullptr;
    ProfScope(Profiler &prof, std::string n, cudaStream_t s) : p(prof.enabled ? &prof : nullptr), name(std::move(n)), stream(s)
    {
        if (!p) return;
        t0 = std::chrono::steady_clock::now();
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(stream, &cs) == cudaSuccess && cs == cudaStreamCaptureStatusNone &&
            cudaEventCreate(&a) == cudaSuccess && cudaEventRecord(a, stream) != cudaSuccess) {
            cudaEventDestroy(a);
            a = nullptr;
        }
    }
    ~ProfScope()
    {
        if (!p) return;
        Profiler::Entry &e = p->entries[name];
        e.calls += 1;
        e.host_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        if (a) {
            cudaEvent_t b = nullptr;
            if (cudaEventCreate(&b) == cudaSuccess && cudaEventRecord(b, stream) == cudaSuccess) {
                p->pending.push_back({name, a, b});
                if (p->pending.size() >= 4096) p->resolve();
            } else {
                cudaEventDestroy(a);
                if (b) cudaEventDestroy(b);
            }
        }
    }
};

struct MemProfiler {
    bool enabled = false;
    std::string key;
    struct Entry {
        long long current = 0, peak = 0;
    };
    std::map<std::string, Entry> entries;

    void set_bytes(const std::string &name, long long bytes)
    {
        if (!enabled) return;
        Entry &e = entries[name];
        e.current = bytes;
        if (bytes > e.peak) e.peak = bytes;
    }
    static void line(std::string &s, const char *name, long long cur, long long peak)
    {
        char buf[512];
        const double cm = cur / (1024.0 * 1024.0), pm = peak / (1024.0 * 1024.0);
        std::snprintf(buf, sizeof(buf),
                      "\n  %s: current(sum/max/avg)=%lld/%lld/%lld B (%.3f/%.3f/%.3f MiB), peak(sum/max/avg)=%lld/%lld/%lld B "
                      "(%.3f/%.3f/%.3f MiB)",
                      name, cur, cur, cur, cm, cm, cm, peak, peak, peak, pm, pm, pm);
        s += buf;
    }
    // every entry is device memory; the reference's host_pinned and external_test
    // categories are reported (empty) for the same layout
    void categories(std::string &s) const
    {
        long long c = 0, p = 0;
        for (const auto &kv : entries) {
            c += kv.second.current;
            p += kv.second.peak;
        }
        line(s, "device", c, p);
        line(s, "host_pinned", 0, 0);
        line(s, "external_test", 0, 0);
    }
    std::string summary() const
    {
        std::string s = "Memory profile:";
        for (const auto &kv : entries) line(s, kv.first.c_str(), kv.second.current, kv.second.peak);
        s += "\nMemory profile categories:";
        categories(s);
        return s + "\n";
    }
    std::string totals() const
    {
        long long c = 0, p = 0;
        for (const auto &kv : entries) {
            c += kv.second.current;
            p += kv.second.peak;
        }
        std::string s = "Memory profile totals:";
        line(s, "total", c, p);
        categories(s);
        return s + "\n";
    }
};

} // namespace fftb
