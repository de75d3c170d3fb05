// Stage tracing: with CICY_TRACE=1 in the environment, each traced scope
// synchronizes the stream on entry and exit and prints its wall time to stderr
// as "[cicy] <name> <ms>".  Off by default (no synchronization added).
#pragma once

#include <cuda_runtime.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>

namespace cicy {

inline bool trace_enabled() {
    static const bool on = [] {
        const char* v = std::getenv("CICY_TRACE");
        return v && v[0] && v[0] != '0';
    }();
    return on;
}

struct TraceScope {
    const char* name;
    cudaStream_t s;
    std::chrono::steady_clock::time_point t0;
    bool on;
    TraceScope(const char* n, cudaStream_t st) : name(n), s(st), on(trace_enabled()) {
        if (on) {
            cudaStreamSynchronize(s);
            t0 = std::chrono::steady_clock::now();
        }
    }
    ~TraceScope() {
        if (on) {
            cudaStreamSynchronize(s);
            double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
            std::fprintf(stderr, "[cicy] %-28s %9.3f ms\n", name, ms);
        }
    }
};

}  // namespace cicy

#define CICY_TRACE_CAT2(a, b) a##b
#define CICY_TRACE_CAT(a, b) CICY_TRACE_CAT2(a, b)
#define CICY_TRACE(name, stream) ::cicy::TraceScope CICY_TRACE_CAT(trace_scope_, __LINE__)(name, stream)

namespace cicy {

// Sequence of traced sections: mark("x") prints the time since the previous mark.
struct TraceSeq {
    cudaStream_t s;
    bool on;
    std::chrono::steady_clock::time_point t;
    explicit TraceSeq(cudaStream_t st) : s(st), on(trace_enabled()) {
        if (on) {
            cudaStreamSynchronize(s);
            t = std::chrono::steady_clock::now();
        }
    }
    void mark(const char* name) {
        if (!on) return;
        cudaStreamSynchronize(s);
        auto now = std::chrono::steady_clock::now();
        std::fprintf(stderr, "[cicy] %-28s %9.3f ms\n", name, std::chrono::duration<double, std::milli>(now - t).count());
        t = now;
    }
};

}  // namespace cicy
