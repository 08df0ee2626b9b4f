// common.cuh -- shared definitions of the B200 hot-path library (status codes,
// launch accounting, error plumbing).
#pragma once
#include <cuda_runtime.h>
#include <cstdio>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/obl.h"

namespace obl {

// Per-context launch recorder.  Every kernel the library launches goes through
// Recorder::begin/end: it counts launches and, when timing is enabled, brackets the
// launch with a pair of CUDA events on the launching stream so that per-kernel device
// time can be reported without a profiler.
struct Recorder {
    long long launches = 0;
    bool timing = false;
    struct Rec { const char *name; cudaEvent_t a, b; };
    std::vector<Rec> recs;
    std::vector<cudaEvent_t> pool;

    cudaEvent_t ev()
    {
        if (!pool.empty()) { cudaEvent_t e = pool.back(); pool.pop_back(); return e; }
        cudaEvent_t e;
        cudaEventCreate(&e);
        return e;
    }
    void begin(const char *name, cudaStream_t s)
    {
        ++launches;
        if (!timing) return;
        Rec r{name, ev(), ev()};
        cudaEventRecord(r.a, s);
        recs.push_back(r);
    }
    void end(cudaStream_t s)
    {
        if (!timing || recs.empty()) return;
        cudaEventRecord(recs.back().b, s);
    }
    void release()
    {
        for (auto &r : recs) { pool.push_back(r.a); pool.push_back(r.b); }
        recs.clear();
    }
    ~Recorder()
    {
        for (auto &r : recs) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
        for (auto e : pool) cudaEventDestroy(e);
    }
};

struct LaunchScope {
    Recorder &r; cudaStream_t s;
    LaunchScope(Recorder &r_, const char *name, cudaStream_t s_) : r(r_), s(s_) { r.begin(name, s); }
    ~LaunchScope() { r.end(s); }
};

} // namespace obl
