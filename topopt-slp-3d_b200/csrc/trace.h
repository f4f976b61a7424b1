// Tracing of the library's entry points.
//
// * NVTX ranges (header-only NVTX 3): every entry point of tosp.h opens a
//   range named after the MATLAB function it replaces, so Nsight timelines show
//   SetupGMG / SolveMG / Grad / ApplyFilter / serving ticks over the kernels.
//   Without a profiler attached the calls cost a few nanoseconds.
// * Metrics: when the environment variable TOSP_METRICS names a file, each
//   solve and each served request appends one JSON line to it (wall time,
//   iterations, relative residual, status; for requests also queue time and
//   precision).  Off when the variable is unset.
#pragma once

#include <nvtx3/nvToolsExt.h>

#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <string>

namespace tosp {

struct TraceRange {
    explicit TraceRange(const char *name) { nvtxRangePushA(name); }
    ~TraceRange() { nvtxRangePop(); }
    TraceRange(const TraceRange &) = delete;
    TraceRange &operator=(const TraceRange &) = delete;
};

// Appends `json` (one object, no newline) as a line of the TOSP_METRICS file.
inline void metrics_line(const std::string &json) {
    static std::mutex mu;
    static const char *path = std::getenv("TOSP_METRICS");
    if (!path || !*path) return;
    std::lock_guard<std::mutex> lk(mu);
    if (FILE *f = std::fopen(path, "a")) {
        std::fputs(json.c_str(), f);
        std::fputc('\n', f);
        std::fclose(f);
    }
}

inline bool metrics_on() {
    static const char *path = std::getenv("TOSP_METRICS");
    return path && *path;
}

}  // namespace tosp
