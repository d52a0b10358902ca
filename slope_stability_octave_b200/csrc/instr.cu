// Live kernel timing for roofline reporting: when enabled, every `sample`-th launch of an
// instrumented kernel kind is bracketed by a pair of CUDA events on its own stream; the
// read-out synchronises, sums the elapsed times and resets.  Launch counts are exact.
#include <cuda_runtime.h>

#include <mutex>
#include <vector>

#include "instr.cuh"
#include "sg_common.cuh"

namespace sg {

struct InstrState {
    std::mutex mu;
    bool on = false;
    int sample = 1;
    int64_t launches[IK_COUNT] = {0};
    int64_t units[IK_COUNT] = {0};
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> timed[IK_COUNT];
    std::vector<cudaEvent_t> pool;
};

static InstrState &state() {
    static InstrState s;
    return s;
}

static cudaEvent_t take_event(InstrState &s) {
    if (!s.pool.empty()) {
        cudaEvent_t e = s.pool.back();
        s.pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

static thread_local int t_redirect_from = -1, t_redirect_to = -1;

InstrRedirect::InstrRedirect(int from, int to) : saved_from(t_redirect_from), saved_to(t_redirect_to) {
    t_redirect_from = from;
    t_redirect_to = to;
}
InstrRedirect::~InstrRedirect() {
    t_redirect_from = saved_from;
    t_redirect_to = saved_to;
}

static thread_local bool t_suspended = false;
InstrSuspend::InstrSuspend() : saved(t_suspended) { t_suspended = true; }
InstrSuspend::~InstrSuspend() { t_suspended = saved; }

InstrToken instr_begin(int kind, cudaStream_t st) {
    InstrState &s = state();
    InstrToken t;
    if (!s.on || t_suspended) return t;
    if (kind == t_redirect_from) kind = t_redirect_to;
    std::lock_guard<std::mutex> g(s.mu);
    const int64_t c = s.launches[kind]++;
    if (c % s.sample != 0) return t;
    t.kind = kind;
    t.a = take_event(s);
    t.b = take_event(s);
    if (t.a) cudaEventRecord(t.a, st);
    return t;
}

void instr_units(int kind, int64_t units) {
    InstrState &s = state();
    if (!s.on || t_suspended || kind < 0 || kind >= IK_COUNT) return;
    std::lock_guard<std::mutex> g(s.mu);
    s.units[kind] += units;
}

void instr_end(const InstrToken &t, cudaStream_t st) {
    if (t.kind < 0 || !t.a || !t.b) return;
    InstrState &s = state();
    cudaEventRecord(t.b, st);
    std::lock_guard<std::mutex> g(s.mu);
    s.timed[t.kind].push_back({t.a, t.b});
}

}  // namespace sg

using namespace sg;

extern "C" int sg_instr_enable(int on, int sample) {
    InstrState &s = state();
    std::lock_guard<std::mutex> g(s.mu);
    s.on = on != 0;
    s.sample = sample > 0 ? sample : 1;
    return SG_OK;
}

// units[k] = the work units recorded for kind k since the last sg_instr_read (not reset here).
extern "C" int sg_instr_units(int64_t *units, int32_t cap) {
    InstrState &s = state();
    SG_CHECK_ARG(units && cap >= 0, "bad argument");
    std::lock_guard<std::mutex> g(s.mu);
    for (int k = 0; k < IK_COUNT && k < cap; ++k) units[k] = s.units[k];
    return SG_OK;
}

// ms[k] = summed duration of the timed launches of kind k, timed[k] = their number,
// launches[k] = all launches of kind k since the last read.  Resets the counters.
extern "C" int sg_instr_read(double *ms, int64_t *timed, int64_t *launches, int32_t cap) {
    InstrState &s = state();
    SG_CUDA(cudaDeviceSynchronize());
    std::lock_guard<std::mutex> g(s.mu);
    for (int k = 0; k < IK_COUNT; ++k) {
        double tot = 0.0;
        for (auto &pr : s.timed[k]) {
            float m = 0.f;
            if (cudaEventElapsedTime(&m, pr.first, pr.second) == cudaSuccess) tot += m;
            s.pool.push_back(pr.first);
            s.pool.push_back(pr.second);
        }
        if (k < cap) {
            if (ms) ms[k] = tot;
            if (timed) timed[k] = (int64_t)s.timed[k].size();
            if (launches) launches[k] = s.launches[k];
        }
        s.timed[k].clear();
        s.launches[k] = 0;
        s.units[k] = 0;
    }
    return SG_OK;
}
