// Optional launch timing: when enabled, CUDA events are recorded on the
// launching stream around every kernel of the selected classes, and
// lq_profile_read sums their durations.  Off by default (no events recorded).
#include <mutex>

#include "lq_internal.h"

namespace lq {

namespace {
struct Pending {
    int cls;
    cudaEvent_t a, b;
};
std::mutex g_mu;
bool g_on = false;
std::vector<Pending> g_pending;
std::vector<cudaEvent_t> g_pool;
double g_ms[kProfClasses] = {0};
long g_count[kProfClasses] = {0};
thread_local cudaEvent_t t_begin = nullptr;
thread_local int t_cls = -1;
// Brackets nest (a renormalising gate runs the norm reduction inside its own
// bracket): only the outermost one records events; inner ones count toward it.
thread_local int t_depth = 0;
// Bumped by lq_profile_enable so a bracket left open across a reset is dropped.
unsigned g_gen = 0;
thread_local unsigned t_gen = 0;

cudaEvent_t take_event() {
    if (!g_pool.empty()) {
        cudaEvent_t e = g_pool.back();
        g_pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
}

void resolve_locked() {
    for (auto &p : g_pending) {
        cudaEventSynchronize(p.b);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, p.a, p.b);
        g_ms[p.cls] += ms;
        g_count[p.cls] += 1;
        g_pool.push_back(p.a);
        g_pool.push_back(p.b);
    }
    g_pending.clear();
}
}  // namespace

bool prof_enabled() { return g_on; }

static bool capturing(cudaStream_t st) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    return cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone;
}

void prof_begin(cudaStream_t st, int cls) {
    if (!g_on || capturing(st)) return;
    std::lock_guard<std::mutex> lk(g_mu);
    if (t_gen != g_gen) {
        t_gen = g_gen;
        t_depth = 0;
        t_begin = nullptr;
    }
    if (t_depth++ > 0) return;
    t_begin = take_event();
    t_cls = cls;
    cudaEventRecord(t_begin, st);
}

void prof_end(cudaStream_t st, int cls) {
    if (!g_on || capturing(st)) return;
    std::lock_guard<std::mutex> lk(g_mu);
    if (t_gen != g_gen || t_depth == 0) return;
    if (--t_depth > 0) return;
    if (!t_begin || t_cls != cls) return;
    cudaEvent_t e = take_event();
    cudaEventRecord(e, st);
    g_pending.push_back({cls, t_begin, e});
    t_begin = nullptr;
    if (g_pending.size() > 4096) resolve_locked();
}

}  // namespace lq

using namespace lq;

extern "C" {

int lq_profile_enable(int on) {
    std::lock_guard<std::mutex> lk(g_mu);
    resolve_locked();
    g_on = on != 0;
    ++g_gen;
    for (int c = 0; c < kProfClasses; ++c) {
        g_ms[c] = 0.0;
        g_count[c] = 0;
    }
    return LQ_OK;
}

int lq_profile_read(int kernel_class, double *total_ms, long long *launches) {
    if (kernel_class < 0 || kernel_class >= kProfClasses)
        return set_error(LQ_ERR_INVALID_ARG, "unknown kernel class %d", kernel_class);
    std::lock_guard<std::mutex> lk(g_mu);
    resolve_locked();
    if (total_ms) *total_ms = g_ms[kernel_class];
    if (launches) *launches = g_count[kernel_class];
    return LQ_OK;
}

}  // extern "C"
