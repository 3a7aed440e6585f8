// Per-launch CUDA-event timing of the library's kernels.
//
// Off by default.  While enabled (iarray_b200_profile_kernels), every launch site that
// holds a KernelTimer records a start and a stop event on the launch's stream; the
// report (iarray_b200_kernel_profile) resolves the pending events and prints, per kernel
// name, the number of launches and their summed device time.  Launch sites pay one
// atomic load when profiling is off.
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/iarray_b200.h"
#include "common.cuh"

namespace iab {

namespace {
struct Pending {
    const char *name;
    cudaEvent_t e0, e1;
};
struct Totals {
    int64_t launches = 0;
    double ms = 0.0;
};
std::atomic<bool> g_on{false};
std::mutex g_mu;
std::vector<Pending> g_pending;
std::map<std::string, Totals> g_totals;

// Folds finished events into the totals; waits for the ones still in flight.
void resolve_locked()
{
    for (const Pending &p : g_pending) {
        float ms = 0.f;
        if (cudaEventSynchronize(p.e1) == cudaSuccess && cudaEventElapsedTime(&ms, p.e0, p.e1) == cudaSuccess) {
            Totals &t = g_totals[p.name];
            t.launches += 1;
            t.ms += ms;
        } else {
            cudaGetLastError();
        }
        cudaEventDestroy(p.e0);
        cudaEventDestroy(p.e1);
    }
    g_pending.clear();
}
}  // namespace

KernelTimer::KernelTimer(const char *name, cudaStream_t st) : name_(name), st_(st)
{
    if (!g_on.load(std::memory_order_relaxed)) return;
    if (cudaEventCreate(&e0_) != cudaSuccess) { cudaGetLastError(); e0_ = nullptr; return; }
    cudaEventRecord(e0_, st_);
}

KernelTimer::~KernelTimer()
{
    if (!e0_) return;
    cudaEvent_t e1 = nullptr;
    if (cudaEventCreate(&e1) != cudaSuccess) { cudaGetLastError(); cudaEventDestroy(e0_); return; }
    cudaEventRecord(e1, st_);
    std::lock_guard<std::mutex> lock(g_mu);
    g_pending.push_back({name_, e0_, e1});
}

bool kprof_enable(bool on)
{
    return g_on.exchange(on);
}

}  // namespace iab

INA_API(ina_rc_t) iarray_b200_profile_kernels(int on)
{
    std::lock_guard<std::mutex> lock(iab::g_mu);
    iab::resolve_locked();
    if (on) iab::g_totals.clear();
    iab::g_on.store(on != 0);
    return INA_SUCCESS;
}

INA_API(ina_rc_t) iarray_b200_kernel_profile(char *buf, int64_t cap, int64_t *len)
{
    if (!len || cap < 0) return INA_RC_ERROR_BIT | (ina_rc_t)INA_ERR_INVALID_ARGUMENT;
    std::string out;
    {
        std::lock_guard<std::mutex> lock(iab::g_mu);
        iab::resolve_locked();
        char line[256];
        for (const auto &kv : iab::g_totals) {
            snprintf(line, sizeof line, "%s %lld %.6f\n", kv.first.c_str(), (long long)kv.second.launches, kv.second.ms);
            out += line;
        }
    }
    *len = (int64_t)out.size();
    if (!buf) return INA_SUCCESS;
    if (cap < (int64_t)out.size() + 1) return INA_RC_ERROR_BIT | (ina_rc_t)IARRAY_ERR_TOO_SMALL_BUFFER;
    memcpy(buf, out.c_str(), out.size() + 1);
    return INA_SUCCESS;
}
