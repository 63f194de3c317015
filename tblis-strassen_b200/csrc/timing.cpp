#include "timing.hpp"

#include <atomic>
#include <mutex>
#include <vector>

#include "tblis_stra_b200.h"

namespace tsb {
namespace {

struct Record { int kind; cudaEvent_t start, stop; };

std::atomic<bool> g_on{false};
std::mutex g_mu;
std::vector<Record> g_records;
thread_local cudaEvent_t t_open[KK_COUNT] = {};

}  // namespace

bool timing_enabled() { return g_on.load(std::memory_order_relaxed); }

void timing_begin(int kind, cudaStream_t stream)
{
    if (!timing_enabled()) return;
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) { cudaGetLastError(); return; }
    cudaEventRecord(e, stream);
    t_open[kind] = e;
}

void timing_end(int kind, cudaStream_t stream)
{
    if (!timing_enabled() || !t_open[kind]) return;
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) { cudaGetLastError(); return; }
    cudaEventRecord(e, stream);
    std::lock_guard<std::mutex> lk(g_mu);
    g_records.push_back({kind, t_open[kind], e});
    t_open[kind] = nullptr;
}

}  // namespace tsb

extern "C" {

int tblis_stra_set_kernel_timing(int on)
{
    std::lock_guard<std::mutex> lk(tsb::g_mu);
    for (auto& r : tsb::g_records) { cudaEventDestroy(r.start); cudaEventDestroy(r.stop); }
    tsb::g_records.clear();
    tsb::g_on.store(on != 0);
    return TBLIS_STRA_SUCCESS;
}

int tblis_stra_kernel_timing(int kind, unsigned long long* launches, double* total_ms)
{
    if (kind < 0 || kind >= tsb::KK_COUNT) return TBLIS_STRA_ERR_ARG;
    std::lock_guard<std::mutex> lk(tsb::g_mu);
    unsigned long long n = 0;
    double ms = 0.0;
    for (auto& r : tsb::g_records)
    {
        if (r.kind != kind) continue;
        if (cudaEventSynchronize(r.stop) != cudaSuccess) return TBLIS_STRA_ERR_CUDA;
        float x = 0.f;
        if (cudaEventElapsedTime(&x, r.start, r.stop) != cudaSuccess) return TBLIS_STRA_ERR_CUDA;
        ms += x;
        n++;
    }
    if (launches) *launches = n;
    if (total_ms) *total_ms = ms;
    return TBLIS_STRA_SUCCESS;
}

}  // extern "C"
