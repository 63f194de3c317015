// Batched contractions: many independent contractions (uneven index bundles
// and extents) planned once and executed as grouped persistent launches
// captured in one CUDA graph.  The reference has no batched Strassen API (its
// batched tensors, src/tensor/, are upstream TBLIS TTM code); this is the
// grouped form of the same contraction, with the Strassen level of each
// problem chosen by a measured-time autotuner.
//
//   create:  plan every problem (bundle analysis, scatter vectors), upload all
//            tables into one device buffer, pick each problem's level
//            (given, or autotuned), group FP64 problems by kernel
//            configuration, and capture into a CUDA graph: one grouped launch
//            of the fused kernel per configuration (every product of every
//            problem of that group in one persistent grid), the set/scale
//            launches of alpha == 0 problems, and, for FP32 problems, each
//            problem's split-BF16 sequence on preallocated workspace;
//   execute: cudaGraphLaunch on the caller's stream.
//
// Autotuner: for a problem with level -1, each level in {0, 1, 2} is timed
// with CUDA events in a grouped launch holding enough copies of the problem to
// fill the GPU (its cost inside a full grouped launch, not its latency alone),
// writing into scratch memory; the fastest level wins.  Results are cached per
// process by a size signature (type, m, n, k rounded to 1/4 octave, batch,
// loader mappings).
#include "tblis_stra_b200.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <vector>

#include "kernels.cuh"
#include "plan.hpp"

namespace tsb {

// capi.cpp
int run_fp32_enqueue(int level, const GemmView& g, const int64_t* const tables[9], const float* A,
                     const float* B, float* C, cudaStream_t st, int sms, void* ws, size_t ws_bytes,
                     int terms, int* err);
size_t fp32_workspace_bytes(int level, const GemmView& g, int terms);
extern std::atomic<unsigned long long> g_launches;

namespace {

struct Prob
{
    GemmView g;
    const void* A; const void* B; void* C;
    size_t tab_off[9];        // element offsets of the 9 scatter vectors in the table buffer
    int level;
    int family_terms, H;
};

int terms_of_level(int level) { return level == 0 ? 1 : level == 1 ? 2 : 4; }

// Default fused-kernel configuration per level in grouped launches (the
// 8-warp tiles keep the per-problem descriptor in registers without spills).
int group_config(int level) { return level == 2 ? 1 : 2; }

bool device_ptr(const void* p)
{
    cudaPointerAttributes attr;
    if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) { cudaGetLastError(); return false; }
    return attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged;
}

DmmaArgs make_args(const Prob& pr, const int64_t* tab, int level, double* C_override, int64_t c_shift)
{
    const GemmView& g = pr.g;
    const ProductTable& t = product_table(level);
    DmmaArgs a;
    std::memset(&a, 0, sizeof a);
    a.A = static_cast<const double*>(pr.A);
    a.B = static_cast<const double*>(pr.B);
    a.C = C_override ? C_override - c_shift : static_cast<double*>(pr.C);
    a.rsA = tab + pr.tab_off[0]; a.rsC = tab + pr.tab_off[1]; a.csB = tab + pr.tab_off[2];
    a.csC = tab + pr.tab_off[3]; a.ksA = tab + pr.tab_off[4]; a.ksB = tab + pr.tab_off[5];
    a.bA = tab + pr.tab_off[6]; a.bB = tab + pr.tab_off[7]; a.bC = tab + pr.tab_off[8];
    a.m = g.m; a.n = g.n; a.k = g.k; a.mC = g.m; a.nC = g.n; a.batch = g.batch;
    const int H = t.H;
    a.ms = (g.m + H - 1) / H; a.ns = (g.n + H - 1) / H; a.ks = (g.k + H - 1) / H;
    a.alpha = g.alpha; a.beta = g.beta;
    a.a_kfast = (g.unit_ksA != 0 && (g.unit_rsA == 0 || g.unit_ksA < g.unit_rsA)) ? 1 : 0;
    a.b_kfast = (g.unit_ksB != 0 && (g.unit_csB == 0 || g.unit_ksB < g.unit_csB)) ? 1 : 0;
    a.nprod = (int)t.prod.size();
    a.H = a.Hc = H;
    for (int p = 0; p < a.nprod; p++)
    {
        const Product& q = t.prod[p];
        DevProduct& d = a.prod[p];
        d.na = q.na; d.nb = q.nb; d.nc = q.nc;
        for (int i = 0; i < 4; i++)
        {
            d.a_r[i] = q.a[i].r; d.a_c[i] = q.a[i].c; d.a_s[i] = q.a[i].sign;
            d.b_r[i] = q.b[i].r; d.b_c[i] = q.b[i].c; d.b_s[i] = q.b[i].sign;
            d.c_r[i] = q.c[i].r; d.c_c[i] = q.c[i].c; d.c_s[i] = q.c[i].sign;
            d.c_first[i] = q.c_first[i];
        }
    }
    int bm = 128, bn = 128;
    dmma_tile_shape(terms_of_level(level), H, H, group_config(level), &bm, &bn);
    a.tiles_m = (int)((a.ms + bm - 1) / bm);
    a.tiles_n = (int)((a.ns + bn - 1) / bn);
    a.work = a.batch * (int64_t)a.tiles_m * a.tiles_n;
    return a;
}

// Upload a group of descriptors and launch it (one grouped persistent grid).
struct GroupBuffers
{
    void* mem = nullptr;
    GroupBuffers() = default;
    GroupBuffers(const GroupBuffers&) = delete;
    GroupBuffers& operator=(const GroupBuffers&) = delete;
    GroupBuffers(GroupBuffers&& o) noexcept : mem(o.mem) { o.mem = nullptr; }
    ~GroupBuffers() { if (mem) cudaFree(mem); }
};

// Upload a group's descriptors and work prefix (before any capture).
int upload_group(const std::vector<DmmaArgs>& args, GroupBuffers& buf, DmmaGroupArgs& g)
{
    std::memset(&g, 0, sizeof g);
    if (args.empty()) return TBLIS_STRA_SUCCESS;
    std::vector<int64_t> prefix(args.size() + 1, 0);
    for (size_t i = 0; i < args.size(); i++) prefix[i + 1] = prefix[i] + args[i].work;
    const size_t bytes_args = args.size() * sizeof(DmmaArgs);
    const size_t bytes = bytes_args + prefix.size() * sizeof(int64_t);
    if (cudaMalloc(&buf.mem, bytes) != cudaSuccess) { cudaGetLastError(); buf.mem = nullptr; return TBLIS_STRA_ERR_ALLOC; }
    std::vector<unsigned char> host(bytes);
    std::memcpy(host.data(), args.data(), bytes_args);
    std::memcpy(host.data() + bytes_args, prefix.data(), prefix.size() * sizeof(int64_t));
    if (cudaMemcpy(buf.mem, host.data(), bytes, cudaMemcpyHostToDevice) != cudaSuccess) return TBLIS_STRA_ERR_CUDA;
    g.probs = static_cast<const DmmaArgs*>(buf.mem);
    g.prefix = reinterpret_cast<const int64_t*>(static_cast<unsigned char*>(buf.mem) + bytes_args);
    g.nprob = (int)args.size();
    g.total = prefix.back();
    return TBLIS_STRA_SUCCESS;
}

// One grouped persistent grid over an uploaded group (capturable).
int launch_group(const DmmaGroupArgs& g, int level, cudaStream_t st, int sms)
{
    if (g.nprob == 0 || g.total == 0) return TBLIS_STRA_SUCCESS;
    const int H = product_table(level).H;
    if (launch_dmma_grouped(g, terms_of_level(level), H, H, group_config(level), st, sms) != cudaSuccess)
        return TBLIS_STRA_ERR_CUDA;
    return TBLIS_STRA_SUCCESS;
}

std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int, int64_t, int, int>, int> g_tune_cache;

std::tuple<int, int, int, int, int64_t, int, int> tune_key(const GemmView& g)
{
    auto q = [](int64_t x) { return x <= 0 ? -1 : (int)std::lround(4.0 * std::log2((double)x)); };
    const int ak = (g.unit_ksA != 0 && (g.unit_rsA == 0 || g.unit_ksA < g.unit_rsA)) ? 1 : 0;
    const int bk = (g.unit_ksB != 0 && (g.unit_csB == 0 || g.unit_ksB < g.unit_csB)) ? 1 : 0;
    return std::make_tuple(g.type, q(g.m), q(g.n), q(g.k), g.batch, ak, bk);
}

}  // namespace

struct BatchPlan
{
    int device = 0;
    int count = 0;
    void* tables = nullptr;                 // all scatter vectors
    void* fp32_ws = nullptr;                // split-BF16 workspace (largest problem)
    int* err = nullptr;
    GroupBuffers groups[3];
    std::vector<int> levels;
    cudaStream_t cap = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    unsigned long long nodes = 0;
    ~BatchPlan()
    {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (cap) cudaStreamDestroy(cap);
        if (tables) cudaFree(tables);
        if (fp32_ws) cudaFree(fp32_ws);
        if (err) cudaFree(err);
    }
};

namespace {

// Time one level of one FP64 problem inside a grouped launch of `copies`
// replicas (all writing to `scratch`); milliseconds per replica.
double time_level(const Prob& pr, const int64_t* tab, int level, double* scratch, int sms)
{
    DmmaArgs one = make_args(pr, tab, level, scratch, pr.g.lo[2]);
    if (one.work <= 0) return 0.0;
    const int64_t fill = (int64_t)sms * 2;
    const int copies = (int)std::max<int64_t>(1, std::min<int64_t>(64, (fill + one.work - 1) / one.work));
    std::vector<DmmaArgs> args(copies, one);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double best = 1e30;
    GroupBuffers gb;
    DmmaGroupArgs g;
    if (upload_group(args, gb, g)) return 1e30;
    for (int rep = 0; rep < 3; rep++)
    {
        cudaEventRecord(e0, nullptr);
        if (launch_group(g, level, nullptr, sms)) { best = 1e30; break; }
        cudaEventRecord(e1, nullptr);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0) best = std::min(best, (double)ms / copies);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return best;
}

int choose_level(const Prob& pr, const int64_t* tab, double* scratch, int sms)
{
    if (pr.g.type != TYPE_DOUBLE) return 0;   // FP32 problems run level 0 unless given
    const auto key = tune_key(pr.g);
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) return it->second;
    }
    int best = 0;
    double best_t = 1e30;
    const int64_t mn = std::min(pr.g.m, std::min(pr.g.n, pr.g.k));
    for (int level = 0; level <= 2; level++)
    {
        if (level > 0 && mn < (int64_t)128 << level) break;   // blocks below one tile
        const double t = time_level(pr, tab, level, scratch, sms);
        if (t < best_t) { best_t = t; best = level; }
    }
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache[key] = best;
    return best;
}

}  // namespace

int batch_create(int count, const tblis_stra_problem* problems, BatchPlan** out)
{
    *out = nullptr;
    if (count < 0 || (count > 0 && !problems)) return TBLIS_STRA_ERR_ARG;
    auto plan = new BatchPlan();
    std::unique_ptr<BatchPlan> guard(plan);
    if (cudaGetDevice(&plan->device) != cudaSuccess) { cudaGetLastError(); return TBLIS_STRA_ERR_NO_DEVICE; }
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, plan->device);
    plan->count = count;

    // 1. plan every problem
    std::vector<Prob> probs(count);
    size_t total_tab = 0;
    int64_t max_c_span = 1;
    for (int i = 0; i < count; i++)
    {
        const tblis_stra_problem& q = problems[i];
        if (q.level < -1 || q.level > 2) return TBLIS_STRA_ERR_ARG;
        int s = plan_contraction(q.A, q.idx_A, q.B, q.idx_B, q.C, q.idx_C, probs[i].g, true);
        if (s) return s;
        Prob& pr = probs[i];
        pr.A = q.A->data; pr.B = q.B->data; pr.C = q.C->data;
        const size_t es = pr.g.type == TYPE_FLOAT ? 4 : 8;
        const tblis_tensor* T[3] = {q.A, q.B, q.C};
        for (int t = 0; t < 3; t++)
        {
            if (pr.g.hi[t] < pr.g.lo[t]) continue;
            if (!T[t]->data) return TBLIS_STRA_ERR_NULL;
            if (reinterpret_cast<uintptr_t>(T[t]->data) % es) return TBLIS_STRA_ERR_ARG;
            if (!device_ptr(T[t]->data)) return TBLIS_STRA_ERR_ARG;   // batches take device memory only
        }
        max_c_span = std::max<int64_t>(max_c_span, pr.g.hi[2] - pr.g.lo[2] + 1);
        const std::vector<int64_t>* v[9] = {&pr.g.rsA, &pr.g.rsC, &pr.g.csB, &pr.g.csC, &pr.g.ksA,
                                            &pr.g.ksB, &pr.g.bA, &pr.g.bB, &pr.g.bC};
        for (int j = 0; j < 9; j++) { pr.tab_off[j] = total_tab; total_tab += std::max<size_t>(v[j]->size(), 1); }
        pr.level = q.level;
    }

    // 2. one device buffer for all scatter vectors
    std::vector<int64_t> host(std::max<size_t>(total_tab, 1), 0);
    for (auto& pr : probs)
    {
        const std::vector<int64_t>* v[9] = {&pr.g.rsA, &pr.g.rsC, &pr.g.csB, &pr.g.csC, &pr.g.ksA,
                                            &pr.g.ksB, &pr.g.bA, &pr.g.bB, &pr.g.bC};
        for (int j = 0; j < 9; j++) std::copy(v[j]->begin(), v[j]->end(), host.begin() + (ptrdiff_t)pr.tab_off[j]);
    }
    if (cudaMalloc(&plan->tables, host.size() * 8) != cudaSuccess) { cudaGetLastError(); plan->tables = nullptr; return TBLIS_STRA_ERR_ALLOC; }
    if (cudaMemcpy(plan->tables, host.data(), host.size() * 8, cudaMemcpyHostToDevice) != cudaSuccess) return TBLIS_STRA_ERR_CUDA;
    const int64_t* tab = static_cast<const int64_t*>(plan->tables);

    // 3. levels (autotuned where -1)
    bool need_tune = false;
    for (auto& pr : probs) need_tune |= (pr.level < 0);
    double* scratch = nullptr;
    if (need_tune)
    {
        if (cudaMalloc(&scratch, (size_t)max_c_span * sizeof(double)) != cudaSuccess) { cudaGetLastError(); return TBLIS_STRA_ERR_ALLOC; }
        cudaMemset(scratch, 0, (size_t)max_c_span * sizeof(double));
    }
    plan->levels.resize(count);
    for (int i = 0; i < count; i++)
    {
        Prob& pr = probs[i];
        const bool trivial = pr.g.m == 0 || pr.g.n == 0 || pr.g.batch == 0 || pr.g.alpha == 0.0 || pr.g.k == 0;
        if (pr.level < 0) pr.level = trivial ? 0 : choose_level(pr, tab, scratch, sms);
        plan->levels[i] = pr.level;
    }
    if (scratch) cudaFree(scratch);
    cudaDeviceSynchronize();
    if (cudaGetLastError() != cudaSuccess) return TBLIS_STRA_ERR_CUDA;

    // FP32 workspace: the largest problem's split-BF16 buffers (problems run in turn).
    size_t ws = 0;
    for (auto& pr : probs)
        if (pr.g.type == TYPE_FLOAT) ws = std::max(ws, fp32_workspace_bytes(pr.level, pr.g, 6));
    if (ws)
    {
        if (cudaMalloc(&plan->fp32_ws, ws) != cudaSuccess) { cudaGetLastError(); plan->fp32_ws = nullptr; return TBLIS_STRA_ERR_ALLOC; }
    }
    if (cudaMalloc(&plan->err, sizeof(int)) != cudaSuccess) { cudaGetLastError(); plan->err = nullptr; return TBLIS_STRA_ERR_ALLOC; }
    cudaMemset(plan->err, 0, sizeof(int));

    // 4. descriptors per FP64 group, uploaded before capture
    DmmaGroupArgs gargs[3];
    for (int lv = 0; lv < 3; lv++)
    {
        std::vector<DmmaArgs> grp;
        for (auto& pr : probs)
        {
            if (pr.g.type != TYPE_DOUBLE || pr.level != lv) continue;
            if (pr.g.m == 0 || pr.g.n == 0 || pr.g.batch == 0 || pr.g.alpha == 0.0 || pr.g.k == 0) continue;
            grp.push_back(make_args(pr, tab, lv, nullptr, 0));
        }
        const int s = upload_group(grp, plan->groups[lv], gargs[lv]);
        if (s) return s;
    }

    // 5. capture the graph: alpha == 0 problems, FP32 problems (each in turn
    // on the shared workspace), then one grouped launch per FP64 level.
    if (cudaStreamCreateWithFlags(&plan->cap, cudaStreamNonBlocking) != cudaSuccess) return TBLIS_STRA_ERR_CUDA;
    const unsigned long long launches0 = g_launches.load();
    if (cudaStreamBeginCapture(plan->cap, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return TBLIS_STRA_ERR_CUDA;
    int status = TBLIS_STRA_SUCCESS;
    for (auto& pr : probs)
    {
        if (status) break;
        if (pr.g.m == 0 || pr.g.n == 0 || pr.g.batch == 0) continue;
        if (pr.g.alpha == 0.0 || pr.g.k == 0)
        {
            if (pr.g.type == TYPE_DOUBLE)
            {
                ScaleArgs sa{static_cast<double*>(pr.C), tab + pr.tab_off[1], tab + pr.tab_off[3], tab + pr.tab_off[8],
                             pr.g.m, pr.g.n, pr.g.batch, pr.g.beta};
                if (launch_scale(sa, plan->cap) != cudaSuccess) status = TBLIS_STRA_ERR_CUDA;
            }
            else
            {
                ScaleF32Args sa{static_cast<float*>(pr.C), tab + pr.tab_off[1], tab + pr.tab_off[3], tab + pr.tab_off[8],
                                pr.g.m, pr.g.n, pr.g.batch, (float)pr.g.beta};
                if (launch_scale_f32(sa, plan->cap) != cudaSuccess) status = TBLIS_STRA_ERR_CUDA;
            }
            continue;
        }
        if (pr.g.type == TYPE_FLOAT)
        {
            const int64_t* t9[9];
            for (int j = 0; j < 9; j++) t9[j] = tab + pr.tab_off[j];
            status = run_fp32_enqueue(pr.level, pr.g, t9, static_cast<const float*>(pr.A),
                                      static_cast<const float*>(pr.B), static_cast<float*>(pr.C),
                                      plan->cap, sms, plan->fp32_ws, ws, 6, plan->err);
        }
    }
    for (int lv = 0; lv < 3 && !status; lv++) status = launch_group(gargs[lv], lv, plan->cap, sms);
    const cudaError_t ec = cudaStreamEndCapture(plan->cap, &plan->graph);
    if (status) return status;
    if (ec != cudaSuccess) { cudaGetLastError(); return TBLIS_STRA_ERR_CUDA; }
    if (cudaGraphInstantiate(&plan->exec, plan->graph, 0) != cudaSuccess) { cudaGetLastError(); return TBLIS_STRA_ERR_CUDA; }
    plan->nodes = g_launches.load() - launches0;
    g_launches -= plan->nodes;   // counted at every execute instead
    *out = guard.release();
    return TBLIS_STRA_SUCCESS;
}

void batch_destroy(BatchPlan* plan) { delete plan; }

int batch_levels(const BatchPlan* plan, int* levels)
{
    if (!plan || !levels) return TBLIS_STRA_ERR_NULL;
    std::copy(plan->levels.begin(), plan->levels.end(), levels);
    return TBLIS_STRA_SUCCESS;
}

int batch_execute(BatchPlan* plan, cudaStream_t st)
{
    if (!plan) return TBLIS_STRA_ERR_NULL;
    if (!plan->exec) return TBLIS_STRA_SUCCESS;
    if (cudaGraphLaunch(plan->exec, st) != cudaSuccess) { cudaGetLastError(); return TBLIS_STRA_ERR_CUDA; }
    g_launches += plan->nodes;
    return TBLIS_STRA_SUCCESS;
}

}  // namespace tsb

extern "C" {

int tblis_stra_batch_create(int count, const tblis_stra_problem* problems, tblis_stra_batch* batch)
{
    if (!batch) return TBLIS_STRA_ERR_NULL;
    tsb::BatchPlan* p = nullptr;
    const int s = tsb::batch_create(count, problems, &p);
    *batch = reinterpret_cast<tblis_stra_batch>(p);
    return s;
}

int tblis_stra_batch_execute(tblis_stra_batch batch, void* stream)
{
    return tsb::batch_execute(reinterpret_cast<tsb::BatchPlan*>(batch), static_cast<cudaStream_t>(stream));
}

int tblis_stra_batch_levels(tblis_stra_batch batch, int* levels)
{
    return tsb::batch_levels(reinterpret_cast<const tsb::BatchPlan*>(batch), levels);
}

void tblis_stra_batch_destroy(tblis_stra_batch batch)
{
    tsb::batch_destroy(reinterpret_cast<tsb::BatchPlan*>(batch));
}

}  // extern "C"
