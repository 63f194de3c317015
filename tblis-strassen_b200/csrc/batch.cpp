// Batched contractions: many independent contractions (uneven index bundles
// and extents) planned once and captured in one CUDA graph.  The reference has
// no batched Strassen API (its batched tensors, src/tensor/, are upstream
// TBLIS TTM code); this is the grouped form of the same contraction, with the
// Strassen level, variant and tile shape of each problem chosen by a
// measured-time autotuner.
//
//   create:  plan every problem (bundle analysis, scatter vectors), upload all
//            tables into one device buffer, choose each problem's schedule
//            (level, variant, tile shape), then capture into a CUDA graph:
//              main stream   the C = beta*C launches of trivial problems; one
//                            grouped fused launch per (level, tile shape); the
//                            problem-by-problem packed schedules; one grouped
//                            packed GEMM per chunk of packed L = 0 problems;
//              pack stream   the pack launches of every chunk, two chunk
//                            workspaces in turn (chunk i's packing waits for
//                            chunk i-2's GEMM), so packing overlaps the GEMMs;
//              two branches  FP32 problems (split-BF16), balanced by flops,
//                            each branch with its own workspace;
//   execute: cudaGraphLaunch on the caller's stream.
//
// Autotuner: every candidate schedule of a problem is timed with CUDA events
// on the problem's own operands, writing to scratch memory.  Grouped
// schedules are timed in a grouped launch holding enough copies of the
// problem to fill the GPU twice (their cost inside a full grouped launch,
// not their latency alone); problem-by-problem schedules run alone.  The
// fastest candidate wins (a later one by a 2 % margin); the choice is
// cached per process by a size signature (type, m, n, k rounded to the
// nearest power of two, batch, requested level, allowed schedules), so
// problems of one size class share one set of timings.
#include "tblis_stra_b200.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <mutex>
#include <tuple>
#include <vector>

#include "kernels.cuh"
#include "memkind.hpp"
#include "plan.hpp"
#include "schedule.hpp"

namespace tsb {

extern std::atomic<unsigned long long> g_launches;

namespace {

enum Variant
{
    V_FUSED = TBLIS_STRA_BATCH_FUSED,
    V_FUSED_SMALL = TBLIS_STRA_BATCH_FUSED_SMALL,
    V_PGROUP = TBLIS_STRA_BATCH_PACKED_GROUPED,
    V_PACKED = TBLIS_STRA_BATCH_PACKED,
    V_SPLIT = TBLIS_STRA_BATCH_SPLIT,
    V_SCALE = TBLIS_STRA_BATCH_SCALE,
    V_SGROUP = TBLIS_STRA_BATCH_SPLIT_GROUPED
};

#define TSB_CU(x) do { const cudaError_t e_ = (x); \
    if (e_ != cudaSuccess) { note_cuda_error(#x, e_, __FILE__, __LINE__); return TBLIS_STRA_ERR_CUDA; } } while (0)

constexpr int FP32_TERMS = 6;

// Schedules the tuner may pick (bit v = variant v), per thread.
constexpr unsigned ALL_VARIANTS = (1u << V_FUSED) | (1u << V_FUSED_SMALL) | (1u << V_PGROUP) | (1u << V_PACKED) |
                                  (1u << V_SPLIT) | (1u << V_SGROUP);
thread_local unsigned t_variant_mask = ALL_VARIANTS;
// Packed operands per chunk of grouped packed problems (two chunk workspaces
// in turn); TBLIS_STRA_BATCH_CHUNK_BYTES overrides it at create time.
size_t chunk_bytes()
{
    const char* s = std::getenv("TBLIS_STRA_BATCH_CHUNK_BYTES");
    const long long v = s ? std::atoll(s) : 0;
    return v > 0 ? (size_t)v : (size_t)2 << 30;
}

struct Prob
{
    GemmView g;
    const void* A; const void* B; void* C;
    size_t tab_off[9];        // element offsets of the 9 scatter vectors in the table buffer
    size_t mtab_off[3] = {0, 0, 0};   // M_p tables of the product-parallel form at L = 1, 2
    bool mcol = false;        // M_p layout (column-major)
    int level_req;            // -1 or 0..2
    int level = 0, variant = V_SCALE;
    bool empty = false;       // nothing to write (m, n or batch zero)
    bool scale = false;       // alpha == 0 or k == 0: C = beta*C
    void tables(const int64_t* tab, const int64_t* out[9]) const
    {
        for (int j = 0; j < 9; j++) out[j] = tab + tab_off[j];
    }
    double flops() const { return 2.0 * (double)g.m * (double)g.n * (double)g.k * (double)g.batch; }
};

int terms_of_level(int level) { return level == 0 ? 1 : level == 1 ? 2 : 4; }

// Fused-kernel configuration of a grouped variant at a level (-1: none).
// The 8-warp 128 x 128 and the 64 x 64 tiles keep the per-problem descriptor
// in registers in grouped launches; L = 1 has no 64 x 64 instance.
int fused_config(int variant, int level)
{
    if (variant == V_FUSED) return 2;
    if (variant == V_FUSED_SMALL) return level == 1 ? -1 : 1;
    return -1;
}

DmmaArgs make_args(const Prob& pr, const int64_t* tab, int level, int config, double* C_override,
                   int64_t c_shift)
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
    dmma_tile_shape(terms_of_level(level), H, H, config, &bm, &bn);
    a.tiles_m = (int)((a.ms + bm - 1) / bm);
    a.tiles_n = (int)((a.ns + bn - 1) / bn);
    a.work = a.batch * (int64_t)a.tiles_m * a.tiles_n;
    return a;
}

// Owned device allocation (cudaMalloc; freed with its owner).
struct DevBuf
{
    void* p = nullptr;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p(o.p) { o.p = nullptr; }
    ~DevBuf() { if (p) cudaFree(p); }
    int alloc(size_t bytes)
    {
        if (std::max<size_t>(bytes, 16) > alloc_limit_bytes()) return TBLIS_STRA_ERR_ALLOC;
        if (cudaMalloc(&p, std::max<size_t>(bytes, 16)) != cudaSuccess) { cudaGetLastError(); p = nullptr; return TBLIS_STRA_ERR_ALLOC; }
        return TBLIS_STRA_SUCCESS;
    }
};

// Descriptors + work prefix of one grouped launch, written into `mem`
// (capacity `cap` bytes) and complete on return.
template <class Desc>
size_t descs_bytes(size_t n) { return (n * sizeof(Desc) + 15) / 16 * 16 + (n + 1) * sizeof(int64_t); }

template <class Desc>
int fill_descs(const std::vector<Desc>& d, const std::vector<int64_t>& work, void* mem, size_t cap,
               const Desc*& probs, const int64_t*& prefix, int64_t& total)
{
    std::vector<int64_t> pre(d.size() + 1, 0);
    for (size_t i = 0; i < d.size(); i++) pre[i + 1] = pre[i] + work[i];
    const size_t bytes_d = (d.size() * sizeof(Desc) + 15) / 16 * 16;
    const size_t bytes = descs_bytes<Desc>(d.size());
    if (bytes > cap) return TBLIS_STRA_ERR_ALLOC;
    std::vector<unsigned char> host(bytes, 0);
    std::memcpy(host.data(), d.data(), d.size() * sizeof(Desc));
    std::memcpy(host.data() + bytes_d, pre.data(), pre.size() * sizeof(int64_t));
    int s = upload_complete(mem, host.data(), bytes);
    if (s) return s;
    probs = static_cast<const Desc*>(mem);
    prefix = reinterpret_cast<const int64_t*>(static_cast<unsigned char*>(mem) + bytes_d);
    total = pre.back();
    return TBLIS_STRA_SUCCESS;
}

// The same into a new allocation owned by `buf`.
template <class Desc>
int upload_descs(const std::vector<Desc>& d, const std::vector<int64_t>& work, DevBuf& buf,
                 const Desc*& probs, const int64_t*& prefix, int64_t& total)
{
    const size_t bytes = descs_bytes<Desc>(d.size());
    int s = buf.alloc(bytes);
    if (s) return s;
    return fill_descs(d, work, buf.p, bytes, probs, prefix, total);
}

// Grouped-launch arguments of fused / packed descriptors: into `buf` (new
// allocation) or, with buf == nullptr, into the existing `mem` of `cap` bytes.
int upload_fused(const std::vector<DmmaArgs>& args, DevBuf* buf, DmmaGroupArgs& g, void* mem = nullptr,
                 size_t cap = 0)
{
    std::memset(&g, 0, sizeof g);
    if (args.empty()) return TBLIS_STRA_SUCCESS;
    std::vector<int64_t> work(args.size());
    for (size_t i = 0; i < args.size(); i++) work[i] = args[i].work;
    g.nprob = (int)args.size();
    return buf ? upload_descs(args, work, *buf, g.probs, g.prefix, g.total)
               : fill_descs(args, work, mem, cap, g.probs, g.prefix, g.total);
}

int upload_packed(const std::vector<PackedGemmArgs>& args, DevBuf* buf, PackedGroupArgs& g,
                  void* mem = nullptr, size_t cap = 0)
{
    std::memset(&g, 0, sizeof g);
    if (args.empty()) return TBLIS_STRA_SUCCESS;
    std::vector<int64_t> work(args.size());
    for (size_t i = 0; i < args.size(); i++) work[i] = args[i].batch * args[i].tiles_m * args[i].tiles_n;
    g.nprob = (int)args.size();
    return buf ? upload_descs(args, work, *buf, g.probs, g.prefix, g.total)
               : fill_descs(args, work, mem, cap, g.probs, g.prefix, g.total);
}

int upload_split(const std::vector<SplitGemmArgs>& args, DevBuf* buf, SplitGroupArgs& g,
                 void* mem = nullptr, size_t cap = 0)
{
    std::memset(&g, 0, sizeof g);
    if (args.empty()) return TBLIS_STRA_SUCCESS;
    std::vector<int64_t> work(args.size());
    for (size_t i = 0; i < args.size(); i++) work[i] = args[i].batch * args[i].tiles_m * args[i].tiles_n;
    g.nprob = (int)args.size();
    return buf ? upload_descs(args, work, *buf, g.probs, g.prefix, g.total)
               : fill_descs(args, work, mem, cap, g.probs, g.prefix, g.total);
}

int launch_fused_group(const DmmaGroupArgs& g, int level, int config, cudaStream_t st, int sms)
{
    if (g.nprob == 0 || g.total == 0) return TBLIS_STRA_SUCCESS;
    const int H = product_table(level).H;
    if (launch_dmma_grouped(g, terms_of_level(level), H, H, config, st, sms) != cudaSuccess)
        return TBLIS_STRA_ERR_CUDA;
    return TBLIS_STRA_SUCCESS;
}

// ---- autotuner ----------------------------------------------------------------

struct Choice { int level, variant; };

using TuneKey = std::tuple<int, int, int, int, int64_t, int, unsigned>;
std::mutex g_tune_mu;
std::map<TuneKey, Choice> g_tune_cache;

TuneKey tune_key(const Prob& pr)
{
    const GemmView& g = pr.g;
    auto q = [](int64_t x) { return x <= 0 ? -1 : (int)std::lround(std::log2((double)x)); };
    return std::make_tuple(g.type, q(g.m), q(g.n), q(g.k), g.batch, pr.level_req, t_variant_mask);
}

// Candidate schedules of a problem.  With the level left to the tuner, a
// Strassen level is tried only when its blocks are at least 1024 long in
// every dimension (below that the extra passes over C cost more than the
// products save), and 64 x 64 tiles at L = 0 only when m or n is below 1024.
// FP64 candidates are limited to the thread's variant mask; when the mask
// leaves none, the pruning is dropped.
std::vector<Choice> candidates(const Prob& pr, bool prune = true)
{
    std::vector<Choice> c;
    const GemmView& g = pr.g;
    auto add = [&](int L, int v) {
        if ((t_variant_mask >> v) & 1u) c.push_back({L, v});
    };
    const int64_t mnk = std::min(g.m, std::min(g.n, g.k));
    for (int L = 0; L <= 2; L++)
    {
        if (pr.level_req >= 0 && L != pr.level_req) continue;
        if (prune && pr.level_req < 0 && L > 0 && mnk < ((int64_t)1024 << L)) continue;
        if (g.type == TYPE_FLOAT)
        {
            if (!pack_geom(L, g).fits) continue;
            if (L == 0) add(0, V_SGROUP);
            add(L, V_SPLIT);
            continue;
        }
        const bool packable = pack_geom(L, g).fits;
        if (L == 0)
        {
            if (packable) add(0, V_PGROUP);
            add(0, V_FUSED);
            if (!prune || std::min(g.m, g.n) < 1024 || pr.level_req == 0) add(0, V_FUSED_SMALL);
            if (packable) add(0, V_PACKED);
        }
        else
        {
            if (packable) add(L, V_PACKED);
            add(L, V_FUSED);
            if (L == 2) add(L, V_FUSED_SMALL);
        }
    }
    if (c.empty() && prune) return candidates(pr, false);
    return c;
}

// Workspace of one problem's schedule: the product-parallel form where it
// applies (packed FP64 and split FP32 at L >= 1), else the grouped sums.
size_t schedule_workspace_bytes(const Prob& pr, const Choice& x, int sms)
{
    if (x.variant == V_SPLIT || x.variant == V_SGROUP)
        return use_product_parallel(x.level, pr.g, sms, true, FP32_TERMS)
                   ? fp32_parallel_workspace_bytes(x.level, pr.g, FP32_TERMS)
                   : fp32_group_workspace_bytes(x.level, pr.g, FP32_TERMS);
    if (x.variant == V_PACKED && use_product_parallel(x.level, pr.g, sms, false, 0))
        return fp64_parallel_workspace_bytes(x.level, pr.g);
    return fp64_packed_group_workspace_bytes(x.level, pr.g);
}

constexpr int MAX_COPIES = 64;

struct Tuner
{
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    DevBuf scratch;            // scratch C (largest C span)
    DevBuf ws;                 // packed / split workspace (largest candidate)
    size_t ws_bytes = 0;
    DevBuf desc;               // grouped-launch descriptors of the copies
    size_t desc_cap = 0;
    int* err = nullptr;
    int sms = 148;
    int timings = 0;
    ~Tuner()
    {
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (st) cudaStreamDestroy(st);
    }
    int init(size_t c_bytes, size_t w_bytes, int* err_flag, int nsm)
    {
        sms = nsm;
        err = err_flag;
        if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return TBLIS_STRA_ERR_CUDA;
        if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return TBLIS_STRA_ERR_CUDA;
        int s;
        if ((s = scratch.alloc(c_bytes))) return s;
        if (cudaMemset(scratch.p, 0, c_bytes) != cudaSuccess) return TBLIS_STRA_ERR_CUDA;
        ws_bytes = w_bytes;
        desc_cap = std::max(std::max(descs_bytes<DmmaArgs>(MAX_COPIES), descs_bytes<PackedGemmArgs>(MAX_COPIES)),
                            descs_bytes<SplitGemmArgs>(MAX_COPIES));
        if ((s = desc.alloc(desc_cap))) return s;
        return ws.alloc(w_bytes);
    }
    int failures = 0;
    std::string first_failure;
    const char* what = "";
    // One timed run after one warm-up; 1e30 on failure (kept as a detail).
    template <class F> double time(F&& fn)
    {
        double best = 1e30;
        for (int rep = 0; rep < 2; rep++)
        {
            cudaEventRecord(e0, st);
            const int s = fn();
            if (s)
            {
                const cudaError_t e = cudaGetLastError();
                fail(std::string("status ") + std::to_string(s) + " " + cudaGetErrorName(e));
                cudaStreamSynchronize(st);
                return 1e30;
            }
            cudaEventRecord(e1, st);
            const cudaError_t e = cudaEventSynchronize(e1);
            if (e != cudaSuccess) { cudaGetLastError(); fail(cudaGetErrorName(e)); return 1e30; }
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (rep > 0) best = std::min(best, (double)ms);
        }
        timings++;
        return best;
    }
    void fail(const std::string& why)
    {
        if (failures++ == 0) first_failure = std::string("autotuning ") + what + ": " + why;
    }
    int copies_for(int64_t work) const
    {
        const int64_t fill = (int64_t)sms * 2;
        return (int)std::max<int64_t>(1, std::min<int64_t>(MAX_COPIES, (fill + work - 1) / work));
    }

    double time_choice(const Prob& pr, const int64_t* tab, const Choice& c)
    {
        const int64_t* tb[9];
        pr.tables(tab, tb);
        const int64_t shift = pr.g.lo[2];
        if (c.variant == V_FUSED || c.variant == V_FUSED_SMALL)
        {
            const int config = fused_config(c.variant, c.level);
            DmmaArgs one = make_args(pr, tab, c.level, config, static_cast<double*>(scratch.p), shift);
            if (one.work <= 0) return 0.0;
            const int copies = copies_for(one.work);
            std::vector<DmmaArgs> args(copies, one);
            DmmaGroupArgs g;
            if (upload_fused(args, nullptr, g, desc.p, desc_cap)) return 1e30;
            return time([&] { return launch_fused_group(g, c.level, config, st, sms); }) / copies;
        }
        if (c.variant == V_PGROUP)
        {
            const PackGeom pg = pack_geom(0, pr.g);
            double* S = static_cast<double*>(ws.p);
            double* T = S + pg.s_elems;
            const Product& p0 = product_table(0).prod[0];
            const double pack_ms = time([&] {
                return enqueue_pack_product(p0, pr.g, pg, tb, static_cast<const double*>(pr.A),
                                            static_cast<const double*>(pr.B), S, T, st);
            });
            PackedGemmArgs one = packed_product_args(0, p0, pr.g, pg, tb, S, T,
                                                     static_cast<double*>(scratch.p) - shift, err);
            const int copies = copies_for(one.batch * one.tiles_m * one.tiles_n);
            std::vector<PackedGemmArgs> args(copies, one);
            PackedGroupArgs g;
            if (upload_packed(args, nullptr, g, desc.p, desc_cap)) return 1e30;
            g.err = err;
            g.wait_limit = wait_limit_cycles();
            const double gemm_ms = time([&] {
                return launch_packed_gemm_grouped(g, st, sms) == cudaSuccess ? 0 : (int)TBLIS_STRA_ERR_CUDA;
            });
            return pack_ms + gemm_ms / copies;
        }
        if (c.variant == V_PACKED && use_product_parallel(c.level, pr.g, sms, false, 0))
            return time([&] {
                return run_fp64_parallel_enqueue(c.level, pr.g, tb, static_cast<const double*>(pr.A),
                                                 static_cast<const double*>(pr.B),
                                                 static_cast<double*>(scratch.p) - shift, st, sms, ws.p, ws_bytes,
                                                 tab + pr.mtab_off[c.level], pr.mcol, err);
            });
        if (c.variant == V_PACKED)
            return time([&] {
                return run_fp64_packed_enqueue(c.level, pr.g, tb, static_cast<const double*>(pr.A),
                                               static_cast<const double*>(pr.B),
                                               static_cast<double*>(scratch.p) - shift, st, sms, ws.p, ws_bytes,
                                               err);
            });
        if (c.variant == V_SGROUP)
        {
            SplitGemmArgs one{};
            float* Cs = static_cast<float*>(scratch.p) - shift;
            const double prep_ms = time([&] {
                return run_fp32_enqueue(0, pr.g, tb, static_cast<const float*>(pr.A), static_cast<const float*>(pr.B),
                                        Cs, st, sms, ws.p, ws_bytes, FP32_TERMS, err, &one, true);
            });
            std::vector<SplitGemmArgs> args(copies_for(one.batch * one.tiles_m * one.tiles_n), one);
            SplitGroupArgs g;
            if (upload_split(args, nullptr, g, desc.p, desc_cap)) return 1e30;
            g.err = err;
            g.wait_limit = wait_limit_cycles();
            const double gemm_ms = time([&] {
                return launch_split_gemm_grouped(g, one.planes, st, sms) == cudaSuccess ? 0 : (int)TBLIS_STRA_ERR_CUDA;
            });
            return prep_ms + gemm_ms / (double)args.size();
        }
        if (c.variant == V_SPLIT && use_product_parallel(c.level, pr.g, sms, true, FP32_TERMS))
            return time([&] {
                return run_fp32_parallel_enqueue(c.level, pr.g, tb, static_cast<const float*>(pr.A),
                                                 static_cast<const float*>(pr.B),
                                                 static_cast<float*>(scratch.p) - shift, st, sms, ws.p, ws_bytes,
                                                 FP32_TERMS, tab + pr.mtab_off[c.level], pr.mcol, err);
            });
        if (c.variant == V_SPLIT)
            return time([&] {
                return run_fp32_enqueue(c.level, pr.g, tb, static_cast<const float*>(pr.A),
                                        static_cast<const float*>(pr.B),
                                        static_cast<float*>(scratch.p) - shift, st, sms, ws.p, ws_bytes,
                                        FP32_TERMS, err);
            });
        return 1e30;
    }

    Choice choose(const Prob& pr, const int64_t* tab)
    {
        const std::vector<Choice> cand = candidates(pr);
        if (cand.size() == 1) return cand[0];
        const TuneKey key = tune_key(pr);
        {
            std::lock_guard<std::mutex> lk(g_tune_mu);
            auto it = g_tune_cache.find(key);
            if (it != g_tune_cache.end()) return it->second;
        }
        // A later candidate must beat the best so far by 2 %: its timing
        // stands for every problem of the size class, so near ties go to the
        // earlier candidate, which is the grouped launch at L = 0 (timed as a
        // share of a full launch, whose tail it removes for the whole chunk)
        // and the lower level otherwise (less rounding error).
        Choice best = cand[0];
        double best_t = 1e30;
        static const char* names[] = {"fused", "fused_small", "packed_grouped", "packed", "split", "scale",
                                      "split_grouped"};
        for (const Choice& c : cand)
        {
            what = names[c.variant];
            const double t = time_choice(pr, tab, c) * (best_t < 1e30 ? 1.02 : 1.0);
            if (t < best_t) { best_t = t; best = c; }
        }
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune_cache[key] = best;
        return best;
    }
};

}  // namespace

struct BatchPlan
{
    int device = 0;
    int count = 0;
    DevBuf tables;                          // all scatter vectors
    DevBuf err;                             // split-BF16 wait-timeout flag
    DevBuf chunk_ws[2];                     // packed operands of grouped chunks
    DevBuf seq_ws;                          // problem-by-problem packed schedule
    DevBuf f32_ws[2];                       // split-BF16 branches
    std::vector<DevBuf> descs;              // grouped-launch descriptors
    std::vector<int> levels, variants;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    unsigned long long nodes = 0;
    double create_s = 0.0, tune_s = 0.0;
    int timings = 0;
    ~BatchPlan()
    {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
    }
};

namespace {

// Streams and events used only while capturing.
struct CaptureStreams
{
    cudaStream_t main = nullptr, pack = nullptr, f32[2] = {nullptr, nullptr};
    std::vector<cudaEvent_t> events;
    ~CaptureStreams()
    {
        for (cudaEvent_t e : events) cudaEventDestroy(e);
        for (cudaStream_t s : {main, pack, f32[0], f32[1]})
            if (s) cudaStreamDestroy(s);
    }
    cudaEvent_t event()
    {
        cudaEvent_t e = nullptr;
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) { cudaGetLastError(); return nullptr; }
        events.push_back(e);
        return e;
    }
};

#define TSB_TRY(x) do { const int s_ = (x); if (s_) return s_; } while (0)

size_t round256(size_t x) { return (x + 255) / 256 * 256; }

size_t pgroup_bytes(const GemmView& g)
{
    const PackGeom pg = pack_geom(0, g);
    return round256(pg.s_elems * sizeof(double)) + round256(pg.t_elems * sizeof(double));
}

}  // namespace

int batch_create(int count, const tblis_stra_problem* problems, BatchPlan** out)
{
    const auto t_start = std::chrono::steady_clock::now();
    *out = nullptr;
    clear_detail();
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
            if (mem_kind(T[t]->data, plan->device) != MemKind::LOCAL) return TBLIS_STRA_ERR_ARG;   // this GPU's memory only
        }
        max_c_span = std::max<int64_t>(max_c_span, pr.g.hi[2] - pr.g.lo[2] + 1);
        const std::vector<int64_t>* v[9] = {&pr.g.rsA, &pr.g.rsC, &pr.g.csB, &pr.g.csC, &pr.g.ksA,
                                            &pr.g.ksB, &pr.g.bA, &pr.g.bB, &pr.g.bC};
        for (int j = 0; j < 9; j++) { pr.tab_off[j] = total_tab; total_tab += std::max<size_t>(v[j]->size(), 1); }
        pr.mcol = m_tables_col_major(pr.g);
        for (int L = 1; L <= 2; L++)
        {
            const int H = product_table(L).H;
            const int64_t nb = (int64_t)product_table(L).prod.size() * pr.g.batch;
            pr.mtab_off[L] = total_tab;
            total_tab += (size_t)std::max<int64_t>((pr.g.m + H - 1) / H + (pr.g.n + H - 1) / H + nb, 1);
        }
        pr.level_req = q.level;
        pr.empty = pr.g.m == 0 || pr.g.n == 0 || pr.g.batch == 0;
        pr.scale = !pr.empty && (pr.g.alpha == 0.0 || pr.g.k == 0);
    }

    // 2. one device buffer for all scatter vectors
    std::vector<int64_t> host(std::max<size_t>(total_tab, 1), 0);
    for (auto& pr : probs)
    {
        const std::vector<int64_t>* v[9] = {&pr.g.rsA, &pr.g.rsC, &pr.g.csB, &pr.g.csC, &pr.g.ksA,
                                            &pr.g.ksB, &pr.g.bA, &pr.g.bB, &pr.g.bC};
        for (int j = 0; j < 9; j++) std::copy(v[j]->begin(), v[j]->end(), host.begin() + (ptrdiff_t)pr.tab_off[j]);
        for (int L = 1; L <= 2; L++)
        {
            const int H = product_table(L).H;
            const int64_t nb = (int64_t)product_table(L).prod.size() * pr.g.batch;
            dense_m_tables((pr.g.m + H - 1) / H, (pr.g.n + H - 1) / H, nb, pr.mcol,
                           host.data() + pr.mtab_off[L]);
        }
    }
    TSB_TRY(plan->tables.alloc(host.size() * 8));
    TSB_TRY(upload_complete(plan->tables.p, host.data(), host.size() * 8));
    const int64_t* tab = static_cast<const int64_t*>(plan->tables.p);
    TSB_TRY(plan->err.alloc(sizeof(int)));
    const int zero = 0;
    TSB_TRY(upload_complete(plan->err.p, &zero, sizeof(int)));
    int* err = static_cast<int*>(plan->err.p);

    // 3. schedules (autotuned where there is a choice)
    const auto t_tune = std::chrono::steady_clock::now();
    {
        size_t tune_ws = 0;
        bool need = false;
        for (auto& pr : probs)
        {
            if (pr.empty || pr.scale) continue;
            const std::vector<Choice> c = candidates(pr);
            if (c.size() < 2) continue;
            need = true;
            for (const Choice& x : c)
                tune_ws = std::max(tune_ws, schedule_workspace_bytes(pr, x, sms));
        }
        Tuner tuner;
        if (need) TSB_TRY(tuner.init((size_t)max_c_span * sizeof(double), tune_ws, err, sms));
        for (auto& pr : probs)
        {
            if (pr.empty || pr.scale) { pr.variant = V_SCALE; pr.level = 0; continue; }
            const std::vector<Choice> c = candidates(pr);
            if (c.empty()) return t_variant_mask == ALL_VARIANTS ? TBLIS_STRA_ERR_TOO_LARGE : TBLIS_STRA_ERR_ARG;
            const Choice ch = c.size() == 1 ? c[0] : tuner.choose(pr, tab);
            pr.level = ch.level;
            pr.variant = ch.variant;
        }
        if (need)
        {
            const cudaError_t e = cudaStreamSynchronize(tuner.st);
            if (e != cudaSuccess || tuner.failures)
            {
                if (e != cudaSuccess) cudaGetLastError();
                // a failed candidate is skipped; a failed stream is an error
                if (e != cudaSuccess)
                {
                    note_detail(tuner.first_failure + "; then " + cudaGetErrorName(e));
                    return TBLIS_STRA_ERR_CUDA;
                }
            }
        }
        plan->timings = tuner.timings;
    }
    plan->tune_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_tune).count();
    TSB_CU(cudaDeviceSynchronize());
    TSB_TRY(upload_complete(plan->err.p, &zero, sizeof(int)));
    for (auto& pr : probs) { plan->levels.push_back(pr.level); plan->variants.push_back(pr.variant); }

    // 4. workspaces and descriptors (all before capture)
    // 4a. fused groups by (level, tile configuration)
    std::map<std::pair<int, int>, std::vector<DmmaArgs>> fused;
    for (auto& pr : probs)
        if (pr.variant == V_FUSED || pr.variant == V_FUSED_SMALL)
        {
            const int config = fused_config(pr.variant, pr.level);
            fused[{pr.level, config}].push_back(make_args(pr, tab, pr.level, config, nullptr, 0));
        }
    std::vector<std::tuple<int, int, DmmaGroupArgs>> fused_groups;
    for (auto& kv : fused)
    {
        plan->descs.emplace_back();
        DmmaGroupArgs g;
        TSB_TRY(upload_fused(kv.second, &plan->descs.back(), g));
        fused_groups.emplace_back(kv.first.first, kv.first.second, g);
    }
    // 4b. problem-by-problem packed schedules share one workspace
    size_t seq_bytes = 0;
    for (auto& pr : probs)
        if (pr.variant == V_PACKED) seq_bytes = std::max(seq_bytes, schedule_workspace_bytes(pr, {pr.level, pr.variant}, sms));
    if (seq_bytes) TSB_TRY(plan->seq_ws.alloc(seq_bytes));
    // 4c. chunks of grouped problems: FP64 packed (V_PGROUP) and FP32 split
    // (V_SGROUP) problems, each kind in consecutive chunks of at most
    // chunk_bytes() of workspace (unless one problem needs more), packed into
    // two chunk workspaces in turn.
    struct Chunk
    {
        bool fp32 = false;
        std::vector<int> probs;
        std::vector<void*> ws;          // per problem: FP64 S (T follows), FP32 split workspace
        PackedGroupArgs pg{};
        SplitGroupArgs sg{};
    };
    auto chunk_need_of = [&](const Prob& pr) {
        return pr.variant == V_PGROUP ? pgroup_bytes(pr.g) : round256(fp32_workspace_bytes(0, pr.g, FP32_TERMS));
    };
    std::vector<Chunk> chunks;
    size_t chunk_need = 0;
    {
        const size_t cap = chunk_bytes();
        for (int kind = 0; kind < 2; kind++)
        {
            size_t used = 0;
            bool open = false;
            for (int i = 0; i < count; i++)
            {
                if (probs[i].variant != (kind ? V_SGROUP : V_PGROUP)) continue;
                const size_t need = chunk_need_of(probs[i]);
                if (!open || (used > 0 && used + need > cap))
                {
                    chunks.emplace_back();
                    chunks.back().fp32 = kind == 1;
                    used = 0;
                    open = true;
                }
                chunks.back().probs.push_back(i);
                used += need;
                chunk_need = std::max(chunk_need, used);
            }
        }
    }
    for (size_t b = 0; b < std::min<size_t>(chunks.size(), 2); b++) TSB_TRY(plan->chunk_ws[b].alloc(chunk_need));
    for (size_t c = 0; c < chunks.size(); c++)
    {
        Chunk& ch = chunks[c];
        unsigned char* base = static_cast<unsigned char*>(plan->chunk_ws[c % 2].p);
        size_t off = 0;
        std::vector<PackedGemmArgs> pargs;
        std::vector<SplitGemmArgs> sargs;
        for (int i : ch.probs)
        {
            const Prob& pr = probs[i];
            const int64_t* tb[9];
            pr.tables(tab, tb);
            ch.ws.push_back(base + off);
            if (!ch.fp32)
            {
                const PackGeom pg = pack_geom(0, pr.g);
                double* S = reinterpret_cast<double*>(base + off);
                double* T = reinterpret_cast<double*>(base + off + round256(pg.s_elems * sizeof(double)));
                pargs.push_back(packed_product_args(0, product_table(0).prod[0], pr.g, pg, tb, S, T,
                                                    static_cast<double*>(pr.C), err));
            }
            else
            {
                SplitGemmArgs a{};
                TSB_TRY(run_fp32_enqueue(0, pr.g, tb, static_cast<const float*>(pr.A), static_cast<const float*>(pr.B),
                                         static_cast<float*>(pr.C), nullptr, sms, base + off, chunk_need_of(pr),
                                         FP32_TERMS, err, &a, false));
                sargs.push_back(a);
            }
            off += chunk_need_of(pr);
        }
        plan->descs.emplace_back();
        if (!ch.fp32)
        {
            TSB_TRY(upload_packed(pargs, &plan->descs.back(), ch.pg));
            ch.pg.err = err;
            ch.pg.wait_limit = wait_limit_cycles();
        }
        else
        {
            TSB_TRY(upload_split(sargs, &plan->descs.back(), ch.sg));
            ch.sg.err = err;
            ch.sg.wait_limit = wait_limit_cycles();
        }
    }
    // 4d. FP32 problems on two branches balanced by flops
    std::vector<int> f32_list[2];
    {
        double load[2] = {0.0, 0.0};
        size_t need[2] = {0, 0};
        for (int i = 0; i < count; i++)
        {
            if (probs[i].variant != V_SPLIT) continue;
            const int b = load[0] <= load[1] ? 0 : 1;
            f32_list[b].push_back(i);
            load[b] += probs[i].flops();
            need[b] = std::max(need[b], schedule_workspace_bytes(probs[i], {probs[i].level, V_SPLIT}, sms));
        }
        for (int b = 0; b < 2; b++)
            if (need[b]) TSB_TRY(plan->f32_ws[b].alloc(need[b]));
    }

    // 5. capture
    CaptureStreams cs;
    TSB_CU(cudaStreamCreateWithFlags(&cs.main, cudaStreamNonBlocking));
    const bool use_pack = !chunks.empty();
    const bool use_f32[2] = {!f32_list[0].empty(), !f32_list[1].empty()};
    if (use_pack) TSB_CU(cudaStreamCreateWithFlags(&cs.pack, cudaStreamNonBlocking));
    for (int b = 0; b < 2; b++)
        if (use_f32[b]) TSB_CU(cudaStreamCreateWithFlags(&cs.f32[b], cudaStreamNonBlocking));
    std::vector<cudaEvent_t> ev_pack(chunks.size()), ev_gemm(chunks.size());
    for (size_t c = 0; c < chunks.size(); c++)
    {
        ev_pack[c] = cs.event();
        ev_gemm[c] = cs.event();
        if (!ev_pack[c] || !ev_gemm[c]) return TBLIS_STRA_ERR_CUDA;
    }
    cudaEvent_t ev_fork = cs.event(), ev_f32[2] = {cs.event(), cs.event()};
    if (!ev_fork || !ev_f32[0] || !ev_f32[1]) return TBLIS_STRA_ERR_CUDA;

    // Stream order of the pack stream: chunk c's packing waits for chunk
    // c-2's GEMM (same workspace); the main stream's GEMM of chunk c waits
    // for its packing.  Both are enqueued in chunk order, the pack launches
    // of chunk c before the GEMM of chunk c-1, so that GEMM's event exists
    // when chunk c+1 needs it.
    auto enqueue_pack = [&](size_t c) -> int {
        if (c >= 2) TSB_CU(cudaStreamWaitEvent(cs.pack, ev_gemm[c - 2], 0));
        const Chunk& ch = chunks[c];
        for (size_t j = 0; j < ch.probs.size(); j++)
        {
            const Prob& pr = probs[ch.probs[j]];
            const int64_t* tb[9];
            pr.tables(tab, tb);
            if (!ch.fp32)
            {
                const PackGeom pg = pack_geom(0, pr.g);
                double* S = static_cast<double*>(ch.ws[j]);
                double* T = reinterpret_cast<double*>(static_cast<unsigned char*>(ch.ws[j]) +
                                                      round256(pg.s_elems * sizeof(double)));
                TSB_TRY(enqueue_pack_product(product_table(0).prod[0], pr.g, pg, tb,
                                             static_cast<const double*>(pr.A), static_cast<const double*>(pr.B),
                                             S, T, cs.pack));
            }
            else
            {
                SplitGemmArgs unused{};
                TSB_TRY(run_fp32_enqueue(0, pr.g, tb, static_cast<const float*>(pr.A),
                                         static_cast<const float*>(pr.B), static_cast<float*>(pr.C), cs.pack, sms,
                                         ch.ws[j], chunk_need_of(pr), FP32_TERMS, err, &unused, true));
            }
        }
        TSB_CU(cudaEventRecord(ev_pack[c], cs.pack));
        return TBLIS_STRA_SUCCESS;
    };
    auto enqueue_gemm = [&](size_t c) -> int {
        TSB_CU(cudaStreamWaitEvent(cs.main, ev_pack[c], 0));
        if (!chunks[c].fp32) TSB_CU(launch_packed_gemm_grouped(chunks[c].pg, cs.main, sms));
        else TSB_CU(launch_split_gemm_grouped(chunks[c].sg, FP32_TERMS == 6 ? 3 : 2, cs.main, sms));
        TSB_CU(cudaEventRecord(ev_gemm[c], cs.main));
        return TBLIS_STRA_SUCCESS;
    };

    auto capture = [&]() -> int {
        TSB_CU(cudaEventRecord(ev_fork, cs.main));
        if (use_pack) TSB_CU(cudaStreamWaitEvent(cs.pack, ev_fork, 0));
        for (int b = 0; b < 2; b++)
            if (use_f32[b]) TSB_CU(cudaStreamWaitEvent(cs.f32[b], ev_fork, 0));

        // FP32 branches
        for (int b = 0; b < 2; b++)
        {
            for (int i : f32_list[b])
            {
                const Prob& pr = probs[i];
                const int64_t* tb[9];
                pr.tables(tab, tb);
                if (use_product_parallel(pr.level, pr.g, sms, true, FP32_TERMS))
                    TSB_TRY(run_fp32_parallel_enqueue(pr.level, pr.g, tb, static_cast<const float*>(pr.A),
                                                      static_cast<const float*>(pr.B), static_cast<float*>(pr.C),
                                                      cs.f32[b], sms, plan->f32_ws[b].p,
                                                      fp32_parallel_workspace_bytes(pr.level, pr.g, FP32_TERMS),
                                                      FP32_TERMS, tab + pr.mtab_off[pr.level], pr.mcol, err));
                else
                    TSB_TRY(run_fp32_enqueue(pr.level, pr.g, tb, static_cast<const float*>(pr.A),
                                             static_cast<const float*>(pr.B), static_cast<float*>(pr.C),
                                             cs.f32[b], sms, plan->f32_ws[b].p,
                                             fp32_group_workspace_bytes(pr.level, pr.g, FP32_TERMS), FP32_TERMS,
                                             err));
            }
            if (use_f32[b]) TSB_CU(cudaEventRecord(ev_f32[b], cs.f32[b]));
        }
        // the first two chunks pack while the main stream runs the rest
        for (size_t c = 0; c < std::min<size_t>(chunks.size(), 2); c++) TSB_TRY(enqueue_pack(c));

        for (auto& pr : probs)
        {
            if (pr.variant != V_SCALE || pr.empty) continue;
            if (pr.g.type == TYPE_DOUBLE)
            {
                ScaleArgs sa{static_cast<double*>(pr.C), tab + pr.tab_off[1], tab + pr.tab_off[3],
                             tab + pr.tab_off[8], pr.g.m, pr.g.n, pr.g.batch, pr.g.beta};
                TSB_CU(launch_scale(sa, cs.main));
            }
            else
            {
                ScaleF32Args sa{static_cast<float*>(pr.C), tab + pr.tab_off[1], tab + pr.tab_off[3],
                                tab + pr.tab_off[8], pr.g.m, pr.g.n, pr.g.batch, (float)pr.g.beta};
                TSB_CU(launch_scale_f32(sa, cs.main));
            }
        }
        for (auto& fg : fused_groups)
            TSB_TRY(launch_fused_group(std::get<2>(fg), std::get<0>(fg), std::get<1>(fg), cs.main, sms));
        for (auto& pr : probs)
        {
            if (pr.variant != V_PACKED) continue;
            const int64_t* tb[9];
            pr.tables(tab, tb);
            if (use_product_parallel(pr.level, pr.g, sms, false, 0))
                TSB_TRY(run_fp64_parallel_enqueue(pr.level, pr.g, tb, static_cast<const double*>(pr.A),
                                                  static_cast<const double*>(pr.B), static_cast<double*>(pr.C),
                                                  cs.main, sms, plan->seq_ws.p,
                                                  fp64_parallel_workspace_bytes(pr.level, pr.g),
                                                  tab + pr.mtab_off[pr.level], pr.mcol, err));
            else
                TSB_TRY(run_fp64_packed_enqueue(pr.level, pr.g, tb, static_cast<const double*>(pr.A),
                                                static_cast<const double*>(pr.B), static_cast<double*>(pr.C),
                                                cs.main, sms, plan->seq_ws.p,
                                                fp64_packed_group_workspace_bytes(pr.level, pr.g), err));
        }
        for (size_t c = 0; c < chunks.size(); c++)
        {
            TSB_TRY(enqueue_gemm(c));
            if (c + 2 < chunks.size()) TSB_TRY(enqueue_pack(c + 2));
        }
        for (int b = 0; b < 2; b++)
            if (use_f32[b]) TSB_CU(cudaStreamWaitEvent(cs.main, ev_f32[b], 0));
        return TBLIS_STRA_SUCCESS;
    };

    const unsigned long long launches0 = g_launches.load();
    TSB_CU(cudaStreamBeginCapture(cs.main, cudaStreamCaptureModeThreadLocal));
    const int status = capture();
    const cudaError_t ec = cudaStreamEndCapture(cs.main, &plan->graph);
    if (status) { cudaGetLastError(); return status; }
    if (ec != cudaSuccess) { cudaGetLastError(); return TBLIS_STRA_ERR_CUDA; }
    TSB_CU(cudaGraphInstantiate(&plan->exec, plan->graph, 0));
    plan->nodes = g_launches.load() - launches0;
    g_launches -= plan->nodes;   // counted at every execute instead
    plan->create_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
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

int batch_schedule(const BatchPlan* plan, int* variants)
{
    if (!plan || !variants) return TBLIS_STRA_ERR_NULL;
    std::copy(plan->variants.begin(), plan->variants.end(), variants);
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
    // batches plan with Strassen whatever algorithm the thread has selected
    const int alg = tsb::thread_algorithm();
    tsb::set_thread_algorithm(0);
    const int s = tsb::batch_create(count, problems, &p);
    tsb::set_thread_algorithm(alg);
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

int tblis_stra_batch_schedule(tblis_stra_batch batch, int* schedules)
{
    return tsb::batch_schedule(reinterpret_cast<const tsb::BatchPlan*>(batch), schedules);
}

int tblis_stra_set_batch_schedules(unsigned mask)
{
    if (mask == 0 || (mask & ~tsb::ALL_VARIANTS)) return TBLIS_STRA_ERR_ARG;
    tsb::t_variant_mask = mask;
    return TBLIS_STRA_SUCCESS;
}

unsigned tblis_stra_get_batch_schedules(void) { return tsb::t_variant_mask; }

int tblis_stra_batch_stats(tblis_stra_batch batch, double* create_s, double* tune_s, int* timings)
{
    auto* p = reinterpret_cast<const tsb::BatchPlan*>(batch);
    if (!p) return TBLIS_STRA_ERR_NULL;
    if (create_s) *create_s = p->create_s;
    if (tune_s) *tune_s = p->tune_s;
    if (timings) *timings = p->timings;
    return TBLIS_STRA_SUCCESS;
}

void tblis_stra_batch_destroy(tblis_stra_batch batch)
{
    tsb::batch_destroy(reinterpret_cast<tsb::BatchPlan*>(batch));
}

}  // extern "C"
