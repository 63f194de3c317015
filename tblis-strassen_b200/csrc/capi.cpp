// extern "C" boundary of the library and the host-side driver behind it.
//
//   tblis_tensor_mult              replaces src/iface/3t/mult.cxx:15
//   stra_tblis_tensor_mult         replaces src/stra_iface/3t/stra_mult.cxx:26
//   stra_tblis_tensor_mult_2level  replaces src/stra_iface/3t/stra_mult_2level.cxx:26
//   tblis_matrix_mult, stra_tblis_matrix_mult[_naive|_ab][_2level]
//                                  replace src/iface/3m and src/stra_iface/3m
//
// Each call: plan the contraction (plan.cpp), fetch or build the device copy of
// its scatter vectors (cached per shape/stride/label signature), stage host
// operands through device memory when needed (pipelined in chunks when all
// three are on the host and large), and enqueue the kernels of the requested
// level and variant on the caller's stream:
//   ABC   packed schedule: per group of 7 products (L >= 1) one pass packs
//         the operand sums into tile order, then per product the packed DMMA
//         GEMM adds +-alpha*S*T into its C blocks; with too little workspace
//         one product at a time, and with none the fully fused kernel (one
//         persistent launch running every product);
//   AB    per product: pack the sums, packed GEMM into one M buffer, then a
//         scatter-add of M into its C blocks;
//   Naive per product: sum-gather dense S and T, pack them, packed GEMM
//         M = S*T, scatter-add;
//   FP32  the split-BF16 schedule on tcgen05 (bf16_split.cu).
// After the call C->scalar is 1 and C->conj 0, as the reference leaves them
// (src/stra_iface/3t/stra_mult.cxx:251-252).
#include "tblis_stra_b200.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "kernels.cuh"
#include "memkind.hpp"
#include "plan.hpp"
#include "schedule.hpp"

extern "C" {
const tblis_comm* const tblis_single = reinterpret_cast<const tblis_comm*>(&tblis_single);
}

namespace tsb {
namespace {

thread_local int t_impl = 1;
thread_local cudaStream_t t_stream = nullptr;
thread_local int t_status = TBLIS_STRA_SUCCESS;
thread_local size_t t_ws_limit = SIZE_MAX;   // device workspace the ABC schedule may use
thread_local int t_fp32_terms = 6;           // split-BF16 product terms for FP32 (3 or 6)
thread_local int t_product_parallel = -1;    // product-parallel ABC: -1 auto, 0 never, 1 when it fits
thread_local long long t_wait_limit = 0;     // pipeline wait bound in SM cycles (0: the kernels' default)
thread_local bool t_wait_inject = false;     // pipeline waits run out whatever the state of their phase
thread_local size_t t_alloc_limit = SIZE_MAX;  // largest single device allocation a call may make
unsigned g_num_threads = 1;
thread_local std::string t_detail;           // what the last failing CUDA call was

// ---- device tables (cached) ------------------------------------------------

struct DevPlan
{
    int device = -1;
    void* mem = nullptr;
    size_t bytes = 0;
    const int64_t *rsA, *rsC, *csB, *csC, *ksA, *ksB, *bA, *bB, *bC;
    // M_p tables of the product-parallel schedule per level, made on first use
    mutable std::mutex mt_mu;
    mutable void* mtab[3] = {nullptr, nullptr, nullptr};
    ~DevPlan()
    {
        if (mem) cudaFree(mem);
        for (void* p : mtab)
            if (p) cudaFree(p);
    }
};

std::mutex g_cache_mu;
std::list<std::pair<std::string, std::shared_ptr<DevPlan>>> g_cache;   // MRU first
constexpr size_t CACHE_MAX = 32;

std::string plan_key(int device, const tblis_tensor* const T[3], const label_type* const I[3])
{
    std::string k;
    auto put = [&](const void* p, size_t n) { k.append(static_cast<const char*>(p), n); };
    put(&device, sizeof device);
    for (int t = 0; t < 3; t++)
    {
        put(&T[t]->type, sizeof T[t]->type);
        put(&T[t]->ndim, sizeof T[t]->ndim);
        if (T[t]->ndim)
        {
            put(T[t]->len, sizeof(len_type) * T[t]->ndim);
            put(T[t]->stride, sizeof(stride_type) * T[t]->ndim);
            put(I[t], sizeof(label_type) * T[t]->ndim);
        }
    }
    return k;
}

int upload_plan(const GemmView& g, int device, std::shared_ptr<DevPlan>& out)
{
    auto dp = std::make_shared<DevPlan>();
    dp->device = device;
    const std::vector<int64_t>* parts[9] = {&g.rsA, &g.rsC, &g.csB, &g.csC, &g.ksA, &g.ksB,
                                            &g.bA, &g.bB, &g.bC};
    size_t total = 0;
    for (auto* v : parts) total += std::max<size_t>(v->size(), 1);
    std::vector<int64_t> host(total, 0);
    size_t off[9], pos = 0;
    for (int i = 0; i < 9; i++)
    {
        off[i] = pos;
        std::copy(parts[i]->begin(), parts[i]->end(), host.begin() + (ptrdiff_t)pos);
        pos += std::max<size_t>(parts[i]->size(), 1);
    }
    dp->bytes = total * sizeof(int64_t);
    if (dp->bytes > t_alloc_limit) return TBLIS_STRA_ERR_ALLOC;
    if (cudaMalloc(&dp->mem, dp->bytes) != cudaSuccess) { cudaGetLastError(); dp->mem = nullptr; return TBLIS_STRA_ERR_ALLOC; }
    const int s = upload_complete(dp->mem, host.data(), dp->bytes);
    if (s) return s;
    const int64_t* base = static_cast<const int64_t*>(dp->mem);
    dp->rsA = base + off[0]; dp->rsC = base + off[1]; dp->csB = base + off[2];
    dp->csC = base + off[3]; dp->ksA = base + off[4]; dp->ksB = base + off[5];
    dp->bA = base + off[6]; dp->bB = base + off[7]; dp->bC = base + off[8];
    out = dp;
    return TBLIS_STRA_SUCCESS;
}

int get_plan(const tblis_tensor* const T[3], const label_type* const I[3], int device,
             GemmView& g, std::shared_ptr<DevPlan>& dp)
{
    std::string key = plan_key(device, T, I);
    {
        std::lock_guard<std::mutex> lk(g_cache_mu);
        for (auto it = g_cache.begin(); it != g_cache.end(); ++it)
            if (it->first == key)
            {
                dp = it->second;
                g_cache.splice(g_cache.begin(), g_cache, it);
                // scalars and sizes still come from a (scatter-free) re-plan
                return plan_contraction(T[0], I[0], T[1], I[1], T[2], I[2], g, false);
            }
    }
    int st = plan_contraction(T[0], I[0], T[1], I[1], T[2], I[2], g, true);
    if (st) return st;
    st = upload_plan(g, device, dp);
    if (st) return st;
    std::lock_guard<std::mutex> lk(g_cache_mu);
    g_cache.emplace_front(key, dp);
    while (g_cache.size() > CACHE_MAX) g_cache.pop_back();
    return TBLIS_STRA_SUCCESS;
}

// Device copy of the M_p tables of plan t at `level` (made once per plan and
// level; the layout follows C's faster bundle, fixed by the plan).
int plan_m_tables(const DevPlan& t, int level, int64_t ms, int64_t ns, int64_t nb, bool col_major,
                  const int64_t*& out)
{
    std::lock_guard<std::mutex> lk(t.mt_mu);
    if (!t.mtab[level])
    {
        std::vector<int64_t> h((size_t)(ms + ns + nb));
        dense_m_tables(ms, ns, nb, col_major, h.data());
        void* d = nullptr;
        if (h.size() * sizeof(int64_t) > t_alloc_limit) return TBLIS_STRA_ERR_ALLOC;
        if (cudaMalloc(&d, h.size() * sizeof(int64_t)) != cudaSuccess) { cudaGetLastError(); return TBLIS_STRA_ERR_ALLOC; }
        const int s = upload_complete(d, h.data(), h.size() * sizeof(int64_t));
        if (s) { cudaFree(d); return s; }
        t.mtab[level] = d;
    }
    out = static_cast<const int64_t*>(t.mtab[level]);
    return TBLIS_STRA_SUCCESS;
}

// Whether the product-parallel form beats running each group's products
// tile by tile (M's local index must fit 32 bits).  At L = 2 it does at every
// size measured: a product's C tiles spread over up to 4 blocks, and with
// products side by side each is written once (as M) and combined in one
// pass.  So it does for the split-BF16 GEMM at L = 1 (16384^3, 6 terms: 200 ->
// 234 TFLOP/s), whose drain epilogue of up to 2 C tiles per product competes
// with the MMAs of the next.  For FP64 at L = 1 it does when the last wave of
// one product's `tiles` on `sms` SMs leaves more than a tenth of the launch
// idle (fewer tiles than SMs included).
bool parallel_pays(int level, bool fp32, int64_t tiles, int sms, int64_t ms, int64_t ns)
{
    if (ms * ns >= ((int64_t)1 << 31)) return false;
    if (level >= 2 || fp32) return true;
    const int64_t rounds = (tiles + sms - 1) / sms;
    return rounds * sms * 10 > tiles * 11;
}

int num_sms(int device)
{
    static std::mutex mu;
    static std::map<int, int> cache;
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find(device);
    if (it != cache.end()) return it->second;
    int v = 148;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device);
    cache[device] = v;
    return v;
}


// The library's own stream-ordered memory pool per device.  Its release
// threshold is unlimited, so memory freed by one call is reused by the next
// without returning to the driver at every synchronisation.
cudaMemPool_t library_pool(int device)
{
    static std::mutex mu;
    static std::map<int, cudaMemPool_t> pools;
    std::lock_guard<std::mutex> lk(mu);
    auto it = pools.find(device);
    if (it != pools.end()) return it->second;
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaMemPool_t pool = nullptr;
    if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) { cudaGetLastError(); return nullptr; }
    uint64_t threshold = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold);
    pools[device] = pool;
    return pool;
}

// Stream-ordered device scratch (packed operands, AB / Naive temporaries, staging).
struct Scratch
{
    void* p = nullptr;
    cudaStream_t s = nullptr;
    ~Scratch() { if (p) cudaFreeAsync(p, s); }
    int alloc(size_t bytes, cudaStream_t st)
    {
        s = st;
        if (bytes == 0) bytes = 16;
        if (bytes > t_alloc_limit) return TBLIS_STRA_ERR_ALLOC;
        int device = 0;
        if (cudaGetDevice(&device) != cudaSuccess) { cudaGetLastError(); return TBLIS_STRA_ERR_NO_DEVICE; }
        cudaMemPool_t pool = library_pool(device);
        cudaError_t e = pool ? cudaMallocFromPoolAsync(&p, bytes, pool, st) : cudaMallocAsync(&p, bytes, st);
        if (e != cudaSuccess) { cudaGetLastError(); p = nullptr; return TBLIS_STRA_ERR_ALLOC; }
        return TBLIS_STRA_SUCCESS;
    }
};

DevProduct to_dev(const Product& p)
{
    DevProduct d{};
    d.na = p.na; d.nb = p.nb; d.nc = p.nc;
    for (int i = 0; i < 4; i++)
    {
        d.a_r[i] = p.a[i].r; d.a_c[i] = p.a[i].c; d.a_s[i] = p.a[i].sign;
        d.b_r[i] = p.b[i].r; d.b_c[i] = p.b[i].c; d.b_s[i] = p.b[i].sign;
        d.c_r[i] = p.c[i].r; d.c_c[i] = p.c[i].c; d.c_s[i] = p.c[i].sign;
        d.c_first[i] = p.c_first[i];
    }
    return d;
}

int max_terms(const ProductTable& t)
{
    int m = 1;
    for (auto& p : t.prod) m = std::max<int>(m, std::max<int>(p.na, p.nb));
    return m;
}

inline int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }

#define TSB_CUDA(x) do { const cudaError_t e_ = (x); \
    if (e_ != cudaSuccess) { note_cuda_error(#x, e_, __FILE__, __LINE__); return TBLIS_STRA_ERR_CUDA; } } while (0)

// Dense row-major temporaries of the AB / Naive variants: offset tables.
struct DenseTables
{
    Scratch mem;
    const int64_t* rows = nullptr;   // i * ld
    const int64_t* cols = nullptr;   // j
    const int64_t* bat = nullptr;    // b * rows_n * ld
    int build(int64_t nr, int64_t ld, int64_t nbat, cudaStream_t st)
    {
        std::vector<int64_t> h((size_t)(nr + ld + nbat));
        for (int64_t i = 0; i < nr; i++) h[(size_t)i] = i * ld;
        for (int64_t j = 0; j < ld; j++) h[(size_t)(nr + j)] = j;
        for (int64_t b = 0; b < nbat; b++) h[(size_t)(nr + ld + b)] = b * nr * ld;
        int s = mem.alloc(h.size() * 8, st);
        if (s) return s;
        TSB_CUDA(cudaMemcpyAsync(mem.p, h.data(), h.size() * 8, cudaMemcpyHostToDevice, st));
        TSB_CUDA(cudaStreamSynchronize(st));   // h is a local buffer
        rows = static_cast<const int64_t*>(mem.p);
        cols = rows + nr;
        bat = cols + ld;
        return TBLIS_STRA_SUCCESS;
    }
};

DmmaArgs base_args(const GemmView& g, const DevPlan& t, const double* A, const double* B, double* C)
{
    DmmaArgs a;
    std::memset(&a, 0, sizeof a);
    a.A = A; a.B = B; a.C = C;
    a.rsA = t.rsA; a.ksA = t.ksA; a.ksB = t.ksB; a.csB = t.csB; a.rsC = t.rsC; a.csC = t.csC;
    a.bA = t.bA; a.bB = t.bB; a.bC = t.bC;
    a.m = g.m; a.n = g.n; a.k = g.k; a.mC = g.m; a.nC = g.n;
    a.batch = g.batch;
    a.alpha = g.alpha; a.beta = g.beta;
    // Consecutive threads walk the operand dimension with the smaller stride.
    a.a_kfast = (g.unit_ksA != 0 && (g.unit_rsA == 0 || g.unit_ksA < g.unit_rsA)) ? 1 : 0;
    a.b_kfast = (g.unit_ksB != 0 && (g.unit_csB == 0 || g.unit_ksB < g.unit_csB)) ? 1 : 0;
    return a;
}

void set_grid(DmmaArgs& a, int64_t ms, int64_t ns, int64_t ks)
{
    a.ms = ms; a.ns = ns; a.ks = ks;
    a.tiles_m = (int)cdiv(ms, 128);
    a.tiles_n = (int)cdiv(ns, 128);
    a.work = a.batch * (int64_t)a.tiles_m * a.tiles_n;
}

// Packed schedule of the ABC variant (see packed_kernels.cu) on pool scratch.
// Blocking calls read back the kernels' wait-timeout flag.
int run_fp64_packed(int level, const GemmView& g, const DevPlan& t, const double* A, const double* B,
                    double* C, cudaStream_t st, int sms, bool blocking, int* shared_err)
{
    // Product-parallel when one product's tiles would leave SMs idle and its
    // workspace is allowed.
    const PackGeom pg = pack_geom(level, g);
    const bool parallel = use_product_parallel(level, g, sms, false, 0);
    const size_t ws_par = parallel ? fp64_parallel_workspace_bytes(level, g) : 0;
    const bool m_col_major = m_tables_col_major(g);
    // A plain contraction with fewer C tiles than SMs: k-split.
    const int P = level == 0 && t_product_parallel != 0 ? ksplit_pieces(g, sms) : 1;
    if (P >= 2 && fp64_ksplit_workspace_bytes(g, P) <= t_ws_limit)
    {
        const int64_t* ktab = nullptr;
        int s;
        if ((s = plan_m_tables(t, 0, g.m, g.n, (int64_t)P * g.batch, m_col_major, ktab))) return s;
        Scratch kbuf, kerr;
        const size_t wsk = fp64_ksplit_workspace_bytes(g, P);
        if ((s = kbuf.alloc(wsk, st))) return s;
        int* err = shared_err;
        if (!err)
        {
            if ((s = kerr.alloc(sizeof(int), st))) return s;
            TSB_CUDA(cudaMemsetAsync(kerr.p, 0, sizeof(int), st));
            err = static_cast<int*>(kerr.p);
        }
        const int64_t* tb[9] = {t.rsA, t.rsC, t.csB, t.csC, t.ksA, t.ksB, t.bA, t.bB, t.bC};
        if ((s = run_fp64_ksplit_enqueue(g, tb, A, B, C, st, sms, kbuf.p, wsk, P, ktab, m_col_major, err))) return s;
        if (blocking && !shared_err)
        {
            int flag = 0;
            TSB_CUDA(cudaMemcpyAsync(&flag, kerr.p, sizeof(int), cudaMemcpyDeviceToHost, st));
            TSB_CUDA(cudaStreamSynchronize(st));
            if (flag) return TBLIS_STRA_ERR_TIMEOUT;
        }
        return TBLIS_STRA_SUCCESS;
    }
    const int64_t* mtab = nullptr;
    int s;
    if (parallel && (s = plan_m_tables(t, level, pg.ms, pg.ns, (int64_t)product_table(level).prod.size() * g.batch,
                                       m_col_major, mtab)))
        return s;
    const size_t ws_group = fp64_packed_group_workspace_bytes(level, g);
    const size_t ws = parallel ? ws_par : ws_group <= t_ws_limit ? ws_group : fp64_packed_workspace_bytes(level, g);
    Scratch buf, errbuf;
    if ((s = buf.alloc(ws, st))) return s;
    int* err = shared_err;
    if (!err)
    {
        if ((s = errbuf.alloc(sizeof(int), st))) return s;
        TSB_CUDA(cudaMemsetAsync(errbuf.p, 0, sizeof(int), st));
        err = static_cast<int*>(errbuf.p);
    }
    const int64_t* tb[9] = {t.rsA, t.rsC, t.csB, t.csC, t.ksA, t.ksB, t.bA, t.bB, t.bC};
    s = parallel ? run_fp64_parallel_enqueue(level, g, tb, A, B, C, st, sms, buf.p, ws, mtab, m_col_major, err)
                 : run_fp64_packed_enqueue(level, g, tb, A, B, C, st, sms, buf.p, ws, err);
    if (s) return s;
    if (blocking && !shared_err)
    {
        int flag = 0;
        TSB_CUDA(cudaMemcpyAsync(&flag, errbuf.p, sizeof(int), cudaMemcpyDeviceToHost, st));
        TSB_CUDA(cudaStreamSynchronize(st));
        if (flag) return TBLIS_STRA_ERR_TIMEOUT;
    }
    return TBLIS_STRA_SUCCESS;
}

// Naive's explicit operand sums of product pr as dense temporaries
// S (ms x ks, k fastest) and T (ks x ns, n fastest) per batch entry
// (straprim_naive2, src/stra_internal/3t/straprim_common.hpp:70-157).
int enqueue_sum_gather(const Product& pr, const GemmView& g, const DevPlan& t, int64_t ms, int64_t ns,
                       int64_t ks, const double* A, const double* B, double* S, double* T, cudaStream_t st)
{
    SumGatherArgs sa{};
    sa.X = A; sa.rsX = t.rsA; sa.csX = t.ksA; sa.bX = t.bA;
    sa.rows_full = g.m; sa.cols_full = g.k; sa.rows = ms; sa.cols = ks;
    sa.batch = g.batch; sa.nt = pr.na; sa.out = S;
    for (int i = 0; i < pr.na; i++) { sa.t_r[i] = pr.a[i].r; sa.t_c[i] = pr.a[i].c; sa.t_s[i] = pr.a[i].sign; }
    TSB_CUDA(launch_sum_gather(sa, st));
    SumGatherArgs sb{};
    sb.X = B; sb.rsX = t.ksB; sb.csX = t.csB; sb.bX = t.bB;
    sb.rows_full = g.k; sb.cols_full = g.n; sb.rows = ks; sb.cols = ns;
    sb.batch = g.batch; sb.nt = pr.nb; sb.out = T;
    for (int i = 0; i < pr.nb; i++) { sb.t_r[i] = pr.b[i].r; sb.t_c[i] = pr.b[i].c; sb.t_s[i] = pr.b[i].sign; }
    TSB_CUDA(launch_sum_gather(sb, st));
    return TBLIS_STRA_SUCCESS;
}

// Naive product pr on the packed GEMM: its dense sums S and T (tables St,
// Tt), then those packed in tile order into PS and PT.
int enqueue_naive_product(const Product& pr, const GemmView& g, const DevPlan& t, const PackGeom& pg,
                          const double* A, const double* B, double* S, double* T, const DenseTables& St,
                          const DenseTables& Tt, double* PS, double* PT, cudaStream_t st)
{
    int s = enqueue_sum_gather(pr, g, t, pg.ms, pg.ns, pg.ks, A, B, S, T, st);
    if (s) return s;
    PackArgs pa{};
    pa.X = S; pa.rs = St.rows; pa.ks = St.cols; pa.bX = St.bat;
    pa.rows_full = pg.ms; pa.k_full = pg.ks; pa.rows_blk = pg.ms; pa.k_blk = pg.ks;
    pa.nt = 1; pa.t_s[0] = 1;
    pa.tiles = pg.tm; pa.k_pad = pg.k_pad; pa.batch = g.batch; pa.kfast = 1; pa.out = PS;
    TSB_CUDA(launch_pack(pa, st));
    PackArgs pb{};
    pb.X = T; pb.rs = Tt.cols; pb.ks = Tt.rows; pb.bX = Tt.bat;
    pb.rows_full = pg.ns; pb.k_full = pg.ks; pb.rows_blk = pg.ns; pb.k_blk = pg.ks;
    pb.nt = 1; pb.t_s[0] = 1;
    pb.tiles = pg.tn; pb.k_pad = pg.k_pad; pb.batch = g.batch; pb.kfast = 0; pb.out = PT;
    TSB_CUDA(launch_pack(pb, st));
    return TBLIS_STRA_SUCCESS;
}

// shared_err (may be null): a device flag of the caller's that the kernels'
// timed-out waits set; the caller then reads it, and `blocking` checks none.
int run_fp64(int level, int impl, const GemmView& g, const DevPlan& t,
             const double* A, const double* B, double* C, cudaStream_t st, int device, bool blocking,
             int* shared_err = nullptr)
{
    if (g.m == 0 || g.n == 0 || g.batch == 0) return TBLIS_STRA_SUCCESS;
    if (g.alpha == 0.0 || g.k == 0)
    {
        ScaleArgs s{C, t.rsC, t.csC, t.bC, g.m, g.n, g.batch, g.beta};
        TSB_CUDA(launch_scale(s, st));
        return TBLIS_STRA_SUCCESS;
    }
    const ProductTable& tab = product_table(level);
    const int H = tab.H;
    const int64_t ms = cdiv(g.m, H), ns = cdiv(g.n, tab.Hn), ks = cdiv(g.k, tab.Hk);
    const int sms = num_sms(device);

    if (level == 0 || impl == 1)
    {
        // Packed schedule (per product: pack the operand sums, GEMM with the
        // +-M update in its epilogue) when its workspace is allowed; else the
        // fully fused kernel, which needs none.
        const PackGeom pg = pack_geom(level, g);
        if (pg.fits && fp64_packed_workspace_bytes(level, g) <= t_ws_limit)
            return run_fp64_packed(level, g, t, A, B, C, st, sms, blocking, shared_err);
        DmmaArgs a = base_args(g, t, A, B, C);
        set_grid(a, ms, ns, ks);
        a.nprod = (int)tab.prod.size();
        a.H = a.Hc = H;
        a.Hk = tab.Hk; a.Hn = tab.Hn;
        for (int p = 0; p < a.nprod; p++) a.prod[p] = to_dev(tab.prod[p]);
        // The producer/consumer fused kernel; the earlier all-warps kernel
        // where it cannot run these arguments.
        Scratch ferr;
        int* err = shared_err;
        int s;
        if (!err && blocking)
        {
            if ((s = ferr.alloc(sizeof(int), st))) return s;
            TSB_CUDA(cudaMemsetAsync(ferr.p, 0, sizeof(int), st));
            err = static_cast<int*>(ferr.p);
        }
        cudaError_t e = launch_fused(a, st, sms, err, wait_limit_cycles(), &g);
        if (e == cudaErrorNotSupported)
        {
            if (tab.Hk != H || tab.Hn != H) return TBLIS_STRA_ERR_UNSUPPORTED;   // square grids only there
            e = launch_dmma(a, max_terms(tab), st, sms);
        }
        TSB_CUDA(e);
        if (blocking && !shared_err)
        {
            int flag = 0;
            TSB_CUDA(cudaMemcpyAsync(&flag, ferr.p, sizeof(int), cudaMemcpyDeviceToHost, st));
            TSB_CUDA(cudaStreamSynchronize(st));
            if (flag) return TBLIS_STRA_ERR_TIMEOUT;
        }
        return TBLIS_STRA_SUCCESS;
    }

    // AB / Naive with room for every product's M: the sums of all products
    // packed (AB straight from A and B; Naive from its dense temporaries S and
    // T, formed product by product), one GEMM launch over all products into
    // their M_p, then one pass adds sum_p W[h][p] M_p into every C block.
    const PackGeom pgp = pack_geom(level, g);
    if (pgp.fits && t_product_parallel != 0 && pgp.ms * pgp.ns < ((int64_t)1 << 31) &&
        fp64_parallel_workspace_bytes(level, g) + (impl == 3 ? (size_t)(g.batch * (ms + ns) * ks) * 8 : 0) <=
            t_ws_limit)
    {
        const bool col_major = m_tables_col_major(g);
        const int np = (int)tab.prod.size();
        const int64_t* mtab = nullptr;
        int s;
        if ((s = plan_m_tables(t, level, pgp.ms, pgp.ns, (int64_t)np * g.batch, col_major, mtab))) return s;
        Scratch wsbuf, errbuf;
        const size_t ws = fp64_parallel_workspace_bytes(level, g);
        if ((s = wsbuf.alloc(ws, st))) return s;
        int* err = shared_err;
        if (!err)
        {
            if ((s = errbuf.alloc(sizeof(int), st))) return s;
            TSB_CUDA(cudaMemsetAsync(errbuf.p, 0, sizeof(int), st));
            err = static_cast<int*>(errbuf.p);
        }
        const int64_t* tb[9] = {t.rsA, t.rsC, t.csB, t.csC, t.ksA, t.ksB, t.bA, t.bB, t.bC};
        if (impl == 2)
        {
            if ((s = run_fp64_parallel_enqueue(level, g, tb, A, B, C, st, sms, wsbuf.p, ws, mtab, col_major, err)))
                return s;
        }
        else
        {
            Scratch Sd, Td;
            DenseTables St, Tt;
            if ((s = Sd.alloc((size_t)(g.batch * ms * ks) * sizeof(double), st))) return s;
            if ((s = Td.alloc((size_t)(g.batch * ks * ns) * sizeof(double), st))) return s;
            if ((s = St.build(ms, ks, g.batch, st))) return s;
            if ((s = Tt.build(ks, ns, g.batch, st))) return s;
            double* PS = static_cast<double*>(wsbuf.p);
            double* PT = PS + (size_t)np * pgp.s_elems;
            for (int p = 0; p < np; p++)
            {
                const Product& pr = tab.prod[(size_t)p];
                if ((s = enqueue_naive_product(pr, g, t, pgp, A, B, static_cast<double*>(Sd.p),
                                               static_cast<double*>(Td.p), St, Tt,
                                               PS + (size_t)p * pgp.s_elems, PT + (size_t)p * pgp.t_elems, st)))
                    return s;
            }
            if ((s = enqueue_products_and_combine(level, g, tb, C, st, sms, wsbuf.p, mtab, col_major, err)))
                return s;
        }
        if (blocking && !shared_err)
        {
            int flag = 0;
            TSB_CUDA(cudaMemcpyAsync(&flag, errbuf.p, sizeof(int), cudaMemcpyDeviceToHost, st));
            TSB_CUDA(cudaStreamSynchronize(st));
            if (flag) return TBLIS_STRA_ERR_TIMEOUT;
        }
        return TBLIS_STRA_SUCCESS;
    }

    // AB / Naive: one M buffer (ms x ns per batch entry), products in order.
    // The product M = S T runs on the packed GEMM: AB packs the operand sums
    // straight from A and B (as ABC does); Naive first forms them as dense
    // temporaries S and T (sum_gather) and packs those.  The GEMM writes M
    // (beta = 0), then scatter_add adds +-alpha*M into the product's C blocks.
    // Sizes beyond the pack grids use the gather-based kernel for M.
    Scratch Mbuf;
    int s = Mbuf.alloc((size_t)(g.batch * ms * ns) * sizeof(double), st);
    if (s) return s;
    double* M = static_cast<double*>(Mbuf.p);
    DenseTables Mt;
    if ((s = Mt.build(ms, ns, g.batch, st))) return s;

    Scratch Sbuf, Tbuf;
    DenseTables St, Tt;
    if (impl == 3)
    {
        if ((s = Sbuf.alloc((size_t)(g.batch * ms * ks) * sizeof(double), st))) return s;
        if ((s = Tbuf.alloc((size_t)(g.batch * ks * ns) * sizeof(double), st))) return s;
        if ((s = St.build(ms, ks, g.batch, st))) return s;
        if ((s = Tt.build(ks, ns, g.batch, st))) return s;
    }
    const PackGeom pg = pack_geom(level, g);
    Scratch Pbuf, errbuf;
    double* PS = nullptr;
    double* PT = nullptr;
    int* err = shared_err;
    if (pg.fits)
    {
        if ((s = Pbuf.alloc((pg.s_elems + pg.t_elems) * sizeof(double), st))) return s;
        PS = static_cast<double*>(Pbuf.p);
        PT = PS + pg.s_elems;
        if (!err)
        {
            if ((s = errbuf.alloc(sizeof(int), st))) return s;
            TSB_CUDA(cudaMemsetAsync(errbuf.p, 0, sizeof(int), st));
            err = static_cast<int*>(errbuf.p);
        }
    }
    const int64_t* tb[9] = {t.rsA, t.rsC, t.csB, t.csC, t.ksA, t.ksB, t.bA, t.bB, t.bC};

    for (const Product& pr : tab.prod)
    {
        if (impl == 3 && !pg.fits)
        {
            if ((s = enqueue_sum_gather(pr, g, t, ms, ns, ks, A, B, static_cast<double*>(Sbuf.p),
                                        static_cast<double*>(Tbuf.p), st)))
                return s;
        }
        if (pg.fits)
        {
            if (impl == 2)
            {
                if ((s = enqueue_pack_product(pr, g, pg, tb, A, B, PS, PT, st))) return s;
            }
            else
            {
                if ((s = enqueue_naive_product(pr, g, t, pg, A, B, static_cast<double*>(Sbuf.p),
                                               static_cast<double*>(Tbuf.p), St, Tt, PS, PT, st)))
                    return s;
            }
            PackedGemmArgs ga{};
            ga.S[0] = PS; ga.T[0] = PT; ga.C = M;
            ga.rsC = Mt.rows; ga.csC = Mt.cols; ga.bC = Mt.bat;
            ga.m = ms; ga.n = ns; ga.ms = ms; ga.ns = ns; ga.k_pad = pg.k_pad;
            ga.tiles_m = pg.tm; ga.tiles_n = pg.tn; ga.batch = g.batch;
            ga.alpha = 1.0; ga.beta = 0.0;
            ga.nprod = 1; ga.H = 1;
            ga.nc[0] = 1; ga.c_s[0][0] = 1; ga.c_first[0][0] = 1;
            ga.err = err;
            ga.wait_limit = wait_limit_cycles();
            TSB_CUDA(launch_packed_gemm(ga, st, sms));
        }
        else
        {
            DmmaArgs a;
            int terms = 1;
            if (impl == 2)
            {
                a = base_args(g, t, A, B, M);
                set_grid(a, ms, ns, ks);
                a.H = H;
                DevProduct d = to_dev(pr);
                terms = std::max<int>(pr.na, pr.nb);
                d.nc = 1; d.c_r[0] = 0; d.c_c[0] = 0; d.c_s[0] = 1; d.c_first[0] = 1;
                a.prod[0] = d;
            }
            else
            {
                std::memset(&a, 0, sizeof a);
                a.A = static_cast<const double*>(Sbuf.p); a.B = static_cast<const double*>(Tbuf.p); a.C = M;
                a.rsA = St.rows; a.ksA = St.cols; a.bA = St.bat;
                a.ksB = Tt.rows; a.csB = Tt.cols; a.bB = Tt.bat;
                a.m = ms; a.n = ns; a.k = ks; a.batch = g.batch;
                a.a_kfast = 1; a.b_kfast = 0;
                set_grid(a, ms, ns, ks);
                a.H = 1;
                DevProduct d{};
                d.na = d.nb = d.nc = 1; d.a_s[0] = d.b_s[0] = d.c_s[0] = 1; d.c_first[0] = 1;
                a.prod[0] = d;
            }
            a.rsC = Mt.rows; a.csC = Mt.cols; a.bC = Mt.bat;
            a.mC = ms; a.nC = ns; a.Hc = 1;
            a.alpha = 1.0; a.beta = 0.0;
            a.nprod = 1;
            TSB_CUDA(launch_dmma(a, terms, st, sms));
        }

        ScatterAddArgs sc{};
        sc.C = C; sc.rsC = t.rsC; sc.csC = t.csC; sc.bC = t.bC;
        sc.m = g.m; sc.n = g.n; sc.ms = ms; sc.ns = ns; sc.batch = g.batch;
        sc.M = M; sc.alpha = g.alpha; sc.beta = g.beta; sc.nc = pr.nc;
        for (int q = 0; q < pr.nc; q++)
        {
            sc.c_r[q] = pr.c[q].r; sc.c_c[q] = pr.c[q].c; sc.c_s[q] = pr.c[q].sign;
            sc.c_first[q] = pr.c_first[q];
        }
        TSB_CUDA(launch_scatter_add(sc, st));
    }
    if (errbuf.p && blocking)
    {
        int flag = 0;
        TSB_CUDA(cudaMemcpyAsync(&flag, errbuf.p, sizeof(int), cudaMemcpyDeviceToHost, st));
        TSB_CUDA(cudaStreamSynchronize(st));
        if (flag) return TBLIS_STRA_ERR_TIMEOUT;
    }
    return TBLIS_STRA_SUCCESS;
}

}  // namespace

PackGeom pack_geom(int level, const GemmView& g)
{
    const ProductTable& tab = product_table(level);
    PackGeom p;
    p.ms = cdiv(g.m, tab.H); p.ns = cdiv(g.n, tab.Hn); p.ks = cdiv(g.k, tab.Hk);
    p.k_pad = cdiv(p.ks, PACK_KSTEP) * PACK_KSTEP;
    p.tm = cdiv(p.ms, PACK_TILE); p.tn = cdiv(p.ns, PACK_TILE);
    p.s_elems = (size_t)(g.batch * p.tm * p.k_pad * PACK_TILE);
    p.t_elems = (size_t)(g.batch * p.tn * p.k_pad * PACK_TILE);
    // pack grids: (k_pad / 32, 2 * tiles, batch)
    p.fits = 2 * p.tm <= 65535 && 2 * p.tn <= 65535 && g.batch <= 65535 && g.batch * p.tm <= 65535 &&
             g.batch * p.tn <= 65535;
    return p;
}

size_t fp64_packed_workspace_bytes(int level, const GemmView& g)
{
    const PackGeom p = pack_geom(level, g);
    return (p.s_elems + p.t_elems) * sizeof(double);
}

size_t fp64_packed_group_workspace_bytes(int level, const GemmView& g)
{
    const size_t one = fp64_packed_workspace_bytes(level, g);
    return level >= 1 && pack_group(level, 0, 0) ? 7 * one : one;
}

namespace {

// Pack the 7 sums of product group G of one operand (0 = A, 1 = B) into out[].
int enqueue_pack_group(int level, int operand, int G, const GemmView& g, const PackGeom& pg,
                       const int64_t* const tb[9], const double* X, double* const out[7], cudaStream_t st)
{
    const PackGroup* grp = pack_group(level, operand, G);
    if (!grp) return TBLIS_STRA_ERR_UNSUPPORTED;
    PackMultiArgs a{};
    a.X = X;
    if (operand == 0)
    {
        a.rs = tb[0]; a.ks = tb[4]; a.bX = tb[6];
        a.rows_full = g.m; a.rows_blk = pg.ms; a.tiles = pg.tm;
        a.kfast = g.unit_ksA != 0 && (g.unit_rsA == 0 || g.unit_ksA < g.unit_rsA);
    }
    else
    {
        a.rs = tb[2]; a.ks = tb[5]; a.bX = tb[7];
        a.rows_full = g.n; a.rows_blk = pg.ns; a.tiles = pg.tn;
        a.kfast = g.unit_ksB != 0 && (g.unit_csB == 0 || g.unit_ksB < g.unit_csB);
    }
    a.k_full = g.k; a.k_blk = pg.ks; a.k_pad = pg.k_pad; a.batch = g.batch;
    a.nt = grp->nt;
    for (int c = 0; c < grp->nt; c++)
    {
        a.t_s[c] = grp->t_s[c];
        for (int j = 0; j < 4; j++)
        {
            // block (row[j/2], col[j%2]) of the operand; B is packed n-major
            const int br = grp->row[c][j / 2], bc = grp->col[c][j % 2];
            a.prow[c][j] = (int8_t)(operand == 0 ? br : bc);
            a.pk[c][j] = (int8_t)(operand == 0 ? bc : br);
        }
    }
    a.nout = 7;
    for (int q = 0; q < 7; q++)
    {
        a.o_n[q] = grp->o_n[q];
        for (int i = 0; i < grp->o_n[q]; i++) { a.o_j[q][i] = grp->o_j[q][i]; a.o_s[q][i] = grp->o_s[q][i]; }
        a.out[q] = out[q];
    }
    TSB_CUDA(launch_pack_multi(a, st));
    return TBLIS_STRA_SUCCESS;
}

}  // namespace

int enqueue_pack_product(const Product& pr, const GemmView& g, const PackGeom& pg,
                         const int64_t* const tb[9], const double* A, const double* B,
                         double* S, double* T, cudaStream_t st)
{
    const bool a_kfast = g.unit_ksA != 0 && (g.unit_rsA == 0 || g.unit_ksA < g.unit_rsA);
    const bool b_kfast = g.unit_ksB != 0 && (g.unit_csB == 0 || g.unit_ksB < g.unit_csB);
    PackArgs pa{};
    pa.X = A; pa.rs = tb[0]; pa.ks = tb[4]; pa.bX = tb[6];
    pa.rows_full = g.m; pa.k_full = g.k; pa.rows_blk = pg.ms; pa.k_blk = pg.ks;
    pa.nt = pr.na;
    for (int i = 0; i < pr.na; i++) { pa.t_r[i] = pr.a[i].r; pa.t_c[i] = pr.a[i].c; pa.t_s[i] = pr.a[i].sign; }
    pa.tiles = pg.tm; pa.k_pad = pg.k_pad; pa.batch = g.batch; pa.kfast = a_kfast; pa.out = S;
    TSB_CUDA(launch_pack(pa, st));
    PackArgs pb{};
    pb.X = B; pb.rs = tb[2]; pb.ks = tb[5]; pb.bX = tb[7];
    pb.rows_full = g.n; pb.k_full = g.k; pb.rows_blk = pg.ns; pb.k_blk = pg.ks;
    pb.nt = pr.nb;
    for (int i = 0; i < pr.nb; i++) { pb.t_r[i] = pr.b[i].c; pb.t_c[i] = pr.b[i].r; pb.t_s[i] = pr.b[i].sign; }
    pb.tiles = pg.tn; pb.k_pad = pg.k_pad; pb.batch = g.batch; pb.kfast = b_kfast; pb.out = T;
    TSB_CUDA(launch_pack(pb, st));
    return TBLIS_STRA_SUCCESS;
}

PackedGemmArgs packed_gemm_base(int level, const GemmView& g, const PackGeom& pg, const int64_t* const tb[9],
                                double* C, int* err)
{
    PackedGemmArgs ga{};
    ga.err = err;
    ga.wait_limit = wait_limit_cycles();
    ga.C = C;
    ga.rsC = tb[1]; ga.csC = tb[3]; ga.bC = tb[8];
    ga.m = g.m; ga.n = g.n; ga.ms = pg.ms; ga.ns = pg.ns; ga.k_pad = pg.k_pad;
    ga.tiles_m = pg.tm; ga.tiles_n = pg.tn; ga.batch = g.batch;
    ga.alpha = g.alpha; ga.beta = g.beta;
    ga.H = product_table(level).H;
    ga.Hn = product_table(level).Hn;
    ga.nprod = 0;
    return ga;
}

void packed_gemm_add(PackedGemmArgs& a, const Product& pr, const double* S, const double* T)
{
    const int p = a.nprod++;
    a.S[p] = S; a.T[p] = T;
    a.nc[p] = pr.nc;
    for (int q = 0; q < pr.nc; q++)
    {
        a.c_r[p][q] = pr.c[q].r; a.c_c[p][q] = pr.c[q].c; a.c_s[p][q] = pr.c[q].sign;
        a.c_first[p][q] = pr.c_first[q];
    }
}

PackedGemmArgs packed_product_args(int level, const Product& pr, const GemmView& g, const PackGeom& pg,
                                   const int64_t* const tb[9], const double* S, const double* T,
                                   double* C, int* err)
{
    PackedGemmArgs ga = packed_gemm_base(level, g, pg, tb, C, err);
    packed_gemm_add(ga, pr, S, T);
    return ga;
}

// S and T are reused for every product, in stream order.
int run_fp64_packed_enqueue(int level, const GemmView& g, const int64_t* const tb[9],
                            const double* A, const double* B, double* C, cudaStream_t st, int sms,
                            void* ws, size_t ws_bytes, int* err)
{
    const PackGeom pg = pack_geom(level, g);
    if (!pg.fits) return TBLIS_STRA_ERR_TOO_LARGE;
    if (ws_bytes < (pg.s_elems + pg.t_elems) * sizeof(double)) return TBLIS_STRA_ERR_ALLOC;
    const ProductTable& tab = product_table(level);
    if (level >= 1 && fp64_packed_group_workspace_bytes(level, g) > fp64_packed_workspace_bytes(level, g) &&
        ws_bytes >= fp64_packed_group_workspace_bytes(level, g))
    {
        // Grouped sums: per group of 7 products, one pass over A and one over
        // B form all 14 operand sums, then the 7 GEMMs in product order.
        double* S[7];
        double* T[7];
        for (int q = 0; q < 7; q++)
        {
            S[q] = static_cast<double*>(ws) + (size_t)q * pg.s_elems;
            T[q] = static_cast<double*>(ws) + 7 * pg.s_elems + (size_t)q * pg.t_elems;
        }
        const int groups = (int)tab.prod.size() / 7;
        for (int G = 0; G < groups; G++)
        {
            int s;
            if ((s = enqueue_pack_group(level, 0, G, g, pg, tb, A, S, st))) return s;
            if ((s = enqueue_pack_group(level, 1, G, g, pg, tb, B, T, st))) return s;
            // one launch runs the group's 7 products tile by tile: a CTA owns a
            // tile position across them, so their C tiles stay in L2
            PackedGemmArgs ga = packed_gemm_base(level, g, pg, tb, C, err);
            for (int q = 0; q < 7; q++) packed_gemm_add(ga, tab.prod[(size_t)(G * 7 + q)], S[q], T[q]);
            TSB_CUDA(launch_packed_gemm(ga, st, sms));
        }
        return TBLIS_STRA_SUCCESS;
    }
    double* S = static_cast<double*>(ws);
    double* T = S + pg.s_elems;
    for (const Product& pr : tab.prod)
    {
        int s = enqueue_pack_product(pr, g, pg, tb, A, B, S, T, st);
        if (s) return s;
        TSB_CUDA(launch_packed_gemm(packed_product_args(level, pr, g, pg, tb, S, T, C, err), st, sms));
    }
    return TBLIS_STRA_SUCCESS;
}

size_t fp64_parallel_workspace_bytes(int level, const GemmView& g)
{
    const PackGeom pg = pack_geom(level, g);
    const size_t np = product_table(level).prod.size();
    const size_t st = (np * (pg.s_elems + pg.t_elems) * sizeof(double) + 255) / 256 * 256;
    return st + np * (size_t)(g.batch * pg.ms * pg.ns) * sizeof(double);
}

void dense_m_tables(int64_t ms, int64_t ns, int64_t nb, bool col_major, int64_t* out)
{
    for (int64_t i = 0; i < ms; i++) out[i] = col_major ? i : i * ns;
    for (int64_t j = 0; j < ns; j++) out[ms + j] = col_major ? j * ms : j;
    for (int64_t b = 0; b < nb; b++) out[ms + ns + b] = b * ms * ns;
}

// The products' sums are packed back to back (S_p = S + p * s_elems), so the
// GEMM sees product p, batch entry b as batch entry p * batch + b of one
// problem of 7^L * batch entries writing M_p = M + p * batch * ms * ns.
int run_fp64_parallel_enqueue(int level, const GemmView& g, const int64_t* const tb[9],
                              const double* A, const double* B, double* C, cudaStream_t st, int sms,
                              void* ws, size_t ws_bytes, const int64_t* mtab, bool col_major, int* err)
{
    if (level < 1) return TBLIS_STRA_ERR_ARG;
    const PackGeom pg = pack_geom(level, g);
    if (!pg.fits) return TBLIS_STRA_ERR_TOO_LARGE;
    if (ws_bytes < fp64_parallel_workspace_bytes(level, g)) return TBLIS_STRA_ERR_ALLOC;
    const ProductTable& tab = product_table(level);
    const int np = (int)tab.prod.size();
    double* S = static_cast<double*>(ws);
    double* T = S + (size_t)np * pg.s_elems;
    int s;
    if (pack_group(level, 0, 0))
    {
        for (int G = 0; G < np / 7; G++)
        {
            double* outS[7];
            double* outT[7];
            for (int q = 0; q < 7; q++)
            {
                outS[q] = S + (size_t)(G * 7 + q) * pg.s_elems;
                outT[q] = T + (size_t)(G * 7 + q) * pg.t_elems;
            }
            if ((s = enqueue_pack_group(level, 0, G, g, pg, tb, A, outS, st))) return s;
            if ((s = enqueue_pack_group(level, 1, G, g, pg, tb, B, outT, st))) return s;
        }
    }
    else
    {
        for (int p = 0; p < np; p++)
            if ((s = enqueue_pack_product(tab.prod[(size_t)p], g, pg, tb, A, B, S + (size_t)p * pg.s_elems,
                                          T + (size_t)p * pg.t_elems, st)))
                return s;
    }
    return enqueue_products_and_combine(level, g, tb, C, st, sms, ws, mtab, col_major, err);
}

// The GEMM over all products (their sums packed back to back at the start
// of ws) into M_p, then the combine launch.
int enqueue_products_and_combine(int level, const GemmView& g, const int64_t* const tb[9], double* C,
                                 cudaStream_t st, int sms, void* ws, const int64_t* mtab, bool col_major,
                                 int* err)
{
    const PackGeom pg = pack_geom(level, g);
    const ProductTable& tab = product_table(level);
    const int np = (int)tab.prod.size();
    double* S = static_cast<double*>(ws);
    double* T = S + (size_t)np * pg.s_elems;
    double* M = reinterpret_cast<double*>(static_cast<char*>(ws) +
                                          ((size_t)np * (pg.s_elems + pg.t_elems) * sizeof(double) + 255) / 256 * 256);
    PackedGemmArgs ga{};
    ga.err = err;
    ga.wait_limit = wait_limit_cycles();
    ga.C = M;
    ga.rsC = mtab; ga.csC = mtab + pg.ms; ga.bC = mtab + pg.ms + pg.ns;
    ga.m = pg.ms; ga.n = pg.ns; ga.ms = pg.ms; ga.ns = pg.ns; ga.k_pad = pg.k_pad;
    ga.tiles_m = pg.tm; ga.tiles_n = pg.tn; ga.batch = (int64_t)np * g.batch;
    ga.alpha = 1.0; ga.beta = 0.0;
    ga.H = 1; ga.nprod = 1;
    ga.S[0] = S; ga.T[0] = T;
    ga.nc[0] = 1; ga.c_s[0][0] = 1; ga.c_first[0][0] = 1;
    TSB_CUDA(launch_packed_gemm(ga, st, sms));

    CombineArgs c{};
    c.C = C; c.rsC = tb[1]; c.csC = tb[3]; c.bC = tb[8];
    c.m = g.m; c.n = g.n; c.ms = pg.ms; c.ns = pg.ns; c.batch = g.batch;
    c.M = M; c.m_pstride = g.batch * pg.ms * pg.ns;
    c.alpha = g.alpha; c.beta = g.beta;
    c.H = tab.H; c.col_major = col_major ? 1 : 0;
    if (np > MAX_COMBINE_PRODUCTS) return TBLIS_STRA_ERR_UNSUPPORTED;
    c.np = np;
    for (int p = 0; p < np; p++)
    {
        const Product& pr = tab.prod[(size_t)p];
        c.nt[p] = (int8_t)pr.nc;
        for (int q = 0; q < pr.nc; q++)
        {
            c.th[p][q] = (int8_t)(pr.c[q].r * tab.H + pr.c[q].c);
            c.ts[p][q] = pr.c[q].sign;
        }
    }
    TSB_CUDA(launch_combine(c, st));
    return TBLIS_STRA_SUCCESS;
}

// ---- k-split plain contraction (L = 0, few tiles) ----------------------------
//
// When the C tiles of a plain contraction are fewer than the SMs, the summed
// range is cut into P pieces of kq (a multiple of the pack k-step): piece p is
// packed as the "product" A(:, piece p) B(piece p, :), the P pieces run side by
// side in one GEMM launch into their own M_p (batch entry p * batch + b), and
// the combine pass forms C = alpha * sum_p M_p + beta * C in FP64 in piece
// order.  No counterpart in the reference, whose threads split the loops of
// the one GEMM instead.

PackGeom ksplit_geom(const GemmView& g, int P)
{
    PackGeom p;
    p.ms = g.m; p.ns = g.n;
    p.ks = cdiv(cdiv(g.k, P), PACK_KSTEP) * PACK_KSTEP;
    p.k_pad = p.ks;
    p.tm = cdiv(p.ms, PACK_TILE); p.tn = cdiv(p.ns, PACK_TILE);
    p.s_elems = (size_t)(g.batch * p.tm * p.k_pad * PACK_TILE);
    p.t_elems = (size_t)(g.batch * p.tn * p.k_pad * PACK_TILE);
    p.fits = 2 * p.tm <= 65535 && 2 * p.tn <= 65535 && g.batch <= 65535 && g.batch * p.tm <= 65535 &&
             g.batch * p.tn <= 65535;
    return p;
}

int ksplit_pieces(const GemmView& g, int sms)
{
    const int64_t tiles = g.batch * cdiv(g.m, PACK_TILE) * cdiv(g.n, PACK_TILE);
    if (tiles >= sms || g.k < 1024 || g.m * g.n >= ((int64_t)1 << 31)) return 1;
    int64_t P = cdiv(2 * (int64_t)sms, tiles);
    P = std::min<int64_t>(P, g.k / 512);
    P = std::min<int64_t>(P, MAX_COMBINE_PRODUCTS);
    return (int)std::max<int64_t>(P, 1);
}

size_t fp64_ksplit_workspace_bytes(const GemmView& g, int P)
{
    const PackGeom pg = ksplit_geom(g, P);
    const size_t st = ((size_t)P * (pg.s_elems + pg.t_elems) * sizeof(double) + 255) / 256 * 256;
    return st + (size_t)P * (size_t)(g.batch * g.m * g.n) * sizeof(double);
}

int run_fp64_ksplit_enqueue(const GemmView& g, const int64_t* const tb[9], const double* A, const double* B,
                            double* C, cudaStream_t st, int sms, void* ws, size_t ws_bytes, int P,
                            const int64_t* mtab, bool col_major, int* err)
{
    if (P < 2 || P > MAX_COMBINE_PRODUCTS) return TBLIS_STRA_ERR_ARG;
    const PackGeom pg = ksplit_geom(g, P);
    if (!pg.fits) return TBLIS_STRA_ERR_TOO_LARGE;
    if (ws_bytes < fp64_ksplit_workspace_bytes(g, P)) return TBLIS_STRA_ERR_ALLOC;
    double* S = static_cast<double*>(ws);
    double* T = S + (size_t)P * pg.s_elems;
    double* M = reinterpret_cast<double*>(static_cast<char*>(ws) +
                                          ((size_t)P * (pg.s_elems + pg.t_elems) * sizeof(double) + 255) / 256 * 256);
    // One pack launch per operand over all P * kq summed indices, each piece
    // written as its own batch entries (kpiece).
    for (int operand = 0; operand < 2; operand++)
    {
        PackArgs pa{};
        if (operand == 0)
        {
            pa.X = A; pa.rs = tb[0]; pa.ks = tb[4]; pa.bX = tb[6];
            pa.rows_full = g.m; pa.rows_blk = g.m; pa.tiles = pg.tm; pa.out = S;
            pa.kfast = g.unit_ksA != 0 && (g.unit_rsA == 0 || g.unit_ksA < g.unit_rsA);
        }
        else
        {
            pa.X = B; pa.rs = tb[2]; pa.ks = tb[5]; pa.bX = tb[7];
            pa.rows_full = g.n; pa.rows_blk = g.n; pa.tiles = pg.tn; pa.out = T;
            pa.kfast = g.unit_ksB != 0 && (g.unit_csB == 0 || g.unit_ksB < g.unit_csB);
        }
        pa.k_full = g.k; pa.k_blk = (int64_t)P * pg.ks;
        pa.nt = 1; pa.t_r[0] = 0; pa.t_c[0] = 0; pa.t_s[0] = 1;
        pa.k_pad = (int64_t)P * pg.k_pad; pa.batch = g.batch; pa.kpiece = pg.k_pad;
        TSB_CUDA(launch_pack(pa, st));
    }
    PackedGemmArgs ga{};
    ga.err = err;
    ga.wait_limit = wait_limit_cycles();
    ga.C = M;
    ga.rsC = mtab; ga.csC = mtab + g.m; ga.bC = mtab + g.m + g.n;
    ga.m = g.m; ga.n = g.n; ga.ms = g.m; ga.ns = g.n; ga.k_pad = pg.k_pad;
    ga.tiles_m = pg.tm; ga.tiles_n = pg.tn; ga.batch = (int64_t)P * g.batch;
    ga.alpha = 1.0; ga.beta = 0.0;
    ga.H = 1; ga.nprod = 1;
    ga.S[0] = S; ga.T[0] = T;
    ga.nc[0] = 1; ga.c_s[0][0] = 1; ga.c_first[0][0] = 1;
    TSB_CUDA(launch_packed_gemm(ga, st, sms));

    CombineArgs c{};
    c.C = C; c.rsC = tb[1]; c.csC = tb[3]; c.bC = tb[8];
    c.m = g.m; c.n = g.n; c.ms = g.m; c.ns = g.n; c.batch = g.batch;
    c.M = M; c.m_pstride = g.batch * g.m * g.n;
    c.alpha = g.alpha; c.beta = g.beta;
    c.H = 1; c.col_major = col_major ? 1 : 0;
    c.np = P;
    for (int p = 0; p < P; p++) { c.nt[p] = 1; c.th[p][0] = 0; c.ts[p][0] = 1; }
    TSB_CUDA(launch_combine(c, st));
    return TBLIS_STRA_SUCCESS;
}

// Host -> device copy that has landed when this returns.  cudaMemcpy from
// pageable memory may return before its DMA completes, and kernels on
// non-blocking streams are not ordered after it, so tables read by such
// kernels go through a private non-blocking stream per device, synchronised.
long long wait_limit_cycles()
{
    if (!t_wait_inject) return t_wait_limit;
    return t_wait_limit > 0 ? -t_wait_limit : -1000;
}
size_t alloc_limit_bytes() { return t_alloc_limit; }

int upload_complete(void* dst, const void* src, size_t bytes)
{
    static std::mutex mu;
    static std::map<int, cudaStream_t> streams;
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) { cudaGetLastError(); return TBLIS_STRA_ERR_NO_DEVICE; }
    cudaStream_t st = nullptr;
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = streams.find(device);
        if (it == streams.end())
        {
            if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess)
            {
                cudaGetLastError();
                return TBLIS_STRA_ERR_CUDA;
            }
            streams[device] = st;
        }
        else st = it->second;
    }
    TSB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st));
    TSB_CUDA(cudaStreamSynchronize(st));
    return TBLIS_STRA_SUCCESS;
}

void note_cuda_error(const char* what, cudaError_t e, const char* file, int line)
{
    const char* base = std::strrchr(file, '/');
    t_detail = std::string(base ? base + 1 : file) + ":" + std::to_string(line) + " " + what + ": " +
               cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    cudaGetLastError();
}

void note_detail(const std::string& what) { t_detail = what; }

void clear_detail() { t_detail.clear(); }

// FP32 contraction: split-BF16 tcgen05 path (bf16_split.cu), Strassen products
// in stream order like the packed FP64 schedule.  Workspace layout: row and
// column scales, A planes, B planes.
size_t fp32_workspace_bytes(int level, const GemmView& g, int terms)
{
    const ProductTable& tab = product_table(level);
    const int H = tab.H;
    const int64_t ms = cdiv(g.m, H), ns = cdiv(g.n, H), ks = cdiv(g.k, H);
    const int64_t nk = cdiv(ks, SPLIT_K);
    const int64_t tm = cdiv(ms, SPLIT_TILE), tn = cdiv(ns, SPLIT_TILE);
    const int P = terms == 3 ? 2 : 3;
    const size_t blk = (size_t)SPLIT_TILE * SPLIT_K * 2;
    const size_t sc = ((size_t)g.batch * (ms + ns) * 2 * sizeof(float) + 255) / 256 * 256;
    return sc + (size_t)P * g.batch * (tm + tn) * nk * blk;
}

size_t fp32_group_workspace_bytes(int level, const GemmView& g, int terms)
{
    const size_t one = fp32_workspace_bytes(level, g, terms);
    if (level < 1 || !pack_group(level, 0, 0)) return one;
    const int H = product_table(level).H;
    const int64_t ms = cdiv(g.m, H), ns = cdiv(g.n, H);
    const size_t sc = ((size_t)g.batch * (ms + ns) * 2 * sizeof(float) + 255) / 256 * 256;
    return sc + 7 * (one - sc);
}

namespace {

// The split sums of product group G of one operand (0 = A, 1 = B) from one
// pass over it, scaled by `scale` and split into P bf16 planes at out[q].
int enqueue_split_pack_group(int level, int operand, int G, const GemmView& g, const int64_t* const tb[9],
                             const float* X, const float* scale, int P, void* const out[7], cudaStream_t st)
{
    const PackGroup* grp = pack_group(level, operand, G);
    if (!grp) return TBLIS_STRA_ERR_UNSUPPORTED;
    const int H = product_table(level).H;
    const int64_t ms = cdiv(g.m, H), ns = cdiv(g.n, H), ks = cdiv(g.k, H);
    SplitPackMultiArgs m{};
    m.X = X;
    if (operand == 0)
    {
        m.rs = tb[0]; m.ks = tb[4]; m.bX = tb[6];
        m.rows_full = g.m; m.rows_blk = ms; m.tiles = cdiv(ms, SPLIT_TILE);
        m.kfast = g.unit_ksA != 0 && (g.unit_rsA == 0 || g.unit_ksA < g.unit_rsA);
    }
    else
    {
        m.rs = tb[2]; m.ks = tb[5]; m.bX = tb[7];
        m.rows_full = g.n; m.rows_blk = ns; m.tiles = cdiv(ns, SPLIT_TILE);
        m.kfast = g.unit_ksB != 0 && (g.unit_csB == 0 || g.unit_ksB < g.unit_csB);
    }
    m.scale = scale;
    m.k_full = g.k; m.k_blk = ks; m.nk = cdiv(ks, SPLIT_K); m.batch = g.batch; m.planes = P;
    m.nt = grp->nt;
    for (int c = 0; c < grp->nt; c++)
    {
        m.t_s[c] = grp->t_s[c];
        for (int j = 0; j < 4; j++)
        {
            // block (row[j/2], col[j%2]) of the operand; B is packed n-major
            const int br = grp->row[c][j / 2], bc = grp->col[c][j % 2];
            m.prow[c][j] = (int8_t)(operand == 0 ? br : bc);
            m.pk[c][j] = (int8_t)(operand == 0 ? bc : br);
        }
    }
    m.nout = 7;
    for (int q = 0; q < 7; q++)
    {
        m.o_n[q] = grp->o_n[q];
        for (int i = 0; i < grp->o_n[q]; i++) { m.o_j[q][i] = grp->o_j[q][i]; m.o_s[q][i] = grp->o_s[q][i]; }
        m.out[q] = out[q];
    }
    TSB_CUDA(launch_split_pack_multi(m, st));
    return TBLIS_STRA_SUCCESS;
}

}  // namespace

int run_fp32_enqueue(int level, const GemmView& g, const int64_t* const tb[9], const float* A,
                     const float* B, float* C, cudaStream_t st, int sms, void* ws, size_t ws_bytes,
                     int terms, int* err, SplitGemmArgs* defer, bool enqueue)
{
    // tb: rsA, rsC, csB, csC, ksA, ksB, bA, bB, bC
    if (defer && level != 0) return TBLIS_STRA_ERR_ARG;
    const ProductTable& tab = product_table(level);
    const int H = tab.H;
    const int64_t ms = cdiv(g.m, H), ns = cdiv(g.n, H), ks = cdiv(g.k, H);
    const int64_t nk = cdiv(ks, SPLIT_K);
    const int64_t tm = cdiv(ms, SPLIT_TILE), tn = cdiv(ns, SPLIT_TILE);
    if (g.batch * tm > 65535 || g.batch * tn > 65535 || nk > 2147483647) return TBLIS_STRA_ERR_TOO_LARGE;
    if (ws_bytes < fp32_workspace_bytes(level, g, terms)) return TBLIS_STRA_ERR_ALLOC;
    const bool grouped = level >= 1 && fp32_group_workspace_bytes(level, g, terms) > fp32_workspace_bytes(level, g, terms) &&
                         ws_bytes >= fp32_group_workspace_bytes(level, g, terms);
    const int P = terms == 3 ? 2 : 3;
    const size_t blk = (size_t)SPLIT_TILE * SPLIT_K * 2;
    const size_t sc = ((size_t)g.batch * (ms + ns) * 2 * sizeof(float) + 255) / 256 * 256;
    float* scaleA = static_cast<float*>(ws);
    float* invA = scaleA + g.batch * ms;
    float* scaleB = invA + g.batch * ms;
    float* invB = scaleB + g.batch * ns;
    void* planesA = static_cast<char*>(ws) + sc;
    void* planesB = static_cast<char*>(planesA) + (size_t)P * g.batch * tm * nk * blk;

    if (enqueue)
    {
        SplitScaleArgs sa{A, tb[0], tb[4], tb[6], g.m, g.k, ms, H, g.batch, scaleA, invA};
        TSB_CUDA(launch_split_scale(sa, st));
        SplitScaleArgs sb{B, tb[2], tb[5], tb[7], g.n, g.k, ns, H, g.batch, scaleB, invB};
        TSB_CUDA(launch_split_scale(sb, st));
    }

    const bool a_kfast = g.unit_ksA != 0 && (g.unit_rsA == 0 || g.unit_ksA < g.unit_rsA);
    const bool b_kfast = g.unit_ksB != 0 && (g.unit_csB == 0 || g.unit_ksB < g.unit_csB);
    static const int8_t TA6[6] = {0, 0, 1, 0, 1, 2}, TB6[6] = {0, 1, 0, 2, 1, 0};
    // One GEMM launch over `n` products that share the tile grid: each CTA
    // runs all of them for its tile position, in the order given.
    auto gemm = [&](const Product* const* prs, const void* const* pA, const void* const* pB, int n) -> int {
        SplitGemmArgs ga{};
        ga.C = C;
        ga.rsC = tb[1]; ga.csC = tb[3]; ga.bC = tb[8];
        ga.invA = invA; ga.invB = invB;
        ga.m = g.m; ga.n = g.n; ga.ms = ms; ga.ns = ns; ga.nk = nk;
        ga.tiles_m = tm; ga.tiles_n = tn; ga.batch = g.batch;
        ga.alpha = (float)g.alpha; ga.beta = (float)g.beta;
        ga.nprod = n; ga.H = H;
        for (int p = 0; p < n; p++)
        {
            const Product& pr = *prs[p];
            ga.A[p] = pA[p]; ga.B[p] = pB[p];
            ga.nc[p] = (int8_t)pr.nc;
            for (int q = 0; q < pr.nc; q++)
            {
                ga.c_r[p][q] = pr.c[q].r; ga.c_c[p][q] = pr.c[q].c; ga.c_s[p][q] = pr.c[q].sign;
                ga.c_first[p][q] = pr.c_first[q];
            }
        }
        ga.planes = P;
        ga.nterms = P == 3 ? 6 : 3;
        for (int i = 0; i < 6; i++) { ga.ta[i] = TA6[i]; ga.tb[i] = TB6[i]; }
        ga.err = err;
        ga.wait_limit = wait_limit_cycles();
        if (defer) { *defer = ga; return TBLIS_STRA_SUCCESS; }
        TSB_CUDA(launch_split_gemm(ga, st, sms));
        return TBLIS_STRA_SUCCESS;
    };
    if (grouped)
    {
        // Per group of 7 products: one pass over A and one over B form the 14
        // split sums (7 plane sets each), then one GEMM launch runs the 7
        // products in product order for each tile position.
        const size_t bytesA = (size_t)P * g.batch * tm * nk * blk, bytesB = (size_t)P * g.batch * tn * nk * blk;
        char* base = static_cast<char*>(ws) + sc;
        void* outA[7];
        void* outB[7];
        for (int q = 0; q < 7; q++)
        {
            outA[q] = base + q * bytesA;
            outB[q] = base + 7 * bytesA + q * bytesB;
        }
        for (int G = 0; G < (int)tab.prod.size() / 7; G++)
        {
            for (int operand = 0; operand < 2; operand++)
            {
                const int s = enqueue_split_pack_group(level, operand, G, g, tb, operand == 0 ? A : B,
                                                       operand == 0 ? scaleA : scaleB, P,
                                                       operand == 0 ? outA : outB, st);
                if (s) return s;
            }
            const Product* prs[7];
            for (int q = 0; q < 7; q++) prs[q] = &tab.prod[(size_t)(G * 7 + q)];
            const int s = gemm(prs, outA, outB, 7);
            if (s) return s;
        }
        return TBLIS_STRA_SUCCESS;
    }
    for (const Product& pr : tab.prod)
    {
        SplitPackArgs pa{};
        pa.X = A; pa.rs = tb[0]; pa.ks = tb[4]; pa.bX = tb[6];
        pa.rows_full = g.m; pa.k_full = g.k; pa.rows_blk = ms; pa.k_blk = ks;
        pa.nt = pr.na;
        for (int i = 0; i < pr.na; i++) { pa.t_r[i] = pr.a[i].r; pa.t_c[i] = pr.a[i].c; pa.t_s[i] = pr.a[i].sign; }
        pa.scale = scaleA; pa.tiles = tm; pa.nk = nk; pa.batch = g.batch; pa.planes = P;
        pa.kfast = a_kfast; pa.out = planesA;
        if (enqueue) TSB_CUDA(launch_split_pack(pa, st));
        SplitPackArgs pb{};
        pb.X = B; pb.rs = tb[2]; pb.ks = tb[5]; pb.bX = tb[7];
        pb.rows_full = g.n; pb.k_full = g.k; pb.rows_blk = ns; pb.k_blk = ks;
        pb.nt = pr.nb;
        for (int i = 0; i < pr.nb; i++) { pb.t_r[i] = pr.b[i].c; pb.t_c[i] = pr.b[i].r; pb.t_s[i] = pr.b[i].sign; }
        pb.scale = scaleB; pb.tiles = tn; pb.nk = nk; pb.batch = g.batch; pb.planes = P;
        pb.kfast = b_kfast; pb.out = planesB;
        if (enqueue) TSB_CUDA(launch_split_pack(pb, st));
        const Product* one = &pr;
        const void* pA1 = planesA;
        const void* pB1 = planesB;
        const int s = gemm(&one, &pA1, &pB1, 1);
        if (s) return s;
    }
    return TBLIS_STRA_SUCCESS;
}

size_t fp32_parallel_workspace_bytes(int level, const GemmView& g, int terms)
{
    const int H = product_table(level).H;
    const size_t np = product_table(level).prod.size();
    const int64_t ms = cdiv(g.m, H), ns = cdiv(g.n, H), ks = cdiv(g.k, H);
    const int64_t nk = cdiv(ks, SPLIT_K);
    const size_t blk = (size_t)SPLIT_TILE * SPLIT_K * 2;
    const int P = terms == 3 ? 2 : 3;
    const size_t sc = ((size_t)g.batch * (ms + ns) * 2 * sizeof(float) + 255) / 256 * 256;
    const size_t planes = np * P * (size_t)g.batch * (cdiv(ms, SPLIT_TILE) + cdiv(ns, SPLIT_TILE)) * nk * blk;
    return sc + planes + np * (size_t)(g.batch * ms * ns) * sizeof(float);
}

bool use_product_parallel(int level, const GemmView& g, int sms, bool fp32, int terms)
{
    if (level < 1 || t_product_parallel == 0 || thread_algorithm() != 0) return false;
    const int H = product_table(level).H;
    const int64_t ms = cdiv(g.m, H), ns = cdiv(g.n, H);
    if (ms * ns >= ((int64_t)1 << 31)) return false;
    int64_t tiles;
    if (fp32)
    {
        if (!pack_group(level, 0, 0) || fp32_parallel_workspace_bytes(level, g, terms) > t_ws_limit) return false;
        tiles = g.batch * cdiv(ms, SPLIT_TILE) * cdiv(ns, SPLIT_TILE);
    }
    else
    {
        const PackGeom pg = pack_geom(level, g);
        if (!pg.fits || fp64_parallel_workspace_bytes(level, g) > t_ws_limit) return false;
        tiles = g.batch * pg.tm * pg.tn;
    }
    return t_product_parallel == 1 || parallel_pays(level, fp32, tiles, sms, ms, ns);
}

bool m_tables_col_major(const GemmView& g)
{
    return g.unit_rsC != 0 && (g.unit_csC == 0 || g.unit_rsC <= g.unit_csC);
}

// Product-parallel split-BF16 schedule (L >= 1): row and column scales, the
// split sums of every product (plane set p of A at planesA + p * bytesA, of B
// likewise), one GEMM launch over all products (batch entry p * batch + b
// reads plane set p) into M_p, then one combine launch into C.
int run_fp32_parallel_enqueue(int level, const GemmView& g, const int64_t* const tb[9], const float* A,
                              const float* B, float* C, cudaStream_t st, int sms, void* ws, size_t ws_bytes,
                              int terms, const int64_t* mtab, bool col_major, int* err)
{
    if (level < 1) return TBLIS_STRA_ERR_ARG;
    const ProductTable& tab = product_table(level);
    const int H = tab.H;
    const int np = (int)tab.prod.size();
    const int64_t ms = cdiv(g.m, H), ns = cdiv(g.n, H), ks = cdiv(g.k, H);
    const int64_t nk = cdiv(ks, SPLIT_K);
    const int64_t tm = cdiv(ms, SPLIT_TILE), tn = cdiv(ns, SPLIT_TILE);
    if (g.batch * tm > 65535 || g.batch * tn > 65535 || nk > 2147483647) return TBLIS_STRA_ERR_TOO_LARGE;
    if (ws_bytes < fp32_parallel_workspace_bytes(level, g, terms)) return TBLIS_STRA_ERR_ALLOC;
    const int P = terms == 3 ? 2 : 3;
    const size_t blk = (size_t)SPLIT_TILE * SPLIT_K * 2;
    const size_t sc = ((size_t)g.batch * (ms + ns) * 2 * sizeof(float) + 255) / 256 * 256;
    float* scaleA = static_cast<float*>(ws);
    float* invA = scaleA + g.batch * ms;
    float* scaleB = invA + g.batch * ms;
    float* invB = scaleB + g.batch * ns;
    const size_t bytesA = (size_t)P * g.batch * tm * nk * blk, bytesB = (size_t)P * g.batch * tn * nk * blk;
    char* planesA = static_cast<char*>(ws) + sc;
    char* planesB = planesA + np * bytesA;
    float* M = reinterpret_cast<float*>(planesB + np * bytesB);

    SplitScaleArgs sa{A, tb[0], tb[4], tb[6], g.m, g.k, ms, H, g.batch, scaleA, invA};
    TSB_CUDA(launch_split_scale(sa, st));
    SplitScaleArgs sb{B, tb[2], tb[5], tb[7], g.n, g.k, ns, H, g.batch, scaleB, invB};
    TSB_CUDA(launch_split_scale(sb, st));

    if (!pack_group(level, 0, 0)) return TBLIS_STRA_ERR_UNSUPPORTED;
    for (int G = 0; G < np / 7; G++)
    {
        void* outA[7];
        void* outB[7];
        for (int q = 0; q < 7; q++)
        {
            outA[q] = planesA + (size_t)(G * 7 + q) * bytesA;
            outB[q] = planesB + (size_t)(G * 7 + q) * bytesB;
        }
        int s;
        if ((s = enqueue_split_pack_group(level, 0, G, g, tb, A, scaleA, P, outA, st))) return s;
        if ((s = enqueue_split_pack_group(level, 1, G, g, tb, B, scaleB, P, outB, st))) return s;
    }

    static const int8_t TA6[6] = {0, 0, 1, 0, 1, 2}, TB6[6] = {0, 1, 0, 2, 1, 0};
    SplitGemmArgs ga{};
    ga.A[0] = planesA; ga.B[0] = planesB; ga.C = M;
    ga.rsC = mtab; ga.csC = mtab + ms; ga.bC = mtab + ms + ns;
    ga.invA = invA; ga.invB = invB;
    ga.m = ms; ga.n = ns; ga.ms = ms; ga.ns = ns; ga.nk = nk;
    ga.tiles_m = tm; ga.tiles_n = tn; ga.batch = (int64_t)np * g.batch; ga.pbatch = g.batch;
    ga.alpha = 1.f; ga.beta = 0.f;
    ga.nprod = 1; ga.H = 1;
    ga.nc[0] = 1; ga.c_s[0][0] = 1; ga.c_first[0][0] = 1;
    ga.planes = P;
    ga.nterms = P == 3 ? 6 : 3;
    for (int i = 0; i < 6; i++) { ga.ta[i] = TA6[i]; ga.tb[i] = TB6[i]; }
    ga.err = err;
    ga.wait_limit = wait_limit_cycles();
    TSB_CUDA(launch_split_gemm(ga, st, sms));

    CombineF32Args c{};
    c.C = C; c.rsC = tb[1]; c.csC = tb[3]; c.bC = tb[8];
    c.m = g.m; c.n = g.n; c.ms = ms; c.ns = ns; c.batch = g.batch;
    c.M = M; c.m_pstride = g.batch * ms * ns;
    c.alpha = g.alpha; c.beta = g.beta;
    c.H = H; c.col_major = col_major ? 1 : 0;
    if (np > MAX_COMBINE_PRODUCTS) return TBLIS_STRA_ERR_UNSUPPORTED;
    c.np = np;
    for (int p = 0; p < np; p++)
    {
        const Product& pr = tab.prod[(size_t)p];
        c.nt[p] = (int8_t)pr.nc;
        for (int q = 0; q < pr.nc; q++)
        {
            c.th[p][q] = (int8_t)(pr.c[q].r * H + pr.c[q].c);
            c.ts[p][q] = pr.c[q].sign;
        }
    }
    TSB_CUDA(launch_combine(c, st));
    return TBLIS_STRA_SUCCESS;
}

// k-split of a plain FP32 contraction (as run_fp64_ksplit_enqueue): the row
// and column scales over the whole summed range, the split planes of each
// piece (plane set p), one split GEMM over P * batch entries into M_p (FP32),
// and the combine pass summing the pieces in FP64.
size_t fp32_ksplit_workspace_bytes(const GemmView& g, int P, int terms)
{
    const int64_t kq = cdiv(cdiv(g.k, P), SPLIT_K) * SPLIT_K;
    const int64_t nk = kq / SPLIT_K;
    const size_t blk = (size_t)SPLIT_TILE * SPLIT_K * 2;
    const int planes = terms == 3 ? 2 : 3;
    const size_t sc = ((size_t)g.batch * (g.m + g.n) * 2 * sizeof(float) + 255) / 256 * 256;
    const size_t pl = (size_t)P * planes * g.batch * (cdiv(g.m, SPLIT_TILE) + cdiv(g.n, SPLIT_TILE)) * nk * blk;
    return sc + pl + (size_t)P * (size_t)(g.batch * g.m * g.n) * sizeof(float);
}

int run_fp32_ksplit_enqueue(const GemmView& g, const int64_t* const tb[9], const float* A, const float* B,
                            float* C, cudaStream_t st, int sms, void* ws, size_t ws_bytes, int terms, int P,
                            const int64_t* mtab, bool col_major, int* err)
{
    if (P < 2 || P > MAX_COMBINE_PRODUCTS) return TBLIS_STRA_ERR_ARG;
    const int64_t kq = cdiv(cdiv(g.k, P), SPLIT_K) * SPLIT_K;
    const int64_t nk = kq / SPLIT_K;
    const int64_t tm = cdiv(g.m, SPLIT_TILE), tn = cdiv(g.n, SPLIT_TILE);
    if (g.batch * tm > 65535 || g.batch * tn > 65535) return TBLIS_STRA_ERR_TOO_LARGE;
    if (ws_bytes < fp32_ksplit_workspace_bytes(g, P, terms)) return TBLIS_STRA_ERR_ALLOC;
    const int planes = terms == 3 ? 2 : 3;
    const size_t blk = (size_t)SPLIT_TILE * SPLIT_K * 2;
    const size_t sc = ((size_t)g.batch * (g.m + g.n) * 2 * sizeof(float) + 255) / 256 * 256;
    float* scaleA = static_cast<float*>(ws);
    float* invA = scaleA + g.batch * g.m;
    float* scaleB = invA + g.batch * g.m;
    float* invB = scaleB + g.batch * g.n;
    const size_t bytesA = (size_t)planes * g.batch * tm * nk * blk, bytesB = (size_t)planes * g.batch * tn * nk * blk;
    char* planesA = static_cast<char*>(ws) + sc;
    char* planesB = planesA + P * bytesA;
    float* M = reinterpret_cast<float*>(planesB + P * bytesB);

    SplitScaleArgs sa{A, tb[0], tb[4], tb[6], g.m, g.k, g.m, 1, g.batch, scaleA, invA};
    TSB_CUDA(launch_split_scale(sa, st));
    SplitScaleArgs sb{B, tb[2], tb[5], tb[7], g.n, g.k, g.n, 1, g.batch, scaleB, invB};
    TSB_CUDA(launch_split_scale(sb, st));
    // One split-pack launch per operand over all P * kq summed indices, each
    // piece written as its own plane set (nkpiece).
    SplitPackArgs pa{};
    pa.X = A; pa.rs = tb[0]; pa.ks = tb[4]; pa.bX = tb[6];
    pa.rows_full = g.m; pa.k_full = g.k; pa.rows_blk = g.m; pa.k_blk = (int64_t)P * kq;
    pa.nt = 1; pa.t_r[0] = 0; pa.t_c[0] = 0; pa.t_s[0] = 1;
    pa.scale = scaleA; pa.tiles = tm; pa.nk = (int64_t)P * nk; pa.nkpiece = nk; pa.batch = g.batch;
    pa.planes = planes; pa.out = planesA;
    pa.kfast = g.unit_ksA != 0 && (g.unit_rsA == 0 || g.unit_ksA < g.unit_rsA);
    TSB_CUDA(launch_split_pack(pa, st));
    SplitPackArgs pb{};
    pb.X = B; pb.rs = tb[2]; pb.ks = tb[5]; pb.bX = tb[7];
    pb.rows_full = g.n; pb.k_full = g.k; pb.rows_blk = g.n; pb.k_blk = (int64_t)P * kq;
    pb.nt = 1; pb.t_r[0] = 0; pb.t_c[0] = 0; pb.t_s[0] = 1;
    pb.scale = scaleB; pb.tiles = tn; pb.nk = (int64_t)P * nk; pb.nkpiece = nk; pb.batch = g.batch;
    pb.planes = planes; pb.out = planesB;
    pb.kfast = g.unit_ksB != 0 && (g.unit_csB == 0 || g.unit_ksB < g.unit_csB);
    TSB_CUDA(launch_split_pack(pb, st));

    static const int8_t TA6[6] = {0, 0, 1, 0, 1, 2}, TB6[6] = {0, 1, 0, 2, 1, 0};
    SplitGemmArgs ga{};
    ga.A[0] = planesA; ga.B[0] = planesB; ga.C = M;
    ga.rsC = mtab; ga.csC = mtab + g.m; ga.bC = mtab + g.m + g.n;
    ga.invA = invA; ga.invB = invB;
    ga.m = g.m; ga.n = g.n; ga.ms = g.m; ga.ns = g.n; ga.nk = nk;
    ga.tiles_m = tm; ga.tiles_n = tn; ga.batch = (int64_t)P * g.batch; ga.pbatch = g.batch;
    ga.alpha = 1.f; ga.beta = 0.f;
    ga.nprod = 1; ga.H = 1;
    ga.nc[0] = 1; ga.c_s[0][0] = 1; ga.c_first[0][0] = 1;
    ga.planes = planes;
    ga.nterms = planes == 3 ? 6 : 3;
    for (int i = 0; i < 6; i++) { ga.ta[i] = TA6[i]; ga.tb[i] = TB6[i]; }
    ga.err = err;
    ga.wait_limit = wait_limit_cycles();
    TSB_CUDA(launch_split_gemm(ga, st, sms));

    CombineF32Args c{};
    c.C = C; c.rsC = tb[1]; c.csC = tb[3]; c.bC = tb[8];
    c.m = g.m; c.n = g.n; c.ms = g.m; c.ns = g.n; c.batch = g.batch;
    c.M = M; c.m_pstride = g.batch * g.m * g.n;
    c.alpha = g.alpha; c.beta = g.beta;
    c.H = 1; c.col_major = col_major ? 1 : 0;
    c.np = P;
    for (int p = 0; p < P; p++) { c.nt[p] = 1; c.th[p][0] = 0; c.ts[p][0] = 1; }
    TSB_CUDA(launch_combine(c, st));
    return TBLIS_STRA_SUCCESS;
}

namespace {

int run_fp32(int level, const GemmView& g, const DevPlan& t, const float* A, const float* B,
             float* C, cudaStream_t st, int device, bool blocking, int* shared_err = nullptr)
{
    if (g.m == 0 || g.n == 0 || g.batch == 0) return TBLIS_STRA_SUCCESS;
    if (g.alpha == 0.0 || g.k == 0)
    {
        ScaleF32Args s{C, t.rsC, t.csC, t.bC, g.m, g.n, g.batch, (float)g.beta};
        TSB_CUDA(launch_scale_f32(s, st));
        return TBLIS_STRA_SUCCESS;
    }
    const int terms = t_fp32_terms;
    Scratch wsbuf, errbuf;
    int s;
    // Product-parallel when one product's 128 x 128 tiles would leave SMs
    // idle and its workspace is allowed (as for FP64).
    const int sms = num_sms(device);
    const int H = product_table(level).H;
    const int64_t* tb[9] = {t.rsA, t.rsC, t.csB, t.csC, t.ksA, t.ksB, t.bA, t.bB, t.bC};
    // A plain contraction with fewer C tiles than SMs: k-split.
    const int P = level == 0 && t_product_parallel != 0 ? ksplit_pieces(g, sms) : 1;
    if (P >= 2 && fp32_ksplit_workspace_bytes(g, P, terms) <= t_ws_limit)
    {
        const int64_t* ktab = nullptr;
        if ((s = plan_m_tables(t, 0, g.m, g.n, (int64_t)P * g.batch, m_tables_col_major(g), ktab))) return s;
        const size_t wsk = fp32_ksplit_workspace_bytes(g, P, terms);
        if ((s = wsbuf.alloc(wsk, st))) return s;
        int* err = shared_err;
        if (!err)
        {
            if ((s = errbuf.alloc(sizeof(int), st))) return s;
            TSB_CUDA(cudaMemsetAsync(errbuf.p, 0, sizeof(int), st));
            err = static_cast<int*>(errbuf.p);
        }
        if ((s = run_fp32_ksplit_enqueue(g, tb, A, B, C, st, sms, wsbuf.p, wsk, terms, P, ktab,
                                         m_tables_col_major(g), err)))
            return s;
        if (blocking && !shared_err)
        {
            int flag = 0;
            TSB_CUDA(cudaMemcpyAsync(&flag, errbuf.p, sizeof(int), cudaMemcpyDeviceToHost, st));
            TSB_CUDA(cudaStreamSynchronize(st));
            if (flag) return TBLIS_STRA_ERR_TIMEOUT;
        }
        return TBLIS_STRA_SUCCESS;
    }
    const bool parallel = use_product_parallel(level, g, sms, true, terms);
    const size_t wsb_par = parallel ? fp32_parallel_workspace_bytes(level, g, terms) : 0;
    const bool m_col_major = m_tables_col_major(g);
    const int64_t* mtab = nullptr;
    if (parallel && (s = plan_m_tables(t, level, cdiv(g.m, H), cdiv(g.n, H),
                                       (int64_t)product_table(level).prod.size() * g.batch, m_col_major, mtab)))
        return s;
    const size_t wsb_group = fp32_group_workspace_bytes(level, g, terms);
    const size_t wsb = parallel ? wsb_par
                       : wsb_group <= t_ws_limit ? wsb_group : fp32_workspace_bytes(level, g, terms);
    if ((s = wsbuf.alloc(wsb, st))) return s;
    int* err = shared_err;
    if (!err)
    {
        if ((s = errbuf.alloc(sizeof(int), st))) return s;
        TSB_CUDA(cudaMemsetAsync(errbuf.p, 0, sizeof(int), st));
        err = static_cast<int*>(errbuf.p);
    }
    s = parallel ? run_fp32_parallel_enqueue(level, g, tb, A, B, C, st, sms, wsbuf.p, wsb, terms, mtab,
                                             m_col_major, err)
                 : run_fp32_enqueue(level, g, tb, A, B, C, st, sms, wsbuf.p, wsb, terms, err);
    if (s) return s;
    if (blocking && !shared_err)
    {
        int flag = 0;
        TSB_CUDA(cudaMemcpyAsync(&flag, errbuf.p, sizeof(int), cudaMemcpyDeviceToHost, st));
        TSB_CUDA(cudaStreamSynchronize(st));
        if (flag) return TBLIS_STRA_ERR_TIMEOUT;
    }
    return TBLIS_STRA_SUCCESS;
}

// ---- pipelined staging of host operands ----------------------------------------
//
// When A, B and C all live in host memory, the call splits the slowest label
// of C that is also in exactly one of A and B into chunks: the other operand is
// copied first, then chunk j of C and of the split operand is copied in while
// chunk j-1 computes, and chunk j of C is copied back while chunk j+1
// computes.  When C's geometry allows it, the other operand is cut in two
// along one of its own C labels as well (chunks (i, j), i outer), so the first
// chunk waits for half of it only.  Each chunk is the same contraction on
// sub-views (the split labels restricted to the chunk's ranges), so every
// chunk is exact and C's chunks are disjoint; beta applies once per element.

struct CopyStreams { cudaStream_t in = nullptr, out = nullptr; };

// Per-device non-blocking streams for the host <-> device copies.
int copy_streams(int device, CopyStreams& cs)
{
    static std::mutex mu;
    static std::map<int, CopyStreams> streams;
    std::lock_guard<std::mutex> lk(mu);
    auto it = streams.find(device);
    if (it != streams.end()) { cs = it->second; return TBLIS_STRA_SUCCESS; }
    CopyStreams c;
    if (cudaStreamCreateWithFlags(&c.in, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c.out, cudaStreamNonBlocking) != cudaSuccess)
    {
        cudaGetLastError();
        return TBLIS_STRA_ERR_CUDA;
    }
    streams[device] = c;
    cs = c;
    return TBLIS_STRA_SUCCESS;
}

// Geometry of the slice [a, b) of the label at position `pos`: the labels
// with smaller strides must tile [0, sigma) densely and those with larger
// strides must be dense among themselves, so the slice is `height` rows of
// (b - a) * sigma elements `pitch` apart, starting at element a * sigma.
bool slice_geometry(const tblis_tensor* T, int pos, int64_t& sigma, int64_t& height, int64_t& pitch)
{
    const int64_t e = T->len[pos];
    sigma = T->stride[pos];
    if (sigma <= 0) return false;
    std::vector<std::pair<int64_t, int64_t>> inner, outer;   // (stride, extent)
    for (unsigned d = 0; d < T->ndim; d++)
    {
        if ((int)d == pos || T->len[d] == 1) continue;
        if (T->stride[d] <= 0 || T->stride[d] == sigma) return false;
        (T->stride[d] < sigma ? inner : outer).emplace_back(T->stride[d], T->len[d]);
    }
    std::sort(inner.begin(), inner.end());
    int64_t run = 1;
    for (auto& x : inner)
    {
        if (x.first != run) return false;
        run *= x.second;
    }
    if (run != sigma) return false;
    std::sort(outer.begin(), outer.end());
    height = 1;
    pitch = sigma * e;
    if (!outer.empty())
    {
        pitch = outer[0].first;
        if (pitch < sigma * e) return false;
        int64_t r = pitch;
        for (auto& x : outer)
        {
            if (x.first != r) return false;
            r *= x.second;
            height *= x.second;
        }
    }
    return true;
}

constexpr size_t PIPELINE_MIN_BYTES = (size_t)64 << 20;
#ifndef TSB_PIPELINE_CHUNKS
#define TSB_PIPELINE_CHUNKS 4
#endif
#ifndef TSB_PIPELINE_CUTS
#define TSB_PIPELINE_CUTS 2
#endif
constexpr int PIPELINE_CHUNKS = TSB_PIPELINE_CHUNKS;   // pieces of the split operand
constexpr int PIPELINE_CUTS = TSB_PIPELINE_CUTS;       // pieces of the other operand (second cut)
constexpr int NOT_PIPELINED = -1;

int run_plan(int level, int impl, const GemmView& g, const DevPlan& t, void* const dptr[3], cudaStream_t st,
             int device, int* shared_err)
{
    if (g.type == TYPE_FLOAT)
        return run_fp32(level, g, t, static_cast<const float*>(dptr[0]), static_cast<const float*>(dptr[1]),
                        static_cast<float*>(dptr[2]), st, device, false, shared_err);
    return run_fp64(level, impl, g, t, static_cast<const double*>(dptr[0]), static_cast<const double*>(dptr[1]),
                    static_cast<double*>(dptr[2]), st, device, false, shared_err);
}

int mult_pipelined(int level, int impl, const tblis_tensor* const T[3], const label_type* const I[3],
                   const GemmView& g, int device, cudaStream_t st)
{
    const size_t es = g.type == TYPE_FLOAT ? sizeof(float) : sizeof(double);
    size_t bytes = 0;
    for (int t = 0; t < 3; t++)
    {
        if (g.hi[t] < g.lo[t] || g.lo[t] != 0 || !T[t]->data || mem_kind(T[t]->data, device) != MemKind::HOST)
            return NOT_PIPELINED;
        for (unsigned d = 0; d < T[t]->ndim; d++)
            for (unsigned e = d + 1; e < T[t]->ndim; e++)
                if (I[t][d] == I[t][e]) return NOT_PIPELINED;            // diagonal labels
        bytes += (size_t)(g.hi[t] + 1) * es;
    }
    if (bytes < PIPELINE_MIN_BYTES) return NOT_PIPELINED;

    // The split label: in C and in exactly one of A, B; largest C stride first.
    auto find = [](const tblis_tensor* X, const label_type* ix, label_type c) {
        for (unsigned d = 0; d < X->ndim; d++)
            if (ix[d] == c) return (int)d;
        return -1;
    };
    std::vector<int> cand;
    for (unsigned d = 0; d < T[2]->ndim; d++)
    {
        const int pa = find(T[0], I[0], I[2][d]), pb = find(T[1], I[1], I[2][d]);
        if ((pa < 0) != (pb < 0) && T[2]->len[d] >= 2) cand.push_back((int)d);
    }
    std::sort(cand.begin(), cand.end(), [&](int x, int y) { return T[2]->stride[x] > T[2]->stride[y]; });
    int pc = -1, op = -1, px = -1;
    int64_t sc = 0, hc = 0, pitc = 0, sx = 0, hx = 0, pitx = 0;
    for (int d : cand)
    {
        const int pa = find(T[0], I[0], I[2][d]);
        const int o = pa >= 0 ? 0 : 1;
        const int p = pa >= 0 ? pa : find(T[1], I[1], I[2][d]);
        if (slice_geometry(T[2], d, sc, hc, pitc) && slice_geometry(T[o], p, sx, hx, pitx))
        {
            pc = d; op = o; px = p;
            break;
        }
    }
    if (pc < 0) return NOT_PIPELINED;
    const int whole = 1 - op;                 // the operand not cut along pc
    const int64_t extent = T[2]->len[pc];
    const int chunks = (int)std::min<int64_t>(PIPELINE_CHUNKS, extent);

    // Second cut, of the other operand: a C label qc of that operand only whose
    // C stride sits next to pc's (inner * extent == outer, the outer one C's
    // last), so block (i, j) of C is one 2-D copy: rows of (inner range) *
    // inner stride elements, one per outer index.
    int qc = -1, pw = -1;
    int64_t sw = 0, hw = 0, pitw = 0;
    for (unsigned d = 0; d < T[2]->ndim && qc < 0; d++)
    {
        const int pa = find(T[0], I[0], I[2][d]), pb = find(T[1], I[1], I[2][d]);
        const int pwhole = whole == 0 ? pa : pb, pother = whole == 0 ? pb : pa;
        if ((int)d == pc || pwhole < 0 || pother >= 0 || T[2]->len[d] < 2) continue;
        const int inner = T[2]->stride[d] < T[2]->stride[pc] ? (int)d : pc;
        const int outer = inner == pc ? (int)d : pc;
        int64_t si, hi, pi, so, ho, po;
        if (!slice_geometry(T[2], inner, si, hi, pi) || !slice_geometry(T[2], outer, so, ho, po)) continue;
        if (T[2]->stride[inner] * T[2]->len[inner] != T[2]->stride[outer] || ho != 1) continue;
        if (!slice_geometry(T[whole], pwhole, sw, hw, pitw)) continue;
        qc = (int)d;
        pw = pwhole;
    }
    const int halves = qc >= 0 ? (int)std::min<int64_t>(PIPELINE_CUTS, T[2]->len[qc]) : 1;

    CopyStreams cs;
    int s = copy_streams(device, cs);
    if (s) return s;
    Scratch stage[3], errbuf;
    for (int t = 0; t < 3; t++)
        if ((s = stage[t].alloc((size_t)(g.hi[t] + 1) * es, st))) return s;
    if ((s = errbuf.alloc(sizeof(int), st))) return s;
    TSB_CUDA(cudaMemsetAsync(errbuf.p, 0, sizeof(int), st));
    int* err = static_cast<int*>(errbuf.p);

    std::vector<cudaEvent_t> ev;
    auto event = [&]() {
        cudaEvent_t e = nullptr;
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) == cudaSuccess) ev.push_back(e);
        else cudaGetLastError();
        return e;
    };
    struct EvGuard
    {
        std::vector<cudaEvent_t>& v;
        ~EvGuard() { for (cudaEvent_t e : v) cudaEventDestroy(e); }
    } guard{ev};

    auto copy2d = [&](int t, int64_t sigma, int64_t height, int64_t pitch, int64_t a, int64_t b,
                      cudaMemcpyKind kind, cudaStream_t cst) -> int {
        const size_t off = (size_t)(a * sigma) * es, width = (size_t)((b - a) * sigma) * es;
        const size_t pb = std::max((size_t)pitch * es, width);
        char* host = static_cast<char*>(T[t]->data) + off;
        char* dev = static_cast<char*>(stage[t].p) + off;
        if (kind == cudaMemcpyHostToDevice)
            TSB_CUDA(cudaMemcpy2DAsync(dev, pb, host, pb, width, (size_t)height, kind, cst));
        else
            TSB_CUDA(cudaMemcpy2DAsync(host, pb, dev, pb, width, (size_t)height, kind, cst));
        return TBLIS_STRA_SUCCESS;
    };

    // C block (i, j): the pc range of chunk j and, with a second cut, the qc
    // range of half i, as one 2-D copy.
    auto copy_c = [&](const int64_t* rq, const int64_t* rp, cudaMemcpyKind kind, cudaStream_t cst) -> int {
        if (qc < 0) return copy2d(2, sc, hc, pitc, rp[0], rp[1], kind, cst);
        const bool q_inner = T[2]->stride[qc] < T[2]->stride[pc];
        const int64_t* ri = q_inner ? rq : rp;
        const int64_t* ro = q_inner ? rp : rq;
        const int inner = q_inner ? qc : pc, outer = q_inner ? pc : qc;
        const int64_t si = T[2]->stride[inner], so = T[2]->stride[outer];
        const size_t off = (size_t)(ri[0] * si + ro[0] * so) * es;
        const size_t width = (size_t)((ri[1] - ri[0]) * si) * es;
        char* host = static_cast<char*>(T[2]->data) + off;
        char* dev = static_cast<char*>(stage[2].p) + off;
        const size_t pb = (size_t)so * es;
        if (kind == cudaMemcpyHostToDevice)
            TSB_CUDA(cudaMemcpy2DAsync(dev, pb, host, pb, width, (size_t)(ro[1] - ro[0]), kind, cst));
        else
            TSB_CUDA(cudaMemcpy2DAsync(host, pb, dev, pb, width, (size_t)(ro[1] - ro[0]), kind, cst));
        return TBLIS_STRA_SUCCESS;
    };

    cudaEvent_t e0 = event(), e_out = event();
    if (!e0 || !e_out) return TBLIS_STRA_ERR_CUDA;
    TSB_CUDA(cudaEventRecord(e0, st));                    // staging buffers allocated
    TSB_CUDA(cudaStreamWaitEvent(cs.in, e0, 0));
    TSB_CUDA(cudaStreamWaitEvent(cs.out, e0, 0));
    std::vector<int64_t> lo(chunks + 1), lw(halves + 1);
    for (int j = 0; j <= chunks; j++) lo[j] = extent * j / chunks;
    const int64_t ext_w = qc >= 0 ? T[2]->len[qc] : 1;
    for (int i = 0; i <= halves; i++) lw[i] = ext_w * i / halves;
    // Copies in the order the chunks need them: half i of the other operand
    // (all of it without a second cut) before its first chunk, slice j of the
    // split operand with chunk (0, j), C block (i, j) with its chunk.
    const int nck = halves * chunks;
    std::vector<cudaEvent_t> e_in(nck), e_done(nck);
    for (int i = 0; i < halves; i++)
        for (int j = 0; j < chunks; j++)
        {
            const int c = i * chunks + j;
            e_in[c] = event();
            e_done[c] = event();
            if (!e_in[c] || !e_done[c]) return TBLIS_STRA_ERR_CUDA;
            if (j == 0)
            {
                if (qc < 0)
                    TSB_CUDA(cudaMemcpyAsync(stage[whole].p, T[whole]->data, (size_t)(g.hi[whole] + 1) * es,
                                             cudaMemcpyHostToDevice, cs.in));
                else if ((s = copy2d(whole, sw, hw, pitw, lw[i], lw[i + 1], cudaMemcpyHostToDevice, cs.in)))
                    return s;
            }
            if (i == 0 && (s = copy2d(op, sx, hx, pitx, lo[j], lo[j + 1], cudaMemcpyHostToDevice, cs.in)))
                return s;
            if ((s = copy_c(&lw[i], &lo[j], cudaMemcpyHostToDevice, cs.in))) return s;
            TSB_CUDA(cudaEventRecord(e_in[c], cs.in));
        }
    for (int i = 0; i < halves; i++)
        for (int j = 0; j < chunks; j++)
        {
            const int c = i * chunks + j;
            // sub-views: the split labels restricted to the chunk's ranges
            tblis_tensor sub[3];
            std::vector<len_type> len[3];
            void* dptr[3];
            for (int t = 0; t < 3; t++)
            {
                sub[t] = *T[t];
                len[t].assign(T[t]->len, T[t]->len + T[t]->ndim);
                dptr[t] = stage[t].p;
            }
            len[op][px] = lo[j + 1] - lo[j];
            len[2][pc] = lo[j + 1] - lo[j];
            dptr[op] = static_cast<char*>(stage[op].p) + (size_t)(lo[j] * sx) * es;
            size_t coff = (size_t)(lo[j] * T[2]->stride[pc]) * es;
            if (qc >= 0)
            {
                len[whole][pw] = lw[i + 1] - lw[i];
                len[2][qc] = lw[i + 1] - lw[i];
                dptr[whole] = static_cast<char*>(stage[whole].p) + (size_t)(lw[i] * sw) * es;
                coff += (size_t)(lw[i] * T[2]->stride[qc]) * es;
            }
            dptr[2] = static_cast<char*>(stage[2].p) + coff;
            for (int t = 0; t < 3; t++) { sub[t].len = len[t].data(); sub[t].data = dptr[t]; }
            const tblis_tensor* ST[3] = {&sub[0], &sub[1], &sub[2]};
            GemmView gj;
            std::shared_ptr<DevPlan> dpj;
            if ((s = get_plan(ST, I, device, gj, dpj))) return s;
            TSB_CUDA(cudaStreamWaitEvent(st, e_in[c], 0));
            if ((s = run_plan(level, impl, gj, *dpj, dptr, st, device, err))) return s;
            TSB_CUDA(cudaEventRecord(e_done[c], st));
            TSB_CUDA(cudaStreamWaitEvent(cs.out, e_done[c], 0));
            if ((s = copy_c(&lw[i], &lo[j], cudaMemcpyDeviceToHost, cs.out))) return s;
        }
    TSB_CUDA(cudaEventRecord(e_out, cs.out));
    TSB_CUDA(cudaStreamWaitEvent(st, e_out, 0));
    int flag = 0;
    TSB_CUDA(cudaMemcpyAsync(&flag, err, sizeof(int), cudaMemcpyDeviceToHost, st));
    TSB_CUDA(cudaStreamSynchronize(st));
    return flag ? TBLIS_STRA_ERR_TIMEOUT : TBLIS_STRA_SUCCESS;
}

int mult(int level, const tblis_tensor* A, const label_type* idx_A,
         const tblis_tensor* B, const label_type* idx_B,
         tblis_tensor* C, const label_type* idx_C, cudaStream_t st, bool blocking)
{
    clear_detail();
    if (level < 0 || level > 2) return TBLIS_STRA_ERR_ARG;
    const int impl = t_impl;
    if (!A || !B || !C) return TBLIS_STRA_ERR_NULL;
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) { cudaGetLastError(); return TBLIS_STRA_ERR_NO_DEVICE; }

    const tblis_tensor* T[3] = {A, B, C};
    const label_type* I[3] = {idx_A, idx_B, idx_C};
    GemmView g;
    std::shared_ptr<DevPlan> dp;
    int s = get_plan(T, I, device, g, dp);
    if (s) return s;
    const bool fp32 = g.type == TYPE_FLOAT;
    // Fast-multiplication algorithms other than Strassen run the FP64 ABC
    // variant (packed product by product, or the fused kernel).
    if (level >= 1 && thread_algorithm() != 0 &&
        (fp32 || impl != 1 || !fmm_table(thread_algorithm(), level)))
        return TBLIS_STRA_ERR_UNSUPPORTED;
    const size_t es = fp32 ? sizeof(float) : sizeof(double);

    // Every element access is an aligned load or store of the element size.
    for (int t = 0; t < 3; t++)
        if (reinterpret_cast<uintptr_t>(T[t]->data) % es) return TBLIS_STRA_ERR_ARG;

    // All operands on the host and large enough: pipelined staging.
    if (g.m > 0 && g.n > 0 && g.batch > 0 && g.alpha != 0.0 && g.k > 0)
    {
        s = mult_pipelined(level, impl, T, I, g, device, st);
        if (s != NOT_PIPELINED)
        {
            if (s) return s;
            if (fp32) { float one = 1.0f; std::memcpy(C->scalar, &one, sizeof one); }
            else { double one = 1.0; std::memcpy(C->scalar, &one, sizeof one); }
            C->conj = 0;
            return TBLIS_STRA_SUCCESS;
        }
    }

    // Stage host operands through device memory.
    void* dptr[3] = {A->data, B->data, C->data};
    Scratch stage[3];
    bool staged[3] = {false, false, false};
    for (int t = 0; t < 3; t++)
    {
        if (g.hi[t] < g.lo[t]) continue;            // empty tensor
        if (!T[t]->data) return TBLIS_STRA_ERR_NULL;
        const MemKind mk = mem_kind(T[t]->data, device);
        if (mk == MemKind::OTHER_DEVICE) return TBLIS_STRA_ERR_ARG;   // another GPU's memory
        if (mk == MemKind::LOCAL) continue;
        const size_t n = (size_t)(g.hi[t] - g.lo[t] + 1);
        if ((s = stage[t].alloc(n * es, st))) return s;
        const char* hsrc = static_cast<const char*>(T[t]->data) + g.lo[t] * (int64_t)es;
        TSB_CUDA(cudaMemcpyAsync(stage[t].p, hsrc, n * es, cudaMemcpyHostToDevice, st));
        dptr[t] = static_cast<char*>(stage[t].p) - g.lo[t] * (int64_t)es;
        staged[t] = true;
    }

    if (fp32)
        s = run_fp32(level, g, *dp, static_cast<const float*>(dptr[0]), static_cast<const float*>(dptr[1]),
                     static_cast<float*>(dptr[2]), st, device,
                     blocking || staged[0] || staged[1] || staged[2]);
    else
        s = run_fp64(level, impl, g, *dp, static_cast<const double*>(dptr[0]),
                     static_cast<const double*>(dptr[1]), static_cast<double*>(dptr[2]), st, device,
                     blocking || staged[0] || staged[1] || staged[2]);
    if (s) return s;

    if (staged[2])
    {
        const size_t n = (size_t)(g.hi[2] - g.lo[2] + 1);
        char* hdst = static_cast<char*>(C->data) + g.lo[2] * (int64_t)es;
        TSB_CUDA(cudaMemcpyAsync(hdst, stage[2].p, n * es, cudaMemcpyDeviceToHost, st));
    }
    if (blocking || staged[0] || staged[1] || staged[2])
        TSB_CUDA(cudaStreamSynchronize(st));

    if (fp32)
    {
        float one = 1.0f;
        std::memcpy(C->scalar, &one, sizeof one);
    }
    else
    {
        double one = 1.0;
        std::memcpy(C->scalar, &one, sizeof one);
    }
    C->conj = 0;
    return TBLIS_STRA_SUCCESS;
}

// Matrix-level calls: the 2-D special case of the contraction,
// C(i,j) = alpha A(i,k) B(k,j) + beta C(i,j), with the variant given by the
// entry point (src/stra_iface/3m/stra_mult.cxx:14-56 checks the same shapes
// and calls internal::stra_mult / stra_mult_naive / stra_mult_ab).
int matrix_mult(int level, int impl, const tblis_matrix* A, const tblis_matrix* B, tblis_matrix* C)
{
    if (!A || !B || !C) return TBLIS_STRA_ERR_NULL;
    if (A->type != B->type || A->type != C->type) return TBLIS_STRA_ERR_TYPE;
    if (A->conj || B->conj || C->conj) return TBLIS_STRA_ERR_CONJ;
    if (A->m != C->m || B->n != C->n || A->n != B->m) return TBLIS_STRA_ERR_EXTENT;
    len_type la[2] = {A->m, A->n}, lb[2] = {B->m, B->n}, lc[2] = {C->m, C->n};
    stride_type sa[2] = {A->rs, A->cs}, sb[2] = {B->rs, B->cs}, sc[2] = {C->rs, C->cs};
    tblis_tensor tA{A->type, 0, {0}, A->data, 2, la, sa};
    tblis_tensor tB{B->type, 0, {0}, B->data, 2, lb, sb};
    tblis_tensor tC{C->type, 0, {0}, C->data, 2, lc, sc};
    std::memcpy(tA.scalar, A->scalar, sizeof tA.scalar);
    std::memcpy(tB.scalar, B->scalar, sizeof tB.scalar);
    std::memcpy(tC.scalar, C->scalar, sizeof tC.scalar);
    const int saved = t_impl;
    t_impl = impl;
    const int s = mult(level, &tA, "ik", &tB, "kj", &tC, "ij", t_stream, true);
    t_impl = saved;
    if (s == TBLIS_STRA_SUCCESS)
    {
        std::memcpy(C->scalar, tC.scalar, sizeof C->scalar);
        C->conj = 0;
    }
    return s;
}

}  // namespace
}  // namespace tsb

extern "C" {

void tblis_matrix_mult(const tblis_comm*, const tblis_config*, const tblis_matrix* A, const tblis_matrix* B,
                       tblis_matrix* C)
{
    tsb::t_status = tsb::matrix_mult(0, 1, A, B, C);
}

void stra_tblis_matrix_mult(const tblis_comm*, const tblis_config*, const tblis_matrix* A, const tblis_matrix* B,
                            tblis_matrix* C)
{
    tsb::t_status = tsb::matrix_mult(1, 1, A, B, C);
}

void stra_tblis_matrix_mult_naive(const tblis_comm*, const tblis_config*, const tblis_matrix* A,
                                  const tblis_matrix* B, tblis_matrix* C)
{
    tsb::t_status = tsb::matrix_mult(1, 3, A, B, C);
}

void stra_tblis_matrix_mult_ab(const tblis_comm*, const tblis_config*, const tblis_matrix* A,
                               const tblis_matrix* B, tblis_matrix* C)
{
    tsb::t_status = tsb::matrix_mult(1, 2, A, B, C);
}

void stra_tblis_matrix_mult_2level(const tblis_comm*, const tblis_config*, const tblis_matrix* A,
                                   const tblis_matrix* B, tblis_matrix* C)
{
    tsb::t_status = tsb::matrix_mult(2, 1, A, B, C);
}

void stra_tblis_matrix_mult_2level_naive(const tblis_comm*, const tblis_config*, const tblis_matrix* A,
                                         const tblis_matrix* B, tblis_matrix* C)
{
    tsb::t_status = tsb::matrix_mult(2, 3, A, B, C);
}

void stra_tblis_matrix_mult_2level_ab(const tblis_comm*, const tblis_config*, const tblis_matrix* A,
                                      const tblis_matrix* B, tblis_matrix* C)
{
    tsb::t_status = tsb::matrix_mult(2, 2, A, B, C);
}

static void drop_in(int level, const tblis_tensor* A, const label_type* idx_A,
                    const tblis_tensor* B, const label_type* idx_B,
                    tblis_tensor* C, const label_type* idx_C)
{
    tsb::t_status = tsb::mult(level, A, idx_A, B, idx_B, C, idx_C, tsb::t_stream, true);
}

void tblis_tensor_mult(const tblis_comm*, const tblis_config*,
                       const tblis_tensor* A, const label_type* idx_A,
                       const tblis_tensor* B, const label_type* idx_B,
                       tblis_tensor* C, const label_type* idx_C)
{
    drop_in(0, A, idx_A, B, idx_B, C, idx_C);
}

void stra_tblis_tensor_mult(const tblis_comm*, const tblis_config*,
                            const tblis_tensor* A, const label_type* idx_A,
                            const tblis_tensor* B, const label_type* idx_B,
                            tblis_tensor* C, const label_type* idx_C)
{
    drop_in(1, A, idx_A, B, idx_B, C, idx_C);
}

void stra_tblis_tensor_mult_2level(const tblis_comm*, const tblis_config*,
                                   const tblis_tensor* A, const label_type* idx_A,
                                   const tblis_tensor* B, const label_type* idx_B,
                                   tblis_tensor* C, const label_type* idx_C)
{
    drop_in(2, A, idx_A, B, idx_B, C, idx_C);
}

int tblis_stra_mult(int level, const tblis_tensor* A, const label_type* idx_A,
                    const tblis_tensor* B, const label_type* idx_B,
                    tblis_tensor* C, const label_type* idx_C, void* stream)
{
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : tsb::t_stream;
    tsb::t_status = tsb::mult(level, A, idx_A, B, idx_B, C, idx_C, st, false);
    return tsb::t_status;
}

unsigned tblis_get_num_threads(void) { return tsb::g_num_threads; }
void tblis_set_num_threads(unsigned n) { tsb::g_num_threads = n ? n : 1; }

int tblis_stra_set_impl(int impl)
{
    if (impl < 1 || impl > 3) return TBLIS_STRA_ERR_ARG;
    tsb::t_impl = impl;
    return TBLIS_STRA_SUCCESS;
}

int tblis_stra_get_impl(void) { return tsb::t_impl; }

int tblis_stra_set_workspace_limit(size_t bytes)
{
    tsb::t_ws_limit = bytes;
    return TBLIS_STRA_SUCCESS;
}

size_t tblis_stra_get_workspace_limit(void) { return tsb::t_ws_limit; }

int tblis_stra_set_fp32_terms(int terms)
{
    if (terms != 3 && terms != 6) return TBLIS_STRA_ERR_ARG;
    tsb::t_fp32_terms = terms;
    return TBLIS_STRA_SUCCESS;
}

int tblis_stra_get_fp32_terms(void) { return tsb::t_fp32_terms; }

int tblis_stra_set_product_parallel(int mode)
{
    if (mode < -1 || mode > 1) return TBLIS_STRA_ERR_ARG;
    tsb::t_product_parallel = mode;
    return TBLIS_STRA_SUCCESS;
}

int tblis_stra_get_product_parallel(void) { return tsb::t_product_parallel; }

int tblis_stra_measure_dmma_peak(int iterations, double* tflops, double* ms, void* stream)
{
    if (!tflops || !ms) return TBLIS_STRA_ERR_NULL;
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) { cudaGetLastError(); return TBLIS_STRA_ERR_NO_DEVICE; }
    const cudaError_t e = tsb::measure_dmma_peak(iterations, tsb::num_sms(device), static_cast<cudaStream_t>(stream),
                                                 tflops, ms);
    if (e == cudaErrorInvalidValue) return TBLIS_STRA_ERR_ARG;
    if (e != cudaSuccess) { tsb::note_cuda_error("measure_dmma_peak", e, __FILE__, __LINE__); return TBLIS_STRA_ERR_CUDA; }
    return TBLIS_STRA_SUCCESS;
}

int tblis_stra_set_algorithm(int id)
{
    if (!tsb::algorithm_by_id(id) || !tsb::fmm_table(id, 1)) return TBLIS_STRA_ERR_ARG;
    tsb::set_thread_algorithm(id);
    return TBLIS_STRA_SUCCESS;
}
int tblis_stra_get_algorithm(void) { return tsb::thread_algorithm(); }

int tblis_stra_algorithm_info(int id, int* mb, int* kb, int* nb, int* rank, int* levels)
{
    const tsb::FmmAlgorithm* a = tsb::algorithm_by_id(id);
    if (!a) return TBLIS_STRA_ERR_ARG;
    if (mb) *mb = a->mb;
    if (kb) *kb = a->kb;
    if (nb) *nb = a->nb;
    if (rank) *rank = a->rank;
    if (levels) *levels = tsb::fmm_table(id, 2) ? 2 : tsb::fmm_table(id, 1) ? 1 : 0;
    return TBLIS_STRA_SUCCESS;
}

int tblis_stra_register_algorithm(int mb, int kb, int nb, int rank, const int* U, const int* V, const int* W,
                                  int* id)
{
    if (!U || !V || !W || !id) return TBLIS_STRA_ERR_NULL;
    if (mb < 1 || kb < 1 || nb < 1 || rank < 1 || mb > 4 || kb > 4 || nb > 4 || rank > 49)
        return TBLIS_STRA_ERR_ARG;
    tsb::FmmAlgorithm a;
    a.name = "registered";
    a.mb = mb; a.kb = kb; a.nb = nb; a.rank = rank;
    a.U.assign(U, U + mb * kb * rank);
    a.V.assign(V, V + kb * nb * rank);
    a.W.assign(W, W + mb * nb * rank);
    const int r = tsb::register_algorithm(a);
    if (r < 0) return -r;
    *id = r;
    return TBLIS_STRA_SUCCESS;
}

int tblis_stra_set_wait_limit(long long cycles)
{
    if (cycles < 0) return TBLIS_STRA_ERR_ARG;
    tsb::t_wait_limit = cycles;
    return TBLIS_STRA_SUCCESS;
}
long long tblis_stra_get_wait_limit(void) { return tsb::t_wait_limit; }

int tblis_stra_set_wait_injection(int on)
{
    tsb::t_wait_inject = on != 0;
    return TBLIS_STRA_SUCCESS;
}
int tblis_stra_get_wait_injection(void) { return tsb::t_wait_inject ? 1 : 0; }

int tblis_stra_set_alloc_limit(size_t bytes)
{
    tsb::t_alloc_limit = bytes;
    return TBLIS_STRA_SUCCESS;
}
size_t tblis_stra_get_alloc_limit(void) { return tsb::t_alloc_limit; }

int tblis_stra_last_status(void) { return tsb::t_status; }

const char* tblis_stra_last_error_detail(void) { return tsb::t_detail.c_str(); }

const char* tblis_stra_status_string(int s)
{
    switch (s)
    {
        case TBLIS_STRA_SUCCESS:         return "success";
        case TBLIS_STRA_ERR_NULL:        return "null tensor, label, extent or stride pointer";
        case TBLIS_STRA_ERR_TYPE:        return "mismatched or unsupported element type";
        case TBLIS_STRA_ERR_EXTENT:      return "one label with different extents";
        case TBLIS_STRA_ERR_CONJ:        return "conjugation requested on a real type";
        case TBLIS_STRA_ERR_ARG:         return "invalid argument (level, impl, ndim or extent)";
        case TBLIS_STRA_ERR_CUDA:        return "CUDA runtime error";
        case TBLIS_STRA_ERR_ALLOC:       return "device workspace allocation failed";
        case TBLIS_STRA_ERR_TOO_LARGE:   return "sizes beyond the kernels' index range";
        case TBLIS_STRA_ERR_UNSUPPORTED: return "request not supported by this build";
        case TBLIS_STRA_ERR_NO_DEVICE:   return "no usable CUDA device";
        case TBLIS_STRA_ERR_TIMEOUT:     return "a kernel's bounded wait expired";
        default:                         return "unknown status";
    }
}

int tblis_stra_set_stream(void* stream)
{
    tsb::t_stream = static_cast<cudaStream_t>(stream);
    return TBLIS_STRA_SUCCESS;
}

void* tblis_stra_get_stream(void) { return tsb::t_stream; }

unsigned long long tblis_stra_launch_count(void) { return tsb::launches(); }

const char* tblis_stra_version(void) { return "tblis-strassen-b200 0.1.0 (sm_100a)"; }

int tblis_stra_plan_query(const tblis_tensor* A, const label_type* idx_A,
                          const tblis_tensor* B, const label_type* idx_B,
                          const tblis_tensor* C, const label_type* idx_C,
                          int64_t* sizes, double* ab,
                          int64_t* rsA, int64_t* rsC, int64_t* csB, int64_t* csC,
                          int64_t* ksA, int64_t* ksB,
                          int64_t* bA, int64_t* bB, int64_t* bC)
{
    tsb::GemmView g;
    const bool want = rsA || rsC || csB || csC || ksA || ksB || bA || bB || bC;
    int s = tsb::plan_contraction(A, idx_A, B, idx_B, C, idx_C, g, want);
    if (s) return s;
    if (sizes) { sizes[0] = g.m; sizes[1] = g.n; sizes[2] = g.k; sizes[3] = g.batch; }
    if (ab) { ab[0] = g.alpha; ab[1] = g.beta; }
    auto cp = [](int64_t* dst, const std::vector<int64_t>& v) {
        if (dst) std::copy(v.begin(), v.end(), dst);
    };
    cp(rsA, g.rsA); cp(rsC, g.rsC); cp(csB, g.csB); cp(csC, g.csC);
    cp(ksA, g.ksA); cp(ksB, g.ksB); cp(bA, g.bA); cp(bB, g.bB); cp(bC, g.bC);
    return TBLIS_STRA_SUCCESS;
}

int tblis_stra_fused_pairs_query(int level, const tblis_tensor* A, const label_type* idx_A,
                                 const tblis_tensor* B, const label_type* idx_B,
                                 const tblis_tensor* C, const label_type* idx_C, int* pairs, int* tables)
{
    if (level < 0 || level > 2) return TBLIS_STRA_ERR_ARG;
    if (!pairs) return TBLIS_STRA_ERR_NULL;
    tsb::GemmView g;
    int s = tsb::plan_contraction(A, idx_A, B, idx_B, C, idx_C, g, false);
    if (s) return s;
    const tsb::ProductTable& tab = tsb::product_table(level);
    int most = 1;   // blocks in the longest operand sum: 16-k slots up to 2, 8-k slots up to 4
    for (const tsb::Product& p : tab.prod) most = std::max(most, std::max((int)p.na, (int)p.nb));
    const int64_t ms = (g.m + tab.H - 1) / tab.H, ns = (g.n + tab.Hn - 1) / tab.Hn,
                  ks = (g.k + tab.Hk - 1) / tab.Hk;
    *pairs = most <= 4 && tsb::fused_pairs_plan(g, tab.H, tab.Hn, tab.Hk, ms, ns, ks, most <= 2 ? 16 : 8, tables)
                 ? 1
                 : 0;
    return TBLIS_STRA_SUCCESS;
}

}  // extern "C"
