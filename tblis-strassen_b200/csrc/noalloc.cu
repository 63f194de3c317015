// tblis_stra_mult_noalloc: a contraction entry point that allocates no device
// memory.
//
// Who needs it: callers that must not (or cannot) call cudaMalloc -- an
// application whose own memory pool has reserved the whole device so a
// library allocation would fail, a host that forbids plug-ins from allocating
// device memory, or latency-critical code that cannot afford the implicit
// device synchronisation of cudaMalloc/cudaFree.  The regular entry points
// allocate the device copy of each contraction's scatter vectors (cached) and,
// for host operands, staging buffers; this one does neither.
//
// How: the scatter vectors live in one file-scope __device__ array of
// NOALLOC_MAX_ENTRIES int64 values (2 MiB, resident on every GPU that loads the
// library until the process exits).  A contraction needs
// 2*m + 2*n + 2*k + 3*batch entries; larger requests are rejected with
// TBLIS_STRA_ERR_TOO_LARGE.  The vectors are written into the array by a small
// kernel from their mixed-radix form (extents and strides of the folded
// modes, passed by value), so no host buffer is involved.  Only FP64 operands
// and the ABC variant run here (AB and Naive need M/S/T buffers), at level 0,
// 1 or 2; all three operands must be device memory of the current device.
//
// Set-up: the first call on each device (with that device current) looks up
// the array's device address with cudaGetSymbolAddress; make that first call
// before any stream capture begins.  Every call overwrites the whole table it
// uses, so nothing has to start at zero; but all calls share the one array, so
// two calls whose work overlaps on the GPU (different streams without ordering
// between them) race on it.
#include "tblis_stra_b200.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <map>
#include <mutex>

#include "kernels.cuh"
#include "memkind.hpp"
#include "plan.hpp"

namespace tsb {

extern std::atomic<unsigned long long> g_launches;

namespace {

constexpr size_t NOALLOC_MAX_ENTRIES = size_t(1) << 18;   // 2 MiB of int64

__device__ __align__(256) int64_t g_noalloc_scratch[NOALLOC_MAX_ENTRIES];

// Modes per scatter vector: every folded mode has extent >= 2, so a vector of
// at most NOALLOC_MAX_ENTRIES entries has at most 18 of them.
constexpr int GEN_MAX_MODES = 18;

// The nine scatter vectors in mixed-radix form: entry i of vector v (stored at
// out + off[v] + i, i < count[v]) is sum_d digit_d(i) * stride[v][d], digits of
// i over len[v][0..nm[v]) with the first mode fastest.
struct ScatterGenArgs
{
    int64_t* out;
    int64_t off[10];                       // off[9] = total entries
    int nm[9];
    int64_t len[9][GEN_MAX_MODES];
    int64_t stride[9][GEN_MAX_MODES];
};

__global__ void scatter_gen_kernel(const __grid_constant__ ScatterGenArgs a)
{
    const int64_t total = a.off[9];
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x)
    {
        int v = 0;
        while (v < 8 && e >= a.off[v + 1]) v++;
        int64_t i = e - a.off[v], off = 0;
        for (int d = 0; d < a.nm[v]; d++)
        {
            const int64_t l = a.len[v][d];
            const int64_t q = i / l;
            off += (i - q * l) * a.stride[v][d];
            i = q;
        }
        a.out[e] = off;
    }
}

std::mutex g_noalloc_mu;
std::map<int, int64_t*> g_noalloc_ptr;   // device -> address of g_noalloc_scratch

int noalloc_scratch(int device, int64_t** out)
{
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    auto it = g_noalloc_ptr.find(device);
    if (it != g_noalloc_ptr.end()) { *out = it->second; return TBLIS_STRA_SUCCESS; }
    int64_t* p = nullptr;
    cudaError_t err = cudaGetSymbolAddress(reinterpret_cast<void**>(&p), g_noalloc_scratch);
    if (err != cudaSuccess || p == nullptr) { cudaGetLastError(); return TBLIS_STRA_ERR_CUDA; }
    g_noalloc_ptr[device] = p;
    *out = p;
    return TBLIS_STRA_SUCCESS;
}

int noalloc_mult(int level, const tblis_tensor* A, const label_type* idx_A,
                 const tblis_tensor* B, const label_type* idx_B,
                 tblis_tensor* C, const label_type* idx_C, cudaStream_t st)
{
    if (level < 0 || level > 2) return TBLIS_STRA_ERR_ARG;
    GemmView g;
    int s = plan_contraction(A, idx_A, B, idx_B, C, idx_C, g, false);
    if (s) return s;
    if (g.type != TYPE_DOUBLE) return TBLIS_STRA_ERR_UNSUPPORTED;
    const int64_t count[9] = {g.m, g.m, g.n, g.n, g.k, g.k, g.batch, g.batch, g.batch};
    const size_t need = 2 * (size_t)g.m + 2 * (size_t)g.n + 2 * (size_t)g.k + 3 * (size_t)g.batch;
    if (need > NOALLOC_MAX_ENTRIES) return TBLIS_STRA_ERR_TOO_LARGE;
    for (int v = 0; v < 9; v++)
        if (g.mode_len[v].size() > (size_t)GEN_MAX_MODES) return TBLIS_STRA_ERR_TOO_LARGE;

    int device = 0;
    const tblis_tensor* T[3] = {A, B, C};
    bool device_known = false;
    for (int t = 0; t < 3; t++)
    {
        if (g.hi[t] < g.lo[t]) continue;   // empty tensor: never dereferenced
        if (!T[t]->data) return TBLIS_STRA_ERR_NULL;
        if (reinterpret_cast<uintptr_t>(T[t]->data) % sizeof(double)) return TBLIS_STRA_ERR_ARG;
        if (!device_known)
        {
            if (cudaGetDevice(&device) != cudaSuccess) { cudaGetLastError(); return TBLIS_STRA_ERR_NO_DEVICE; }
            device_known = true;
        }
        if (mem_kind(T[t]->data, device) != MemKind::LOCAL) return TBLIS_STRA_ERR_ARG;
    }
    if (g.m == 0 || g.n == 0 || g.batch == 0)
    {
        double one = 1.0;
        std::memcpy(C->scalar, &one, sizeof one);
        C->conj = 0;
        return TBLIS_STRA_SUCCESS;
    }

    int64_t* scratch = nullptr;
    if ((s = noalloc_scratch(device, &scratch))) return s;

    // Write the scatter vectors into the array on the caller's stream.
    ScatterGenArgs gen;
    std::memset(&gen, 0, sizeof gen);
    gen.out = scratch;
    gen.off[0] = 0;
    for (int v = 0; v < 9; v++)
    {
        gen.off[v + 1] = gen.off[v] + count[v];
        gen.nm[v] = (int)g.mode_len[v].size();
        for (int d = 0; d < gen.nm[v]; d++)
        {
            gen.len[v][d] = g.mode_len[v][d];
            gen.stride[v][d] = g.mode_stride[v][d];
        }
    }
    {
        const int threads = 256;
        const int64_t blocks = std::min<int64_t>((gen.off[9] + threads - 1) / threads, 1024);
        scatter_gen_kernel<<<(unsigned)blocks, threads, 0, st>>>(gen);
        if (cudaGetLastError() != cudaSuccess) return TBLIS_STRA_ERR_CUDA;
        g_launches++;
    }

    const int64_t* rsA = scratch + gen.off[0]; const int64_t* rsC = scratch + gen.off[1];
    const int64_t* csB = scratch + gen.off[2]; const int64_t* csC = scratch + gen.off[3];
    const int64_t* ksA = scratch + gen.off[4]; const int64_t* ksB = scratch + gen.off[5];
    const int64_t* bA = scratch + gen.off[6];  const int64_t* bB = scratch + gen.off[7];
    const int64_t* bC = scratch + gen.off[8];
    double* Cd = static_cast<double*>(C->data);

    if (g.alpha == 0.0 || g.k == 0)
    {
        ScaleArgs sa{Cd, rsC, csC, bC, g.m, g.n, g.batch, g.beta};
        if (launch_scale(sa, st) != cudaSuccess) return TBLIS_STRA_ERR_CUDA;
    }
    else
    {
        if (level >= 1 && thread_algorithm() != 0 && !fmm_table(thread_algorithm(), level))
            return TBLIS_STRA_ERR_UNSUPPORTED;
        const ProductTable& tab = product_table(level);
        const int H = tab.H;
        DmmaArgs a;
        std::memset(&a, 0, sizeof a);
        a.A = static_cast<const double*>(A->data);
        a.B = static_cast<const double*>(B->data);
        a.C = Cd;
        a.rsA = rsA; a.ksA = ksA; a.ksB = ksB; a.csB = csB; a.rsC = rsC; a.csC = csC;
        a.bA = bA; a.bB = bB; a.bC = bC;
        a.m = g.m; a.n = g.n; a.k = g.k; a.mC = g.m; a.nC = g.n; a.batch = g.batch;
        a.ms = (g.m + H - 1) / H; a.ns = (g.n + tab.Hn - 1) / tab.Hn; a.ks = (g.k + tab.Hk - 1) / tab.Hk;
        a.tiles_m = (int)((a.ms + 127) / 128);
        a.tiles_n = (int)((a.ns + 127) / 128);
        a.work = a.batch * (int64_t)a.tiles_m * a.tiles_n;
        a.alpha = g.alpha; a.beta = g.beta;
        a.a_kfast = (g.unit_ksA != 0 && (g.unit_rsA == 0 || g.unit_ksA < g.unit_rsA)) ? 1 : 0;
        a.b_kfast = (g.unit_ksB != 0 && (g.unit_csB == 0 || g.unit_ksB < g.unit_csB)) ? 1 : 0;
        a.nprod = (int)tab.prod.size();
        a.H = a.Hc = H;
        a.Hk = tab.Hk; a.Hn = tab.Hn;
        int terms = 1;
        for (int p = 0; p < a.nprod; p++)
        {
            const Product& pr = tab.prod[p];
            DevProduct& d = a.prod[p];
            d.na = pr.na; d.nb = pr.nb; d.nc = pr.nc;
            for (int i = 0; i < 4; i++)
            {
                d.a_r[i] = pr.a[i].r; d.a_c[i] = pr.a[i].c; d.a_s[i] = pr.a[i].sign;
                d.b_r[i] = pr.b[i].r; d.b_c[i] = pr.b[i].c; d.b_s[i] = pr.b[i].sign;
                d.c_r[i] = pr.c[i].r; d.c_c[i] = pr.c[i].c; d.c_s[i] = pr.c[i].sign;
                d.c_first[i] = pr.c_first[i];
            }
            terms = std::max<int>(terms, std::max<int>(pr.na, pr.nb));
        }
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        // No error flag (it would need memory): a bounded wait that runs out
        // still ends the kernel cleanly.
        cudaError_t e = launch_fused(a, st, sms, nullptr, 0, &g);
        if (e == cudaErrorNotSupported)
        {
            if (tab.Hk != H || tab.Hn != H) return TBLIS_STRA_ERR_UNSUPPORTED;
            e = launch_dmma(a, terms, st, sms);
        }
        if (e != cudaSuccess) { cudaGetLastError(); return TBLIS_STRA_ERR_CUDA; }
    }
    double one = 1.0;
    std::memcpy(C->scalar, &one, sizeof one);
    C->conj = 0;
    return TBLIS_STRA_SUCCESS;
}

}  // namespace
}  // namespace tsb

extern "C" int tblis_stra_mult_noalloc(int level,
                                       const tblis_tensor* A, const label_type* idx_A,
                                       const tblis_tensor* B, const label_type* idx_B,
                                       tblis_tensor* C, const label_type* idx_C,
                                       void* stream)
{
    if (!A || !B || !C) return TBLIS_STRA_ERR_NULL;
    return tsb::noalloc_mult(level, A, idx_A, B, idx_B, C, idx_C, static_cast<cudaStream_t>(stream));
}
