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
// TBLIS_STRA_ERR_TOO_LARGE.  Only the ABC variant runs here (AB and Naive need
// M/S/T buffers), at level 0, 1 or 2; all three operands must be device
// memory.
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
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "kernels.cuh"
#include "plan.hpp"

namespace tsb {
namespace {

constexpr size_t NOALLOC_MAX_ENTRIES = size_t(1) << 18;   // 2 MiB of int64

__device__ __align__(256) int64_t g_noalloc_scratch[NOALLOC_MAX_ENTRIES];

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

bool on_device(const void* p)
{
    cudaPointerAttributes attr;
    if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) { cudaGetLastError(); return false; }
    return attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged;
}

int noalloc_mult(int level, const tblis_tensor* A, const label_type* idx_A,
                 const tblis_tensor* B, const label_type* idx_B,
                 tblis_tensor* C, const label_type* idx_C, cudaStream_t st)
{
    if (level < 0 || level > 2) return TBLIS_STRA_ERR_ARG;
    GemmView g;
    int s = plan_contraction(A, idx_A, B, idx_B, C, idx_C, g, true);
    if (s) return s;
    if (g.type != TYPE_DOUBLE) return TBLIS_STRA_ERR_UNSUPPORTED;
    const size_t need = 2 * (size_t)g.m + 2 * (size_t)g.n + 2 * (size_t)g.k + 3 * (size_t)g.batch;
    if (need > NOALLOC_MAX_ENTRIES) return TBLIS_STRA_ERR_TOO_LARGE;
    const tblis_tensor* T[3] = {A, B, C};
    for (int t = 0; t < 3; t++)
    {
        if (g.hi[t] < g.lo[t]) continue;   // empty tensor: never dereferenced
        if (!T[t]->data) return TBLIS_STRA_ERR_NULL;
        if (reinterpret_cast<uintptr_t>(T[t]->data) % sizeof(double)) return TBLIS_STRA_ERR_ARG;
        if (!on_device(T[t]->data)) return TBLIS_STRA_ERR_ARG;
    }
    if (g.m == 0 || g.n == 0 || g.batch == 0)
    {
        double one = 1.0;
        std::memcpy(C->scalar, &one, sizeof one);
        C->conj = 0;
        return TBLIS_STRA_SUCCESS;
    }

    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) { cudaGetLastError(); return TBLIS_STRA_ERR_NO_DEVICE; }
    int64_t* scratch = nullptr;
    if ((s = noalloc_scratch(device, &scratch))) return s;

    // Pack the scatter vectors (host memory) and copy them into the array.
    const std::vector<int64_t>* parts[9] = {&g.rsA, &g.rsC, &g.csB, &g.csC, &g.ksA, &g.ksB,
                                            &g.bA, &g.bB, &g.bC};
    std::vector<int64_t> host;
    host.reserve(need);
    size_t off[9];
    for (int i = 0; i < 9; i++)
    {
        off[i] = host.size();
        host.insert(host.end(), parts[i]->begin(), parts[i]->end());
    }
    if (cudaMemcpyAsync(scratch, host.data(), host.size() * sizeof(int64_t),
                        cudaMemcpyHostToDevice, st) != cudaSuccess)
        return TBLIS_STRA_ERR_CUDA;
    // (pageable source: the call returns once the data is staged, so `host`
    // may be released afterwards)

    const int64_t* rsA = scratch + off[0]; const int64_t* rsC = scratch + off[1];
    const int64_t* csB = scratch + off[2]; const int64_t* csC = scratch + off[3];
    const int64_t* ksA = scratch + off[4]; const int64_t* ksB = scratch + off[5];
    const int64_t* bA = scratch + off[6];  const int64_t* bB = scratch + off[7];
    const int64_t* bC = scratch + off[8];
    double* Cd = static_cast<double*>(C->data);

    if (g.alpha == 0.0 || g.k == 0)
    {
        ScaleArgs sa{Cd, rsC, csC, bC, g.m, g.n, g.batch, g.beta};
        if (launch_scale(sa, st) != cudaSuccess) return TBLIS_STRA_ERR_CUDA;
    }
    else
    {
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
        a.ms = (g.m + H - 1) / H; a.ns = (g.n + H - 1) / H; a.ks = (g.k + H - 1) / H;
        a.tiles_m = (int)((a.ms + 127) / 128);
        a.tiles_n = (int)((a.ns + 127) / 128);
        a.work = a.batch * (int64_t)a.tiles_m * a.tiles_n;
        a.alpha = g.alpha; a.beta = g.beta;
        a.a_kfast = (g.unit_ksA != 0 && (g.unit_rsA == 0 || g.unit_ksA < g.unit_rsA)) ? 1 : 0;
        a.b_kfast = (g.unit_ksB != 0 && (g.unit_csB == 0 || g.unit_ksB < g.unit_csB)) ? 1 : 0;
        a.nprod = (int)tab.prod.size();
        a.H = a.Hc = H;
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
        if (launch_dmma(a, terms, st, sms) != cudaSuccess) return TBLIS_STRA_ERR_CUDA;
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
