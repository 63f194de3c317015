// Packed-operand path of the FP64 contraction: the B200 form of the
// reference's ABC schedule.
//
// The reference's ABC variant packs the signed Strassen sums of the A and B
// blocks into contiguous buffers while packing (stra_pack_{two,four}_*,
// src/kernels/3m/gemm.hpp:504-816, 1344-1917; stra_packm.hpp:367-683) and
// fuses C_p += coeff_p * alpha * AB into its micro-kernel
// (src/stra_nodes/stra_gemm_ukr.hpp:622-940).  Here, per Strassen product:
//
//   pack_kernel          S = sum_i u_i A_i and T = sum_j v_j B_j gathered
//                        through the scatter vectors into tile order (HBM bound);
//   packed_gemm_kernel   DMMA GEMM on S and T whose epilogue adds +-alpha*S*T
//                        into the product's C blocks (beta on first touch).
//
// Forming each sum once per element in HBM costs about 1 % of the GEMM time at
// NIm = NJn = NPk = 16384, while summing inside the GEMM costs shared-memory
// bandwidth on every fragment read; the GEMM's loader becomes a plain copy of
// contiguous 16-byte chunks.
#include "kernels.cuh"
#include "tile_layout.cuh"
#include "timing.hpp"

#include <atomic>
#include <cstdlib>

namespace tsb {

extern std::atomic<unsigned long long> g_launches;

namespace {

// ---- pack ---------------------------------------------------------------------

constexpr int PK_K = 32;          // k values per pack CTA
constexpr int PK_THREADS = 256;

__global__ void __launch_bounds__(PK_THREADS)
pack_kernel(const __grid_constant__ PackArgs a)
{
    __shared__ double buf[PACK_TILE][PK_K + 1];
    __shared__ int64_t rowoff[4][PACK_TILE];     // per term: batch + row offset (or invalid)
    __shared__ int64_t koff[4][PK_K];            // per term: k offset (or invalid)
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int64_t k0 = (int64_t)blockIdx.x * PK_K;
    const int64_t t = blockIdx.y;
    const int64_t b = blockIdx.z;
    const int64_t r0 = t * PACK_TILE;
    const int nt = a.nt;

    // Offset tables of this CTA's rows and k values, once per term.
    for (int i = tid; i < nt * PACK_TILE; i += PK_THREADS)
    {
        const int q = i / PACK_TILE, r = i % PACK_TILE;
        const int64_t lr = r0 + r, gr = a.t_r[q] * a.rows_blk + lr;
        rowoff[q][r] = (lr < a.rows_blk && gr < a.rows_full) ? a.bX[b] + a.rs[gr] : OFF_INVALID;
    }
    for (int i = tid; i < nt * PK_K; i += PK_THREADS)
    {
        const int q = i / PK_K, kk = i % PK_K;
        const int64_t lk = k0 + kk, gk = a.t_c[q] * a.k_blk + lk;
        koff[q][kk] = (lk < a.k_blk && gk < a.k_full) ? a.ks[gk] : OFF_INVALID;
    }
    __syncthreads();

    // Gather and sum: with kfast the 32 lanes of a warp walk 32 consecutive k
    // of one row, else 32 consecutive rows of one k.  Terms outermost, so all
    // loads of one term are independent and in flight together.
    constexpr int E = PACK_TILE * PK_K / PK_THREADS;
    double v[E];
#pragma unroll
    for (int x = 0; x < E; x++) v[x] = 0.0;
    for (int q = 0; q < nt; q++)
    {
        const bool neg = a.t_s[q] < 0;
#pragma unroll
        for (int x = 0; x < E; x++)
        {
            const int r = a.kfast ? warp + 8 * x : lane + 32 * (x & 3);
            const int kk = a.kfast ? lane : warp + 8 * (x >> 2);
            const int64_t ro = rowoff[q][r], ko = koff[q][kk];
            if (ro != OFF_INVALID && ko != OFF_INVALID)
            {
                const double e = a.X[ro + ko];
                v[x] += neg ? -e : e;
            }
        }
    }
#pragma unroll
    for (int x = 0; x < E; x++)
    {
        const int r = a.kfast ? warp + 8 * x : lane + 32 * (x & 3);
        const int kk = a.kfast ? lane : warp + 8 * (x >> 2);
        buf[r][kk] = v[x];
    }
    __syncthreads();
    // Write tile rows (one k each) in the swizzled order: 128 consecutive
    // doubles per k, so every warp store is contiguous.
    double* out = a.out + ((b * a.tiles + t) * a.k_pad + k0) * PACK_TILE;
#pragma unroll 4
    for (int x = 0; x < PACK_TILE * PK_K / PK_THREADS; x++)
    {
        const int r = lane + 32 * (x & 3);
        const int kk = warp + 8 * (x >> 2);
        if (k0 + kk < a.k_pad)
            out[(int64_t)kk * PACK_TILE + tile_pos((int)((k0 + kk) & 7), r, 0)] = buf[r][kk];
    }
}

// ---- packed GEMM ------------------------------------------------------------------

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" :: "r"(dst), "l"(src));
}

__device__ __forceinline__ void cp_async_commit()
{
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}

template <int N>
__device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;\n" :: "n"(N) : "memory");
}

__device__ __forceinline__ void dmma(double (&c)[4], double a0, double a1, double b0)
{
    asm("mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 "
        "{%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
        : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
        : "d"(a0), "d"(a1), "d"(b0));
}

template <int BK_, int STAGES_, int WM_, int WN_>
struct PCfg
{
    static constexpr int BM = PACK_TILE, BN = PACK_TILE, BK = BK_, STAGES = STAGES_;
    static constexpr int WM = WM_, WN = WN_, NT = 32 * WM * WN;
    static constexpr int WTM = BM / WM, WTN = BN / WN, MI = WTM / 16, NI = WTN / 8;
    static constexpr size_t stage_bytes = size_t(BK) * (BM + BN) * 8;
    static constexpr size_t smem = STAGES * stage_bytes + size_t(4) * (BM + BN) * 8;
    static_assert(PACK_KSTEP % BK == 0 || BK % PACK_KSTEP == 0, "k-step compatible with packing");
    static_assert(BK % 8 == 0, "swizzle period");
    static_assert((BK * BM / 2) % NT == 0, "16-byte chunks per thread");
};

// One output tile (work item w of the problem `a`) of the packed GEMM.
template <class K>
__device__ __forceinline__ void packed_tile(const PackedGemmArgs& a, int64_t w, unsigned char* smem)
{
    constexpr int BM = K::BM, BN = K::BN, BK = K::BK, NT = K::NT, STAGES = K::STAGES;
    constexpr int MI = K::MI, NI = K::NI;
    double* As = reinterpret_cast<double*>(smem);
    double* Bs = As + STAGES * BK * BM;
    int64_t* rowC = reinterpret_cast<int64_t*>(Bs + STAGES * BK * BN);
    int64_t* colC = rowC + 4 * BM;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t4 = lane & 3;
    const int wm = (warp / K::WN) * K::WTM;
    const int wn = (warp % K::WN) * K::WTN;
    const int64_t tiles = a.tiles_m * a.tiles_n;
    const int64_t nk = a.k_pad / BK;

    {
        const int64_t b = w / tiles;
        const int64_t tw = w - b * tiles;
        const int64_t GROUP = 8;
        const int64_t group = tw / (GROUP * a.tiles_n);
        const int64_t first_m = group * GROUP;
        const int64_t gsize = (a.tiles_m - first_m) < GROUP ? (a.tiles_m - first_m) : GROUP;
        const int64_t tm = first_m + (tw % gsize);
        const int64_t tn = (tw % (GROUP * a.tiles_n)) / gsize;

        __syncthreads();   // previous tile's epilogue done with the tables
        for (int i = tid; i < 4 * BM; i += NT)
        {
            const int q = i / BM, r = i % BM;
            const int64_t loc = tm * BM + r;
            const int64_t gi = (q < a.nc ? a.c_r[q] : 0) * a.ms + loc;
            rowC[i] = (q < a.nc && loc < a.ms && gi < a.m) ? a.bC[b] + a.rsC[gi] : OFF_INVALID;
        }
        for (int i = tid; i < 4 * BN; i += NT)
        {
            const int q = i / BN, c = i % BN;
            const int64_t loc = tn * BN + c;
            const int64_t gj = (q < a.nc ? a.c_c[q] : 0) * a.ns + loc;
            colC[i] = (q < a.nc && loc < a.ns && gj < a.n) ? a.csC[gj] : OFF_INVALID;
        }

        const double* Sb = a.S + ((b * a.tiles_m + tm) * a.k_pad) * BM;
        const double* Tb = a.T + ((b * a.tiles_n + tn) * a.k_pad) * BN;
        auto copy_stage = [&](int64_t s) {
            const int buf = (int)(s % STAGES);
            const double* sa = Sb + s * BK * BM;
            const double* sb = Tb + s * BK * BN;
            const uint32_t da = smem_u32(As + buf * BK * BM);
            const uint32_t db = smem_u32(Bs + buf * BK * BN);
#pragma unroll
            for (int c = tid; c < BK * BM / 2; c += NT) cp_async16(da + c * 16, sa + 2 * c);
#pragma unroll
            for (int c = tid; c < BK * BN / 2; c += NT) cp_async16(db + c * 16, sb + 2 * c);
        };

        for (int64_t s = 0; s < STAGES - 1; s++)
        {
            if (s < nk) copy_stage(s);
            cp_async_commit();
        }

        double acc[MI][NI][4];
#pragma unroll
        for (int mi = 0; mi < MI; mi++)
#pragma unroll
            for (int ni = 0; ni < NI; ni++)
#pragma unroll
                for (int e = 0; e < 4; e++) acc[mi][ni][e] = 0.0;

        auto load_frags = [&](const double* Ab, const double* Bb, int k4,
                              double (&af)[MI][2], double (&bf)[NI]) {
            const int kr = k4 + t4;
            const int pg = 2 * ((g + swz_c(kr)) & 7);
#pragma unroll
            for (int mi = 0; mi < MI; mi++)
            {
                const double2 v = *reinterpret_cast<const double2*>(Ab + kr * BM + wm + mi * 16 + pg);
                af[mi][0] = v.x; af[mi][1] = v.y;
            }
#pragma unroll
            for (int nj = 0; nj < NI / 2; nj++)
            {
                const double2 v = *reinterpret_cast<const double2*>(Bb + kr * BN + wn + nj * 16 + pg);
                bf[2 * nj] = v.x; bf[2 * nj + 1] = v.y;
            }
        };

        for (int64_t s = 0; s < nk; s++)
        {
            cp_async_wait<STAGES - 2>();
            __syncthreads();
            if (s + STAGES - 1 < nk) copy_stage(s + STAGES - 1);
            cp_async_commit();
            const int buf = (int)(s % STAGES);
            const double* Ab = As + buf * BK * BM;
            const double* Bb = Bs + buf * BK * BN;
            double af[2][MI][2], bf[2][NI];
            load_frags(Ab, Bb, 0, af[0], bf[0]);
#pragma unroll
            for (int q = 0; q < BK / 4; q++)
            {
                const int cur = q & 1;
                if (q + 1 < BK / 4) load_frags(Ab, Bb, (q + 1) * 4, af[cur ^ 1], bf[cur ^ 1]);
#pragma unroll
                for (int mi = 0; mi < MI; mi++)
#pragma unroll
                    for (int ni = 0; ni < NI; ni++)
                        dmma(acc[mi][ni], af[cur][mi][0], af[cur][mi][1], bf[cur][ni]);
            }
        }
        cp_async_wait<0>();

        // Epilogue: C_q = (first ? beta*C_q : C_q) + sign_q*alpha*S*T.  All
        // loads of C are issued before the stores so their latencies overlap.
        for (int q = 0; q < a.nc; q++)
        {
            const int64_t* rt = rowC + q * BM;
            const int64_t* ct = colC + q * BN;
            const double coef = a.c_s[q] < 0 ? -a.alpha : a.alpha;
            const bool first = a.c_first[q] != 0;
            const bool read_c = !first || a.beta != 0.0;
            const double cb = first ? a.beta : 1.0;
#pragma unroll
            for (int mi = 0; mi < MI; mi++)
            {
                double cv[2][NI][2];
#pragma unroll
                for (int hr = 0; hr < 2; hr++)
                {
                    const int64_t ro = rt[wm + mi * 16 + g + hr * 8];
#pragma unroll
                    for (int ni = 0; ni < NI; ni++)
#pragma unroll
                        for (int hc = 0; hc < 2; hc++)
                        {
                            const int64_t co = ct[wn + ni * 8 + t4 * 2 + hc];
                            cv[hr][ni][hc] = (read_c && ro != OFF_INVALID && co != OFF_INVALID)
                                                 ? a.C[ro + co] : 0.0;
                        }
                }
#pragma unroll
                for (int hr = 0; hr < 2; hr++)
                {
                    const int64_t ro = rt[wm + mi * 16 + g + hr * 8];
                    if (ro == OFF_INVALID) continue;
#pragma unroll
                    for (int ni = 0; ni < NI; ni++)
#pragma unroll
                        for (int hc = 0; hc < 2; hc++)
                        {
                            const int64_t co = ct[wn + ni * 8 + t4 * 2 + hc];
                            if (co == OFF_INVALID) continue;
                            a.C[ro + co] = coef * acc[mi][ni][hr * 2 + hc] + cb * cv[hr][ni][hc];
                        }
                }
            }
        }
    }
}

template <class K>
__global__ void __launch_bounds__(K::NT, 1)
packed_gemm_kernel(const __grid_constant__ PackedGemmArgs a)
{
    extern __shared__ __align__(128) unsigned char smem[];
    const int64_t work = a.batch * a.tiles_m * a.tiles_n;
    for (int64_t w = blockIdx.x; w < work; w += gridDim.x) packed_tile<K>(a, w, smem);
}

// Grouped form: one persistent grid over the tiles of many problems (each
// with its own packed S and T); work item w belongs to the problem p with
// prefix[p] <= w < prefix[p + 1].  The problem's descriptor is staged in
// shared memory whenever a CTA moves to another problem.
template <class K>
__global__ void __launch_bounds__(K::NT, 1)
packed_gemm_grouped_kernel(const __grid_constant__ PackedGroupArgs g)
{
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ PackedGemmArgs desc;
    static_assert(sizeof(PackedGemmArgs) % 8 == 0, "descriptor copied as 8-byte words");
    int cur = -1;
    for (int64_t w = blockIdx.x; w < g.total; w += gridDim.x)
    {
        int lo = 0, hi = g.nprob - 1;
        while (lo < hi)
        {
            const int mid = (lo + hi + 1) >> 1;
            if (g.prefix[mid] <= w) lo = mid; else hi = mid - 1;
        }
        if (lo != cur)
        {
            __syncthreads();   // the previous tile no longer reads the descriptor
            const int64_t* src = reinterpret_cast<const int64_t*>(g.probs + lo);
            int64_t* dst = reinterpret_cast<int64_t*>(&desc);
            for (int i = threadIdx.x; i < (int)(sizeof(PackedGemmArgs) / 8); i += blockDim.x) dst[i] = src[i];
            __syncthreads();
            cur = lo;
        }
        packed_tile<K>(desc, w - g.prefix[lo], smem);
    }
}

template <class K>
cudaError_t launch_packed_cfg(const PackedGemmArgs& a, cudaStream_t stream, int num_sms)
{
    static_assert(K::smem <= 227 * 1024, "shared memory budget");
    if (a.k_pad % K::BK) return cudaErrorInvalidValue;
    auto kern = packed_gemm_kernel<K>;
    cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)K::smem);
    if (err != cudaSuccess) return err;
    const int64_t work = a.batch * a.tiles_m * a.tiles_n;
    int per_sm = 0;
    err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, K::NT, K::smem);
    if (err != cudaSuccess) return err;
    if (per_sm < 1) per_sm = 1;
    int64_t grid = (int64_t)num_sms * per_sm;
    if (work < grid) grid = work;
    timing_begin(KK_PACKED_GEMM, stream);
    kern<<<(unsigned)grid, K::NT, K::smem, stream>>>(a);
    timing_end(KK_PACKED_GEMM, stream);
    return cudaGetLastError();
}

template <class K>
cudaError_t launch_packed_grouped_cfg(const PackedGroupArgs& g, cudaStream_t stream, int num_sms)
{
    constexpr size_t static_smem = sizeof(PackedGemmArgs);
    static_assert(K::smem + static_smem <= 227 * 1024, "shared memory budget");
    auto kern = packed_gemm_grouped_kernel<K>;
    cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)K::smem);
    if (err != cudaSuccess) return err;
    int per_sm = 0;
    err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, K::NT, K::smem);
    if (err != cudaSuccess) return err;
    if (per_sm < 1) per_sm = 1;
    int64_t grid = (int64_t)num_sms * per_sm;
    if (g.total < grid) grid = g.total;
    timing_begin(KK_PACKED_GEMM, stream);
    kern<<<(unsigned)grid, K::NT, K::smem, stream>>>(g);
    timing_end(KK_PACKED_GEMM, stream);
    return cudaGetLastError();
}

using PG0 = PCfg<32, 3, 4, 4>;   // 16 warps of 32 x 32, k-step 32
using PG1 = PCfg<16, 6, 4, 4>;
using PG2 = PCfg<16, 4, 4, 4>;
using PG3 = PCfg<16, 4, 2, 4>;   // 8 warps of 64 x 32

}  // namespace

cudaError_t launch_pack(const PackArgs& a, cudaStream_t stream)
{
    if (a.batch <= 0 || a.tiles <= 0 || a.k_pad <= 0) return cudaSuccess;
    if (a.k_pad % PK_K && a.k_pad % PACK_KSTEP) return cudaErrorInvalidValue;
    dim3 grid((unsigned)((a.k_pad + PK_K - 1) / PK_K), (unsigned)a.tiles, (unsigned)a.batch);
    if (a.tiles > 65535 || a.batch > 65535) return cudaErrorInvalidValue;
    timing_begin(KK_PACK, stream);
    pack_kernel<<<grid, PK_THREADS, 0, stream>>>(a);
    timing_end(KK_PACK, stream);
    cudaError_t err = cudaGetLastError();
    if (err == cudaSuccess) g_launches++;
    return err;
}

cudaError_t launch_packed_gemm(const PackedGemmArgs& a, cudaStream_t stream, int num_sms, int config)
{
    if (a.batch <= 0 || a.tiles_m <= 0 || a.tiles_n <= 0) return cudaSuccess;
    if (a.nc < 1 || a.nc > 4) return cudaErrorInvalidValue;
    if (config < 0)
    {
        static const int env = [] {
            const char* s = std::getenv("TBLIS_STRA_PACKED_CONFIG");
            return s ? std::atoi(s) : -1;
        }();
        config = env;
    }
    cudaError_t err;
    switch (config)
    {
        case 1:  err = launch_packed_cfg<PG1>(a, stream, num_sms); break;
        case 2:  err = launch_packed_cfg<PG2>(a, stream, num_sms); break;
        case 3:  err = launch_packed_cfg<PG3>(a, stream, num_sms); break;
        default: err = launch_packed_cfg<PG0>(a, stream, num_sms); break;
    }
    if (err == cudaSuccess) g_launches++;
    return err;
}

cudaError_t launch_packed_gemm_grouped(const PackedGroupArgs& g, cudaStream_t stream, int num_sms)
{
    if (g.nprob <= 0 || g.total <= 0) return cudaSuccess;
    const cudaError_t err = launch_packed_grouped_cfg<PG0>(g, stream, num_sms);
    if (err == cudaSuccess) g_launches++;
    return err;
}

}  // namespace tsb
