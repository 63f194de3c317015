// FP64 Strassen / plain contraction kernel for sm_100a (B200) on the FP64
// tensor cores (DMMA, mma.sync m16n8k4 f64; tcgen05 has no f64 kind).
//
// What it replaces in the reference (one kernel for all of it):
//   * the GEMM control tree nc/kc/mc/nr/mr (src/stra_nodes/stra_partm.hpp:12-131);
//   * the fused Strassen packing sum_i coeff_i * A_i, sum_j coeff_j * B_j
//     (stra_pack_{two,four}_*, src/kernels/3m/gemm.hpp:504-816, 1344-1917) --
//     here the raw blocks are gathered through the scatter vectors into shared
//     memory with cp.async and summed while being read into MMA fragments;
//   * the micro-kernel C_p += coeff_p * alpha * A*B for up to 4 C blocks
//     (stra_gemm_ukr_{two,four}, src/stra_nodes/stra_gemm_ukr.hpp:622-940) --
//     here the epilogue of each product;
//   * the per-product loop M0..M6 / M0..M48 with barriers between products
//     (src/stra_internal/3t/stra_mult.cxx:426-590) -- here every CTA owns one
//     tile position of the block grid and runs all products for it in order,
//     so C blocks shared by several products need no atomics and no barrier,
//     and beta is applied exactly once (by the first product touching a block).
//
// Tile shapes are template parameters (BM x BN per CTA, k-step BK, WM x WN
// warps each owning a (BM/WM) x (BN/WN) tile of m16n8k4 fragments, STAGES deep
// cp.async ring).  Shared-memory tiles are stored k-major, rows g and g+8 of
// each 16-row group (columns for B) adjacent and swizzled per k (tile_pos), so
// every fragment pair a thread needs is one 128-bit load and both the loads and
// the cp.async writes are free of bank conflicts.
// A persistent grid walks (batch, tile) work items.
#include "kernels.cuh"
#include "tile_layout.cuh"
#include "timing.hpp"

#include <atomic>

namespace tsb {

namespace {

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void cp_async8(uint32_t dst, const void* src, int src_bytes)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n"
                 :: "r"(dst), "l"(src), "r"(src_bytes));
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

template <int BM_, int BN_, int BK_, int WM_, int WN_, int STAGES_, int NA_, int NB_, int MINB_, int HM_>
struct Cfg
{
    static constexpr int BM = BM_, BN = BN_, BK = BK_, WM = WM_, WN = WN_;
    static constexpr int STAGES = STAGES_, NA = NA_, NB = NB_, MINB = MINB_;
    static constexpr int HMAX = HM_;                       // largest block grid side H
    static constexpr int NT = 32 * WM * WN;
    static constexpr int WTM = BM / WM, WTN = BN / WN;     // warp tile
    static constexpr int MI = WTM / 16, NI = WTN / 8;      // fragments per warp
    static constexpr int LDA = BM, LDB = BN;               // rows 128-byte aligned (swizzled)
    static constexpr int R = STAGES + 1;                   // k-offset table ring
    static constexpr size_t a_bytes = size_t(STAGES) * NA * BK * LDA * 8;
    static constexpr size_t b_bytes = size_t(STAGES) * NB * BK * LDB * 8;
    static constexpr size_t tab_bytes = size_t(HMAX) * (BM + BM + BN + BN) * 8;
    static constexpr size_t k_bytes = size_t(R) * HMAX * BK * 8 * 2;
    static constexpr size_t smem = a_bytes + b_bytes + tab_bytes + k_bytes;
    static_assert(WTM % 16 == 0 && WTN % 16 == 0, "warp tile must hold whole fragment pairs");
    static_assert(BK % 8 == 0, "k-step is a multiple of 8 (loader lane map)");
    static_assert(BM % 16 == 0 && BN % 16 == 0, "tiles are whole 16-row groups");
    static_assert(2 * HMAX * BK <= NT, "one thread per k-table entry");
    static_assert((BK * BM) % NT == 0 && (BK * BN) % NT == 0, "loader covers the tile");
};

// One (batch, tile) work item of a contraction: all of its Strassen products.
template <class K, bool KA, bool KB>
__device__ __forceinline__ void dmma_tile(const DmmaArgs& args, int64_t w, unsigned char* smem)
{
    constexpr int BM = K::BM, BN = K::BN, BK = K::BK, NT = K::NT;
    constexpr int NA = K::NA, NB = K::NB, STAGES = K::STAGES, R = K::R;
    constexpr int LDA = K::LDA, LDB = K::LDB, MI = K::MI, NI = K::NI;
    constexpr int HMAX = K::HMAX;
    double* As = reinterpret_cast<double*>(smem);
    double* Bs = reinterpret_cast<double*>(smem + K::a_bytes);
    int64_t* rowA = reinterpret_cast<int64_t*>(smem + K::a_bytes + K::b_bytes);
    int64_t* rowC = rowA + HMAX * BM;
    int64_t* colB = rowC + HMAX * BM;
    int64_t* colC = colB + HMAX * BN;
    int64_t* kA = colC + HMAX * BN;           // [R][HMAX][BK]
    int64_t* kB = kA + R * HMAX * BK;         // [R][HMAX][BK]

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int g = lane >> 2;         // groupID
    const int t4 = lane & 3;         // threadID_in_group
    const int wm = (warp / K::WN) * K::WTM;
    const int wn = (warp % K::WN) * K::WTN;

    const int64_t tiles = (int64_t)args.tiles_m * args.tiles_n;
    const int64_t nk = (args.ks + BK - 1) / BK;
    const int H = args.H;
    const int Hc = args.Hc;

        const int64_t b = w / tiles;
        const int64_t tw = w - b * tiles;
        // Grouped raster (8 tile rows per group) so concurrent CTAs share panels in L2.
        const int64_t GROUP = 8;
        const int64_t group = tw / (GROUP * args.tiles_n);
        const int64_t first_m = group * GROUP;
        const int64_t gsize = (args.tiles_m - first_m) < GROUP ? (args.tiles_m - first_m) : GROUP;
        const int64_t ti = first_m + (tw % gsize);
        const int64_t tj = (tw % (GROUP * args.tiles_n)) / gsize;
        const int64_t tm0 = ti * BM;
        const int64_t tn0 = tj * BN;

        __syncthreads();   // previous work item done with the tables
        const int64_t offA = args.bA[b], offB = args.bB[b], offC = args.bC[b];
        for (int i = tid; i < HMAX * BM; i += NT)
        {
            const int h = i / BM, r = i % BM;
            const int64_t loc = tm0 + r, gi = h * args.ms + loc;
            rowA[i] = (h < H && loc < args.ms && gi < args.m) ? offA + args.rsA[gi] : OFF_INVALID;
            rowC[i] = (h < Hc && loc < args.ms && gi < args.mC) ? offC + args.rsC[gi] : OFF_INVALID;
        }
        for (int i = tid; i < HMAX * BN; i += NT)
        {
            const int h = i / BN, c = i % BN;
            const int64_t loc = tn0 + c, gj = h * args.ns + loc;
            colB[i] = (h < H && loc < args.ns && gj < args.n) ? offB + args.csB[gj] : OFF_INVALID;
            colC[i] = (h < Hc && loc < args.ns && gj < args.nC) ? args.csC[gj] : OFF_INVALID;
        }

        for (int p = 0; p < args.nprod; p++)
        {
            const DevProduct& P = args.prod[p];
            const int na = P.na, nb = P.nb;

            // k offset table of one stage: kX[slot][h][kk] for every k part h;
            // threads [0, HMAX*BK) fill A entries, [HMAX*BK, 2*HMAX*BK) B entries.
            auto load_ktab = [&](int64_t stage, int64_t& v) {
                const int e = tid % (HMAX * BK);
                const int h = e / BK, kk = e % BK;
                const int64_t kl = stage * BK + kk, gk = h * args.ks + kl;
                const bool ok = (h < H && kl < args.ks && gk < args.k);
                v = OFF_INVALID;
                if (ok)
                {
                    if (tid < HMAX * BK) v = args.ksA[gk];
                    else if (tid < 2 * HMAX * BK) v = args.ksB[gk];
                }
            };
            auto store_ktab = [&](int64_t stage, int64_t v) {
                const int sl = (int)(stage % R);
                if (tid < HMAX * BK)           kA[sl * HMAX * BK + tid] = v;
                else if (tid < 2 * HMAX * BK)  kB[sl * HMAX * BK + tid - HMAX * BK] = v;
            };

            // Loader.  Element x of A term i lands on tile (row r, k kk); with
            // KA consecutive threads walk k (coalesced when A is contiguous
            // along k), otherwise rows.  B likewise with KB.
            constexpr int EA = BK * BM / NT;        // A elements per thread per term
            constexpr int EB = BK * BN / NT;
            constexpr int EPS = NA * EA + NB * EB;  // elements per thread per stage
            constexpr int Q = BK / 4;               // k4 steps per stage
            constexpr int CH = (EPS + Q - 1) / Q;   // loader elements per k4 step
            uint32_t rA[NA], rB[NB];                // row/col table of each term (smem)
            int kofA[NA], kofB[NB];                 // its k part (offset into a k table)
            uint32_t dA[NA], dB[NB];                // its tile in stage buffer 0 (smem)
#pragma unroll
            for (int i = 0; i < NA; i++)
            {
                rA[i] = smem_u32(rowA + (i < na ? P.a_r[i] : 0) * BM);
                kofA[i] = (i < na ? P.a_c[i] : 0) * BK;
                dA[i] = smem_u32(As + (size_t)i * BK * LDA);
            }
#pragma unroll
            for (int j = 0; j < NB; j++)
            {
                rB[j] = smem_u32(colB + (j < nb ? P.b_c[j] : 0) * BN);
                kofB[j] = (j < nb ? P.b_r[j] : 0) * BK;
                dB[j] = smem_u32(Bs + (size_t)j * BK * LDB);
            }
            auto lds64 = [](uint32_t addr) {
                int64_t v;
                asm volatile("ld.shared.s64 %0, [%1];\n" : "=l"(v) : "r"(addr));
                return v;
            };
            auto issue_elem = [&](int j, int buf, const int64_t* kAs, const int64_t* kBs) {
                if (j < NA * EA)
                {
                    const int i = j / EA, x = j % EA;
                    if (i < na)
                    {
                        int kk, r;
                        lane_map<BK, BM>(KA, tid + x * NT, kk, r);
                        const int64_t ro = lds64(rA[i] + r * 8);
                        const int64_t ko = kAs[kofA[i] + kk];
                        const bool ok = (ro != OFF_INVALID) & (ko != OFF_INVALID);
                        const uint32_t dst = dA[i] + (uint32_t)(buf * NA * BK * LDA + tile_pos(kk, r, LDA)) * 8;
                        cp_async8(dst, ok ? args.A + (ro + ko) : args.A, ok ? 8 : 0);
                    }
                }
                else
                {
                    const int jj = j - NA * EA;
                    const int i = jj / EB, x = jj % EB;
                    if (i < nb)
                    {
                        int kk, c;
                        lane_map<BK, BN>(KB, tid + x * NT, kk, c);
                        const int64_t co = lds64(rB[i] + c * 8);
                        const int64_t ko = kBs[kofB[i] + kk];
                        const bool ok = (co != OFF_INVALID) & (ko != OFF_INVALID);
                        const uint32_t dst = dB[i] + (uint32_t)(buf * NB * BK * LDB + tile_pos(kk, c, LDB)) * 8;
                        cp_async8(dst, ok ? args.B + (ko + co) : args.B, ok ? 8 : 0);
                    }
                }
            };
            auto issue_stage = [&](int64_t stage) {
                const int buf = (int)(stage % STAGES);
                const int sl = (int)(stage % R);
#pragma unroll
                for (int j = 0; j < EPS; j++)
                    issue_elem(j, buf, kA + sl * HMAX * BK, kB + sl * HMAX * BK);
            };

            __syncthreads();   // previous product's last stage fully consumed
            // Prologue: k tables for stages 0..STAGES-1, then data for 0..STAGES-2.
            for (int64_t s = 0; s < STAGES; s++)
            {
                int64_t v;
                load_ktab(s, v);
                store_ktab(s, v);
            }
            __syncthreads();
            for (int64_t s = 0; s < STAGES - 1; s++)
            {
                if (s < nk) issue_stage(s);
                cp_async_commit();
            }

            double acc[MI][NI][4];
#pragma unroll
            for (int mi = 0; mi < MI; mi++)
#pragma unroll
                for (int ni = 0; ni < NI; ni++)
#pragma unroll
                    for (int e = 0; e < 4; e++) acc[mi][ni][e] = 0.0;

            // Each operand sum is formed as x_0 + sum_i rel_i * x_i with
            // rel_i = sign_i * sign_0 in {+1, -1} (one exact FMA per term);
            // sign_0 of A and B moves into the C coefficient.
            double ra[NA], rb[NB];
#pragma unroll
            for (int i = 0; i < NA; i++) ra[i] = (i < na && P.a_s[i] * P.a_s[0] < 0) ? -1.0 : 1.0;
#pragma unroll
            for (int j = 0; j < NB; j++) rb[j] = (j < nb && P.b_s[j] * P.b_s[0] < 0) ? -1.0 : 1.0;
            const bool lead_neg = (P.a_s[0] * P.b_s[0]) < 0;

            // Fragments of one k4 step: signed sums over the terms, read as
            // 128-bit pairs from the permuted layouts.
            auto load_frags = [&](const double* Ab, const double* Bb, int k4,
                                  double (&af)[MI][2], double (&bf)[NI]) {
                const int kr = k4 + t4;
                const int pg = 2 * ((g + swz_c(kr)) & 7);   // swizzled pair of rows g, g+8
#pragma unroll
                for (int mi = 0; mi < MI; mi++)
                {
                    const int pos = kr * LDA + wm + mi * 16 + pg;
                    double2 v = *reinterpret_cast<const double2*>(Ab + pos);
                    double x0 = v.x, x1 = v.y;
#pragma unroll
                    for (int i = 1; i < NA; i++)
                    {
                        if (i < na)
                        {
                            double2 u = *reinterpret_cast<const double2*>(Ab + (size_t)i * BK * LDA + pos);
                            x0 = fma(ra[i], u.x, x0);
                            x1 = fma(ra[i], u.y, x1);
                        }
                    }
                    af[mi][0] = x0; af[mi][1] = x1;
                }
#pragma unroll
                for (int nj = 0; nj < NI / 2; nj++)
                {
                    const int pos = kr * LDB + wn + nj * 16 + pg;
                    double2 v = *reinterpret_cast<const double2*>(Bb + pos);
                    double y0 = v.x, y1 = v.y;
#pragma unroll
                    for (int j = 1; j < NB; j++)
                    {
                        if (j < nb)
                        {
                            double2 u = *reinterpret_cast<const double2*>(Bb + (size_t)j * BK * LDB + pos);
                            y0 = fma(rb[j], u.x, y0);
                            y1 = fma(rb[j], u.y, y1);
                        }
                    }
                    bf[2 * nj] = y0; bf[2 * nj + 1] = y1;
                }
            };

            for (int64_t s = 0; s < nk; s++)
            {
                cp_async_wait<STAGES - 2>();
                __syncthreads();
                // This stage refills buffer (s+STAGES-1) % STAGES, whose k table
                // is ready, spread over the k4 steps between the DMMA batches;
                // the k table of stage s+STAGES is fetched into a register.
                const int64_t sn = s + STAGES - 1;
                const bool refill = sn < nk;
                const int nbuf = (int)(sn % STAGES);
                const int nsl = (int)(sn % R);
                const int64_t* kAs = kA + nsl * HMAX * BK;
                const int64_t* kBs = kB + nsl * HMAX * BK;
                int64_t kv;
                load_ktab(s + STAGES, kv);

                const int buf = (int)(s % STAGES);
                const double* Ab = As + (size_t)buf * NA * BK * LDA;
                const double* Bb = Bs + (size_t)buf * NB * BK * LDB;
                double af[2][MI][2], bf[2][NI];
                load_frags(Ab, Bb, 0, af[0], bf[0]);
#pragma unroll
                for (int q = 0; q < Q; q++)
                {
                    const int cur = q & 1;
                    if (q + 1 < Q) load_frags(Ab, Bb, (q + 1) * 4, af[cur ^ 1], bf[cur ^ 1]);
#pragma unroll
                    for (int mi = 0; mi < MI; mi++)
#pragma unroll
                        for (int ni = 0; ni < NI; ni++)
                            dmma(acc[mi][ni], af[cur][mi][0], af[cur][mi][1], bf[cur][ni]);
                    if (refill)
                    {
#pragma unroll
                        for (int c = 0; c < CH; c++)
                            if (q * CH + c < EPS) issue_elem(q * CH + c, nbuf, kAs, kBs);
                    }
                }
                cp_async_commit();
                store_ktab(s + STAGES, kv);
            }
            cp_async_wait<0>();

            // Epilogue: C_q = (first ? beta*C_q : C_q) + sign_q*alpha*M for each target.
            for (int q = 0; q < P.nc; q++)
            {
                const int64_t* rt = rowC + P.c_r[q] * BM;
                const int64_t* ct = colC + P.c_c[q] * BN;
                const double coef = ((P.c_s[q] < 0) != lead_neg) ? -args.alpha : args.alpha;
                const bool first = P.c_first[q] != 0;
                const double beta = args.beta;
#pragma unroll
                for (int mi = 0; mi < MI; mi++)
                {
#pragma unroll
                    for (int hr = 0; hr < 2; hr++)
                    {
                        const int64_t ro = rt[wm + mi * 16 + g + hr * 8];
                        if (ro == OFF_INVALID) continue;
#pragma unroll
                        for (int ni = 0; ni < NI; ni++)
                        {
#pragma unroll
                            for (int hc = 0; hc < 2; hc++)
                            {
                                const int64_t co = ct[wn + ni * 8 + t4 * 2 + hc];
                                if (co == OFF_INVALID) continue;
                                double* ptr = args.C + ro + co;
                                double v = coef * acc[mi][ni][hr * 2 + hc];
                                if (!first) v += *ptr;
                                else if (beta != 0.0) v += beta * *ptr;
                                *ptr = v;
                            }
                        }
                    }
                }
            }
        }
}

template <class K, bool KA, bool KB>
__global__ void __launch_bounds__(K::NT, K::MINB)
stra_dmma_kernel(const __grid_constant__ DmmaArgs args)
{
    extern __shared__ __align__(128) unsigned char smem[];
    for (int64_t w = blockIdx.x; w < args.work; w += gridDim.x)
        dmma_tile<K, KA, KB>(args, w, smem);
}

// Grouped launch: the work items of many contractions (one descriptor each,
// in global memory) in one persistent grid; work item w belongs to the
// problem p with prefix[p] <= w < prefix[p+1].
template <class K>
__global__ void __launch_bounds__(K::NT, K::MINB)
stra_dmma_grouped_kernel(const __grid_constant__ DmmaGroupArgs g)
{
    extern __shared__ __align__(128) unsigned char smem[];
    for (int64_t w = blockIdx.x; w < g.total; w += gridDim.x)
    {
        int lo = 0, hi = g.nprob - 1;
        while (lo < hi)
        {
            const int mid = (lo + hi + 1) >> 1;
            if (g.prefix[mid] <= w) lo = mid; else hi = mid - 1;
        }
        const DmmaArgs& a = g.probs[lo];
        const int64_t local = w - g.prefix[lo];
        if (a.a_kfast)
        {
            if (a.b_kfast) dmma_tile<K, true, true>(a, local, smem);
            else           dmma_tile<K, true, false>(a, local, smem);
        }
        else
        {
            if (a.b_kfast) dmma_tile<K, false, true>(a, local, smem);
            else           dmma_tile<K, false, false>(a, local, smem);
        }
    }
}

template <class K>
cudaError_t launch_cfg(const DmmaArgs& in, cudaStream_t stream, int num_sms)
{
    static_assert(K::smem <= 227 * 1024, "shared memory budget");
    auto kern = in.a_kfast ? (in.b_kfast ? stra_dmma_kernel<K, true, true> : stra_dmma_kernel<K, true, false>)
                           : (in.b_kfast ? stra_dmma_kernel<K, false, true> : stra_dmma_kernel<K, false, false>);
    cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)K::smem);
    if (err != cudaSuccess) return err;
    DmmaArgs args = in;
    args.tiles_m = (int)((args.ms + K::BM - 1) / K::BM);
    args.tiles_n = (int)((args.ns + K::BN - 1) / K::BN);
    args.work = args.batch * (int64_t)args.tiles_m * args.tiles_n;
    if (args.work <= 0) return cudaSuccess;
    int per_sm = 0;
    err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, K::NT, K::smem);
    if (err != cudaSuccess) return err;
    if (per_sm < 1) per_sm = 1;
    int64_t grid = (int64_t)num_sms * per_sm;
    if (args.work < grid) grid = args.work;
    timing_begin(KK_FUSED, stream);
    kern<<<(unsigned)grid, K::NT, K::smem, stream>>>(args);
    timing_end(KK_FUSED, stream);
    return cudaGetLastError();
}

// Tile configurations: <BM, BN, BK, WM, WN, STAGES, NA, NB, min CTAs per SM, H max>.
// 16 warps of 32 x 32 per SM keep the DMMA pipe fed (the register file then
// holds 128 registers per thread); 1 CTA of 512 threads or 4 CTAs of 128.
// Plain products on a 1 x 1 grid (ABC at level 0):
using P0 = Cfg<128, 128, 16, 4, 4, 3, 1, 1, 1, 1>;
using P1 = Cfg<64, 64, 16, 2, 2, 3, 1, 1, 4, 1>;
using P2 = Cfg<128, 128, 16, 2, 4, 3, 1, 1, 1, 1>;
// Single-term products on a block grid (AB / Naive GEMMs):
using G0 = Cfg<128, 128, 16, 4, 4, 3, 1, 1, 1, 4>;
// Two-term sums (level 1):
using T0 = Cfg<128, 128, 8, 4, 4, 6, 2, 2, 1, 2>;
using T1 = Cfg<128, 128, 16, 4, 4, 3, 2, 2, 1, 2>;
using T2 = Cfg<128, 128, 8, 2, 4, 4, 2, 2, 1, 2>;
// Four-term sums (level 2):
using F0 = Cfg<128, 128, 8, 4, 4, 3, 4, 4, 1, 4>;
using F1 = Cfg<64, 64, 8, 2, 2, 3, 4, 4, 2, 4>;
using F2 = Cfg<128, 128, 8, 2, 4, 3, 4, 4, 1, 4>;

template <class K>
cudaError_t launch_group_cfg(const DmmaGroupArgs& g, cudaStream_t stream, int num_sms)
{
    static_assert(K::smem <= 227 * 1024, "shared memory budget");
    auto kern = stra_dmma_grouped_kernel<K>;
    cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)K::smem);
    if (err != cudaSuccess) return err;
    if (g.total <= 0 || g.nprob <= 0) return cudaSuccess;
    int per_sm = 0;
    err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, K::NT, K::smem);
    if (err != cudaSuccess) return err;
    if (per_sm < 1) per_sm = 1;
    int64_t grid = (int64_t)num_sms * per_sm;
    if (g.total < grid) grid = g.total;
    timing_begin(KK_FUSED, stream);
    kern<<<(unsigned)grid, K::NT, K::smem, stream>>>(g);
    timing_end(KK_FUSED, stream);
    return cudaGetLastError();
}

// Configuration family for a request: P* (plain, 1 x 1 grid), G0 (single
// terms on a grid), T* (two-term sums, grid <= 2), F* (up to four terms).
int config_family(int terms, int H, int Hc)
{
    if (terms <= 1 && H <= 1 && Hc <= 1) return 0;
    if (terms <= 1) return 1;
    if (terms <= 2 && H <= 2 && Hc <= 2) return 2;
    return 3;
}

// FP64 tensor-pipe ceiling: every warp issues `iters` rounds of 8
// independent m16n8k4 DMMAs on register operands (no memory traffic), so the
// pipe, not the operand feed, sets the rate.  The result is stored only if it
// equals an impossible value (the operands are non-negative, so the sum is),
// which keeps the loop alive.
__device__ double g_dmma_peak_sink;

__global__ void __launch_bounds__(512, 2) dmma_peak_kernel(int iters)
{
    double acc[8][4];
#pragma unroll
    for (int j = 0; j < 8; j++)
#pragma unroll
        for (int e = 0; e < 4; e++) acc[j][e] = 0.0;
    const double a0 = 1e-3 * (threadIdx.x & 31), a1 = 2e-3, b0 = 1e-3 * blockIdx.x;
    for (int i = 0; i < iters; i++)
    {
#pragma unroll
        for (int j = 0; j < 8; j++) dmma(acc[j], a0, a1, b0);
    }
    double t = 0.0;
#pragma unroll
    for (int j = 0; j < 8; j++) t += acc[j][0] + acc[j][1] + acc[j][2] + acc[j][3];
    if (t == -1.0) g_dmma_peak_sink = t;
}

}  // namespace

std::atomic<unsigned long long> g_launches{0};

cudaError_t measure_dmma_peak(int iters, int num_sms, cudaStream_t stream, double* tflops, double* ms)
{
    if (iters <= 0 || num_sms <= 0) return cudaErrorInvalidValue;
    const int per_sm = 2, threads = 512;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t err = cudaEventCreate(&e0);
    if (err == cudaSuccess) err = cudaEventCreate(&e1);
    if (err == cudaSuccess)
    {
        dmma_peak_kernel<<<num_sms * per_sm, threads, 0, stream>>>(iters);   // warm-up
        cudaEventRecord(e0, stream);
        dmma_peak_kernel<<<num_sms * per_sm, threads, 0, stream>>>(iters);
        cudaEventRecord(e1, stream);
        err = cudaEventSynchronize(e1);
    }
    float t = 0.f;
    if (err == cudaSuccess) err = cudaEventElapsedTime(&t, e0, e1);
    if (err == cudaSuccess) err = cudaGetLastError();
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (err != cudaSuccess) return err;
    g_launches += 2;
    const double flops = 2.0 * 16 * 8 * 4 * 8.0 * (double)iters * (threads / 32) * (double)num_sms * per_sm;
    *ms = t;
    *tflops = flops / (t * 1e-3) / 1e12;
    return cudaSuccess;
}

void dmma_tile_shape(int terms, int H, int Hc, int config, int* bm, int* bn)
{
    int m = 128, n = 128;
    switch (config_family(terms, H, Hc))
    {
        case 0: if (config == 1) { m = P1::BM; n = P1::BN; } else if (config == 2) { m = P2::BM; n = P2::BN; }
                else { m = P0::BM; n = P0::BN; } break;
        case 1: m = G0::BM; n = G0::BN; break;
        case 2: if (config == 1) { m = T1::BM; n = T1::BN; } else if (config == 2) { m = T2::BM; n = T2::BN; }
                else { m = T0::BM; n = T0::BN; } break;
        default: if (config == 1) { m = F1::BM; n = F1::BN; } else if (config == 2) { m = F2::BM; n = F2::BN; }
                 else { m = F0::BM; n = F0::BN; } break;
    }
    *bm = m;
    *bn = n;
}

cudaError_t launch_dmma_grouped(const DmmaGroupArgs& g, int terms, int H, int Hc, int config,
                                cudaStream_t stream, int num_sms)
{
    if (terms > 4 || H > 4 || Hc > 4) return cudaErrorInvalidValue;
    cudaError_t err;
    switch (config_family(terms, H, Hc))
    {
        case 0: err = config == 1 ? launch_group_cfg<P1>(g, stream, num_sms)
                    : config == 2 ? launch_group_cfg<P2>(g, stream, num_sms)
                                  : launch_group_cfg<P0>(g, stream, num_sms); break;
        case 1: err = launch_group_cfg<G0>(g, stream, num_sms); break;
        case 2: err = config == 1 ? launch_group_cfg<T1>(g, stream, num_sms)
                    : config == 2 ? launch_group_cfg<T2>(g, stream, num_sms)
                                  : launch_group_cfg<T0>(g, stream, num_sms); break;
        default: err = config == 1 ? launch_group_cfg<F1>(g, stream, num_sms)
                     : config == 2 ? launch_group_cfg<F2>(g, stream, num_sms)
                                   : launch_group_cfg<F0>(g, stream, num_sms); break;
    }
    if (err == cudaSuccess) g_launches++;
    return err;
}

unsigned long long launches() { return g_launches.load(); }

cudaError_t launch_dmma(const DmmaArgs& args, int terms, cudaStream_t stream, int num_sms, int config)
{
    if (args.batch <= 0 || args.ms <= 0 || args.ns <= 0) return cudaSuccess;
    if (terms > 4 || args.H > 4 || args.Hc > 4) return cudaErrorInvalidValue;
    cudaError_t err;
    if (terms <= 1 && args.H <= 1 && args.Hc <= 1)
    {
        switch (config)
        {
            case 1:  err = launch_cfg<P1>(args, stream, num_sms); break;
            case 2:  err = launch_cfg<P2>(args, stream, num_sms); break;
            default: err = launch_cfg<P0>(args, stream, num_sms); break;
        }
    }
    else if (terms <= 1)
    {
        err = launch_cfg<G0>(args, stream, num_sms);   // block grid up to 4 x 4
    }
    else if (terms <= 2 && args.H <= 2 && args.Hc <= 2)
    {
        switch (config)
        {
            case 1:  err = launch_cfg<T1>(args, stream, num_sms); break;
            case 2:  err = launch_cfg<T2>(args, stream, num_sms); break;
            default: err = launch_cfg<T0>(args, stream, num_sms); break;
        }
    }
    else
    {
        // up to 4 terms per sum on a block grid up to 4 x 4
        switch (config)
        {
            case 1:  err = launch_cfg<F1>(args, stream, num_sms); break;
            case 2:  err = launch_cfg<F2>(args, stream, num_sms); break;
            default: err = launch_cfg<F0>(args, stream, num_sms); break;
        }
    }
    if (err == cudaSuccess) g_launches++;
    return err;
}

}  // namespace tsb
