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
// Tile: 128 x 128 per CTA, k-step 8, 8 warps as 2 (m) x 4 (n), 64 x 32 per warp
// (4 x 4 m16n8k4 fragments).  A persistent grid walks (batch, tile) work items.
#include "kernels.cuh"

#include <atomic>

namespace tsb {

namespace {

constexpr int BM = 128;
constexpr int BN = 128;
constexpr int BK = 8;
constexpr int NT = 256;
constexpr int PAD = 4;            // doubles; row pitch 132*8 B = 32 mod 128 B: conflict-free fragments
constexpr int LDA = BM + PAD;
constexpr int LDB = BN + PAD;
constexpr int HMAX = 4;

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void cp_async8(uint32_t dst, const void* src, int src_bytes)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n"
                 :: "r"(dst), "l"(src), "r"(src_bytes) : "memory");
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
    asm volatile("mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 "
                 "{%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
                 : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
                 : "d"(a0), "d"(a1), "d"(b0));
}

// Flip the sign of x when mask has the sign bit set (integer op, no FP64 multiply).
__device__ __forceinline__ double apply_sign(double x, long long mask)
{
    return __longlong_as_double(__double_as_longlong(x) ^ mask);
}

template <int NA, int NB, int STAGES>
struct Smem
{
    static constexpr int R = STAGES + 1;   // ring of per-stage k offset tables
    static constexpr size_t a_bytes = size_t(STAGES) * NA * BK * LDA * 8;
    static constexpr size_t b_bytes = size_t(STAGES) * NB * BK * LDB * 8;
    static constexpr size_t tab_bytes = size_t(HMAX) * (BM + BM + BN + BN) * 8;
    static constexpr size_t k_bytes = size_t(R) * HMAX * BK * 8 * 2;
    static constexpr size_t total = a_bytes + b_bytes + tab_bytes + k_bytes;
};

template <int NA, int NB, int STAGES>
__global__ void __launch_bounds__(NT, 1)
stra_dmma_kernel(const __grid_constant__ DmmaArgs args)
{
    using S = Smem<NA, NB, STAGES>;
    extern __shared__ __align__(128) unsigned char smem[];
    double* As = reinterpret_cast<double*>(smem);
    double* Bs = reinterpret_cast<double*>(smem + S::a_bytes);
    int64_t* rowA = reinterpret_cast<int64_t*>(smem + S::a_bytes + S::b_bytes);
    int64_t* rowC = rowA + HMAX * BM;
    int64_t* colB = rowC + HMAX * BM;
    int64_t* colC = colB + HMAX * BN;
    int64_t* kA = colC + HMAX * BN;           // [R][HMAX][BK]
    int64_t* kB = kA + S::R * HMAX * BK;      // [R][HMAX][BK]

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int g = lane >> 2;         // groupID
    const int t4 = lane & 3;         // threadID_in_group
    const int wm = (warp >> 2) * 64; // 2 warps along m
    const int wn = (warp & 3) * 32;  // 4 warps along n

    const int64_t tiles = (int64_t)args.tiles_m * args.tiles_n;
    const int64_t nk = (args.ks + BK - 1) / BK;
    const int H = args.H;
    const int Hc = args.Hc;

    for (int64_t w = blockIdx.x; w < args.work; w += gridDim.x)
    {
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

            // k offset table of one stage: kX[slot][h][kk] for every k part h.
            auto load_ktab = [&](int64_t stage, int64_t& va, int64_t& vb, int& sl, int& idx) {
                // thread tid < HMAX*BK fills A entry, tid in [HMAX*BK, 2*HMAX*BK) fills B.
                const int e = tid % (HMAX * BK);
                const int h = e / BK, kk = e % BK;
                const int64_t kl = stage * BK + kk, gk = h * args.ks + kl;
                const bool ok = (h < H && kl < args.ks && gk < args.k);
                sl = (int)(stage % S::R);
                idx = e;
                if (tid < HMAX * BK)       va = ok ? args.ksA[gk] : OFF_INVALID;
                else if (tid < 2 * HMAX * BK) vb = ok ? args.ksB[gk] : OFF_INVALID;
            };
            auto store_ktab = [&](int sl, int idx, int64_t va, int64_t vb) {
                if (tid < HMAX * BK)           kA[sl * HMAX * BK + idx] = va;
                else if (tid < 2 * HMAX * BK)  kB[sl * HMAX * BK + idx] = vb;
            };

            // Issue the cp.async gathers of one stage (all A and B terms).
            auto issue_stage = [&](int64_t stage) {
                const int buf = (int)(stage % STAGES);
                const int sl = (int)(stage % S::R);
                const int64_t* kAs = kA + sl * HMAX * BK;
                const int64_t* kBs = kB + sl * HMAX * BK;
#pragma unroll
                for (int i = 0; i < NA; i++)
                {
                    if (i < na)
                    {
                        const int64_t* rtab = rowA + P.a_r[i] * BM;
                        const int64_t* ktab = kAs + P.a_c[i] * BK;
                        double* dst = As + ((size_t)buf * NA + i) * BK * LDA;
#pragma unroll
                        for (int x = 0; x < BK * BM / NT; x++)
                        {
                            const int e = tid + x * NT;
                            const int r = args.a_kfast ? e / BK : e % BM;
                            const int kk = args.a_kfast ? e % BK : e / BM;
                            const int64_t ro = rtab[r], ko = ktab[kk];
                            const bool ok = (ro != OFF_INVALID) && (ko != OFF_INVALID);
                            const double* src = ok ? args.A + ro + ko : args.A;
                            cp_async8(smem_u32(dst + kk * LDA + r), src, ok ? 8 : 0);
                        }
                    }
                }
#pragma unroll
                for (int j = 0; j < NB; j++)
                {
                    if (j < nb)
                    {
                        const int64_t* ctab = colB + P.b_c[j] * BN;
                        const int64_t* ktab = kBs + P.b_r[j] * BK;
                        double* dst = Bs + ((size_t)buf * NB + j) * BK * LDB;
#pragma unroll
                        for (int x = 0; x < BK * BN / NT; x++)
                        {
                            const int e = tid + x * NT;
                            const int c = args.b_kfast ? e / BK : e % BN;
                            const int kk = args.b_kfast ? e % BK : e / BN;
                            const int64_t co = ctab[c], ko = ktab[kk];
                            const bool ok = (co != OFF_INVALID) && (ko != OFF_INVALID);
                            const double* src = ok ? args.B + ko + co : args.B;
                            cp_async8(smem_u32(dst + kk * LDB + c), src, ok ? 8 : 0);
                        }
                    }
                }
            };

            __syncthreads();   // previous product's last stage fully consumed
            // Prologue: k tables for stages 0..STAGES-1, then data for 0..STAGES-2.
            for (int64_t s = 0; s < STAGES; s++)
            {
                int64_t va = 0, vb = 0; int sl = 0, idx = 0;
                load_ktab(s, va, vb, sl, idx);
                store_ktab(sl, idx, va, vb);
            }
            __syncthreads();
            for (int64_t s = 0; s < STAGES - 1; s++)
            {
                if (s < nk) issue_stage(s);
                cp_async_commit();
            }

            double acc[4][4][4];
#pragma unroll
            for (int mi = 0; mi < 4; mi++)
#pragma unroll
                for (int ni = 0; ni < 4; ni++)
#pragma unroll
                    for (int e = 0; e < 4; e++) acc[mi][ni][e] = 0.0;

            long long sa[NA], sb[NB];
#pragma unroll
            for (int i = 0; i < NA; i++) sa[i] = (i < na && P.a_s[i] < 0) ? (long long)0x8000000000000000ull : 0ll;
#pragma unroll
            for (int j = 0; j < NB; j++) sb[j] = (j < nb && P.b_s[j] < 0) ? (long long)0x8000000000000000ull : 0ll;

            for (int64_t s = 0; s < nk; s++)
            {
                cp_async_wait<STAGES - 2>();
                __syncthreads();
                // Refill: data of stage s+STAGES-1 (its k table is ready), and
                // fetch the k table of stage s+STAGES into registers.
                const int64_t sn = s + STAGES - 1;
                if (sn < nk) issue_stage(sn);
                cp_async_commit();
                int64_t va = 0, vb = 0; int sl = 0, idx = 0;
                load_ktab(s + STAGES, va, vb, sl, idx);

                const int buf = (int)(s % STAGES);
                const double* Ab = As + (size_t)buf * NA * BK * LDA;
                const double* Bb = Bs + (size_t)buf * NB * BK * LDB;
#pragma unroll
                for (int k4 = 0; k4 < BK; k4 += 4)
                {
                    double af[4][2], bf[4];
                    const int kr = k4 + t4;
#pragma unroll
                    for (int mi = 0; mi < 4; mi++)
                    {
                        const int r0 = wm + mi * 16 + g;
                        double x0 = apply_sign(Ab[kr * LDA + r0], sa[0]);
                        double x1 = apply_sign(Ab[kr * LDA + r0 + 8], sa[0]);
#pragma unroll
                        for (int i = 1; i < NA; i++)
                        {
                            if (i < na)
                            {
                                const double* Ai = Ab + (size_t)i * BK * LDA;
                                x0 += apply_sign(Ai[kr * LDA + r0], sa[i]);
                                x1 += apply_sign(Ai[kr * LDA + r0 + 8], sa[i]);
                            }
                        }
                        af[mi][0] = x0; af[mi][1] = x1;
                    }
#pragma unroll
                    for (int ni = 0; ni < 4; ni++)
                    {
                        const int c0 = wn + ni * 8 + g;
                        double y = apply_sign(Bb[kr * LDB + c0], sb[0]);
#pragma unroll
                        for (int j = 1; j < NB; j++)
                        {
                            if (j < nb)
                            {
                                const double* Bj = Bb + (size_t)j * BK * LDB;
                                y += apply_sign(Bj[kr * LDB + c0], sb[j]);
                            }
                        }
                        bf[ni] = y;
                    }
#pragma unroll
                    for (int mi = 0; mi < 4; mi++)
#pragma unroll
                        for (int ni = 0; ni < 4; ni++)
                            dmma(acc[mi][ni], af[mi][0], af[mi][1], bf[ni]);
                }
                store_ktab(sl, idx, va, vb);
            }
            cp_async_wait<0>();

            // Epilogue: C_q = (first ? beta*C_q : C_q) + sign_q*alpha*M for each target.
            for (int q = 0; q < P.nc; q++)
            {
                const int64_t* rt = rowC + P.c_r[q] * BM;
                const int64_t* ct = colC + P.c_c[q] * BN;
                const double coef = P.c_s[q] < 0 ? -args.alpha : args.alpha;
                const bool first = P.c_first[q] != 0;
                const double beta = args.beta;
#pragma unroll
                for (int mi = 0; mi < 4; mi++)
                {
#pragma unroll
                    for (int hr = 0; hr < 2; hr++)
                    {
                        const int64_t ro = rt[wm + mi * 16 + g + hr * 8];
                        if (ro == OFF_INVALID) continue;
#pragma unroll
                        for (int ni = 0; ni < 4; ni++)
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
}

template <int NA, int NB, int STAGES>
cudaError_t launch_instance(const DmmaArgs& args, cudaStream_t stream, int num_sms)
{
    using S = Smem<NA, NB, STAGES>;
    auto kern = stra_dmma_kernel<NA, NB, STAGES>;
    static_assert(S::total <= 227 * 1024, "shared memory budget");
    cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::total);
    if (err != cudaSuccess) return err;
    int64_t grid = args.work < num_sms ? args.work : num_sms;
    if (grid < 1) grid = 1;
    kern<<<(unsigned)grid, NT, S::total, stream>>>(args);
    return cudaGetLastError();
}

}  // namespace

std::atomic<unsigned long long> g_launches{0};

unsigned long long launches() { return g_launches.load(); }

cudaError_t launch_dmma(const DmmaArgs& args, int terms, cudaStream_t stream, int num_sms)
{
    if (args.work <= 0) return cudaSuccess;
    cudaError_t err;
    if (terms <= 1)      err = launch_instance<1, 1, 8>(args, stream, num_sms);
    else if (terms <= 2) err = launch_instance<2, 2, 6>(args, stream, num_sms);
    else                 err = launch_instance<4, 4, 3>(args, stream, num_sms);
    if (err == cudaSuccess) g_launches++;
    return err;
}

}  // namespace tsb
