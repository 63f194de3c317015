// Fully fused FP64 ABC Strassen kernel: all 7^L products of a contraction in
// one persistent launch, no workspace.
//
// What it replaces in the reference (src/stra_internal/3t/stra_mult.cxx:308-605
// and its 2-level form): the per-product control tree with fused packing
// (stra_pack_{two,four}_*, src/kernels/3m/gemm.hpp:504-816, 1344-1917) and the
// micro-kernel that adds +-M into up to 4 C blocks (stra_gemm_ukr_{two,four},
// src/stra_nodes/stra_gemm_ukr.hpp:622-940).
//
// Warp roles (384 threads per CTA, one CTA per SM, persistent over
// (batch, 128 x 128 tile) work items; every CTA runs all products of its tile
// in order, so C blocks shared by products need no atomics and beta is
// applied once, by the first product touching a block):
//
//   producer warpgroup (warps 0-3, registers cut with setmaxnreg): fills a
//     3-slot ring, one k-step per slot, through the scatter vectors, in one of
//     two modes:
//       RAW (sums of at most 2 blocks: L <= 1): cp.async gathers of the raw
//         blocks of each operand sum (16 k per slot) into the swizzled k-major
//         fragment layout (tile_pos); the slot's "full" mbarrier completes when
//         the copies land (cp.async.mbarrier.arrive), so the producer never
//         waits on data and runs ahead to the next slot;
//       SUM (up to 4 blocks: L = 2): the blocks are loaded into registers,
//         S = sum_i u_i A_i and T = sum_j v_j B_j are formed once per staged
//         tile (32 k per slot) and stored into the slot.
//   consumer warpgroups (warps 4-11): 2 x 4 warps of 64 x 32 (m16n8k4 DMMA
//     fragments read as 128-bit pairs; in RAW mode the 2 blocks' fragments are
//     summed with their signs as they are read); after a slot is read each warp
//     arrives on its "empty" mbarrier; after the last k-step of a product the
//     epilogue adds +-alpha*S*T into the product's C blocks.
//
// Measured at 16384^3 (no-workspace calls, effective TFLOP/s): RAW L=0 33.1,
// L=1 19.8 on the headline contraction's layout (30.9 at L=1 on k-major GEMM
// operands), SUM L=2 10.1; both modes are bound by the element-wise gathers
// through the scatter vectors (8-byte requests to L2).  Where the unit-stride
// modes of A and B are contracted modes, the element-pair form
// (fused_pairs.cu: 16-byte pair copies or tensor-map boxes into a planned
// conflict-free layout) runs instead: 33.3, 32.2 and 23.9 at L=0, 1 and 2
// there.
//
// The producer runs up to 3 k-steps ahead, across product and tile
// boundaries.  Every wait is bounded; a wait that runs out makes both roles
// leave their loops at the next tile (a collective OR over each role's named
// barrier); RAW-mode producers then let their own copies land before the CTA
// ends.
#include "fused_common.cuh"
#include "mbarrier.cuh"
#include "tile_layout.cuh"
#include "timing.hpp"

#include <atomic>

namespace tsb {

extern std::atomic<unsigned long long> g_launches;

namespace {

using namespace fused;

constexpr int FBK_MAX = 32;
constexpr int PCH = 16;                  // SUM mode: producer elements per batch of loads

// Per-mode geometry.  Register split: threads x launch registers is the CTA's
// pool; the producer gives back what the consumers take (checked against the
// compiled count on the host before every launch; both splits compile without
// spills).
template <bool RAW>
struct FMode
{
    static constexpr int BK = RAW ? 16 : 32;               // k per ring slot
    static constexpr int NT = RAW ? 2 : 1;                 // blocks per operand held in a slot
    static constexpr int PE = BK * FT / PT;                // elements of one operand block per producer thread
    static constexpr int KENT = 2 * FHMAX * BK / PT;       // k-table entries per producer thread
    static constexpr int PROD_REGS = RAW ? 80 : 128;
    static constexpr int CONS_REGS = RAW ? 200 : 184;
    static constexpr size_t SLOT_DOUBLES = size_t(BK) * FT * 2 * NT;
    static_assert(2 * FHMAX * BK == KENT * PT, "k-table entries split evenly over the producers");
    static_assert(RAW || PE % PCH == 0, "producer batches cover a block");
};

constexpr size_t RING_BYTES = FSTAGES * size_t(FBK_MAX) * FT * 2 * 8;   // either mode's 3 slots
static_assert(FSTAGES * FMode<true>::SLOT_DOUBLES * 8 == RING_BYTES &&
              FSTAGES * FMode<false>::SLOT_DOUBLES * 8 == RING_BYTES, "both modes fill the ring");
constexpr size_t TAB_BYTES = size_t(4) * FHMAX * FT * 8                 // rowA, colB, rowC, colC
                             + size_t(2) * FHMAX * FBK_MAX * 8;         // k tables of A and B
constexpr size_t FUSED_SMEM = RING_BYTES + TAB_BYTES + sizeof(FusedCtrl);
static_assert(FUSED_SMEM <= 227 * 1024, "shared memory budget");

// SUM mode: one operand sum of one ring slot: X(r, k) = sum_t sign_t * X[row_t(r) + k_t(k)]
// over the terms of the product's sum, stored at tile_pos(k, r).  `rows` is
// the row (column) offset table [FHMAX][FT] of the tile, `ktab` this k-step's
// k offset table [FHMAX][BK]; invalid entries read as zero.  The loads of two
// terms are issued together, so a thread keeps 2 * PCH loads in flight (the
// gathers are latency-bound, not bandwidth-bound).
template <bool KFAST, int BK>
__device__ __forceinline__ void produce_tile(const double* __restrict__ X, const int64_t* rows, const int64_t* ktab,
                                             int nt, const int8_t* t_row, const int8_t* t_k, const int8_t* t_s,
                                             double* dst, int ptid)
{
    constexpr int PE = BK * FT / PT;
#pragma unroll 1
    for (int c0 = 0; c0 < PE; c0 += PCH)
    {
        double v[PCH];
#pragma unroll
        for (int e = 0; e < PCH; e++) v[e] = 0.0;
#pragma unroll 1
        for (int t = 0; t < nt; t += 2)
        {
            const bool two = t + 1 < nt;
            const int64_t* rt0 = rows + t_row[t] * FT;
            const int64_t* kt0 = ktab + t_k[t] * BK;
            const int64_t* rt1 = rows + t_row[two ? t + 1 : t] * FT;
            const int64_t* kt1 = ktab + t_k[two ? t + 1 : t] * BK;
            const double s0 = t_s[t] < 0 ? -1.0 : 1.0;
            const double s1 = two ? (t_s[t + 1] < 0 ? -1.0 : 1.0) : 0.0;
            double x0[PCH], x1[PCH];
#pragma unroll
            for (int e = 0; e < PCH; e++)
            {
                int kk, r;
                lane_map<BK, FT>(KFAST, ptid + (c0 + e) * PT, kk, r);
                const int64_t ro0 = rt0[r], ko0 = kt0[kk], ro1 = rt1[r], ko1 = kt1[kk];
                x0[e] = (ro0 != OFF_INVALID && ko0 != OFF_INVALID) ? __ldg(X + (ro0 + ko0)) : 0.0;
                x1[e] = (two && ro1 != OFF_INVALID && ko1 != OFF_INVALID) ? __ldg(X + (ro1 + ko1)) : 0.0;
            }
            // exact: s0, s1 are +-1 or 0
#pragma unroll
            for (int e = 0; e < PCH; e++) v[e] += s0 * x0[e] + s1 * x1[e];
        }
#pragma unroll
        for (int e = 0; e < PCH; e++)
        {
            int kk, r;
            lane_map<BK, FT>(KFAST, ptid + (c0 + e) * PT, kk, r);
            dst[tile_pos(kk, r, FT)] = v[e];
        }
    }
}

__device__ __forceinline__ void cp_async8(uint32_t dst, const void* src, int src_bytes)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" :: "r"(dst), "l"(src), "r"(src_bytes));
}

// RAW mode: the raw blocks of one operand sum into a slot, block t at
// dst + t * BK * FT, element (r, k) at tile_pos(k, r); invalid entries are
// zero-filled (source size 0).
template <bool KFAST, int BK>
__device__ __forceinline__ void issue_tiles(const double* __restrict__ X, const int64_t* rows, const int64_t* ktab,
                                            int nt, const int8_t* t_row, const int8_t* t_k, double* dst, int ptid)
{
    constexpr int PE = BK * FT / PT;
    for (int t = 0; t < nt; t++)
    {
        const int64_t* rt = rows + t_row[t] * FT;
        const int64_t* kt = ktab + t_k[t] * BK;
        const uint32_t base = smem_addr(dst + (size_t)t * BK * FT);
#pragma unroll
        for (int e = 0; e < PE; e++)
        {
            int kk, r;
            lane_map<BK, FT>(KFAST, ptid + e * PT, kk, r);
            const int64_t ro = rt[r], ko = kt[kk];
            const bool ok = ro != OFF_INVALID && ko != OFF_INVALID;
            cp_async8(base + (uint32_t)tile_pos(kk, r, FT) * 8, ok ? X + (ro + ko) : X, ok ? 8 : 0);
        }
    }
}

template <bool RAW, bool KA, bool KB>
__global__ void __launch_bounds__(FTHREADS, 1)
stra_fused_kernel(const __grid_constant__ DmmaArgs a, int* err, long long limit)
{
    using M = FMode<RAW>;
    constexpr int BK = M::BK;
    extern __shared__ __align__(128) unsigned char smem[];
    double* ring = reinterpret_cast<double*>(smem);
    int64_t* rowA = reinterpret_cast<int64_t*>(smem + RING_BYTES);
    int64_t* colB = rowA + FHMAX * FT;
    int64_t* rowC = colB + FHMAX * FT;
    int64_t* colC = rowC + FHMAX * FT;
    int64_t* kA = colC + FHMAX * FT;         // [FHMAX][BK]
    int64_t* kB = kA + FHMAX * BK;           // [FHMAX][BK]
    FusedCtrl* ctl = reinterpret_cast<FusedCtrl*>(colC + FHMAX * FT + 2 * FHMAX * FBK_MAX);
    volatile int* abort_flag = &ctl->abort;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0)
    {
        for (int s = 0; s < FSTAGES; s++)
        {
            mbar_init(smem_addr(&ctl->full[s]), PT);
            mbar_init(smem_addr(&ctl->empty[s]), NCW);
        }
        ctl->abort = 0;
        mbar_init_fence();
    }
    __syncthreads();

    const int64_t tiles = (int64_t)a.tiles_m * a.tiles_n;
    const int64_t work = a.batch * tiles;
    const int64_t nk = (a.ks + BK - 1) / BK;
    const int H = a.H;                           // block rows of A and C
    const int Hk = a.Hk > 0 ? a.Hk : a.H;        // block columns of A, rows of B
    const int Hn = a.Hn > 0 ? a.Hn : a.H;        // block columns of B and C

    if (warp < NPW)
    {
        // ---------------- producer warpgroup ----------------
        asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;\n" :: "n"(M::PROD_REGS));
        const int ptid = tid;
        // This thread's entries of the k offset tables kA, kB for k-step s
        // (KENT of them): they depend on the k-step only (not on the product or
        // the tile), so the next k-step's are loaded while the current one is
        // produced.
        auto ktab_entry = [&](int64_t s, int j) -> int64_t {
            const int i = ptid + j * PT;
            const int op = i / (FHMAX * BK), e = i % (FHMAX * BK);
            const int h = e / BK, kk = e % BK;
            const int64_t kl = s * BK + kk, gk = h * a.ks + kl;
            if (!(h < Hk && kl < a.ks && gk < a.k)) return OFF_INVALID;
            return op == 0 ? a.ksA[gk] : a.ksB[gk];
        };
        int64_t kv[M::KENT];
#pragma unroll
        for (int j = 0; j < M::KENT; j++) kv[j] = nk > 0 ? ktab_entry(0, j) : OFF_INVALID;
        uint32_t it = 0;
        bool ok = true;      // this thread's waits so far
        bool stop = false;   // set only right after a collective check, so uniform
        // Every exit is taken right after a collective OR over the producers'
        // named barrier; a thread whose wait ran out keeps walking the same
        // loop (producing nothing) until the next one.
        for (int64_t w = blockIdx.x; w < work && !stop; w += gridDim.x)
        {
            if (bar_any<1, PT>(!ok)) break;
            int64_t b, tm, tn;
            decode_work(a, w, b, tm, tn);
            const int64_t offA = a.bA[b], offB = a.bB[b];
            for (int i = ptid; i < FHMAX * FT; i += PT)
            {
                const int h = i / FT, r = i % FT;
                const int64_t li = tm * FT + r, gi = h * a.ms + li;
                rowA[i] = (h < H && li < a.ms && gi < a.m) ? offA + a.rsA[gi] : OFF_INVALID;
                const int64_t lj = tn * FT + r, gj = h * a.ns + lj;
                colB[i] = (h < Hn && lj < a.ns && gj < a.n) ? offB + a.csB[gj] : OFF_INVALID;
            }
            for (int p = 0; p < a.nprod && !stop; p++)
            {
                const DevProduct& P = a.prod[p];
                for (int64_t s = 0; s < nk; s++)
                {
                    // All producers are done with the last k-step's tables (and
                    // the tile's row tables are complete); a wait that ran out
                    // in any of them ends the loops for all of them.
                    if (bar_any<1, PT>(!ok)) { stop = true; break; }
#pragma unroll
                    for (int j = 0; j < M::KENT; j++) kA[ptid + j * PT] = kv[j];   // kA, kB: one array
                    bar_sync<1, PT>();
                    {
                        const int64_t sn = s + 1 < nk ? s + 1 : 0;
#pragma unroll
                        for (int j = 0; j < M::KENT; j++) kv[j] = ktab_entry(sn, j);
                    }
                    const uint32_t slot = it % FSTAGES;
                    const uint32_t use = it / FSTAGES;   // earlier uses of this slot
                    it++;
                    if (!ok || (use > 0 && !mbar_wait(smem_addr(&ctl->empty[slot]), (use & 1) ^ 1, abort_flag, err,
                                                      1, limit)))
                    {
                        ok = false;
                        continue;
                    }
                    double* S = ring + slot * M::SLOT_DOUBLES;
                    double* T = S + M::NT * BK * FT;
                    if constexpr (RAW)
                    {
                        issue_tiles<KA, BK>(a.A, rowA, kA, P.na, P.a_r, P.a_c, S, ptid);
                        issue_tiles<KB, BK>(a.B, colB, kB, P.nb, P.b_c, P.b_r, T, ptid);
                        // the slot's full barrier completes when every producer's copies have landed
                        asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];\n"
                                     :: "r"(smem_addr(&ctl->full[slot])) : "memory");
                    }
                    else
                    {
                        produce_tile<KA, BK>(a.A, rowA, kA, P.na, P.a_r, P.a_c, P.a_s, S, ptid);
                        produce_tile<KB, BK>(a.B, colB, kB, P.nb, P.b_c, P.b_r, P.b_s, T, ptid);
                        mbar_arrive(smem_addr(&ctl->full[slot]));   // release: the stores above are visible
                    }
                }
            }
        }
        if constexpr (RAW)
            asm volatile("cp.async.wait_all;\n" ::: "memory");   // this thread's copies land before it leaves
    }
    else
    {
        // ---------------- consumer warpgroups ----------------
        asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;\n" :: "n"(M::CONS_REGS));
        const int ctid = tid - PT;
        const int cw = warp - NPW;
        const int g = lane >> 2, t4 = lane & 3;
        const int wm = (cw / CWN) * WTM;
        const int wn = (cw % CWN) * WTN;
        uint32_t cit = 0;
        bool ok = true;
        for (int64_t w = blockIdx.x; w < work; w += gridDim.x)
        {
            if (bar_any<2, CT>(!ok)) break;
            int64_t b, tm, tn;
            decode_work(a, w, b, tm, tn);
            fill_c_tables(a, b, tm, tn, rowC, colC, ctid);
            bar_sync<2, CT>();

            for (int p = 0; p < a.nprod && ok; p++)
            {
                double acc[MI][NI][4];
#pragma unroll
                for (int mi = 0; mi < MI; mi++)
#pragma unroll
                    for (int ni = 0; ni < NI; ni++)
#pragma unroll
                        for (int e = 0; e < 4; e++) acc[mi][ni][e] = 0.0;

                for (int64_t s = 0; s < nk; s++)
                {
                    const uint32_t slot = cit % FSTAGES;
                    ok = __all_sync(0xffffffffu, mbar_wait(smem_addr(&ctl->full[slot]), (cit / FSTAGES) & 1,
                                                           abort_flag, err, 2, limit));
                    if (!ok) break;
                    const double* Ab = ring + slot * M::SLOT_DOUBLES;
                    const double* Bb = Ab + M::NT * BK * FT;
                    // RAW mode: the second block of a sum, with its sign
                    // relative to the first (the first's sign moves to the
                    // C coefficient, as products' signs multiply)
                    const DevProduct& Pc = a.prod[p];
                    const bool a2 = RAW && Pc.na > 1, b2 = RAW && Pc.nb > 1;
                    const double ra = a2 && (Pc.a_s[1] * Pc.a_s[0] < 0) ? -1.0 : 1.0;
                    const double rb = b2 && (Pc.b_s[1] * Pc.b_s[0] < 0) ? -1.0 : 1.0;
#pragma unroll
                    for (int k4 = 0; k4 < BK; k4 += 4)
                    {
                        const int kr = k4 + t4;
                        const int pg = 2 * ((g + swz_c(kr)) & 7);
                        double af[MI][2], bf[NI];
#pragma unroll
                        for (int mi = 0; mi < MI; mi++)
                        {
                            const int pos = kr * FT + wm + mi * 16 + pg;
                            const double2 v = *reinterpret_cast<const double2*>(Ab + pos);
                            af[mi][0] = v.x; af[mi][1] = v.y;
                            if (a2)
                            {
                                const double2 u = *reinterpret_cast<const double2*>(Ab + BK * FT + pos);
                                af[mi][0] = fma(ra, u.x, af[mi][0]); af[mi][1] = fma(ra, u.y, af[mi][1]);
                            }
                        }
#pragma unroll
                        for (int nj = 0; nj < NI / 2; nj++)
                        {
                            const int pos = kr * FT + wn + nj * 16 + pg;
                            const double2 v = *reinterpret_cast<const double2*>(Bb + pos);
                            bf[2 * nj] = v.x; bf[2 * nj + 1] = v.y;
                            if (b2)
                            {
                                const double2 u = *reinterpret_cast<const double2*>(Bb + BK * FT + pos);
                                bf[2 * nj] = fma(rb, u.x, bf[2 * nj]); bf[2 * nj + 1] = fma(rb, u.y, bf[2 * nj + 1]);
                            }
                        }
#pragma unroll
                        for (int mi = 0; mi < MI; mi++)
#pragma unroll
                            for (int ni = 0; ni < NI; ni++)
                                dmma(acc[mi][ni], af[mi][0], af[mi][1], bf[ni]);
                    }
                    __syncwarp();
                    if (lane == 0) mbar_arrive(smem_addr(&ctl->empty[slot]));
                    cit++;
                }
                if (!ok) break;

                // C_t = (first ? beta*C_t : C_t) + sign_t*alpha*S*T for the
                // product's C blocks t.  RAW mode formed the sums as
                // A_0 +- A_1 (B likewise): the signs of the first blocks
                // multiply into the coefficient.
                const DevProduct& P = a.prod[p];
                const bool lead_neg = RAW && ((P.a_s[0] < 0) != (P.b_s[0] < 0));
                product_epilogue(a, P, lead_neg, rowC, colC, acc, wm, wn, g, 2 * t4, 2 * t4 + 1);
            }
        }
    }
}

}  // namespace

cudaError_t launch_fused(const DmmaArgs& in, cudaStream_t stream, int num_sms, int* err, long long wait_limit,
                         const GemmView* g)
{
    if (in.batch <= 0 || in.ms <= 0 || in.ns <= 0) return cudaSuccess;
    if (g)
    {
        const cudaError_t e = launch_fused_pairs(in, *g, stream, num_sms, err, wait_limit);
        if (e != cudaErrorNotSupported) return e;
    }
    // direct C updates on grids of up to 4 x 4 blocks only
    if (in.H < 1 || in.H > FHMAX || in.Hc != in.H || in.mC != in.m || in.nC != in.n) return cudaErrorNotSupported;
    if (in.Hk < 0 || in.Hk > FHMAX || in.Hn < 0 || in.Hn > FHMAX) return cudaErrorNotSupported;
    if (in.nprod < 1 || in.nprod > MAX_PRODUCTS) return cudaErrorInvalidValue;
    // RAW mode when every operand sum has at most 2 blocks (L <= 1), else SUM
    bool raw = true;
    for (int p = 0; p < in.nprod; p++)
        if (in.prod[p].na > FMode<true>::NT || in.prod[p].nb > FMode<true>::NT) raw = false;
    using Kern = void (*)(DmmaArgs, int*, long long);
    Kern kern;
    if (raw)
        kern = in.a_kfast ? (in.b_kfast ? stra_fused_kernel<true, true, true> : stra_fused_kernel<true, true, false>)
                          : (in.b_kfast ? stra_fused_kernel<true, false, true> : stra_fused_kernel<true, false, false>);
    else
        kern = in.a_kfast ? (in.b_kfast ? stra_fused_kernel<false, true, true> : stra_fused_kernel<false, true, false>)
                          : (in.b_kfast ? stra_fused_kernel<false, false, true> : stra_fused_kernel<false, false, false>);
    // The register split must fit the pool the CTA is launched with.
    const size_t need = raw ? (size_t)FMode<true>::PROD_REGS * PT + (size_t)FMode<true>::CONS_REGS * CT
                            : (size_t)FMode<false>::PROD_REGS * PT + (size_t)FMode<false>::CONS_REGS * CT;
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, reinterpret_cast<const void*>(kern));
    if (e != cudaSuccess) return e;
    if ((size_t)fa.numRegs * FTHREADS < need) return cudaErrorNotSupported;
    e = cudaFuncSetAttribute(reinterpret_cast<const void*>(kern), cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)FUSED_SMEM);
    if (e != cudaSuccess) return e;
    DmmaArgs args = in;
    args.tiles_m = (int)((args.ms + FT - 1) / FT);
    args.tiles_n = (int)((args.ns + FT - 1) / FT);
    args.work = args.batch * (int64_t)args.tiles_m * args.tiles_n;
    if (args.work <= 0) return cudaSuccess;
    int64_t grid = num_sms;
    if (args.work < grid) grid = args.work;
    timing_begin(KK_FUSED, stream);
    kern<<<(unsigned)grid, FTHREADS, FUSED_SMEM, stream>>>(args, err, wait_cycles(wait_limit));
    timing_end(KK_FUSED, stream);
    e = cudaGetLastError();
    if (e == cudaSuccess) g_launches++;
    return e;
}

}  // namespace tsb
