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
//                        through the scatter vectors into tile order (HBM bound;
//                        `kpiece` writes the pieces of a k-split as batch
//                        entries);
//   pack_multi_kernel    the 7 sums of a product group in one pass (L >= 1);
//   packed_gemm_ws_kernel DMMA GEMM on S and T (bulk-copy operand ring on
//                        mbarriers, no block barrier in the k loop) whose
//                        epilogue adds +-alpha*S*T into the product's C blocks
//                        (beta on first touch), for up to 7 products per tile
//                        position; in the product-parallel and k-split forms
//                        it sees every product (piece) as a batch entry and
//                        writes its own M; packed_gemm_grouped_kernel the
//                        same over many problems' tiles.
//
// Forming each sum once per element in HBM costs about 1 % of the GEMM time at
// NIm = NJn = NPk = 16384, while summing inside the GEMM costs shared-memory
// bandwidth on every fragment read; the GEMM's loader becomes a plain copy of
// contiguous 16-byte chunks.
#include "kernels.cuh"
#include "mbarrier.cuh"
#include "tile_layout.cuh"
#include "timing.hpp"

#include <atomic>

namespace tsb {

extern std::atomic<unsigned long long> g_launches;

namespace {

// ---- pack ---------------------------------------------------------------------

constexpr int PK_K = 32;          // k values per pack CTA
constexpr int PK_THREADS = 256;
constexpr int PK_ROWS = PACK_TILE / 2;   // rows per pack CTA: half a tile

// Pack CTAs cover 64 rows x 32 k (half of a 128-row tile: blockIdx.y = 2 *
// tile + half), so their shared memory and registers stay small and several
// CTAs per SM overlap one CTA's gathers with another's writes.  Element e of a
// thread: with kfast the 32 lanes of a warp walk 32 consecutive k of one row,
// else 32 consecutive rows of one k.
constexpr int PK_E = PK_ROWS * PK_K / PK_THREADS;
__device__ __forceinline__ int pk_row(bool kfast, int warp, int lane, int e)
{
    return kfast ? warp + 8 * e : lane + 32 * (e & 1);
}
__device__ __forceinline__ int pk_k(bool kfast, int warp, int lane, int e)
{
    return kfast ? lane : warp + 8 * (e >> 1);
}

// Write buf (rows [64 half, 64 half + 64) of the tile, PK_K k) in the tile's
// swizzled order: per k a row of 128 consecutive doubles, so warp stores are
// contiguous.
__device__ __forceinline__ void pk_write(const double (*buf)[PK_K + 1], double* out, int64_t k0, int64_t k_pad,
                                         int half, int warp, int lane)
{
#pragma unroll
    for (int e = 0; e < PK_E; e++)
    {
        const int r = lane + 32 * (e & 1);
        const int kk = warp + 8 * (e >> 1);
        if (k0 + kk < k_pad)
            out[(int64_t)kk * PACK_TILE + tile_pos((int)((k0 + kk) & 7), half * PK_ROWS + r, 0)] = buf[r][kk];
    }
}

__global__ void __launch_bounds__(PK_THREADS)
pack_kernel(const __grid_constant__ PackArgs a)
{
    __shared__ double buf[PK_ROWS][PK_K + 1];
    __shared__ int64_t rowoff[4][PK_ROWS];       // per term: batch + row offset (or invalid)
    __shared__ int64_t koff[4][PK_K];            // per term: k offset (or invalid)
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int64_t k0 = (int64_t)blockIdx.x * PK_K;
    const int64_t t = blockIdx.y >> 1;
    const int half = blockIdx.y & 1;
    const int64_t b = blockIdx.z;
    const int64_t r0 = t * PACK_TILE + half * PK_ROWS;
    const int nt = a.nt;
    const bool kfast = a.kfast != 0;

    // Offset tables of this CTA's rows and k values, once per term.
    for (int i = tid; i < nt * PK_ROWS; i += PK_THREADS)
    {
        const int q = i / PK_ROWS, r = i % PK_ROWS;
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

    // Gather and sum, terms outermost, so all loads of one term are
    // independent and in flight together.
    double v[PK_E];
#pragma unroll
    for (int e = 0; e < PK_E; e++) v[e] = 0.0;
    for (int q = 0; q < nt; q++)
    {
        const bool neg = a.t_s[q] < 0;
#pragma unroll
        for (int e = 0; e < PK_E; e++)
        {
            const int64_t ro = rowoff[q][pk_row(kfast, warp, lane, e)], ko = koff[q][pk_k(kfast, warp, lane, e)];
            if (ro != OFF_INVALID && ko != OFF_INVALID)
            {
                const double x = a.X[ro + ko];
                v[e] += neg ? -x : x;
            }
        }
    }
#pragma unroll
    for (int e = 0; e < PK_E; e++) buf[pk_row(kfast, warp, lane, e)][pk_k(kfast, warp, lane, e)] = v[e];
    __syncthreads();
    double* dst;
    if (a.kpiece > 0)
    {
        const int64_t p = k0 / a.kpiece;
        dst = a.out + (((p * a.batch + b) * a.tiles + t) * a.kpiece + (k0 - p * a.kpiece)) * PACK_TILE;
    }
    else
        dst = a.out + ((b * a.tiles + t) * a.k_pad + k0) * PACK_TILE;
    pk_write(buf, dst, k0, a.k_pad, half, warp, lane);
}

// Seven sums of one product group per pass (L >= 1): each CTA reads its
// 64-row x 32-k window of every block of the group's coarse sum once, forms
// the four sub-block sums X_j in registers, then writes each output's signed
// combination through the shared-memory transpose of pack_kernel.  At L=2 this
// reads each block of A (and B) once per group instead of once per product
// that uses it: 48 instead of 144 block reads per operand.
__global__ void __launch_bounds__(PK_THREADS)
pack_multi_kernel(const __grid_constant__ PackMultiArgs a)
{
    __shared__ double buf[PK_ROWS][PK_K + 1];
    __shared__ int64_t rowoff[8][PK_ROWS];       // per block (t, j): batch + row offset (or invalid)
    __shared__ int64_t koff[8][PK_K];            // per block (t, j): k offset (or invalid)
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int64_t k0 = (int64_t)blockIdx.x * PK_K;
    const int64_t t = blockIdx.y >> 1;
    const int half = blockIdx.y & 1;
    const int64_t b = blockIdx.z;
    const int64_t r0 = t * PACK_TILE + half * PK_ROWS;
    const int nblk = a.nt * 4;
    const bool kfast = a.kfast != 0;

    for (int i = tid; i < nblk * PK_ROWS; i += PK_THREADS)
    {
        const int q = i / PK_ROWS, r = i % PK_ROWS;
        const int64_t lr = r0 + r, gr = a.prow[q >> 2][q & 3] * a.rows_blk + lr;
        rowoff[q][r] = (lr < a.rows_blk && gr < a.rows_full) ? a.bX[b] + a.rs[gr] : OFF_INVALID;
    }
    for (int i = tid; i < nblk * PK_K; i += PK_THREADS)
    {
        const int q = i / PK_K, kk = i % PK_K;
        const int64_t lk = k0 + kk, gk = a.pk[q >> 2][q & 3] * a.k_blk + lk;
        koff[q][kk] = (lk < a.k_blk && gk < a.k_full) ? a.ks[gk] : OFF_INVALID;
    }
    __syncthreads();

    double x[4][PK_E];
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
        for (int e = 0; e < PK_E; e++) x[j][e] = 0.0;
    for (int c = 0; c < a.nt; c++)
    {
        const bool neg = a.t_s[c] < 0;
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int e = 0; e < PK_E; e++)
            {
                const int64_t ro = rowoff[c * 4 + j][pk_row(kfast, warp, lane, e)];
                const int64_t ko = koff[c * 4 + j][pk_k(kfast, warp, lane, e)];
                if (ro != OFF_INVALID && ko != OFF_INVALID)
                {
                    const double v = a.X[ro + ko];
                    x[j][e] += neg ? -v : v;
                }
            }
    }
    for (int o = 0; o < a.nout; o++)
    {
        int cf[4];
#pragma unroll
        for (int j = 0; j < 4; j++)
            cf[j] = (a.o_n[o] > 0 && a.o_j[o][0] == j ? a.o_s[o][0] : 0) +
                    (a.o_n[o] > 1 && a.o_j[o][1] == j ? a.o_s[o][1] : 0);
        __syncthreads();   // the previous output's tile has left buf
#pragma unroll
        for (int e = 0; e < PK_E; e++)
        {
            double v = 0.0;
#pragma unroll
            for (int j = 0; j < 4; j++)
                if (cf[j]) v += cf[j] > 0 ? x[j][e] : -x[j][e];
            buf[pk_row(kfast, warp, lane, e)][pk_k(kfast, warp, lane, e)] = v;
        }
        __syncthreads();
        pk_write(buf, a.out[o] + ((b * a.tiles + t) * a.k_pad + k0) * PACK_TILE, k0, a.k_pad, half, warp, lane);
    }
}

// ---- packed GEMM ------------------------------------------------------------------

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

// ---- warp-specialised packed GEMM ----------------------------------------------------
//
// 128 x 128 output tiles of 16 warps with 32 x 32 warp tiles of m16n8k4 DMMA
// fragments, read as 128-bit pairs from the swizzled k-major layout.  The
// operand ring is filled by 1-D bulk copies (one 32 KB copy of S and one of T
// per k-step: a packed tile's k-steps are contiguous) that complete on an
// mbarrier, so the CTA never meets at a block barrier inside the k loop.  Thread 0 also produces: after each
// k-step it refills the slot that step used once all 16 warps have released
// it (one arrival per warp), so warps drift apart by up to STAGES - 1 steps
// and the DMMA pipe does not drain at a block-wide barrier.  The producer
// runs ahead across tile boundaries, loading the next tile's first steps
// during the epilogue.  Every wait is bounded (mbarrier.cuh).

// Thread 0's producer cursor and the ring's barriers (shared memory).
struct WsCtrl
{
    uint64_t full[4], empty[4];    // per ring slot; STAGES <= 4
    int64_t pw, ps, nk;            // producer: work item, k-step within a product, k-steps
    const double* sA;
    const double* sB;
    uint32_t pit;                  // k-steps issued
    int pq, np;                    // producer: product within the work item, products of it
    int abort;
};

// Work sources: one problem (kernel parameter) or a group of problems
// (descriptors in global memory; work item w belongs to the problem p with
// prefix[p] <= w < prefix[p + 1]).
// The parameter is read through a pointer of unknown origin, so its fields
// are loaded where they are used (as the group's descriptors are) instead of
// being held in registers across the k loop.
struct OneProblem
{
    const PackedGemmArgs* a;
    __device__ int64_t total() const { return a->batch * a->tiles_m * a->tiles_n; }
    __device__ const PackedGemmArgs& at(int64_t w, int64_t& local) const
    {
        local = w;
        const PackedGemmArgs* p = a;
        asm volatile("" : "+l"(p));
        return *p;
    }
};

struct ProblemGroup
{
    const PackedGroupArgs& g;
    __device__ int64_t total() const { return g.total; }
    __device__ const PackedGemmArgs& at(int64_t w, int64_t& local) const
    {
        int lo = 0, hi = g.nprob - 1;
        while (lo < hi)
        {
            const int mid = (lo + hi + 1) >> 1;
            if (g.prefix[mid] <= w) lo = mid; else hi = mid - 1;
        }
        local = w - g.prefix[lo];
        return g.probs[lo];
    }
};

// Tile (batch b, row tile tm, column tile tn) of work item w: groups of 8
// row tiles walk the column tiles together so concurrent CTAs share panels.
__device__ __forceinline__ void decode_tile(const PackedGemmArgs& a, int64_t w, int64_t& b, int64_t& tm,
                                            int64_t& tn)
{
    const int64_t tiles = a.tiles_m * a.tiles_n;
    b = w / tiles;
    const int64_t tw = w - b * tiles;
    const int64_t GROUP = 8;
    const int64_t group = tw / (GROUP * a.tiles_n);
    const int64_t first_m = group * GROUP;
    const int64_t gsize = (a.tiles_m - first_m) < GROUP ? (a.tiles_m - first_m) : GROUP;
    tm = first_m + (tw % gsize);
    tn = (tw % (GROUP * a.tiles_n)) / gsize;
}

template <class K>
constexpr size_t ws_smem()
{
    return K::STAGES * K::stage_bytes + size_t(4) * (K::BM + K::BN) * 8 + sizeof(WsCtrl);
}

template <class K, class Src>
__device__ __forceinline__ void packed_ws_body(const Src& src, int* err, long long limit, unsigned char* smem)
{
    constexpr int BM = K::BM, BN = K::BN, BK = K::BK, NT = K::NT, STAGES = K::STAGES;
    constexpr int MI = K::MI, NI = K::NI, NW = NT / 32;
    static_assert(STAGES <= 4, "WsCtrl holds 4 ring slots");
    static_assert((BK * BM * 8) % 16 == 0 && (BK * BN * 8) % 16 == 0, "bulk copies of 16-byte multiples");
    double* As = reinterpret_cast<double*>(smem);
    double* Bs = As + STAGES * BK * BM;
    int64_t* rowC = reinterpret_cast<int64_t*>(Bs + STAGES * BK * BN);
    int64_t* colC = rowC + 4 * BM;
    WsCtrl* ctl = reinterpret_cast<WsCtrl*>(colC + 4 * BN);
    volatile int* abort_flag = &ctl->abort;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t4 = lane & 3;
    const int wm = (warp / K::WN) * K::WTM;
    const int wn = (warp % K::WN) * K::WTN;
    const int64_t total = src.total();

    if (tid == 0)
    {
        for (int s = 0; s < STAGES; s++)
        {
            mbar_init(smem_addr(&ctl->full[s]), 1);
            mbar_init(smem_addr(&ctl->empty[s]), NW);
        }
        ctl->pw = blockIdx.x; ctl->ps = 0; ctl->nk = 0; ctl->pit = 0; ctl->pq = 0; ctl->np = 0; ctl->abort = 0;
        mbar_init_fence();
    }
    __syncthreads();

    // Producer (thread 0): issue the next k-step of this CTA's work sequence
    // into its ring slot, after the warps have released the slot's previous
    // use.  False on a timed-out or aborted wait.
    auto produce = [&]() -> bool {
        while (ctl->pw < total)
        {
            if (ctl->ps == 0)
            {
                int64_t local;
                const PackedGemmArgs& p = src.at(ctl->pw, local);
                int64_t b, tm, tn;
                decode_tile(p, local, b, tm, tn);
                ctl->nk = p.k_pad / BK;
                ctl->np = p.nprod;
                if (ctl->nk == 0) { ctl->pw += gridDim.x; continue; }
                const int q = ctl->pq;
                ctl->sA = p.S[q] + ((b * p.tiles_m + tm) * p.k_pad) * BM;
                ctl->sB = p.T[q] + ((b * p.tiles_n + tn) * p.k_pad) * BN;
            }
            const uint32_t it = ctl->pit, slot = it % STAGES;
            if (it >= (uint32_t)STAGES &&
                !mbar_wait(smem_addr(&ctl->empty[slot]), ((it / STAGES) & 1) ^ 1, abort_flag, err, 1, limit))
                return false;
            const uint32_t full = smem_addr(&ctl->full[slot]);
            mbar_expect_tx(full, (uint32_t)((BK * BM + BK * BN) * 8));
            bulk_copy(smem_addr(As + slot * BK * BM), ctl->sA + ctl->ps * BK * BM, BK * BM * 8, full);
            bulk_copy(smem_addr(Bs + slot * BK * BN), ctl->sB + ctl->ps * BK * BN, BK * BN * 8, full);
            ctl->pit = it + 1;
            if (++ctl->ps == ctl->nk)
            {
                ctl->ps = 0;
                if (++ctl->pq == ctl->np) { ctl->pq = 0; ctl->pw += gridDim.x; }
            }
            return true;
        }
        return true;
    };
    bool ok = true;
    if (tid == 0)
        for (int s = 0; s < STAGES && ok; s++) ok = produce();

    auto load_frags = [&](const double* Ab, const double* Bb, int k4, double (&af)[MI][2], double (&bf)[NI]) {
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

    uint32_t cit = 0;   // k-steps consumed
    for (int64_t w = blockIdx.x; w < total; w += gridDim.x)
    {
        // Every thread takes part in every tile's barriers; a failed wait
        // anywhere ends the loop for all of them here.
        if (__syncthreads_or(!ok)) break;
        int64_t local;
        const PackedGemmArgs& a = src.at(w, local);
        int64_t b, tm, tn;
        decode_tile(a, local, b, tm, tn);
        const int64_t nk = a.k_pad / BK;
        // Offset tables of the tile's rows (columns) in every block row (column)
        // h < H of the C block grid, shared by all products of the work item.
        const int H = a.H, Hn = a.Hn > 0 ? a.Hn : a.H;
        for (int i = tid; i < 4 * BM; i += NT)
        {
            const int h = i / BM, r = i % BM;
            const int64_t loc = tm * BM + r, gi = h * a.ms + loc;
            rowC[i] = (h < H && loc < a.ms && gi < a.m) ? a.bC[b] + a.rsC[gi] : OFF_INVALID;
        }
        for (int i = tid; i < 4 * BN; i += NT)
        {
            const int h = i / BN, c = i % BN;
            const int64_t loc = tn * BN + c, gj = h * a.ns + loc;
            colC[i] = (h < Hn && loc < a.ns && gj < a.n) ? a.csC[gj] : OFF_INVALID;
        }
        __syncthreads();

        for (int p = 0; p < a.nprod && ok && nk > 0; p++)
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
                const uint32_t slot = cit % STAGES;
                // warp-uniform outcome, so the warp stays converged
                ok = __all_sync(0xffffffffu,
                                mbar_wait(smem_addr(&ctl->full[slot]), (cit / STAGES) & 1, abort_flag, err, 2,
                                          limit));
                if (!ok) break;
                const double* Ab = As + slot * BK * BM;
                const double* Bb = Bs + slot * BK * BN;
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
                __syncwarp();
                if (lane == 0) mbar_arrive(smem_addr(&ctl->empty[slot]));
                cit++;
                if (warp == 0)
                {
                    bool pok = true;
                    if (lane == 0) pok = produce();
                    ok = __shfl_sync(0xffffffffu, pok, 0);
                    if (!ok) break;
                }
            }
            if (!ok) break;   // the barrier at the top of the tile loop ends it

            // Epilogue of product p: C_t = (first ? beta*C_t : C_t) +
            // sign_t*alpha*S*T for its C blocks t, all loads of a row pair
            // issued before its stores.
            for (int t = 0; t < a.nc[p]; t++)
            {
                const int64_t* rt = rowC + a.c_r[p][t] * BM;
                const int64_t* ct = colC + a.c_c[p][t] * BN;
                const double coef = a.c_s[p][t] < 0 ? -a.alpha : a.alpha;
                const bool first = a.c_first[p][t] != 0;
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
    // Copies still in flight (after an abort) land before the CTA leaves:
    // bounded waits on the last STAGES k-steps issued.
    if (tid == 0)
    {
        volatile int never = 0;
        const uint32_t pit = ctl->pit;
        for (uint32_t i = (pit > (uint32_t)STAGES ? pit - STAGES : 0); i < pit; i++)
            mbar_wait(smem_addr(&ctl->full[i % STAGES]), (i / STAGES) & 1, &never, nullptr, 0, MBAR_WAIT_LIMIT);
    }
}

template <class K>
__global__ void __launch_bounds__(K::NT, 1)
packed_gemm_ws_kernel(const __grid_constant__ PackedGemmArgs a)
{
    extern __shared__ __align__(128) unsigned char smem[];
    packed_ws_body<K>(OneProblem{&a}, a.err, wait_cycles(a.wait_limit), smem);
}

template <class K>
__global__ void __launch_bounds__(K::NT, 1)
packed_gemm_grouped_kernel(const __grid_constant__ PackedGroupArgs g)
{
    extern __shared__ __align__(128) unsigned char smem[];
    packed_ws_body<K>(ProblemGroup{g}, g.err, wait_cycles(g.wait_limit), smem);
}

template <class K>
cudaError_t launch_packed_ws_cfg(const PackedGemmArgs& a, cudaStream_t stream, int num_sms)
{
    static_assert(ws_smem<K>() <= 227 * 1024, "shared memory budget");
    if (a.k_pad % K::BK) return cudaErrorInvalidValue;
    auto kern = packed_gemm_ws_kernel<K>;
    cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ws_smem<K>());
    if (err != cudaSuccess) return err;
    const int64_t work = a.batch * a.tiles_m * a.tiles_n;
    int64_t grid = num_sms;
    if (work < grid) grid = work;
    timing_begin(KK_PACKED_GEMM, stream);
    kern<<<(unsigned)grid, K::NT, ws_smem<K>(), stream>>>(a);
    timing_end(KK_PACKED_GEMM, stream);
    return cudaGetLastError();
}

template <class K>
cudaError_t launch_packed_grouped_cfg(const PackedGroupArgs& g, cudaStream_t stream, int num_sms)
{
    static_assert(ws_smem<K>() <= 227 * 1024, "shared memory budget");
    auto kern = packed_gemm_grouped_kernel<K>;
    cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ws_smem<K>());
    if (err != cudaSuccess) return err;
    int64_t grid = num_sms;
    if (g.total < grid) grid = g.total;
    timing_begin(KK_PACKED_GEMM, stream);
    kern<<<(unsigned)grid, K::NT, ws_smem<K>(), stream>>>(g);
    timing_end(KK_PACKED_GEMM, stream);
    return cudaGetLastError();
}

using PG0 = PCfg<32, 3, 4, 4>;   // 16 warps of 32 x 32, k-step 32

}  // namespace

cudaError_t launch_pack(const PackArgs& a, cudaStream_t stream)
{
    if (a.batch <= 0 || a.tiles <= 0 || a.k_pad <= 0) return cudaSuccess;
    if (a.k_pad % PK_K && a.k_pad % PACK_KSTEP) return cudaErrorInvalidValue;
    if (a.kpiece < 0 || (a.kpiece > 0 && (a.kpiece % PK_K || a.k_pad % a.kpiece))) return cudaErrorInvalidValue;
    dim3 grid((unsigned)((a.k_pad + PK_K - 1) / PK_K), (unsigned)(2 * a.tiles), (unsigned)a.batch);
    if (2 * a.tiles > 65535 || a.batch > 65535) return cudaErrorInvalidValue;
    timing_begin(KK_PACK, stream);
    pack_kernel<<<grid, PK_THREADS, 0, stream>>>(a);
    timing_end(KK_PACK, stream);
    cudaError_t err = cudaGetLastError();
    if (err == cudaSuccess) g_launches++;
    return err;
}

cudaError_t launch_pack_multi(const PackMultiArgs& a, cudaStream_t stream)
{
    if (a.batch <= 0 || a.tiles <= 0 || a.k_pad <= 0 || a.nout <= 0) return cudaSuccess;
    if (a.k_pad % PK_K || a.nt < 1 || a.nt > 2 || a.nout > 7) return cudaErrorInvalidValue;
    if (2 * a.tiles > 65535 || a.batch > 65535) return cudaErrorInvalidValue;
    dim3 grid((unsigned)(a.k_pad / PK_K), (unsigned)(2 * a.tiles), (unsigned)a.batch);
    timing_begin(KK_PACK, stream);
    pack_multi_kernel<<<grid, PK_THREADS, 0, stream>>>(a);
    timing_end(KK_PACK, stream);
    cudaError_t err = cudaGetLastError();
    if (err == cudaSuccess) g_launches++;
    return err;
}

cudaError_t launch_packed_gemm(const PackedGemmArgs& a, cudaStream_t stream, int num_sms)
{
    if (a.batch <= 0 || a.tiles_m <= 0 || a.tiles_n <= 0) return cudaSuccess;
    if (a.nprod < 1 || a.nprod > MAX_GROUP_PRODUCTS || a.H < 1 || a.H > 4 || a.Hn < 0 || a.Hn > 4)
        return cudaErrorInvalidValue;
    for (int p = 0; p < a.nprod; p++)
        if (a.nc[p] < 1 || a.nc[p] > 4) return cudaErrorInvalidValue;
    const cudaError_t err = launch_packed_ws_cfg<PG0>(a, stream, num_sms);
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
