// Fused FP64 ABC Strassen kernel, element-pair form: all products of a
// contraction in one persistent launch, no workspace, with the block tiles
// of A and B staged in a shared-memory layout planned on the host so that
// every DMMA fragment read is a conflict-free 16-byte load of two k-steps'
// elements (A always; B too when its contiguous k pairs are A's).
//
// What it replaces in the reference: the same per-product control tree and
// micro-kernel as the gather form in fused_kernel.cu
// (src/stra_internal/3t/stra_mult.cxx:308-605, src/kernels/3m/gemm.hpp:504-816,
// src/stra_nodes/stra_gemm_ukr.hpp:622-940), for operands whose
// unit-stride mode is a k mode -- the reference packs such panels with vector
// loads along that mode (src/stra_nodes/stra_packm.hpp:367-683).
//
// Two producers fill the same layout (the host picks one):
//   TMA: where every tile is a box of its operand whose rows are one
//     128-byte run of the unit-stride k mode (each row and k mode's extent
//     divides the tile or is a multiple of it, at most 5 dimensions, the
//     unit-stride k mode at dimension 0), four lanes of one producer warp
//     copy the product's (up to 2 + 2) block tiles, one tensor-map box
//     (cp.async.bulk.tensor) each, on the slot's "full" mbarrier;
//   PAIRS: elsewhere, the producer warpgroup copies each k pair of the
//     unit-stride mode (two consecutive doubles) with one 16-byte cp.async,
//     addressed through the row and k offset tables of the tile (any row
//     layout, ragged blocks included: entries past the extents read as
//     zero); the slot's "full" mbarrier completes when the copies land.
// A ring slot (64 KB) holds the blocks of the product's sums: 128 x 16 tiles,
// up to 2 per operand (Strassen levels 0 and 1), or 128 x 8 tiles, up to 4
// per operand (level 2, whose sums have up to 4 blocks; pair copies only).
// Layout of one 128 x TB tile: row r at TB r doubles; inside a row, the TB k
// in the order of a bit permutation of the slot's k index that puts the pair
// bit at position 0; then the 16-byte chunks of every 128 bytes XORed with
// bits of the row (the TMA swizzle of span 32, 64 or 128 bytes, or none; at
// most 64 for 8-double rows).  The TMA form is limited to layouts a tensor
// map writes densely (dimension 0's box bytes equal to the swizzle span).
//
// Consumers (warps 4-11, 2 x 4 warps of 64 x 32): which k a lane takes in
// which MMA step is a permutation of the slot's TB k (a sum over k may take
// them in any order), chosen with the permutations of each warp's 8 fragment
// rows and columns so that the reads are conflict-free; the blocks of an
// operand sum are read and added with their relative signs; the epilogue adds
// +-alpha * (S T) into the product's C blocks as the gather form does.
//
// Every wait is bounded; after a wait runs out both roles leave their loops
// and the producers let their copies in flight land before the CTA ends.
// No load uses cluster multicast; this kernel runs on one GPU.
#include "fused_common.cuh"
#include "mbarrier.cuh"
#include "plan.hpp"
#include "timing.hpp"

#include <cuda.h>

#include <algorithm>
#include <atomic>
#include <climits>
#include <cstring>
#include <map>
#include <utility>
#include <vector>

namespace tsb {

extern std::atomic<unsigned long long> g_launches;

using namespace fused;

namespace {

constexpr int PROD_TMA = 0, PROD_PAIRS = 1;
// A ring slot holds, per operand, the blocks of the product's sum: 2 tiles of
// 128 x 16 (sums of up to 2 blocks, Strassen levels 0 and 1) or 4 tiles of
// 128 x 8 (up to 4 blocks, level 2), 64 KB either way.  TB, the slot's k, is
// the kernel's template parameter; a tile row holds TB doubles.
constexpr int TBK = 16;                                   // k per ring slot, at most
constexpr int TSLOT_DOUBLES = 2 * 32 * FT;                // A0..A(NT-1) B0..B(NT-1)
template <int TB>
struct SlotShape
{
    static constexpr int NT = 32 / TB;                    // blocks per operand in a slot
    static constexpr int ROW = TB;                        // doubles per tile row in shared memory
    static constexpr int BOX = TB * FT;                   // one tile, doubles
    static constexpr int LPR = TB / 2;                    // producer lanes per tile row (one pair each)
    static constexpr int RPW = 32 / LPR;                  // tile rows per producer warp and pass
    static constexpr int RPP = NPW * RPW;                 // tile rows per pass of the producer warpgroup
    static constexpr int NIP = FT / RPP;                  // passes per tile
    static constexpr int NQ = TB / 8;                     // pairs of MMA k-steps per slot
    static constexpr int KTAB = 2 * FHMAX * TB;           // k-table entries (kA, kB)
    static constexpr int KENT = (KTAB + PT - 1) / PT;     // per producer thread
    static_assert(TB == 8 || TB == 16, "slot k");
    static_assert(2 * NT * BOX == TSLOT_DOUBLES && NIP * RPP == FT, "slot shape");
};
constexpr size_t TRING_BYTES = size_t(FSTAGES) * TSLOT_DOUBLES * 8;
constexpr size_t CTAB_BYTES = size_t(2) * FHMAX * FT * 8;                        // rowC, colC
constexpr size_t PTAB_BYTES = size_t(2) * FHMAX * FT * 8 + size_t(2) * FHMAX * TBK * 8;   // rowA, colB, kA, kB
constexpr size_t PAIRS_SMEM = 1024 + TRING_BYTES + CTAB_BYTES + PTAB_BYTES + sizeof(FusedCtrl);
static_assert(PAIRS_SMEM <= 227 * 1024, "shared memory budget");
constexpr size_t tile_smem(int prod)
{
    return prod == PROD_PAIRS ? PAIRS_SMEM : 1024 + TRING_BYTES + CTAB_BYTES + sizeof(FusedCtrl);
}
// Register splits (threads x launch registers is the pool; checked against
// the compiled count before every launch).
template <int PROD>
struct Regs
{
    static constexpr int PROD_REGS = PROD == PROD_PAIRS ? 80 : 64;
    static constexpr int CONS_REGS = PROD == PROD_PAIRS ? 208 : 216;
};

// How a tile origin gives the box coordinates of one operand (TMA form):
// coordinate d is the sum over its parts p of ((v / div) % mod) * mult (no
// modulus when mod is 0: the top digit of its index), v the origin's row, k
// or batch index as src[d] says.  A dimension has several parts when the
// planner split one mode of the tensor into several.
constexpr int TMA_PARTS = 3;
struct TmaCoords
{
    int ndim;
    int src[5];          // 0: row index (m for A, n for B), 1: k index, 2: batch index
    int nparts[5];
    long long div[5][TMA_PARTS];
    long long mod[5][TMA_PARTS];
    long long mult[5][TMA_PARTS];
};

struct FusedPairs
{
    CUtensorMap map[2];  // A, B (TMA form)
    TmaCoords co[2];
    // Consumer lane tables, in doubles inside a tile, swizzle applied: lane
    // (g, t4) of a warp at tile row (column) 0 reads A's pair of steps 2q,
    // 2q+1 at aoff[lane][q] and B's step j at boff[lane][j] (in pairs: the
    // pair of steps 2q, 2q+1 at boff[lane][2q]); q < TB / 8.  Tile row r + 8 i
    // is 8 i TB doubles further: shifts by multiples of 8 rows commute with
    // the swizzle (spans up to 128 bytes for 16-double rows, 64 for 8).
    int16_t aoff[32][2];
    int16_t boff[32][4];
    int8_t sigA[8];      // fragment row g -> row within its group of 8
    int8_t sigB[8];      // fragment column g -> column within its group of 8
    // PAIRS producer: unswizzled position of each slot k in a tile row, the
    // swizzle span (bytes), the pair bit of the slot k index and the TB / 2
    // pair bases in copy order (consecutive lanes take consecutive pairs).
    int8_t koff[2][TBK];
    int16_t swz[2];
    int8_t pbit[2];
    int8_t pbase[2][8];
};

__device__ __forceinline__ void box_coords(const TmaCoords& co, int64_t row, int64_t k, int64_t b, int (&c)[5])
{
#pragma unroll
    for (int d = 0; d < 5; d++)
    {
        c[d] = 0;
        if (d < co.ndim)
        {
            const int64_t v = co.src[d] == 0 ? row : co.src[d] == 1 ? k : b;
            int64_t x = 0;
            for (int p = 0; p < co.nparts[d]; p++)
            {
                int64_t y = co.div[d][p] == 1 ? v : v / co.div[d][p];
                if (co.mod[d][p]) y %= co.mod[d][p];
                x += y * co.mult[d][p];
            }
            c[d] = (int)x;
        }
    }
}

// One box of `map` at coordinates c into shared memory at dst, completing on
// the mbarrier's transaction count.
__device__ __forceinline__ void tma_box(uint32_t dst, const CUtensorMap* map, const int (&c)[5], int nd,
                                        uint32_t mbar)
{
    const unsigned long long m = reinterpret_cast<unsigned long long>(map);
    switch (nd)
    {
    case 1:
        asm volatile("cp.async.bulk.tensor.1d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                     " [%0], [%1, {%2}], [%3];\n" :: "r"(dst), "l"(m), "r"(c[0]), "r"(mbar) : "memory");
        break;
    case 2:
        asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                     " [%0], [%1, {%2, %3}], [%4];\n"
                     :: "r"(dst), "l"(m), "r"(c[0]), "r"(c[1]), "r"(mbar) : "memory");
        break;
    case 3:
        asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                     " [%0], [%1, {%2, %3, %4}], [%5];\n"
                     :: "r"(dst), "l"(m), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(mbar) : "memory");
        break;
    case 4:
        asm volatile("cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                     " [%0], [%1, {%2, %3, %4, %5}], [%6];\n"
                     :: "r"(dst), "l"(m), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(mbar) : "memory");
        break;
    default:
        asm volatile("cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                     " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];\n"
                     :: "r"(dst), "l"(m), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(c[4]), "r"(mbar)
                     : "memory");
        break;
    }
}

// 16-byte copy global -> shared of which the first `src_bytes` (16, 8 or 0)
// come from src and the rest is zero.
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, int src_bytes)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" :: "r"(dst), "l"(src), "r"(src_bytes));
}

// The 16-byte chunk bits [4, 4 + s) of a byte offset XORed with bits
// [7, 7 + s), s = log2(span / 16): the TMA swizzle of span 32, 64 or 128
// bytes of a tile aligned to its repeat (0: none).
__host__ __device__ __forceinline__ int swizzle(int byte, int span)
{
    if (span == 0) return byte;
    const int s = span == 32 ? 1 : span == 64 ? 2 : 3;
    return byte ^ (((byte >> 7) & ((1 << s) - 1)) << 4);
}

__device__ __forceinline__ double2 ld2(const double* p)
{
    return *reinterpret_cast<const double2*>(p);
}

// x with its sign bit XORed with bit 31 of m (m is 0 or 0x80000000): a
// block's sign relative to the first of its sum, applied exactly.
__device__ __forceinline__ double flip(double x, uint32_t m)
{
    return __hiloint2double(__double2hiint(x) ^ (int)m, __double2loint(x));
}

template <int PROD, bool BPAIR, int TB>
__global__ void __launch_bounds__(FTHREADS, 1)
stra_fused_pair_kernel(const __grid_constant__ DmmaArgs a, const __grid_constant__ FusedPairs tp, int* err,
                       long long limit)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    // The ring on a 1 KB boundary: the swizzle repeats every 8 rows.
    const uint32_t raw = smem_addr(smem_raw);
    unsigned char* smem = smem_raw + (((raw + 1023u) & ~1023u) - raw);
    double* ring = reinterpret_cast<double*>(smem);
    int64_t* rowC = reinterpret_cast<int64_t*>(smem + TRING_BYTES);
    int64_t* colC = rowC + FHMAX * FT;
    int64_t* rowA = colC + FHMAX * FT;       // PAIRS producer tables
    int64_t* colB = rowA + FHMAX * FT;
    int64_t* kA = colB + FHMAX * FT;         // [FHMAX][TB], kB follows (room for TBK)
    int64_t* kB = kA + FHMAX * TB;
    FusedCtrl* ctl = reinterpret_cast<FusedCtrl*>(PROD == PROD_PAIRS ? reinterpret_cast<unsigned char*>(kA + 2 * FHMAX * TBK)
                                                                     : reinterpret_cast<unsigned char*>(rowA));
    volatile int* abort_flag = &ctl->abort;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0)
    {
        for (int s = 0; s < FSTAGES; s++)
        {
            mbar_init(smem_addr(&ctl->full[s]), PROD == PROD_PAIRS ? PT : 1);
            mbar_init(smem_addr(&ctl->empty[s]), NCW);
        }
        ctl->abort = 0;
        mbar_init_fence();
    }
    __syncthreads();

    const int64_t work = a.batch * (int64_t)a.tiles_m * a.tiles_n;
    using SS = SlotShape<TB>;
    constexpr int NT = SS::NT, ROW = SS::ROW, BOX = SS::BOX;
    const int64_t nk = (a.ks + TB - 1) / TB;

    if (warp < NPW)
    {
        asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;\n" :: "n"(Regs<PROD>::PROD_REGS));
        if constexpr (PROD == PROD_TMA)
        {
            // ---------------- producer warp 0: lanes issue the boxes ----------------
            // Lane 0 waits for the slot and posts its byte count; then lanes
            // 0 and 1 copy the A blocks of the product's sum, lanes 2 and 3 the
            // B blocks, each computing its own box coordinates.
            static_assert(TB == TBK, "tensor-map boxes fill 16-k slots");
            if (warp != 0) return;
            if (lane == 0)
                for (int m = 0; m < 2; m++)
                    asm volatile("prefetch.tensormap [%0];\n" :: "l"(reinterpret_cast<unsigned long long>(&tp.map[m]))
                                 : "memory");
            uint32_t it = 0;
            bool ok = true;
            for (int64_t w = blockIdx.x; w < work && ok; w += gridDim.x)
            {
                int64_t b, tm, tn;
                decode_work(a, w, b, tm, tn);
                for (int p = 0; p < a.nprod && ok; p++)
                {
                    const DevProduct& P = a.prod[p];
                    for (int64_t s = 0; s < nk; s++)
                    {
                        const uint32_t slot = it % FSTAGES, use = it / FSTAGES;
                        bool got = true;
                        if (lane == 0 && use > 0)
                            got = mbar_wait(smem_addr(&ctl->empty[slot]), (use & 1) ^ 1, abort_flag, err, 1, limit);
                        ok = __shfl_sync(0xffffffffu, got, 0);
                        if (!ok) break;
                        it++;
                        const uint32_t full = smem_addr(&ctl->full[slot]);
                        if (lane == 0) mbar_expect_tx(full, (uint32_t)((P.na + P.nb) * BOX * 8));
                        __syncwarp();
                        double* S = ring + slot * TSLOT_DOUBLES;
                        int c[5];
                        if (lane < P.na)
                        {
                            box_coords(tp.co[0], P.a_r[lane] * a.ms + tm * FT, P.a_c[lane] * a.ks + s * TB, b, c);
                            tma_box(smem_addr(S + lane * BOX), &tp.map[0], c, tp.co[0].ndim, full);
                        }
                        else if (lane >= NT && lane - NT < P.nb)
                        {
                            const int t = lane - NT;
                            box_coords(tp.co[1], P.b_c[t] * a.ns + tn * FT, P.b_r[t] * a.ks + s * TB, b, c);
                            tma_box(smem_addr(S + (NT + t) * BOX), &tp.map[1], c, tp.co[1].ndim, full);
                        }
                    }
                }
            }
            // Copies in flight land before the CTA leaves: bounded waits on
            // the last uses of the slots.
            if (lane == 0)
            {
                volatile int never = 0;
                for (uint32_t i = it > (uint32_t)FSTAGES ? it - FSTAGES : 0; i < it; i++)
                    mbar_wait(smem_addr(&ctl->full[i % FSTAGES]), (i / FSTAGES) & 1, &never, nullptr, 0,
                              MBAR_WAIT_LIMIT);
            }
            return;
        }
        else
        {
            // ---------------- producer warpgroup: 16-byte pair copies ----------------
            // Thread (warp w, lane l) copies pair kp = l % P of tile rows
            // r0 + (4 * 32 / P) i, r0 = (32 / P) w + l / P, P = TB / 2 pairs
            // per row: a row's pairs go to consecutive lanes (one 16-byte
            // chunk each of one TB-double row).
            const int ptid = tid;
            const int kp = lane % SS::LPR, r0 = warp * SS::RPW + lane / SS::LPR;
            const int klA = tp.pbase[0][kp], klB = tp.pbase[1][kp];
            const int kla2 = klA | (1 << tp.pbit[0]), klb2 = klB | (1 << tp.pbit[1]);
            const int dA = (swizzle((tp.koff[0][klA] + ROW * (r0 & 7)) * 8, tp.swz[0]) >> 3) + ROW * (r0 & ~7);
            const int dB = (swizzle((tp.koff[1][klB] + ROW * (r0 & 7)) * 8, tp.swz[1]) >> 3) + ROW * (r0 & ~7);
            const int H = a.H;
            const int Hk = a.Hk > 0 ? a.Hk : a.H;
            const int Hn = a.Hn > 0 ? a.Hn : a.H;
            // This thread's entries of the k tables kA, kB for k-step s: they
            // depend on the k-step only, so the next step's are loaded while
            // the current one is copied.
            auto ktab_entry = [&](int64_t s, int j) -> int64_t {
                const int i = ptid + j * PT;
                const int op = i / (FHMAX * TB), e = i % (FHMAX * TB);
                const int h = e / TB, kk = e % TB;
                const int64_t kl = s * TB + kk, gk = h * a.ks + kl;
                if (!(i < SS::KTAB && h < Hk && kl < a.ks && gk < a.k)) return OFF_INVALID;
                return op == 0 ? a.ksA[gk] : a.ksB[gk];
            };
            int64_t kv[SS::KENT];
#pragma unroll
            for (int j = 0; j < SS::KENT; j++) kv[j] = nk > 0 ? ktab_entry(0, j) : OFF_INVALID;
            uint32_t it = 0;
            bool ok = true;      // this thread's waits so far
            bool stop = false;   // set only right after a collective check, so uniform
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
                        // All producers are done with the last k-step's tables
                        // (and the tile's row tables are complete); a wait
                        // that ran out in any of them ends the loops for all.
                        if (bar_any<1, PT>(!ok)) { stop = true; break; }
#pragma unroll
                        for (int j = 0; j < SS::KENT; j++)   // kA, kB: one array
                            if (SS::KENT * PT == SS::KTAB || ptid + j * PT < SS::KTAB) kA[ptid + j * PT] = kv[j];
                        bar_sync<1, PT>();
                        {
                            const int64_t sn = s + 1 < nk ? s + 1 : 0;
#pragma unroll
                            for (int j = 0; j < SS::KENT; j++) kv[j] = ktab_entry(sn, j);
                        }
                        const uint32_t slot = it % FSTAGES, use = it / FSTAGES;
                        it++;
                        if (!ok || (use > 0 && !mbar_wait(smem_addr(&ctl->empty[slot]), (use & 1) ^ 1,
                                                                abort_flag, err, 1, limit)))
                        {
                            ok = false;
                            continue;
                        }
                        const uint32_t S = smem_addr(ring + slot * TSLOT_DOUBLES);
                        const uint32_t T = S + NT * BOX * 8;
                        for (int t = 0; t < P.na; t++)
                        {
                            const int64_t* rt = rowA + P.a_r[t] * FT;
                            const int64_t* kt = kA + P.a_c[t] * TB;
                            const int64_t ko = kt[klA];
                            const int nb = kt[kla2] != OFF_INVALID ? 16 : 8;
#pragma unroll
                            for (int i = 0; i < SS::NIP; i++)
                            {
                                const int64_t ro = rt[r0 + SS::RPP * i];
                                const bool v = ro != OFF_INVALID && ko != OFF_INVALID;
                                cp_async16(S + (uint32_t)(t * BOX + dA + SS::RPP * ROW * i) * 8,
                                           v ? a.A + (ro + ko) : a.A, v ? nb : 0);
                            }
                        }
                        for (int t = 0; t < P.nb; t++)
                        {
                            const int64_t* ct = colB + P.b_c[t] * FT;
                            const int64_t* kt = kB + P.b_r[t] * TB;
                            const int64_t ko = kt[klB];
                            const int nb = kt[klb2] != OFF_INVALID ? 16 : 8;
#pragma unroll
                            for (int i = 0; i < SS::NIP; i++)
                            {
                                const int64_t co = ct[r0 + SS::RPP * i];
                                const bool v = co != OFF_INVALID && ko != OFF_INVALID;
                                cp_async16(T + (uint32_t)(t * BOX + dB + SS::RPP * ROW * i) * 8,
                                           v ? a.B + (co + ko) : a.B, v ? nb : 0);
                            }
                        }
                        // the slot's full barrier completes when every producer's copies have landed
                        asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];\n"
                                     :: "r"(smem_addr(&ctl->full[slot])) : "memory");
                    }
                }
            }
            asm volatile("cp.async.wait_all;\n" ::: "memory");   // this thread's copies land before it leaves
            return;
        }
    }

    // ---------------- consumer warpgroups ----------------
    asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;\n" :: "n"(Regs<PROD>::CONS_REGS));
    const int ctid = tid - PT;
    const int cw = warp - NPW;
    const int g = lane >> 2, t4 = lane & 3;
    const int wm = (cw / CWN) * WTM;
    const int wn = (cw % CWN) * WTN;
    const int sa = tp.sigA[g];
    // This lane's reads inside a tile: A's pairs of steps at rows wm + sa
    // (+16 mi, +8 for the fragment's second row), B's steps at columns
    // wn + sigB[g] (+8 ni).
    int a_off[SS::NQ], b_off[2 * SS::NQ];
#pragma unroll
    for (int q = 0; q < SS::NQ; q++) a_off[q] = tp.aoff[lane][q] + wm * ROW;
#pragma unroll
    for (int j = 0; j < 2 * SS::NQ; j++) b_off[j] = tp.boff[lane][j] + wn * ROW;
    const int col0 = tp.sigB[2 * t4], col1 = tp.sigB[2 * t4 + 1];

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
            const DevProduct& P = a.prod[p];
            // the other blocks of a sum, with their signs relative to the
            // first (the first's sign moves to the C coefficient): added as
            // fma(+-1, u, v) with 2 blocks per sum or B read in pairs, as
            // sign-bit flips (fewer registers: no spills) with 4 blocks and B
            // read by element
            constexpr bool FMA_SUMS = TB == 16 || BPAIR;
            const int na = P.na, nb = P.nb;
            uint32_t ma[NT], mb[NT];
            double ra[NT], rb[NT];
#pragma unroll
            for (int t = 1; t < NT; t++)
            {
                ma[t] = t < na && P.a_s[t] * P.a_s[0] < 0 ? 0x80000000u : 0u;
                mb[t] = t < nb && P.b_s[t] * P.b_s[0] < 0 ? 0x80000000u : 0u;
                ra[t] = ma[t] ? -1.0 : 1.0;
                rb[t] = mb[t] ? -1.0 : 1.0;
            }

            for (int64_t s = 0; s < nk; s++)
            {
                const uint32_t slot = cit % FSTAGES;
                ok = __all_sync(0xffffffffu, mbar_wait(smem_addr(&ctl->full[slot]), (cit / FSTAGES) & 1,
                                                             abort_flag, err, 2, limit));
                if (!ok) break;
                const double* Ab = ring + slot * TSLOT_DOUBLES;
                const double* Bb = Ab + NT * BOX;
#pragma unroll
                for (int q = 0; q < SS::NQ; q++)
                {
                    double2 va[MI][2];
#pragma unroll
                    for (int mi = 0; mi < MI; mi++)
#pragma unroll
                        for (int h = 0; h < 2; h++)
                        {
                            const double* pa = Ab + (mi * 16 + h * 8) * ROW + a_off[q];
                            va[mi][h] = ld2(pa);
#pragma unroll
                            for (int t = 1; t < NT; t++)
                                if (t < na)
                                {
                                    const double2 u = ld2(pa + t * BOX);
                                    if (FMA_SUMS)
                                    {
                                        va[mi][h].x = fma(ra[t], u.x, va[mi][h].x);
                                        va[mi][h].y = fma(ra[t], u.y, va[mi][h].y);
                                    }
                                    else
                                    {
                                        va[mi][h].x += flip(u.x, ma[t]);
                                        va[mi][h].y += flip(u.y, ma[t]);
                                    }
                                }
                        }
                    double vb[NI][2];
#pragma unroll
                    for (int ni = 0; ni < NI; ni++)
                    {
                        if (BPAIR)
                        {
                            const double* pb = Bb + ni * 8 * ROW + b_off[2 * q];
                            double2 v = ld2(pb);
#pragma unroll
                            for (int t = 1; t < NT; t++)
                                if (t < nb)
                                {
                                    const double2 u = ld2(pb + t * BOX);
                                    if (FMA_SUMS)
                                    {
                                        v.x = fma(rb[t], u.x, v.x);
                                        v.y = fma(rb[t], u.y, v.y);
                                    }
                                    else
                                    {
                                        v.x += flip(u.x, mb[t]);
                                        v.y += flip(u.y, mb[t]);
                                    }
                                }
                            vb[ni][0] = v.x;
                            vb[ni][1] = v.y;
                        }
                        else
#pragma unroll
                            for (int jj = 0; jj < 2; jj++)
                            {
                                const double* pb = Bb + ni * 8 * ROW + b_off[2 * q + jj];
                                vb[ni][jj] = *pb;
#pragma unroll
                                for (int t = 1; t < NT; t++)
                                    if (t < nb)
                                        vb[ni][jj] = FMA_SUMS ? fma(rb[t], pb[t * BOX], vb[ni][jj])
                                                              : vb[ni][jj] + flip(pb[t * BOX], mb[t]);
                            }
                    }
#pragma unroll
                    for (int jj = 0; jj < 2; jj++)
#pragma unroll
                        for (int mi = 0; mi < MI; mi++)
#pragma unroll
                            for (int ni = 0; ni < NI; ni++)
                                dmma(acc[mi][ni], jj ? va[mi][0].y : va[mi][0].x, jj ? va[mi][1].y : va[mi][1].x,
                                     vb[ni][jj]);
                }
                __syncwarp();
                if (lane == 0) mbar_arrive(smem_addr(&ctl->empty[slot]));
                cit++;
            }
            if (!ok) break;
            const bool lead_neg = (P.a_s[0] < 0) != (P.b_s[0] < 0);
            product_epilogue(a, P, lead_neg, rowC, colC, acc, wm, wn, sa, col0, col1);
        }
    }
}

// ---------------------------------------------------------------- host side

// One layout of an operand's tile in shared memory: slot k kl at position
// koff[kl] of its 16-double row, then the swizzle of span swz.  For the TMA
// form also the tensor map that writes it.
struct Layout
{
    int ndim = 0;        // tensor-map rank (TMA form; 0: pair copies)
    TmaCoords co;
    int64_t len[5], stride[5];
    uint32_t box[5];
    int swz = 0;
    int koff[TBK];
};

// Layouts of the TMA form: the tile of one operand over its row modes (FT
// per tile), k modes (TBK per tile) and batch modes, given as (len, stride)
// lists in the planner's order (first mode fastest), as a box whose k modes
// all precede its row modes (so each tile row holds its 16 k).  Empty when
// the tile is not a box of at most 5 dimensions with dimension 0 a k mode of
// unit stride.  `bit0` receives the slot k bit of dimension 0's lowest digit
// bit (the pair of elements one 16-byte read returns).
std::vector<Layout> tma_layouts(const std::vector<int64_t>* L[3], const std::vector<int64_t>* S[3], int& bit0)
{
    struct Part { int64_t div, mod, mult; };
    struct D { int src; int64_t len, stride; uint32_t box; std::vector<Part> parts; int kpos; };
    std::vector<Layout> out;
    std::vector<D> kb, rb, cd;
    const int64_t tile[3] = {FT, TBK, 1};
    for (int src = 0; src < 3; src++)
    {
        const std::vector<int64_t>& l = *L[src];
        const std::vector<int64_t>& st = *S[src];
        if (l.size() != st.size()) return out;
        int top = -1;
        for (size_t i = 0; i < l.size(); i++)
            if (l[i] > 1) top = (int)i;
        int64_t rem = tile[src], div = 1;
        for (size_t i = 0; i < l.size(); i++)
        {
            if (l[i] <= 1) continue;
            D d{src, l[i], st[i], 1, {Part{div, (int)i == top ? 0 : l[i], 1}}, 0};
            if (rem > 1)
            {
                if (l[i] <= rem)
                {
                    if (rem % l[i]) return out;
                    d.box = (uint32_t)l[i];
                    rem /= l[i];
                }
                else
                {
                    // the top digit may end inside a box: its last box reads
                    // past the extent, as zero
                    if (l[i] % rem && (int)i != top) return out;
                    d.box = (uint32_t)rem;
                    rem = 1;
                }
                (src == 0 ? rb : kb).push_back(d);
            }
            else
                cd.push_back(d);
            div *= l[i];
        }
        if (rem > 1) return out;   // fewer rows (k) than one tile
    }
    {
        int w = 1;
        for (D& d : kb) { d.kpos = w; w *= (int)d.box; }
    }
    int unit = -1;
    for (size_t i = 0; i < kb.size(); i++)
        if (kb[i].stride == 1) unit = (int)i;
    if (unit < 0 || kb[unit].box < 2 || kb.size() > 4) return out;
    bit0 = 0;
    while ((1 << bit0) < kb[unit].kpos) bit0++;
    std::vector<int> rest;
    for (size_t i = 0; i < kb.size(); i++)
        if ((int)i != unit) rest.push_back((int)i);
    do
    {
        std::vector<D> dims;
        dims.push_back(kb[unit]);
        for (int i : rest) dims.push_back(kb[i]);
        for (const D& d : rb) dims.push_back(d);
        // A mode that only carries the origin and continues another mode of
        // the same index in memory (its stride is that mode's extent times
        // stride) joins that mode's dimension as its high digits.
        for (const D& y : cd)
        {
            bool merged = false;
            for (D& x : dims)
                if (x.src == y.src && y.stride == x.len * x.stride && x.parts.size() < TMA_PARTS)
                {
                    Part pt = y.parts[0];
                    pt.mult = x.len;
                    x.parts.push_back(pt);
                    x.len *= y.len;
                    merged = true;
                    break;
                }
            if (!merged) dims.push_back(y);
        }
        bool fits = dims.size() <= 5;
        for (size_t i = 1; fits && i < dims.size(); i++)
            if (dims[i].stride <= 0 || (dims[i].stride * 8) % 16 != 0) fits = false;
        for (size_t i = 0; fits && i < dims.size(); i++)
            if (dims[i].len > ((int64_t)1 << 31)) fits = false;
        if (!fits) continue;
        Layout lay;
        lay.ndim = (int)dims.size();
        std::memset(&lay.co, 0, sizeof lay.co);
        lay.co.ndim = lay.ndim;
        for (int d = 0; d < lay.ndim; d++)
        {
            lay.len[d] = dims[d].len;
            lay.stride[d] = dims[d].stride;
            lay.box[d] = dims[d].box;
            lay.co.src[d] = dims[d].src;
            lay.co.nparts[d] = (int)dims[d].parts.size();
            for (size_t q = 0; q < dims[d].parts.size(); q++)
            {
                lay.co.div[d][q] = dims[d].parts[q].div;
                lay.co.mod[d][q] = dims[d].parts[q].mod;
                lay.co.mult[d][q] = dims[d].parts[q].mult;
            }
        }
        for (int kl = 0; kl < TBK; kl++)
        {
            auto digit = [&](int i) { return (kl / kb[i].kpos) % (int)kb[i].box; };
            int off = digit(unit), m = (int)kb[unit].box;
            for (int i : rest) { off += digit(i) * m; m *= (int)kb[i].box; }
            lay.koff[kl] = off;
        }
        lay.swz = 0;
        out.push_back(lay);
        const int span = (int)kb[unit].box * 8;   // swizzle only where the box stays dense
        if (span == 32 || span == 64 || span == 128)
        {
            lay.swz = span;
            out.push_back(lay);
        }
    } while (std::next_permutation(rest.begin(), rest.end()));
    return out;
}

// Layouts of the pair-copy form for slots of tb k (16 or 8): the pair bit
// at row position 0, the other slot k bits in every order, every swizzle
// span that commutes with shifts by 8 rows (up to 128 bytes for 16-double
// rows, 64 for 8).
std::vector<Layout> pair_layouts(int bit, int tb)
{
    std::vector<Layout> out;
    const int nbits = tb == 16 ? 4 : 3;
    int rest[3], nr = 0;
    for (int b = 0; b < nbits; b++)
        if (b != bit) rest[nr++] = b;
    std::sort(rest, rest + nr);
    do
    {
        for (int span : {0, 32, 64, 128})
        {
            if (span > tb * 8) continue;
            Layout lay;
            std::memset(&lay.co, 0, sizeof lay.co);
            lay.swz = span;
            for (int kl = 0; kl < tb; kl++)
            {
                int pos = (kl >> bit) & 1;
                for (int i = 0; i < nr; i++) pos |= ((kl >> rest[i]) & 1) << (i + 1);
                lay.koff[kl] = pos;
            }
            out.push_back(lay);
        }
    } while (std::next_permutation(rest, rest + nr));
    return out;
}

// Bank conflicts of one operand's reads for a lane mapping kappa(t, j), a
// permutation sig of the 8 fragment rows (columns) and rows of tb doubles:
// 16-byte reads of the pairs (steps 2q, 2q+1) by quarter warps when `pairs`,
// else 8-byte reads of each step by half warps.  Row offsets are multiples of
// 8 rows and do not change the banks.
template <class Kappa>
int read_conflicts(const Layout& lay, const int sig[8], Kappa kappa, bool pairs, int tb)
{
    int cost = 0;
    if (pairs)
    {
        for (int Q = 0; Q < 4; Q++)
            for (int q = 0; q < tb / 8; q++)
            {
                int cnt[8] = {0}, mx = 0;
                for (int g = 2 * Q; g < 2 * Q + 2; g++)
                    for (int t = 0; t < 4; t++)
                    {
                        const int byte = swizzle((lay.koff[kappa(t, 2 * q)] + tb * sig[g]) * 8, lay.swz);
                        mx = std::max(mx, ++cnt[(byte >> 4) & 7]);
                    }
                cost += mx - 1;
            }
    }
    else
    {
        for (int Hh = 0; Hh < 2; Hh++)
            for (int j = 0; j < tb / 4; j++)
            {
                int cnt[16] = {0}, mx = 0;
                for (int g = 4 * Hh; g < 4 * Hh + 4; g++)
                    for (int t = 0; t < 4; t++)
                    {
                        const int byte = swizzle((lay.koff[kappa(t, j)] + tb * sig[g]) * 8, lay.swz);
                        mx = std::max(mx, ++cnt[(byte >> 3) & 15]);
                    }
                cost += mx - 1;
            }
    }
    return cost;
}

// The chosen plan of both operands.
struct Plan
{
    int prod = PROD_PAIRS;
    int tb = TBK;        // k per slot
    Layout la, lb;
    FusedPairs tp;       // lane tables filled (tensor maps and coordinates not yet)
    bool bpair = false;
    int conflicts = 0;
    int bitA = 0, bitB = 0;
};

// Lane tables of the consumers for slots of tb k.  Step j (0 .. tb/4 - 1) of
// lane t (0..3) in a group of tb / 4 MMA k-steps takes slot k kappa(t, j):
// bit 0 of j is A's pair bit (so steps 2q, 2q+1 read one 16-byte pair of A);
// bit 1 of j (16-k slots) and the two bits of t take the other k bits in a
// chosen order.  B is read in pairs as well when its pair bit is A's, else by
// element.  The search takes, for each lane mapping, the layout of each
// operand and the permutation of its fragment rows (columns; permutations of
// the 3 bits of g) with the fewest bank conflicts, and keeps the best mapping.
bool choose_plan(const std::vector<Layout>& LA, int bitA0, const std::vector<Layout>& LB, int bitB0, int tb,
                 Plan& pl)
{
    if (LA.empty() || LB.empty()) return false;
    static const int perm[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
    int sigs[6][8];
    for (int pi = 0; pi < 6; pi++)
        for (int g = 0; g < 8; g++)
            sigs[pi][g] = (((g >> 0) & 1) << perm[pi][0]) | (((g >> 1) & 1) << perm[pi][1]) |
                          (((g >> 2) & 1) << perm[pi][2]);
    const int nbits = tb == 16 ? 4 : 3;
    const bool bpair = bitA0 == bitB0;
    int best = INT_MAX;
    for (int b1 = nbits == 4 ? 0 : -1; b1 < (nbits == 4 ? 4 : 0); b1++)
    {
        if (b1 == bitA0) continue;
        int rest[2], nr = 0;
        for (int b = 0; b < nbits; b++)
            if (b != bitA0 && b != b1) rest[nr++] = b;
        for (int order = 0; order < 2; order++)
        {
            const int t0 = rest[order], t1 = rest[1 - order];
            auto kappa = [&](int t, int j) {
                return ((j & 1) << bitA0) | (b1 >= 0 ? (j >> 1) << b1 : 0) | ((t & 1) << t0) | ((t >> 1) << t1);
            };
            int ca = INT_MAX, cb = INT_MAX, ia = 0, ib = 0, pa = 0, pb = 0;
            for (size_t i = 0; i < LA.size(); i++)
                for (int pi = 0; pi < 6; pi++)
                {
                    const int c = read_conflicts(LA[i], sigs[pi], kappa, true, tb);
                    if (c < ca) { ca = c; ia = (int)i; pa = pi; }
                }
            for (size_t i = 0; i < LB.size(); i++)
                for (int pi = 0; pi < 6; pi++)
                {
                    const int c = read_conflicts(LB[i], sigs[pi], kappa, bpair, tb);
                    if (c < cb) { cb = c; ib = (int)i; pb = pi; }
                }
            if (ca + cb < best)
            {
                best = ca + cb;
                pl.tb = tb;
                pl.la = LA[ia];
                pl.lb = LB[ib];
                pl.bpair = bpair;
                pl.conflicts = best;
                pl.bitA = bitA0;
                pl.bitB = bitB0;
                FusedPairs& tp = pl.tp;
                std::memset(tp.aoff, 0, sizeof tp.aoff);
                std::memset(tp.boff, 0, sizeof tp.boff);
                for (int lane = 0; lane < 32; lane++)
                {
                    const int g = lane >> 2, t = lane & 3;
                    for (int q = 0; q < tb / 8; q++)
                        tp.aoff[lane][q] =
                            (int16_t)(swizzle((pl.la.koff[kappa(t, 2 * q)] + tb * sigs[pa][g]) * 8, pl.la.swz) / 8);
                    for (int j = 0; j < tb / 4; j++)
                        tp.boff[lane][j] =
                            (int16_t)(swizzle((pl.lb.koff[kappa(t, j)] + tb * sigs[pb][g]) * 8, pl.lb.swz) / 8);
                }
                for (int g = 0; g < 8; g++)
                {
                    tp.sigA[g] = (int8_t)sigs[pa][g];
                    tp.sigB[g] = (int8_t)sigs[pb][g];
                }
            }
        }
    }
    return true;
}

// The pair bit of one operand for the pair-copy form with slots of tb k: its
// k modes (planner order) hold a unit-stride mode u (of even extent unless it
// is the top k mode) whose lower modes span 2^b slot k (2^b < tb), so slot k
// kl and kl + 2^b (bit b of kl clear) are adjacent doubles.  Every other
// stride (k, row and batch modes) is even, so each pair starts on 16 bytes
// (with a 16-byte aligned base), and slots start on multiples of tb k (one
// block along k, or block extents of whole slots).  `pbase` receives the tb/2
// pair bases of a slot ordered by their offset in the operand, so that
// consecutive lanes copy neighbouring pairs.
bool pair_bit(const std::vector<int64_t>& kl, const std::vector<int64_t>& ks, const std::vector<int64_t>& rs,
              const std::vector<int64_t>& bs, int Hk, int64_t kblk, int tb, int& bit, int8_t pbase[8])
{
    if (Hk > 1 && kblk % tb) return false;
    int u = -1, top = -1;
    for (size_t i = 0; i < kl.size(); i++)
    {
        if (kl[i] > 1 && ks[i] == 1) u = (int)i;
        if (kl[i] > 1) top = (int)i;
    }
    // an odd extent only on the top k mode: its last pair's partner lies
    // past k and reads as zero
    if (u < 0 || (kl[u] % 2 && u != top)) return false;
    int64_t below = 1;
    for (int i = 0; i < u; i++) below *= kl[i];
    if (below > tb / 2 || (below & (below - 1))) return false;
    for (size_t i = 0; i < kl.size(); i++)
        if ((int)i != u && kl[i] > 1 && ks[i] % 2) return false;
    for (size_t i = 0; i < rs.size(); i++)
        if (rs[i] % 2) return false;
    for (size_t i = 0; i < bs.size(); i++)
        if (bs[i] % 2) return false;
    bit = 0;
    while ((int64_t(1) << bit) < below) bit++;
    // offsets of the pair bases of the first slot (mixed radix over the modes)
    std::vector<std::pair<int64_t, int>> bases;
    for (int k = 0; k < tb; k++)
    {
        if ((k >> bit) & 1) continue;
        int64_t rest = k, off = 0;
        for (size_t i = 0; i < kl.size(); i++)
        {
            off += (rest % kl[i]) * ks[i];
            rest /= kl[i];
        }
        bases.emplace_back(off, k);
    }
    std::stable_sort(bases.begin(), bases.end());
    for (int i = 0; i < 8; i++) pbase[i] = i < tb / 2 ? (int8_t)bases[i].second : 0;
    return true;
}

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// The driver's tensor-map encoder, looked up once through the runtime (no
// link against the driver library).
EncodeTiled encode_tiled()
{
    static EncodeTiled fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
        {
            cudaGetLastError();
            return static_cast<EncodeTiled>(nullptr);
        }
        return reinterpret_cast<EncodeTiled>(p);
    }();
    return fn;
}

bool encode_box(const Layout& lay, const double* base, CUtensorMap& map)
{
    EncodeTiled enc = encode_tiled();
    if (!enc) return false;
    cuuint64_t gdim[5], gstride[4];
    cuuint32_t box[5], estride[5];
    size_t box_elems = 1;
    for (int d = 0; d < lay.ndim; d++)
    {
        gdim[d] = (cuuint64_t)lay.len[d];
        box[d] = lay.box[d];
        box_elems *= lay.box[d];
        estride[d] = 1;
        if (d > 0) gstride[d - 1] = (cuuint64_t)lay.stride[d] * 8;
    }
    // a box is one 16 KB tile, written densely (dimension 0's bytes equal the
    // swizzle span, or no swizzle)
    if (box_elems != (size_t)SlotShape<TBK>::BOX) return false;
    if (lay.swz != 0 && lay.swz != (int)lay.box[0] * 8) return false;
    const CUtensorMapSwizzle sw = lay.swz == 32    ? CU_TENSOR_MAP_SWIZZLE_32B
                                  : lay.swz == 64  ? CU_TENSOR_MAP_SWIZZLE_64B
                                  : lay.swz == 128 ? CU_TENSOR_MAP_SWIZZLE_128B
                                                   : CU_TENSOR_MAP_SWIZZLE_NONE;
    std::memset(&map, 0, sizeof map);
    const CUresult r = enc(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, (cuuint32_t)lay.ndim, const_cast<double*>(base),
                           gdim, gstride, box, estride, CU_TENSOR_MAP_INTERLEAVE_NONE, sw,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

// The plan of both operands for a grid of H x Hk (A), Hk x Hn (B) blocks of
// extents ms, ns, ks and slots of tb k (16: sums of up to 2 blocks, 8: up to
// 4); false when the element-pair kernel does not apply.  Slots of 8 k are
// filled by pair copies only.
// Tensor-map boxes where every tile is a box whose rows are one 128-byte run
// of the operand (16 k of its unit-stride mode: one request per row); 16-byte
// pair copies elsewhere.  Measured at 16384^3 (effective TFLOP/s, L0 / L1):
// k-major GEMM operands (128-byte rows) 34.5 / 34.7 by boxes, 33.4 / 34.2 by
// pairs; the headline contraction's layout (32-byte runs: each box 512 small
// requests) 17.9 / 20.3 by boxes, 33.3 / 32.2 by pairs.
bool plan_operands(const GemmView& g, int H, int Hn, int Hk, int64_t ms, int64_t ns, int64_t ks, int tb, Plan& pl)
{
    if (g.type != TYPE_DOUBLE || (tb != 16 && tb != 8)) return false;
    std::memset(&pl.tp, 0, sizeof pl.tp);
    // Tiles of the TMA form must not cross block boundaries (a grid of one
    // block along an index has none: its ragged end lies past the tensor).
    if (tb == TBK && !((H > 1 && ms % FT) || (Hn > 1 && ns % FT) || (Hk > 1 && ks % TBK)))
    {
        const std::vector<int64_t>* LA[3] = {&g.mode_len[0], &g.mode_len[4], &g.mode_len[6]};
        const std::vector<int64_t>* SA[3] = {&g.mode_stride[0], &g.mode_stride[4], &g.mode_stride[6]};
        const std::vector<int64_t>* LB[3] = {&g.mode_len[2], &g.mode_len[5], &g.mode_len[7]};
        const std::vector<int64_t>* SB[3] = {&g.mode_stride[2], &g.mode_stride[5], &g.mode_stride[7]};
        int bA = -1, bB = -1;
        auto wide = [](std::vector<Layout> v) {
            v.erase(std::remove_if(v.begin(), v.end(), [](const Layout& l) { return l.box[0] != (uint32_t)TBK; }),
                    v.end());
            return v;
        };
        const std::vector<Layout> la = wide(tma_layouts(LA, SA, bA));
        const std::vector<Layout> lb = wide(tma_layouts(LB, SB, bB));
        if (choose_plan(la, bA, lb, bB, TBK, pl))
        {
            pl.prod = PROD_TMA;
            return true;
        }
    }
    int bitA = 0, bitB = 0;
    if (pair_bit(g.mode_len[4], g.mode_stride[4], g.mode_stride[0], g.mode_stride[6], Hk, ks, tb, bitA,
                 pl.tp.pbase[0]) &&
        pair_bit(g.mode_len[5], g.mode_stride[5], g.mode_stride[2], g.mode_stride[7], Hk, ks, tb, bitB,
                 pl.tp.pbase[1]) &&
        choose_plan(pair_layouts(bitA, tb), bitA, pair_layouts(bitB, tb), bitB, tb, pl))
    {
        pl.prod = PROD_PAIRS;
        for (int op = 0; op < 2; op++)
        {
            const Layout& lay = op ? pl.lb : pl.la;
            for (int kl = 0; kl < TBK; kl++) pl.tp.koff[op][kl] = kl < tb ? (int8_t)lay.koff[kl] : 0;
            pl.tp.swz[op] = (int16_t)lay.swz;
        }
        pl.tp.pbit[0] = (int8_t)bitA;
        pl.tp.pbit[1] = (int8_t)bitB;
        return true;
    }
    return false;
}

// Plans by contraction shape (the operands' mode extents and strides, the
// block grid), per calling thread: the layout and lane-table search costs
// about half a millisecond, the kernel at small sizes less.  Failures are
// kept too.  At most 64 entries (cleared when full).
bool cached_plan(const GemmView& g, int H, int Hn, int Hk, int64_t ms, int64_t ns, int64_t ks, int tb, Plan& pl)
{
    thread_local std::map<std::vector<int64_t>, std::pair<bool, Plan>> plans;
    std::vector<int64_t> key = {g.type, H, Hn, Hk, ms, ns, ks, tb};
    for (int v : {0, 2, 4, 5, 6, 7})
    {
        key.push_back((int64_t)g.mode_len[v].size());
        key.insert(key.end(), g.mode_len[v].begin(), g.mode_len[v].end());
        key.insert(key.end(), g.mode_stride[v].begin(), g.mode_stride[v].end());
    }
    auto it = plans.find(key);
    if (it != plans.end())
    {
        pl = it->second.second;
        return it->second.first;
    }
    if (plans.size() >= 64) plans.clear();
    const bool ok = plan_operands(g, H, Hn, Hk, ms, ns, ks, tb, pl);
    plans.emplace(std::move(key), std::make_pair(ok, pl));
    return ok;
}

}  // namespace

bool fused_pairs_plan(const GemmView& g, int H, int Hn, int Hk, int64_t ms, int64_t ns, int64_t ks, int tb,
                      int tables[PAIRS_PLAN_INTS])
{
    Plan pl;
    if (!cached_plan(g, H, Hn, Hk, ms, ns, ks, tb, pl)) return false;
    if (tables)
    {
        int i = 0;
        tables[i++] = pl.conflicts;
        tables[i++] = pl.prod;
        tables[i++] = pl.la.ndim;
        tables[i++] = pl.lb.ndim;
        tables[i++] = pl.bpair ? 1 : 0;
        tables[i++] = pl.la.swz;
        tables[i++] = pl.lb.swz;
        tables[i++] = pl.bitA;
        tables[i++] = pl.bitB;
        for (int l = 0; l < 32; l++)
            for (int q = 0; q < 2; q++) tables[i++] = pl.tp.aoff[l][q];
        for (int l = 0; l < 32; l++)
            for (int j = 0; j < 4; j++) tables[i++] = pl.tp.boff[l][j];
        for (int gg = 0; gg < 8; gg++) tables[i++] = pl.tp.sigA[gg];
        for (int gg = 0; gg < 8; gg++) tables[i++] = pl.tp.sigB[gg];
        for (int kl = 0; kl < TBK; kl++) tables[i++] = pl.la.koff[kl];
        for (int kl = 0; kl < TBK; kl++) tables[i++] = pl.lb.koff[kl];
        for (int p = 0; p < 8; p++) tables[i++] = pl.tp.pbase[0][p];
        for (int p = 0; p < 8; p++) tables[i++] = pl.tp.pbase[1][p];
        tables[i++] = pl.tb;
    }
    return true;
}

cudaError_t launch_fused_pairs(const DmmaArgs& in, const GemmView& g, cudaStream_t stream, int num_sms, int* err,
                               long long wait_limit)
{
    if (in.batch <= 0 || in.ms <= 0 || in.ns <= 0) return cudaSuccess;
    if (in.H < 1 || in.H > FHMAX || in.Hc != in.H || in.mC != in.m || in.nC != in.n) return cudaErrorNotSupported;
    if (in.Hk < 0 || in.Hk > FHMAX || in.Hn < 0 || in.Hn > FHMAX) return cudaErrorNotSupported;
    if (in.nprod < 1 || in.nprod > MAX_PRODUCTS) return cudaErrorInvalidValue;
    int most = 1;   // blocks in the longest operand sum
    for (int p = 0; p < in.nprod; p++) most = std::max(most, (int)std::max(in.prod[p].na, in.prod[p].nb));
    if (most > SlotShape<8>::NT) return cudaErrorNotSupported;
    const int tb = most <= SlotShape<16>::NT ? 16 : 8;
    if (reinterpret_cast<uintptr_t>(in.A) % 16 || reinterpret_cast<uintptr_t>(in.B) % 16)
        return cudaErrorNotSupported;
    const int Hn = in.Hn > 0 ? in.Hn : in.H, Hk = in.Hk > 0 ? in.Hk : in.H;
    Plan pl;
    if (!cached_plan(g, in.H, Hn, Hk, in.ms, in.ns, in.ks, tb, pl)) return cudaErrorNotSupported;
    FusedPairs& tp = pl.tp;
    if (pl.prod == PROD_TMA)
    {
        tp.co[0] = pl.la.co;
        tp.co[1] = pl.lb.co;
        if (!encode_box(pl.la, in.A, tp.map[0]) || !encode_box(pl.lb, in.B, tp.map[1])) return cudaErrorNotSupported;
    }
    using Kern = void (*)(DmmaArgs, FusedPairs, int*, long long);
    Kern kern = pl.prod == PROD_PAIRS
                    ? (pl.tb == 8 ? (pl.bpair ? stra_fused_pair_kernel<PROD_PAIRS, true, 8>
                                              : stra_fused_pair_kernel<PROD_PAIRS, false, 8>)
                                  : (pl.bpair ? stra_fused_pair_kernel<PROD_PAIRS, true, 16>
                                              : stra_fused_pair_kernel<PROD_PAIRS, false, 16>))
                    : (pl.bpair ? stra_fused_pair_kernel<PROD_TMA, true, 16> : stra_fused_pair_kernel<PROD_TMA, false, 16>);
    const size_t need = pl.prod == PROD_PAIRS
                            ? (size_t)Regs<PROD_PAIRS>::PROD_REGS * PT + (size_t)Regs<PROD_PAIRS>::CONS_REGS * CT
                            : (size_t)Regs<PROD_TMA>::PROD_REGS * PT + (size_t)Regs<PROD_TMA>::CONS_REGS * CT;
    const size_t smem = tile_smem(pl.prod);
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, reinterpret_cast<const void*>(kern));
    if (e != cudaSuccess) return e;
    if ((size_t)fa.numRegs * FTHREADS < need) return cudaErrorNotSupported;
    e = cudaFuncSetAttribute(reinterpret_cast<const void*>(kern), cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
    if (e != cudaSuccess) return e;
    DmmaArgs args = in;
    args.tiles_m = (int)((args.ms + FT - 1) / FT);
    args.tiles_n = (int)((args.ns + FT - 1) / FT);
    args.work = args.batch * (int64_t)args.tiles_m * args.tiles_n;
    if (args.work <= 0) return cudaSuccess;
    int64_t grid = num_sms;
    if (args.work < grid) grid = args.work;
    const int kind = pl.prod == PROD_PAIRS ? KK_FUSED_PAIRS : KK_FUSED_TMA;
    timing_begin(kind, stream);
    kern<<<(unsigned)grid, FTHREADS, smem, stream>>>(args, tp, err, wait_cycles(wait_limit));
    timing_end(kind, stream);
    e = cudaGetLastError();
    if (e == cudaSuccess) g_launches++;
    return e;
}

}  // namespace tsb
