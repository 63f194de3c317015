// Split-BF16 path for FP32 contractions on the 5th-generation tensor cores
// (tcgen05, accumulators in TMEM).  No counterpart kernel in the reference,
// which computes FP32 contractions with its CPU micro-kernels; the Strassen
// schedule around it is the reference's ABC one (see packed_kernels.cu).
//
// Per Strassen product:
//   scale_kernel     per local row r (A side) / column c (B side) a power of two
//                    2^-e with 2^-e * max|X(r,:)| in [0.5, 1), taken over all
//                    blocks of that row index, so every block of one signed sum
//                    shares it;
//   split_pack_kernel  S = sum_i u_i A_i in FP32, times the row scale, split
//                    into P bf16 planes hi + mid (+ lo) with x ~ hi + mid + lo,
//                    written as 128 x 64 tiles in the K-major 128-byte-swizzled
//                    layout the tcgen05 shared-memory descriptors read;
//   split_gemm_kernel  for each 128 x 128 C tile, the bf16 products of the plane
//                    pairs (hh, hm, mh for 3 terms; + hl, mm, lh for 6 terms)
//                    accumulate in TMEM (FP32, hi*hi apart from the smaller
//                    correction terms) over chunks of 256 k; drain warps
//                    add each chunk into FP32 registers (keeping the FP32
//                    rounding of the accumulation to chunk length) and finally
//                    write C_q = (first ? beta*C_q : C_q) + sign*alpha*acc
//                    / (row scale * column scale).
//
// At L >= 1, split_pack_multi_kernel forms the 7 split sums of a product group
// from one pass over each operand.  By default one split_gemm_kernel launch
// then runs every product side by side (batch entry p * batch + b reads plane
// set p, `pbatch`) into its own M_p, which the combine pass of aux_kernels.cu
// sums into C; with that form off, one launch per group runs the group's 7
// products in product order for each tile position (nprod, per-product C
// targets), so the C tiles they update stay in L2 between products.  A plain
// contraction on a small grid splits its summed range the same way
// (split_pack_kernel's `nkpiece`).
//
// Warp roles in split_gemm_kernel (192 threads, one CTA per SM):
//   warp 0      one lane issues the bulk copies (cp.async.bulk, 1-D TMA) of
//               each stage's plane tiles into shared memory;
//   warp 1      allocates TMEM; one lane issues tcgen05.mma and commits;
//   warps 2-5   read TMEM (tcgen05.ld), accumulate, write C.
// Every wait on an mbarrier is bounded (about a second of clock cycles); on
// expiry the kernel records an error code and every role returns.
#include "kernels.cuh"
#include "mbarrier.cuh"
#include "timing.hpp"

#include <cuda_bf16.h>

#include <atomic>

namespace tsb {

extern std::atomic<unsigned long long> g_launches;

namespace {

constexpr int ST = SPLIT_TILE;               // 128: tile rows (A side) / columns (B side)
constexpr int SK = SPLIT_K;                  // k per tile block (one 128-byte bf16 row)
constexpr int BLK = ST * SK * 2;             // 16 KB per tile block
constexpr int KCH = 256 / SK;                // k blocks per TMEM accumulation chunk (256 k)
constexpr int ROWB = SK * 2;                 // bytes per block row
static_assert(SK == 32 || SK == 64, "64- or 128-byte swizzled rows");

// Byte offset of element (r, k) in a 128 x SK bf16 block, K-major with the
// swizzle of its row length (16-byte chunk c = k/8 of row r):
//   64-byte rows (SWIZZLE_64B):   chunk c ^ ((r / 2) % 4), 8-row groups of 512 B;
//   128-byte rows (SWIZZLE_128B): chunk c ^ (r % 8),       8-row groups of 1024 B.
__host__ __device__ __forceinline__ int swz(int r, int k)
{
    const int c = SK == 32 ? ((k >> 3) ^ (r >> 1)) & 3 : ((k >> 3) ^ r) & 7;
    return (r >> 3) * (8 * ROWB) + (r & 7) * ROWB + (c << 4) + (k & 7) * 2;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// ---- row scales -------------------------------------------------------------------

__global__ void scale_kernel(const __grid_constant__ SplitScaleArgs a)
{
    const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (wid >= a.batch * a.rows_blk) return;
    const int64_t b = wid / a.rows_blk, r = wid % a.rows_blk;
    float m = 0.f;
    for (int h = 0; h < a.parts; h++)
    {
        const int64_t gr = h * a.rows_blk + r;
        if (gr >= a.rows_full) continue;
        const int64_t base = a.bX[b] + a.rs[gr];
        for (int64_t k = lane; k < a.k_full; k += 32) m = fmaxf(m, fabsf(a.X[base + a.ks[k]]));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0)
    {
        int e = 0;
        if (m > 0.f && isfinite(m)) frexpf(m, &e);
        e = max(-120, min(120, e));
        a.scale[wid] = ldexpf(1.f, -e);
        a.inv[wid] = ldexpf(1.f, e);
    }
}

// ---- split pack -------------------------------------------------------------------

constexpr int PR = ST / 2;

// Split the scaled FP32 values of buf (rows [64 half, 64 half + 64) of one
// 128 x SK block) into bf16 planes hi = bf16(x), mid = bf16(x - hi),
// lo = bf16(x - hi - mid), written as 16-byte chunks (8 k of one row) at
// their swizzled offsets; plane p of the block is at out + p * plane_stride +
// block_off.
__device__ __forceinline__ void write_planes(const float (*buf)[SK + 1], void* out, size_t plane_stride,
                                             size_t block_off, int half, int planes, int tid)
{
    unsigned char* blk = reinterpret_cast<unsigned char*>(out) + block_off;
#pragma unroll
    for (int i = 0; i < PR * (SK / 8) / 256; i++)
    {
        const int q = tid + 256 * i;
        const int r = q / (SK / 8), g = q % (SK / 8);
        // two values per conversion (cvt.rn.bf16x2.f32); the residuals are
        // exact in FP32, and bf16 -> FP32 is a shift
        uint32_t hv[4], mv[4], lv[4];
#pragma unroll
        for (int j = 0; j < 4; j++)
        {
            const float x0 = buf[r][g * 8 + 2 * j], x1 = buf[r][g * 8 + 2 * j + 1];
            const __nv_bfloat162 h = __floats2bfloat162_rn(x0, x1);
            const float a0 = x0 - __low2float(h), a1 = x1 - __high2float(h);
            const __nv_bfloat162 m = __floats2bfloat162_rn(a0, a1);
            const __nv_bfloat162 l = __floats2bfloat162_rn(a0 - __low2float(m), a1 - __high2float(m));
            hv[j] = *reinterpret_cast<const uint32_t*>(&h);
            mv[j] = *reinterpret_cast<const uint32_t*>(&m);
            lv[j] = *reinterpret_cast<const uint32_t*>(&l);
        }
        const int off = swz(half * PR + r, g * 8);
        *reinterpret_cast<uint4*>(blk + off) = make_uint4(hv[0], hv[1], hv[2], hv[3]);
        *reinterpret_cast<uint4*>(blk + plane_stride + off) = make_uint4(mv[0], mv[1], mv[2], mv[3]);
        if (planes > 2)
            *reinterpret_cast<uint4*>(blk + 2 * plane_stride + off) = make_uint4(lv[0], lv[1], lv[2], lv[3]);
    }
}

// Each CTA packs half a tile block (PR = 64 of its 128 rows x SK k), so a
// CTA's shared memory stays small and several CTAs per SM keep loads in flight.

__global__ void __launch_bounds__(256)
split_pack_kernel(const __grid_constant__ SplitPackArgs a)
{
    __shared__ float buf[PR][SK + 1];
    __shared__ int64_t rowoff[4][PR];            // per term: batch + row offset (or invalid)
    __shared__ int64_t koff[4][SK];              // per term: k offset (or invalid)
    __shared__ float rscale[PR];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int64_t c = blockIdx.x;            // k block
    const int64_t t = blockIdx.y >> 1;       // row tile
    const int half = blockIdx.y & 1;         // its rows [64 half, 64 half + 64)
    const int64_t b = blockIdx.z;
    const int64_t r0 = t * ST + half * PR, k0 = c * SK;
    const int nt = a.nt;
    for (int i = tid; i < nt * PR; i += 256)
    {
        const int q = i / PR, r = i % PR;
        const int64_t lr = r0 + r, gr = a.t_r[q] * a.rows_blk + lr;
        rowoff[q][r] = (lr < a.rows_blk && gr < a.rows_full) ? a.bX[b] + a.rs[gr] : OFF_INVALID;
    }
    for (int i = tid; i < nt * SK; i += 256)
    {
        const int q = i / SK, kk = i % SK;
        const int64_t lk = k0 + kk, gk = a.t_c[q] * a.k_blk + lk;
        koff[q][kk] = (lk < a.k_blk && gk < a.k_full) ? a.ks[gk] : OFF_INVALID;
    }
    for (int i = tid; i < PR; i += 256)
        rscale[i] = (r0 + i < a.rows_blk) ? a.scale[b * a.rows_blk + r0 + i] : 0.f;
    __syncthreads();
    // Terms outermost: all loads of one term are independent and in flight.
    // With kfast the 32 lanes of a warp walk 32 consecutive k of one row,
    // else 32 consecutive rows of one k.
    constexpr int E = PR * SK / 256;
    auto row_of = [&](int x) { return a.kfast ? warp + 8 * (x / (SK / 32)) : lane + 32 * (x % (PR / 32)); };
    auto k_of = [&](int x) { return a.kfast ? lane + 32 * (x % (SK / 32)) : warp + 8 * (x / (PR / 32)); };
    float v[E];
#pragma unroll
    for (int x = 0; x < E; x++) v[x] = 0.f;
    for (int q = 0; q < nt; q++)
    {
        const bool neg = a.t_s[q] < 0;
#pragma unroll
        for (int x = 0; x < E; x++)
        {
            const int64_t ro = rowoff[q][row_of(x)], ko = koff[q][k_of(x)];
            if (ro != OFF_INVALID && ko != OFF_INVALID)
            {
                const float e = a.X[ro + ko];
                v[x] += neg ? -e : e;
            }
        }
    }
#pragma unroll
    for (int x = 0; x < E; x++)
    {
        const int r = row_of(x);
        buf[r][k_of(x)] = v[x] * rscale[r];
    }
    __syncthreads();
    if (a.nkpiece > 0)
    {
        const int64_t p = c / a.nkpiece;
        const size_t plane = (size_t)a.batch * a.tiles * a.nkpiece * BLK;
        write_planes(buf, reinterpret_cast<unsigned char*>(a.out) + p * a.planes * plane, plane,
                     ((size_t)(b * a.tiles + t) * a.nkpiece + (c - p * a.nkpiece)) * BLK, half, a.planes, tid);
    }
    else
        write_planes(buf, a.out, (size_t)a.batch * a.tiles * a.nk * BLK,
                     ((size_t)(b * a.tiles + t) * a.nk + c) * BLK, half, a.planes, tid);
}

// Seven split sums of one product group per pass (L >= 1), the FP32 form of
// pack_multi_kernel: the CTA's 64-row x SK window of every block of the
// group's coarse sum is read once, the four sub-block sums X_j stay in
// registers, and each output's signed combination is scaled and split.
__global__ void __launch_bounds__(256)
split_pack_multi_kernel(const __grid_constant__ SplitPackMultiArgs a)
{
    __shared__ float buf[PR][SK + 1];
    __shared__ int64_t rowoff[8][PR];            // per block (t, j): batch + row offset (or invalid)
    __shared__ int64_t koff[8][SK];              // per block (t, j): k offset (or invalid)
    __shared__ float rscale[PR];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int64_t c = blockIdx.x;
    const int64_t t = blockIdx.y >> 1;
    const int half = blockIdx.y & 1;
    const int64_t b = blockIdx.z;
    const int64_t r0 = t * ST + half * PR, k0 = c * SK;
    const int nblk = a.nt * 4;
    for (int i = tid; i < nblk * PR; i += 256)
    {
        const int q = i / PR, r = i % PR;
        const int64_t lr = r0 + r, gr = a.prow[q >> 2][q & 3] * a.rows_blk + lr;
        rowoff[q][r] = (lr < a.rows_blk && gr < a.rows_full) ? a.bX[b] + a.rs[gr] : OFF_INVALID;
    }
    for (int i = tid; i < nblk * SK; i += 256)
    {
        const int q = i / SK, kk = i % SK;
        const int64_t lk = k0 + kk, gk = a.pk[q >> 2][q & 3] * a.k_blk + lk;
        koff[q][kk] = (lk < a.k_blk && gk < a.k_full) ? a.ks[gk] : OFF_INVALID;
    }
    for (int i = tid; i < PR; i += 256)
        rscale[i] = (r0 + i < a.rows_blk) ? a.scale[b * a.rows_blk + r0 + i] : 0.f;
    __syncthreads();
    constexpr int E = PR * SK / 256;
    auto row_of = [&](int x) { return a.kfast ? warp + 8 * (x / (SK / 32)) : lane + 32 * (x % (PR / 32)); };
    auto k_of = [&](int x) { return a.kfast ? lane + 32 * (x % (SK / 32)) : warp + 8 * (x / (PR / 32)); };
    float xs[4][E];
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
        for (int x = 0; x < E; x++) xs[j][x] = 0.f;
    for (int q = 0; q < a.nt; q++)
    {
        const bool neg = a.t_s[q] < 0;
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int x = 0; x < E; x++)
            {
                const int64_t ro = rowoff[q * 4 + j][row_of(x)], ko = koff[q * 4 + j][k_of(x)];
                if (ro != OFF_INVALID && ko != OFF_INVALID)
                {
                    const float e = a.X[ro + ko];
                    xs[j][x] += neg ? -e : e;
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
        for (int x = 0; x < E; x++)
        {
            float v = 0.f;
#pragma unroll
            for (int j = 0; j < 4; j++)
                if (cf[j]) v += cf[j] > 0 ? xs[j][x] : -xs[j][x];
            const int r = row_of(x);
            buf[r][k_of(x)] = v * rscale[r];
        }
        __syncthreads();
        write_planes(buf, a.out[o], (size_t)a.batch * a.tiles * a.nk * BLK,
                     ((size_t)(b * a.tiles + t) * a.nk + c) * BLK, half, a.planes, tid);
    }
}

// ---- tcgen05 GEMM -------------------------------------------------------------------

// Shared-memory descriptor of a 128-row, K-major, swizzled block (swz):
// start >> 4, leading offset 16 B (unused when swizzled), stride 8 rows
// between 8-row groups, fixed 0b001 at bit 46, swizzle mode 4 (64 B rows) or
// 2 (128 B rows) at bit 61.
__device__ __forceinline__ uint64_t sdesc(uint32_t addr)
{
    constexpr uint64_t mode = SK == 32 ? 4 : 2;
    return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)1 << 16) | ((uint64_t)((8 * ROWB) >> 4) << 32) |
           ((uint64_t)1 << 46) | (mode << 61);
}

// Instruction descriptor, kind::f16: D = F32, A = B = BF16, both K-major,
// N = 128 (>> 3 at bit 17), M = 128 (>> 4 at bit 24).
constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((128u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void mma_bf16(uint32_t d, uint64_t ad, uint64_t bd, uint32_t acc)
{
    asm volatile("{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
                 :: "r"(d), "l"(ad), "l"(bd), "r"(IDESC), "r"(acc));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n"
                 :: "r"(mbar) : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32])
{
    uint32_t r[32];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                 "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                 "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                   "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
                   "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
                   "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
                   "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

// Barrier slots of the split GEMM: full[s], empty[s] per ring stage, then
// two accumulator-full, two accumulator-empty and the MMA drain barrier.
constexpr int MAX_STAGES = 6;
constexpr int BAR_FULL = 0, BAR_EMPTY = MAX_STAGES, BAR_ACCF = 2 * MAX_STAGES, BAR_ACCE = 2 * MAX_STAGES + 2,
              BAR_DRAIN = 2 * MAX_STAGES + 4, NBARS = 2 * MAX_STAGES + 5;

template <int P>
struct SG
{
    static constexpr int STAGE_BYTES = 2 * P * BLK;
    static constexpr int STAGES = (192 * 1024) / STAGE_BYTES < MAX_STAGES ? (192 * 1024) / STAGE_BYTES : MAX_STAGES;
    static constexpr int TAB_BYTES = 4 * (ST + ST) * 8 + 2 * ST * 4;
    static constexpr int CTRL_BYTES = 256;
    static constexpr size_t smem = 1024 + size_t(STAGES) * STAGE_BYTES + CTRL_BYTES + TAB_BYTES;
};

// Work sources of the split GEMM: one problem (the kernel parameter, read
// through a pointer of unknown origin so its fields are loaded where used) or
// a group of problems (descriptors in global memory; work item w belongs to
// the problem p with prefix[p] <= w < prefix[p + 1]).  Every role resolves the
// problem of each tile itself, since the roles run tiles apart.
struct OneSplit
{
    const SplitGemmArgs* a;
    __device__ int64_t total() const { return a->batch * a->tiles_m * a->tiles_n; }
    __device__ const SplitGemmArgs& at(int64_t w, int64_t& local) const
    {
        local = w;
        const SplitGemmArgs* p = a;
        asm volatile("" : "+l"(p));
        return *p;
    }
};

struct SplitGroup
{
    const SplitGroupArgs& g;
    __device__ int64_t total() const { return g.total; }
    __device__ const SplitGemmArgs& at(int64_t w, int64_t& local) const
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

// Named barrier 1 over the 128 drain threads with an OR over `flag`: true
// when any of them passes a non-zero flag.
__device__ __forceinline__ bool drain_any(bool flag)
{
    uint32_t out;
    asm volatile("{\n.reg .pred q, p;\nsetp.ne.u32 q, %1, 0;\nbar.red.or.pred p, 1, 128, q;\n"
                 "selp.u32 %0, 1, 0, p;\n}\n" : "=r"(out) : "r"((uint32_t)flag) : "memory");
    return out != 0;
}

template <int P, class Src>
__device__ __forceinline__ void split_gemm_body(const Src& src, int* err, long long limit, unsigned char* smem_raw)
{
    using K = SG<P>;
    // Plane pairs of the product terms (0 = hi, 1 = mid, 2 = lo): hh, hm, mh,
    // then hl, mm, lh with three planes; compile-time so the single issuing
    // thread builds every descriptor from constants.
    constexpr int NTERMS = P == 3 ? 6 : 3;
    constexpr int TERM_A[6] = {0, 0, 1, 0, 1, 2}, TERM_B[6] = {0, 1, 0, 2, 1, 0};
    constexpr int STAGES = K::STAGES;
    unsigned char* smem = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    unsigned char* stages = smem;                           // [STAGES][A planes | B planes]
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + STAGES * K::STAGE_BYTES);
    static_assert(NBARS * 8 + 8 <= K::CTRL_BYTES, "barriers, TMEM slot and abort flag");
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + NBARS);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
    int64_t* rowC = reinterpret_cast<int64_t*>(smem + STAGES * K::STAGE_BYTES + K::CTRL_BYTES);
    int64_t* colC = rowC + 4 * ST;
    float* invr = reinterpret_cast<float*>(colC + 4 * ST);
    float* invc = invr + ST;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    auto bar = [&](int i) { return smem_u32(bars + i); };
    if (tid == 0)
    {
        for (int s = 0; s < STAGES; s++) { mbar_init(bar(BAR_FULL + s), 1); mbar_init(bar(BAR_EMPTY + s), 1); }
        for (int s = 0; s < 2; s++) { mbar_init(bar(BAR_ACCF + s), 1); mbar_init(bar(BAR_ACCE + s), 128); }
        mbar_init(bar(BAR_DRAIN), 1);
        *abort_flag = 0;
        mbar_init_fence();
    }
    if (warp == 1)
    {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;\n"
                     :: "r"(smem_u32(tmem_slot)) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *tmem_slot;

    const int64_t work = src.total();
    auto decode = [&](const SplitGemmArgs& a, int64_t w, int64_t& b, int64_t& tm, int64_t& tn) {
        const int64_t tiles = a.tiles_m * a.tiles_n;
        b = w / tiles;
        const int64_t tw = w - b * tiles;
        const int64_t GROUP = 8;
        const int64_t group = tw / (GROUP * a.tiles_n);
        const int64_t first_m = group * GROUP;
        const int64_t gsize = (a.tiles_m - first_m) < GROUP ? (a.tiles_m - first_m) : GROUP;
        tm = first_m + (tw % gsize);
        tn = (tw % (GROUP * a.tiles_n)) / gsize;
    };

    if (warp == 0)
    {
        if (lane == 0)
        {
            uint32_t it = 0;
            bool ok = true;
            for (int64_t w = blockIdx.x; w < work && ok; w += gridDim.x)
            {
                int64_t local, b, tm, tn;
                const SplitGemmArgs& a = src.at(w, local);
                decode(a, local, b, tm, tn);
                const int64_t nk = a.nk;
                // batch entry b = pp * pbatch + bl: entry bl of the pp-th plane set
                const int64_t pb = a.pbatch > 0 ? a.pbatch : a.batch;
                const int64_t pp = b / pb, bl = b - pp * pb;
                const size_t planeA = (size_t)pb * a.tiles_m * nk * BLK;
                const size_t planeB = (size_t)pb * a.tiles_n * nk * BLK;
                for (int q = 0; q < a.nprod && ok; q++)
                {
                const unsigned char* srcA = reinterpret_cast<const unsigned char*>(a.A[q]) + pp * P * planeA +
                                            ((size_t)(bl * a.tiles_m + tm) * nk) * BLK;
                const unsigned char* srcB = reinterpret_cast<const unsigned char*>(a.B[q]) + pp * P * planeB +
                                            ((size_t)(bl * a.tiles_n + tn) * nk) * BLK;
                for (int64_t c = 0; c < nk; c++, it++)
                {
                    const int s = it % STAGES;
                    const uint32_t ph = (it / STAGES) & 1;
                    if (!mbar_wait(bar(BAR_EMPTY + s), ph ^ 1, abort_flag, err, 1, limit)) { ok = false; break; }
                    mbar_expect_tx(bar(BAR_FULL + s), 2 * P * BLK);
                    const uint32_t dst = smem_u32(stages + s * K::STAGE_BYTES);
#pragma unroll
                    for (int p = 0; p < P; p++)
                    {
                        bulk_copy(dst + p * BLK, srcA + p * planeA + c * BLK, BLK, bar(BAR_FULL + s));
                        bulk_copy(dst + (P + p) * BLK, srcB + p * planeB + c * BLK, BLK, bar(BAR_FULL + s));
                    }
                }
                }
            }
            // Copies still in flight land before the CTA leaves (bounded wait on
            // the full barrier of each of the last STAGES stages issued).
            volatile int never = 0;
            for (uint32_t i = (it > STAGES ? it - STAGES : 0); i < it; i++)
                mbar_wait(bar(BAR_FULL + i % STAGES), (i / STAGES) & 1, &never, nullptr, 0, MBAR_WAIT_LIMIT);
        }
    }
    else if (warp == 1)
    {
        if (lane == 0)
        {
            uint32_t it = 0, u = 0;
            bool ok = true;
            for (int64_t w = blockIdx.x; w < work && ok; w += gridDim.x)
            {
                int64_t local;
                const SplitGemmArgs& a = src.at(w, local);
                const int64_t nk = a.nk;
                for (int q = 0; q < a.nprod && ok; q++)
                {
                uint32_t dcol = 0;
                for (int64_t c = 0; c < nk; c++, it++)
                {
                    if (c % KCH == 0)
                    {
                        const int bacc = u & 1;
                        if (!mbar_wait(bar(BAR_ACCE + bacc), ((u >> 1) & 1) ^ 1, abort_flag, err, 2, limit)) { ok = false; break; }
                        fence_after();
                        dcol = bacc * 2 * ST;
                    }
                    const int s = it % STAGES;
                    if (!mbar_wait(bar(BAR_FULL + s), (it / STAGES) & 1, abort_flag, err, 3, limit)) { ok = false; break; }
                    fence_after();
                    const uint32_t base = smem_u32(stages + s * K::STAGE_BYTES);
#pragma unroll
                    for (int t = 0; t < NTERMS; t++)
                    {
                        const uint64_t ad = sdesc(base + TERM_A[t] * BLK);
                        const uint64_t bd = sdesc(base + (P + TERM_B[t]) * BLK);
                        // hi*hi accumulates in its own TMEM columns; the
                        // smaller correction terms share the next 128.
                        const uint32_t d = tmem + dcol + (t == 0 ? 0 : ST);
                        const bool fresh = (c % KCH == 0) && (t <= 1);
#pragma unroll
                        for (int kk = 0; kk < SK / 16; kk++)
                            mma_bf16(d, ad + 2 * kk, bd + 2 * kk, (fresh && kk == 0) ? 0u : 1u);
                    }
                    mma_commit(bar(BAR_EMPTY + s));
                    if (c % KCH == KCH - 1 || c == nk - 1)
                    {
                        mma_commit(bar(BAR_ACCF + (u & 1)));
                        u++;
                    }
                }
                }
            }
            // Every MMA issued completes before TMEM is freed.
            mma_commit(bar(BAR_DRAIN));
            volatile int never = 0;
            mbar_wait(bar(BAR_DRAIN), 0, &never, nullptr, 0, MBAR_WAIT_LIMIT);
        }
    }
    else
    {
        // Drain warps: thread owns tile row `row` (TMEM lane).
        const int q = warp & 3;
        const int row = q * 32 + lane;
        const int dt = tid - 64;                 // 0..127
        uint32_t u = 0;
        bool ok = true;
        for (int64_t w = blockIdx.x; w < work; w += gridDim.x)
        {
            // Every drain thread takes part in every tile's barrier; a failed
            // wait in any of them ends the loop for all of them here (one
            // that failed in the previous tile skipped the rest of it).
            if (drain_any(!ok)) break;
            int64_t local, b, tm, tn;
            const SplitGemmArgs& a = src.at(w, local);
            decode(a, local, b, tm, tn);
            const int64_t nk = a.nk;
            // Offsets of this tile's rows and columns in each block position
            // of C; every product of the group writes into these.
            for (int h = 0; h < 4; h++)
            {
                const int64_t li = tm * ST + dt, lj = tn * ST + dt;
                const int64_t gi = (int64_t)h * a.ms + li;
                const int64_t gj = (int64_t)h * a.ns + lj;
                rowC[h * ST + dt] = (h < a.H && li < a.ms && gi < a.m) ? a.bC[b] + a.rsC[gi] : OFF_INVALID;
                colC[h * ST + dt] = (h < a.H && lj < a.ns && gj < a.n) ? a.csC[gj] : OFF_INVALID;
            }
            {
                const int64_t pb = a.pbatch > 0 ? a.pbatch : a.batch;
                const int64_t bl = b % pb;
                const int64_t li = tm * ST + dt, lj = tn * ST + dt;
                invr[dt] = li < a.ms ? a.invA[bl * a.ms + li] : 0.f;
                invc[dt] = lj < a.ns ? a.invB[bl * a.ns + lj] : 0.f;
            }
            asm volatile("bar.sync 1, 128;\n" ::: "memory");

            const int64_t nch = (nk + KCH - 1) / KCH;
            for (int p = 0; p < a.nprod && ok; p++)
            {
                float acc[ST];
#pragma unroll
                for (int j = 0; j < ST; j++) acc[j] = 0.f;
                for (int64_t ch = 0; ch < nch; ch++, u++)
                {
                    const int bacc = u & 1;
                    // warp-uniform outcome: the TMEM loads below are warp-collective
                    if (!__all_sync(0xffffffffu, mbar_wait(bar(BAR_ACCF + bacc), (u >> 1) & 1, abort_flag, err, 4,
                                                          limit)))
                    {
                        ok = false;
                        break;
                    }
                    fence_after();
#pragma unroll
                    for (int j = 0; j < ST / 32; j++)
                    {
                        float hh[32], cr[32];
                        const uint32_t ta = tmem + ((uint32_t)(q * 32) << 16) + bacc * 2 * ST + j * 32;
                        tmem_ld32(ta, hh);
                        tmem_ld32(ta + ST, cr);
#pragma unroll
                        for (int i = 0; i < 32; i++) acc[j * 32 + i] += hh[i] + cr[i];
                    }
                    fence_before();
                    mbar_arrive(bar(BAR_ACCE + bacc));
                }
                if (!ok) break;
                // C update in batches of 32 columns: all loads of a batch are
                // issued before any store, so their latencies overlap.
                for (int t = 0; t < a.nc[p]; t++)
                {
                    const int64_t ro = rowC[a.c_r[p][t] * ST + row];
                    if (ro == OFF_INVALID) continue;
                    const int64_t* cc = colC + a.c_c[p][t] * ST;
                    const float coef = (a.c_s[p][t] < 0 ? -a.alpha : a.alpha) * invr[row];
                    const bool first = a.c_first[p][t] != 0;
                    const bool read_c = !first || a.beta != 0.f;
                    const float cb = first ? a.beta : 1.f;
                    float* crow = a.C + ro;
#pragma unroll
                    for (int j0 = 0; j0 < ST; j0 += 32)
                    {
                        float cv[32];
#pragma unroll
                        for (int i = 0; i < 32; i++)
                        {
                            const int64_t co = cc[j0 + i];
                            cv[i] = (read_c && co != OFF_INVALID) ? crow[co] : 0.f;
                        }
#pragma unroll
                        for (int i = 0; i < 32; i++)
                        {
                            const int64_t co = cc[j0 + i];
                            if (co != OFF_INVALID) crow[co] = coef * acc[j0 + i] * invc[j0 + i] + cb * cv[i];
                        }
                    }
                }
            }
        }
    }
    fence_before();
    __syncthreads();
    if (warp == 1)
    {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;\n" :: "r"(tmem) : "memory");
    }
}

template <int P>
__global__ void __launch_bounds__(192, 1)
split_gemm_kernel(const __grid_constant__ SplitGemmArgs a)
{
    extern __shared__ unsigned char smem_raw[];
    split_gemm_body<P>(OneSplit{&a}, a.err, wait_cycles(a.wait_limit), smem_raw);
}

template <int P>
__global__ void __launch_bounds__(192, 1)
split_gemm_grouped_kernel(const __grid_constant__ SplitGroupArgs g)
{
    extern __shared__ unsigned char smem_raw[];
    split_gemm_body<P>(SplitGroup{g}, g.err, wait_cycles(g.wait_limit), smem_raw);
}

template <int P>
cudaError_t launch_split_gemm_p(const SplitGemmArgs& a, cudaStream_t stream, int num_sms)
{
    auto kern = split_gemm_kernel<P>;
    cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SG<P>::smem);
    if (err != cudaSuccess) return err;
    const int64_t work = a.batch * a.tiles_m * a.tiles_n;
    int64_t grid = num_sms;
    if (work < grid) grid = work;
    timing_begin(KK_SPLIT_GEMM, stream);
    kern<<<(unsigned)grid, 192, SG<P>::smem, stream>>>(a);
    timing_end(KK_SPLIT_GEMM, stream);
    return cudaGetLastError();
}

template <int P>
cudaError_t launch_split_grouped_p(const SplitGroupArgs& g, cudaStream_t stream, int num_sms)
{
    auto kern = split_gemm_grouped_kernel<P>;
    cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SG<P>::smem);
    if (err != cudaSuccess) return err;
    int64_t grid = num_sms;
    if (g.total < grid) grid = g.total;
    timing_begin(KK_SPLIT_GEMM, stream);
    kern<<<(unsigned)grid, 192, SG<P>::smem, stream>>>(g);
    timing_end(KK_SPLIT_GEMM, stream);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_split_scale(const SplitScaleArgs& a, cudaStream_t stream)
{
    const int64_t warps = a.batch * a.rows_blk;
    if (warps <= 0) return cudaSuccess;
    const int64_t blocks = (warps * 32 + 255) / 256;
    timing_begin(KK_AUX, stream);
    scale_kernel<<<(unsigned)blocks, 256, 0, stream>>>(a);
    timing_end(KK_AUX, stream);
    cudaError_t err = cudaGetLastError();
    if (err == cudaSuccess) g_launches++;
    return err;
}

cudaError_t launch_split_pack(const SplitPackArgs& a, cudaStream_t stream)
{
    if (a.batch <= 0 || a.tiles <= 0 || a.nk <= 0) return cudaSuccess;
    if (2 * a.tiles > 65535 || a.batch > 65535 || (a.planes != 2 && a.planes != 3)) return cudaErrorInvalidValue;
    if (a.nkpiece < 0 || (a.nkpiece > 0 && a.nk % a.nkpiece)) return cudaErrorInvalidValue;
    dim3 grid((unsigned)a.nk, (unsigned)(2 * a.tiles), (unsigned)a.batch);
    timing_begin(KK_PACK, stream);
    split_pack_kernel<<<grid, 256, 0, stream>>>(a);
    timing_end(KK_PACK, stream);
    cudaError_t err = cudaGetLastError();
    if (err == cudaSuccess) g_launches++;
    return err;
}

cudaError_t launch_split_pack_multi(const SplitPackMultiArgs& a, cudaStream_t stream)
{
    if (a.batch <= 0 || a.tiles <= 0 || a.nk <= 0 || a.nout <= 0) return cudaSuccess;
    if (2 * a.tiles > 65535 || a.batch > 65535 || (a.planes != 2 && a.planes != 3)) return cudaErrorInvalidValue;
    if (a.nt < 1 || a.nt > 2 || a.nout > 7) return cudaErrorInvalidValue;
    dim3 grid((unsigned)a.nk, (unsigned)(2 * a.tiles), (unsigned)a.batch);
    timing_begin(KK_PACK, stream);
    split_pack_multi_kernel<<<grid, 256, 0, stream>>>(a);
    timing_end(KK_PACK, stream);
    cudaError_t err = cudaGetLastError();
    if (err == cudaSuccess) g_launches++;
    return err;
}

// The kernels run the terms hh, hm, mh (+ hl, mm, lh with three planes) in
// this order; a descriptor asking for anything else is rejected.
bool standard_terms(const SplitGemmArgs& a)
{
    static const int8_t TA[6] = {0, 0, 1, 0, 1, 2}, TB[6] = {0, 1, 0, 2, 1, 0};
    if (a.nterms != (a.planes == 3 ? 6 : 3)) return false;
    for (int t = 0; t < a.nterms; t++)
        if (a.ta[t] != TA[t] || a.tb[t] != TB[t]) return false;
    return true;
}

// Products 1..7, block positions 1..4 per dimension, 1..4 targets per
// product, each inside the block grid.
bool split_targets_valid(const SplitGemmArgs& a)
{
    if (a.nprod < 1 || a.nprod > MAX_GROUP_PRODUCTS || a.H < 1 || a.H > 4) return false;
    for (int p = 0; p < a.nprod; p++)
    {
        if (a.nc[p] < 1 || a.nc[p] > 4 || !a.A[p] || !a.B[p]) return false;
        for (int t = 0; t < a.nc[p]; t++)
            if (a.c_r[p][t] < 0 || a.c_r[p][t] >= a.H || a.c_c[p][t] < 0 || a.c_c[p][t] >= a.H) return false;
    }
    return true;
}

cudaError_t launch_split_gemm(const SplitGemmArgs& a, cudaStream_t stream, int num_sms)
{
    if (a.batch <= 0 || a.tiles_m <= 0 || a.tiles_n <= 0 || a.nk <= 0) return cudaSuccess;
    if (!split_targets_valid(a) || !standard_terms(a)) return cudaErrorInvalidValue;
    cudaError_t err = a.planes == 3 ? launch_split_gemm_p<3>(a, stream, num_sms)
                    : a.planes == 2 ? launch_split_gemm_p<2>(a, stream, num_sms)
                                    : cudaErrorInvalidValue;
    if (err == cudaSuccess) g_launches++;
    return err;
}

cudaError_t launch_split_gemm_grouped(const SplitGroupArgs& g, int planes, cudaStream_t stream, int num_sms)
{
    if (g.nprob <= 0 || g.total <= 0) return cudaSuccess;
    cudaError_t err = planes == 3 ? launch_split_grouped_p<3>(g, stream, num_sms)
                    : planes == 2 ? launch_split_grouped_p<2>(g, stream, num_sms)
                                  : cudaErrorInvalidValue;
    if (err == cudaSuccess) g_launches++;
    return err;
}

}  // namespace tsb
