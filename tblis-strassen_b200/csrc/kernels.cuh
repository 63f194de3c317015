// Device-side interfaces shared by the kernels and the host launcher.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace tsb {

// Marks an out-of-range row, column or contracted index in the per-tile
// offset tables: the loader zero-fills it and the epilogue skips it.
constexpr int64_t OFF_INVALID = INT64_MIN;

constexpr int MAX_PRODUCTS = 49;

// One Strassen product on the device: signed sums of up to 4 A blocks
// (row part, k part) and 4 B blocks (k part, col part); the result M is added,
// with sign, into up to 4 C blocks (row part, col part).  c_first marks the
// product that first touches a C block of the tile, where beta is applied.
struct DevProduct
{
    int8_t na, nb, nc, pad;
    int8_t a_r[4], a_c[4], a_s[4];
    int8_t b_r[4], b_c[4], b_s[4];
    int8_t c_r[4], c_c[4], c_s[4], c_first[4];
};

// Arguments of the FP64 Strassen/GEMM kernel.  Element (i, p) of A lives at
// A[bA[b] + rsA[i] + ksA[p]], (p, j) of B at B[bB[b] + ksB[p] + csB[j]] and
// (i, j) of C at C[bC[b] + rsC[i] + csC[j]].  The matrix is cut into an
// H x H grid of blocks of ms x ks (A), ks x ns (B), ms x ns (C); indices past
// m, n, k (the padding of a ragged split) read as zero and are not written.
struct DmmaArgs
{
    const double* A;
    const double* B;
    double* C;
    const int64_t* rsA; const int64_t* ksA;
    const int64_t* ksB; const int64_t* csB;
    const int64_t* rsC; const int64_t* csC;
    const int64_t* bA; const int64_t* bB; const int64_t* bC;
    int64_t m, n, k;        // extents seen by A and B
    int64_t mC, nC;         // extents of the C side (m, n; or ms, ns for an M buffer)
    int64_t ms, ns, ks;     // block extents
    int64_t batch;
    int tiles_m, tiles_n;
    int64_t work;           // batch * tiles_m * tiles_n
    double alpha, beta;
    int a_kfast, b_kfast;   // loader thread mapping: 1 = consecutive threads walk k
    int nprod, H, Hc;       // products; grid parts on the A/B side and the C side
    // Rectangular grids of other fast-multiplication algorithms (fused kernel
    // only): A is H x Hk blocks, B Hk x Hn, C H x Hn; 0 means H.
    int Hk, Hn;
    DevProduct prod[MAX_PRODUCTS];
};

// Grouped launch of the fused kernel: many contractions (one DmmaArgs each,
// with tiles_m, tiles_n and work already set for the chosen configuration)
// in one persistent grid.  prefix[p] = work items before problem p.
struct DmmaGroupArgs
{
    const DmmaArgs* probs;
    const int64_t* prefix;
    int nprob;
    int64_t total;
};

// Elementwise helpers for the AB and Naive variants and for alpha == 0.
struct ScaleArgs
{
    double* C;
    const int64_t* rsC; const int64_t* csC; const int64_t* bC;
    int64_t m, n, batch;
    double beta;
};

struct ScaleF32Args
{
    float* C;
    const int64_t* rsC; const int64_t* csC; const int64_t* bC;
    int64_t m, n, batch;
    float beta;
};

// Dense S = sum_t sign_t * X[block_t]  (rows x cols per batch, row-major) where
// X(i, j) = X[bX[b] + rsX[i] + csX[j]].
struct SumGatherArgs
{
    const double* X;
    const int64_t* rsX; const int64_t* csX; const int64_t* bX;
    int64_t rows_full, cols_full;  // bounds of the full index ranges
    int64_t rows, cols;            // block extents (output is rows x cols)
    int64_t batch;
    int nt;
    int8_t t_r[4], t_c[4], t_s[4];
    double* out;
};

// C[block_q] = (first_q ? beta*C : C) + coef_q * alpha * M for q < nc.
struct ScatterAddArgs
{
    double* C;
    const int64_t* rsC; const int64_t* csC; const int64_t* bC;
    int64_t m, n;                  // full C extents
    int64_t ms, ns;                // block extents (M is ms x ns per batch)
    int64_t batch;
    const double* M;
    double alpha, beta;
    int nc;
    int8_t c_r[4], c_c[4], c_s[4], c_first[4];
};

// Products run side by side into their own M_p (dense ms x ns per batch entry,
// M_p at M + p * m_pstride, column-major when col_major, else row-major), then
// for every C block position h = hr * H + hc:
//   C[h] = alpha * sum_p W[h][p] M_p + beta * C[h]
// where product p adds sign ts[p][t] * M_p into position th[p][t], t < nt[p]
// (sums in FP64, beta * C read only when beta != 0).  Up to 49 products on a
// grid of up to 4 x 4 positions: a level-2 Strassen.  T = double or float.
constexpr int MAX_COMBINE_PRODUCTS = 49;
template <class T>
struct CombineArgsT
{
    T* C;
    const int64_t* rsC; const int64_t* csC; const int64_t* bC;
    int64_t m, n, ms, ns, batch;
    const T* M;
    int64_t m_pstride;
    double alpha, beta;
    int H, col_major, np;
    int8_t nt[MAX_COMBINE_PRODUCTS];
    int8_t th[MAX_COMBINE_PRODUCTS][4], ts[MAX_COMBINE_PRODUCTS][4];
};
using CombineArgs = CombineArgsT<double>;
using CombineF32Args = CombineArgsT<float>;

// ---- packed operands -------------------------------------------------------
//
// A Strassen operand sum (or a plain operand) packed into tile order: for
// batch b, tile t of PACK_TILE rows (A side) or columns (B side) and k in
// [0, k_pad), the PACK_TILE values of that k sit contiguously at
//   out[((b * tiles + t) * k_pad + k) * PACK_TILE + pack_pos(k, r)]
// in exactly the swizzled order the GEMM kernel keeps in shared memory, so a
// pipeline stage is a straight 16-byte-chunk copy.  Rows past the block and k
// past the block are zero.
constexpr int PACK_TILE = 128;
constexpr int PACK_KSTEP = 32;     // k_pad is a multiple of this

struct PackArgs
{
    const double* X;                           // X(i, p) = X[bX[b] + rs[i] + ks[p]]
    const int64_t* rs; const int64_t* ks; const int64_t* bX;
    int64_t rows_full, k_full;                 // bounds of the full index ranges
    int64_t rows_blk, k_blk;                   // block extents
    int nt;                                    // terms of the sum (1..4)
    int8_t t_r[4], t_c[4], t_s[4];             // block row part, k part, sign
    int64_t tiles, k_pad, batch;
    int kfast;                                 // 1: X is contiguous along k
    double* out;
    // 0, or the k length of the pieces of a k-split (a multiple of the pack
    // k-step dividing k_pad): piece p = k / kpiece is written as batch entry
    // p * batch + b of a problem whose k_pad is kpiece.
    int64_t kpiece;
};

// Packed GEMM (S and T packed, PACK_TILE x k_pad tiles): for every 128 x 128 tile position, products q = 0..nprod-1 in
// order: C blocks (c_r, c_c) of product q += c_s * alpha * S_q T_q (beta on
// first touch).  All products share the tile grid and k_pad; a CTA owns a
// tile position across its products, so the C tiles a group of products
// updates stay in L2 between them.
constexpr int MAX_GROUP_PRODUCTS = 7;
struct PackedGemmArgs
{
    const double* S[MAX_GROUP_PRODUCTS];       // packed operand sums, tile order
    const double* T[MAX_GROUP_PRODUCTS];
    double* C;
    const int64_t* rsC; const int64_t* csC; const int64_t* bC;
    int64_t m, n;                              // full C extents
    int64_t ms, ns;                            // block extents
    int64_t k_pad;
    int64_t tiles_m, tiles_n, batch;
    double alpha, beta;
    int nprod;                                 // products per tile position (1..7)
    int H;                                     // block rows of the C grid (1 .. 4)
    int Hn;                                    // block columns of the C grid (0: H)
    int8_t nc[MAX_GROUP_PRODUCTS];             // C blocks per product (1..4)
    int8_t c_r[MAX_GROUP_PRODUCTS][4], c_c[MAX_GROUP_PRODUCTS][4];
    int8_t c_s[MAX_GROUP_PRODUCTS][4], c_first[MAX_GROUP_PRODUCTS][4];
    int* err;                                  // set on a timed-out wait (may be null)
    long long wait_limit;                      // bound on each pipeline wait, SM cycles (0: ~1 s)
};

// Seven packed operand sums in one pass (pack_multi_kernel): the blocks of
// the group's coarse sum are read once; X_j = sum_t sign_t * block(t, j)
// (j = 0..3), output o = sum_i o_s[o][i] * X_{o_j[o][i]}, each written in the
// layout of PackArgs::out.  Block (t, j) sits at packed-row block prow[t][j]
// and k block pk[t][j].
struct PackMultiArgs
{
    const double* X;
    const int64_t* rs; const int64_t* ks; const int64_t* bX;
    int64_t rows_full, k_full;
    int64_t rows_blk, k_blk;
    int nt;                                    // coarse terms (1 or 2)
    int8_t t_s[2];
    int8_t prow[2][4], pk[2][4];
    int nout;                                  // outputs (<= 7)
    int8_t o_n[7], o_j[7][2], o_s[7][2];
    double* out[7];
    int64_t tiles, k_pad, batch;
    int kfast;
};

// Grouped packed GEMM: many problems' tiles in one persistent launch.
struct PackedGroupArgs
{
    const PackedGemmArgs* probs;   // device array [nprob]
    const int64_t* prefix;         // device array [nprob + 1]: work prefix sums
    int nprob;
    int64_t total;
    int* err;                      // set on a timed-out wait (may be null)
    long long wait_limit;          // bound on each pipeline wait, SM cycles (0: ~1 s)
};

// ---- split-BF16 (FP32 contractions on tcgen05) --------------------------------------
//
// Planes: P bf16 planes (hi, mid[, lo]) of a scaled FP32 operand sum, each
// [batch][tiles][nk][128 x 64 block] with blocks in the K-major 128-byte
// swizzled layout; nk = k_pad / 64.
constexpr int SPLIT_TILE = 128;
constexpr int SPLIT_K = 64;

struct SplitScaleArgs
{
    const float* X;                            // X(i, p) = X[bX[b] + rs[i] + ks[p]]
    const int64_t* rs; const int64_t* ks; const int64_t* bX;
    int64_t rows_full, k_full, rows_blk;
    int parts;                                 // row parts of the block grid (H)
    int64_t batch;
    float* scale;                              // [batch][rows_blk] power-of-two multipliers
    float* inv;                                // their inverses
};

struct SplitPackArgs
{
    const float* X;
    const int64_t* rs; const int64_t* ks; const int64_t* bX;
    int64_t rows_full, k_full, rows_blk, k_blk;
    int nt;
    int8_t t_r[4], t_c[4], t_s[4];
    const float* scale;                        // [batch][rows_blk]
    int64_t tiles, nk, batch;
    int planes;                                // 2 (3-term) or 3 (6-term)
    int kfast;
    void* out;                                 // bf16 planes
    // 0, or the k blocks per piece of a k-split (dividing nk): k block c of
    // piece p = c / nkpiece is written as batch entry b of plane set p (plane
    // sets of planes * batch * tiles * nkpiece blocks, one after another).
    int64_t nkpiece;
};

// Seven split sums of one product group in one pass (split_pack_multi_kernel;
// the FP32 counterpart of PackMultiArgs): X_j = sum_t sign_t * block(t, j),
// output o = sum_i o_s[o][i] * X_{o_j[o][i]}, scaled per row and split into
// planes laid out as SplitPackArgs::out.
struct SplitPackMultiArgs
{
    const float* X;
    const int64_t* rs; const int64_t* ks; const int64_t* bX;
    int64_t rows_full, k_full, rows_blk, k_blk;
    int nt;
    int8_t t_s[2];
    int8_t prow[2][4], pk[2][4];
    int nout;
    int8_t o_n[7], o_j[7][2], o_s[7][2];
    const float* scale;                        // [batch][rows_blk]
    int64_t tiles, nk, batch;
    int planes;
    int kfast;
    void* out[7];
};

// Split GEMM: for every 128 x 128 tile position, products q = 0..nprod-1 in
// order (as PackedGemmArgs): C blocks (c_r, c_c) of product q +=
// c_s * alpha * (A_q B_q) / scales, beta on first touch.
struct SplitGemmArgs
{
    const void* A[MAX_GROUP_PRODUCTS];         // bf16 planes of each product's A-side sum
    const void* B[MAX_GROUP_PRODUCTS];         // and B-side sum
    float* C;
    const int64_t* rsC; const int64_t* csC; const int64_t* bC;
    const float* invA;                         // [batch][ms] inverse row scales
    const float* invB;                         // [batch][ns] inverse column scales
    int64_t m, n, ms, ns, nk, tiles_m, tiles_n, batch;
    // Batch entries per plane set (0: batch).  With pbatch < batch, entry
    // b = pp * pbatch + bl reads entry bl of plane set pp, which starts
    // pp * planes * pbatch * tiles * nk blocks after A[q] (B[q]); the row and
    // column scales are those of bl, the C tables those of b.  Products run
    // side by side this way, one plane set each.
    int64_t pbatch;
    float alpha, beta;
    int nprod;                                 // products per tile position (1..7)
    int H;                                     // side of the C block grid (1, 2 or 4)
    int8_t nc[MAX_GROUP_PRODUCTS];
    int8_t c_r[MAX_GROUP_PRODUCTS][4], c_c[MAX_GROUP_PRODUCTS][4];
    int8_t c_s[MAX_GROUP_PRODUCTS][4], c_first[MAX_GROUP_PRODUCTS][4];
    int planes, nterms;
    int8_t ta[6], tb[6];                       // plane pair of each product term
    int* err;                                  // set on a timed-out wait (may be null)
    long long wait_limit;                      // bound on each pipeline wait, SM cycles (0: ~1 s)
};

// Grouped split GEMM: many problems' tiles in one persistent launch (all
// with the same number of planes).
struct SplitGroupArgs
{
    const SplitGemmArgs* probs;    // device array [nprob]
    const int64_t* prefix;         // device array [nprob + 1]: work prefix sums
    int nprob;
    int64_t total;
    int* err;                      // set on a timed-out wait (may be null)
    long long wait_limit;          // bound on each pipeline wait, SM cycles (0: ~1 s)
};

cudaError_t launch_split_scale(const SplitScaleArgs& args, cudaStream_t stream);
cudaError_t launch_split_pack(const SplitPackArgs& args, cudaStream_t stream);
cudaError_t launch_split_pack_multi(const SplitPackMultiArgs& args, cudaStream_t stream);
cudaError_t launch_split_gemm(const SplitGemmArgs& args, cudaStream_t stream, int num_sms);
cudaError_t launch_split_gemm_grouped(const SplitGroupArgs& args, int planes, cudaStream_t stream, int num_sms);

cudaError_t launch_pack(const PackArgs& args, cudaStream_t stream);
cudaError_t launch_pack_multi(const PackMultiArgs& args, cudaStream_t stream);
cudaError_t launch_packed_gemm(const PackedGemmArgs& args, cudaStream_t stream, int num_sms);
cudaError_t launch_packed_gemm_grouped(const PackedGroupArgs& args, cudaStream_t stream, int num_sms);

// Launchers (kernels.cu).  `terms` = largest number of blocks in one sum
// (1, 2 or 4), selecting the kernel instance.  Return a cudaError_t.
// `config` selects a tile configuration (-1: default for `terms`).
cudaError_t launch_dmma(const DmmaArgs& args, int terms, cudaStream_t stream, int num_sms,
                        int config = -1);
// Tile shape (rows x columns per CTA) of the fused-kernel configuration that
// launch_dmma / launch_dmma_grouped pick for these parameters.
void dmma_tile_shape(int terms, int H, int Hc, int config, int* bm, int* bn);
// Fully fused ABC kernel with a producer warpgroup forming the operand sums
// once per staged tile (fused_kernel.cu): C updated directly (Hc == H,
// mC == m, nC == n), H <= 4.  cudaErrorNotSupported when it cannot run
// these arguments (the caller then uses launch_dmma).  `err` (may be null)
// is set when a bounded wait runs out; wait_limit as PackedGemmArgs.  With
// the contraction's plan `g`, the element-pair form (fused_pairs.cu) runs
// where its conditions hold, the gather form elsewhere.
struct GemmView;
cudaError_t launch_fused(const DmmaArgs& args, cudaStream_t stream, int num_sms, int* err, long long wait_limit,
                         const GemmView* g = nullptr);
// The element-pair form alone; cudaErrorNotSupported when its conditions do
// not hold (fused_pairs.cu lists them).
cudaError_t launch_fused_pairs(const DmmaArgs& args, const GemmView& g, cudaStream_t stream, int num_sms, int* err,
                               long long wait_limit);
// Whether the element-pair form applies to a plan cut into an H x Hk (A),
// Hk x Hn (B) grid of blocks of extents ms, ns, ks with ring slots of tb k
// (16 for operand sums of up to 2 blocks, 8 for up to 4; host only).
// `tables` (may be null; PAIRS_PLAN_INTS entries) receives: the bank-conflict
// count of the consumers' reads, the producer (0 tensor-map boxes, 1 16-byte
// pair copies), the tensor-map ranks of A and B (0 for pair copies), 1 when B
// is read in pairs, the swizzle spans of A and B, the pair bits of A and B,
// then the lane offsets aoff[32][2], boff[32][4], sigA[8], sigB[8], the
// unswizzled row positions of the slot's k in A's and B's tiles (16 each,
// the first tb used), the pair bases of A and B in copy order (8 each, the
// first tb / 2 used) and tb.
constexpr int PAIRS_PLAN_INTS = 9 + 64 + 128 + 8 + 8 + 16 + 16 + 8 + 8 + 1;
bool fused_pairs_plan(const GemmView& g, int H, int Hn, int Hk, int64_t ms, int64_t ns, int64_t ks, int tb,
                      int tables[PAIRS_PLAN_INTS]);
cudaError_t launch_dmma_grouped(const DmmaGroupArgs& g, int terms, int H, int Hc, int config,
                                cudaStream_t stream, int num_sms);
cudaError_t launch_scale(const ScaleArgs& args, cudaStream_t stream);
cudaError_t launch_scale_f32(const ScaleF32Args& args, cudaStream_t stream);
cudaError_t launch_sum_gather(const SumGatherArgs& args, cudaStream_t stream);
cudaError_t launch_scatter_add(const ScatterAddArgs& args, cudaStream_t stream);
cudaError_t launch_combine(const CombineArgs& args, cudaStream_t stream);
cudaError_t launch_combine(const CombineF32Args& args, cudaStream_t stream);

// The FP64 tensor-pipe ceiling of this GPU: DMMA throughput of register-only
// m16n8k4 loops over every SM (2 CTAs of 16 warps each), `iters` rounds of 8
// MMAs per warp, timed with CUDA events on `stream` after one warm-up launch.
cudaError_t measure_dmma_peak(int iters, int num_sms, cudaStream_t stream, double* tflops, double* ms);

// Number of kernels this library has launched (all launchers count).
unsigned long long launches();

}  // namespace tsb
