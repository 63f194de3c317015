// Contraction planning: index-bundle analysis of a tblis contraction and its
// reduction to one batched matrix product over scatter vectors.
//
// Behaviour follows the reference's bundle analysis in
// src/iface/3t/mult.cxx:15-146 (identical in src/stra_iface/3t/stra_mult.cxx:26-213):
//   * diagonal(): labels sorted, repeated labels merged by summing strides,
//     extent-1 modes dropped (src/util/tensor.hpp:305-342);
//   * seven label classes ABC, AB, AC, BC, A-only, B-only, C-only
//     (src/iface/3t/mult.cxx:43-86), extents checked equal;
//   * fold(): modes jointly contiguous in every tensor of a class merge
//     (src/util/tensor.hpp:270-303), ordered by the first tensor's stride;
//   * alpha = alpha_A * alpha_B, beta = alpha_C (src/iface/3t/mult.cxx:128-129).
//
// The matrix view is the Block-Scatter-Matrix idea of the reference
// (src/matrix/stra_tensor_view.hpp:427-513, src/matrix/block_scatter_matrix.hpp):
// a row index of the product maps to an element offset through a scatter
// vector.  Where the reference keeps one scatter vector per operand dimension
// and per Strassen sub-block, this plan keeps one per (operand, dimension) over
// the whole flattened bundle; sub-blocks are index ranges into it.
//
// Classes the reference routes through separate code (mult_blas/mult_ref,
// src/internal/3t/mult.cxx:313-473) fold into the same product here:
//   * ABC (batch) and C-only labels become batch modes (A/B stride 0 on C-only:
//     the product is broadcast into every C-only position);
//   * A-only and B-only labels become extra contracted modes with stride 0 in
//     the other operand (a sum over them factorises: sum_a' A * sum_b' B).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "tblis_stra_b200.h"

namespace tsb {

// One class of labels after diagonal() and fold(): extents, labels and, for
// each tensor the class appears in, the strides (same order).
struct Bundle
{
    std::vector<int64_t> len;
    std::vector<label_type> idx;
    std::vector<std::vector<int64_t>> stride;   // one vector per tensor
};

// A batched matrix product  C[b](i,j) = alpha * sum_p A[b](i,p) B[b](p,j) + beta * C[b](i,j)
// with every element addressed as base + row-scatter + col-scatter + batch-scatter.
struct GemmView
{
    int type = TYPE_DOUBLE;
    double alpha = 1.0, beta = 0.0;
    int64_t m = 1, n = 1, k = 1, batch = 1;
    std::vector<int64_t> rsA, rsC;     // length m
    std::vector<int64_t> csB, csC;     // length n
    std::vector<int64_t> ksA, ksB;     // length k
    std::vector<int64_t> bA, bB, bC;   // length batch
    // Stride of the fastest mode of each scatter vector (0 when the bundle is
    // empty), used to choose the loader's thread mapping for coalescing.
    int64_t unit_rsA = 0, unit_ksA = 0, unit_ksB = 0, unit_csB = 0, unit_rsC = 0, unit_csC = 0;
    // Offset span touched in each tensor (elements), for host staging.
    int64_t lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    // The mixed-radix form of the nine scatter vectors, in the order rsA,
    // rsC, csB, csC, ksA, ksB, bA, bB, bC: entry i of vector v is
    // sum_d digit_d(i) * stride[d] with digits of i over len (first mode
    // fastest).  Filled whether or not the vectors themselves are built.
    std::vector<int64_t> mode_len[9], mode_stride[9];
    // Bundles after folding, kept for diagnostics and tests.
    Bundle ABC, AB, AC, BC, A_only, B_only, C_only;
};

// Returns a TBLIS_STRA_* status.  On success `out` describes the product.
int plan_contraction(const tblis_tensor* A, const label_type* idx_A,
                     const tblis_tensor* B, const label_type* idx_B,
                     const tblis_tensor* C, const label_type* idx_C,
                     GemmView& out, bool build_scatter = true);

// Offset span [lo, hi] (elements) covered by a tensor with these extents and
// strides; an empty tensor gives lo = 0, hi = -1.
void tensor_span(unsigned ndim, const len_type* len, const stride_type* stride,
                 int64_t& lo, int64_t& hi);

// ---- Strassen product tables --------------------------------------------

// One term of a signed sum of sub-blocks: block (r, c) of an H x H grid.
struct Term { int8_t r, c, sign; };

struct Product
{
    int8_t na = 0, nb = 0, nc = 0;
    Term a[4], b[4], c[4];
    int8_t c_first[4] = {0, 0, 0, 0};   // 1 when this product is the first to touch that C block
};

struct ProductTable
{
    int level = 0;
    int H = 1;            // block rows of A and C (2^level for Strassen)
    int Hk = 1, Hn = 1;   // block columns of A (= rows of B) and of B and C
    int algorithm = 0;    // registry id of the fast-multiplication algorithm
    std::vector<Product> prod;
};

// A fast matrix-multiplication algorithm <mb, kb, nb; rank>: on an mb x kb
// block grid of A, kb x nb of B and mb x nb of C, product r is
//   M_r = (sum_i U[i][r] A_i) (sum_j V[j][r] B_j),   C_q += W[q][r] M_r,
// block id = row * (grid columns) + column, coefficient matrices row-major
// (rows = block ids, columns = products), the layout of the reference's
// coefficient files (src/stra_internal/3t/strassen:1-14; the generator
// src/stra_internal/3m/my_stra_gen.py takes the same U/V/W for other shapes).
struct FmmAlgorithm
{
    std::string name;
    int mb = 2, kb = 2, nb = 2, rank = 7;
    std::vector<int> U, V, W;
};

// Built-in algorithms: 0 Strassen <2,2,2;7>; 1 the classical <2,2,2;8>;
// 2-4 Strassen beside the classical product on the third block row, column
// or summed slice: <3,2,2;11>, <2,3,2;11>, <2,2,3;11>.  register_algorithm
// adds more (checked: the coefficients must multiply matrices exactly) and
// returns the new id, or a negative TBLIS_STRA_* status.
constexpr int FMM_BUILTIN = 5;
int register_algorithm(const FmmAlgorithm& a);
const FmmAlgorithm* algorithm_by_id(int id);
// The product table of algorithm `id` at `level` (its Kronecker power), or
// nullptr when the kernels cannot run it: block grid beyond 4 x 4, more than
// 49 products, or a sum or C update of more than 4 blocks.
const ProductTable* fmm_table(int id, int level);

// The calling thread's algorithm (tblis_stra_set_algorithm); product_table()
// below serves it at every level >= 1.
void set_thread_algorithm(int id);
int thread_algorithm();

// 〈2,2,2〉 Strassen coefficients (U for A, V for B, W for C; rows = sub-block
// id 0..3 = (id/2, id%2), columns = products), as listed in
// src/stra_internal/3t/strassen:1-14, and their Kronecker square for level 2
// (the 49-product grid of src/stra_internal/3t/stra_mult_2level.cxx:341-1485);
// at level >= 1 with another algorithm selected on the calling thread, that
// algorithm's table (callers check fmm_table() first).
const ProductTable& product_table(int level);
const ProductTable& strassen_table(int level);

// The operand sums of 7 consecutive products (all of L=1, or products
// 7G .. 7G+6 of L=2) in factored form, so one pass over the operand forms all
// seven: X_j = sum_t sign_t * block(row[t][j/2], col[t][j%2]) for the 4
// sub-blocks j of the group's coarse sum, and sum q = sum_i s[q][i] * X_{j[q][i]}.
// Blocks are positions in the H x H grid of the operand as the product table
// addresses it (A: (m-block, k-block); B: (k-block, n-block)).  Expanding
// reproduces product_table(level)'s terms exactly (checked when built).
struct PackGroup
{
    int nt = 0;                  // coarse terms (1 or 2)
    int8_t t_s[2] = {0, 0};
    int8_t row[2][2] = {}, col[2][2] = {};
    int8_t o_n[7] = {}, o_j[7][2] = {}, o_s[7][2] = {};
};
// operand 0 = A, 1 = B; group in [0, 7^(level-1)); nullptr if level is 0 or
// the factored form failed its check against the product table.
const PackGroup* pack_group(int level, int operand, int group);

}  // namespace tsb
