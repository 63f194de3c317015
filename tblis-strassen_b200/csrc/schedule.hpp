// Host-side schedules shared by the single-call entry points (capi.cpp) and
// the batched plans (batch.cpp).  Scatter-vector tables are passed as nine
// device pointers in the order rsA, rsC, csB, csC, ksA, ksB, bA, bB, bC.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <string>

#include "kernels.cuh"
#include "plan.hpp"

namespace tsb {

// The failing CUDA call behind the last TBLIS_STRA_ERR_CUDA of this thread
// (tblis_stra_last_error_detail); note_cuda_error also clears the runtime's
// last-error state.
void note_cuda_error(const char* what, cudaError_t e, const char* file, int line);
void note_detail(const std::string& what);
void clear_detail();

// The calling thread's bound on the pipeline waits of the warp-specialised
// kernels, in SM clock cycles (tblis_stra_set_wait_limit; 0 = the default).
long long wait_limit_cycles();
// The calling thread's ceiling on one device allocation (tblis_stra_set_alloc_limit).
size_t alloc_limit_bytes();

// Host -> device copy complete on return (see capi.cpp).
int upload_complete(void* dst, const void* src, size_t bytes);

// Block and tile geometry of the packed FP64 schedule at one Strassen level.
struct PackGeom
{
    int64_t ms, ns, ks;     // block extents (ceil(m / 2^L) ...)
    int64_t k_pad;          // ks rounded up to the pack k-step
    int64_t tm, tn;         // 128-row tiles of S and T per batch entry
    size_t s_elems, t_elems;
    bool fits;              // pack grid limits hold
};
PackGeom pack_geom(int level, const GemmView& g);

// Bytes of S + T for the packed schedule one product at a time, and for
// the grouped-sum form (L >= 1: the 7 sums of a product group formed in one
// pass, 7 S and 7 T held at once).  run_fp64_packed_enqueue uses the grouped
// form whenever ws_bytes allows it.
size_t fp64_packed_workspace_bytes(int level, const GemmView& g);
size_t fp64_packed_group_workspace_bytes(int level, const GemmView& g);

// Pack product `pr`'s operand sums into S and T (two launches).
int enqueue_pack_product(const Product& pr, const GemmView& g, const PackGeom& pg,
                         const int64_t* const tb[9], const double* A, const double* B,
                         double* S, double* T, cudaStream_t st);

// Descriptor of a packed GEMM over C at `level` with no products yet, and
// appending a product (its operand sums S, T and C blocks; up to 7, run in
// the order added); `err` (device int, may be null) records a timed-out wait.
PackedGemmArgs packed_gemm_base(int level, const GemmView& g, const PackGeom& pg, const int64_t* const tb[9],
                                double* C, int* err);
void packed_gemm_add(PackedGemmArgs& a, const Product& pr, const double* S, const double* T);
// Both for one product.
PackedGemmArgs packed_product_args(int level, const Product& pr, const GemmView& g, const PackGeom& pg,
                                   const int64_t* const tb[9], const double* S, const double* T,
                                   double* C, int* err);

// Whole packed ABC schedule of one FP64 contraction on caller workspace.
int run_fp64_packed_enqueue(int level, const GemmView& g, const int64_t* const tb[9],
                            const double* A, const double* B, double* C, cudaStream_t st, int sms,
                            void* ws, size_t ws_bytes, int* err);

// Product-parallel ABC schedule (L >= 1) on caller workspace: every
// product's sums packed (S_p, T_p), one GEMM launch over all 7^L products
// into M_p (dense ms x ns per batch entry), then one combine launch forming
// each C block from the M_p.  mtab: the M_p row, column and batch tables
// (dense_m_tables); col_major: M's layout.
size_t fp64_parallel_workspace_bytes(int level, const GemmView& g);
int run_fp64_parallel_enqueue(int level, const GemmView& g, const int64_t* const tb[9],
                              const double* A, const double* B, double* C, cudaStream_t st, int sms,
                              void* ws, size_t ws_bytes, const int64_t* mtab, bool col_major, int* err);
// Its second half alone, once the products' sums are packed in ws (S_p at
// ws + p * s_elems doubles, then T_p).
int enqueue_products_and_combine(int level, const GemmView& g, const int64_t* const tb[9], double* C,
                                 cudaStream_t st, int sms, void* ws, const int64_t* mtab, bool col_major,
                                 int* err);
// k-split plain contraction (L = 0): the number of pieces for a grid of
// fewer C tiles than SMs (1: no split), its workspace, and the schedule (P
// packed piece pairs, one GEMM over them into M_p, one combine launch; M
// tables for m x n with P * batch entries).
int ksplit_pieces(const GemmView& g, int sms);
size_t fp64_ksplit_workspace_bytes(const GemmView& g, int P);
int run_fp64_ksplit_enqueue(const GemmView& g, const int64_t* const tb[9], const double* A, const double* B,
                            double* C, cudaStream_t st, int sms, void* ws, size_t ws_bytes, int P,
                            const int64_t* mtab, bool col_major, int* err);
// Host copy of those tables: rows[ms], cols[ns], batch[nb].
void dense_m_tables(int64_t ms, int64_t ns, int64_t nb, bool col_major, int64_t* out);
// M's layout for C's layout: column-major when C's row bundle is the faster.
bool m_tables_col_major(const GemmView& g);
// Whether a contraction at `level` runs product-parallel: the automatic rule
// (L = 2 always; L = 1 when one product's last wave of tiles leaves more than
// a tenth of the SMs idle), the calling thread's setting
// (tblis_stra_set_product_parallel) and its workspace limit.
bool use_product_parallel(int level, const GemmView& g, int sms, bool fp32, int terms);

// Split-BF16 schedule of one FP32 contraction on caller workspace.
size_t fp32_workspace_bytes(int level, const GemmView& g, int terms);
// The same with the 7 split sums of a product group held at once (L >= 1);
// run_fp32_enqueue forms them in one pass whenever ws_bytes allows it.
size_t fp32_group_workspace_bytes(int level, const GemmView& g, int terms);
// Product-parallel split-BF16 schedule (L >= 1; M tables as for FP64).
size_t fp32_parallel_workspace_bytes(int level, const GemmView& g, int terms);
int run_fp32_parallel_enqueue(int level, const GemmView& g, const int64_t* const tb[9], const float* A,
                              const float* B, float* C, cudaStream_t st, int sms, void* ws, size_t ws_bytes,
                              int terms, const int64_t* mtab, bool col_major, int* err);
// With `defer` (L = 0 only) the GEMM is not launched: its descriptor is
// returned for a grouped launch; with enqueue == false nothing is launched at
// all (the descriptor alone, for a plan built before capture).
int run_fp32_enqueue(int level, const GemmView& g, const int64_t* const tb[9], const float* A,
                     const float* B, float* C, cudaStream_t st, int sms, void* ws, size_t ws_bytes,
                     int terms, int* err, SplitGemmArgs* defer = nullptr, bool enqueue = true);

}  // namespace tsb
