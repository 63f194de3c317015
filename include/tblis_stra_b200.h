/*
 * tblis_stra_b200.h -- C ABI of the B200 (sm_100a) Strassen tensor-contraction
 * library.  Drop-in for the contraction entry points of tblis-strassen:
 *
 *     C(idx_C) = alpha * A(idx_A) * B(idx_B) + beta * C(idx_C)
 *
 * with alpha = A->scalar * B->scalar and beta = C->scalar, exactly as the
 * reference reads them (src/iface/3t/mult.cxx:128-129).  Every index label of
 * a tensor names one mode; a label shared by A and B only is contracted, a
 * label shared by A (or B) and C is a free row (column) index, a label in all
 * three is a batch index, and a label in one tensor only is summed (A, B) or
 * broadcast (C).  Repeated labels inside one tensor take the diagonal.
 *
 * Data pointers may be device memory (the fast path: stream-ordered, no
 * copies) or host memory (the library stages through device memory and copies
 * C back; the call is then synchronous).  The three drop-in symbols keep the
 * reference's blocking `void` semantics and record a status readable through
 * tblis_stra_last_status(); tblis_stra_mult() returns the status directly and
 * is asynchronous on device pointers.
 *
 * FP64 (TYPE_DOUBLE) runs on the FP64 tensor cores (DMMA); FP32 (TYPE_FLOAT)
 * runs the split-BF16 tcgen05 path (tblis_stra_set_fp32_terms).  Complex types
 * return TBLIS_STRA_ERR_TYPE.
 */
#ifndef TBLIS_STRA_B200_H
#define TBLIS_STRA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- types (layout-compatible with the reference) ----------------------- */

/* Replaces src/util/basic_types.h:61-63 (configure defaults ptrdiff_t,
 * ptrdiff_t, char; configure.ac:77-110). */
typedef ptrdiff_t len_type;
typedef ptrdiff_t stride_type;
typedef char label_type;

/* Replaces src/util/basic_types.h:52-59. */
typedef enum
{
    TYPE_SINGLE   = 0,
    TYPE_FLOAT    = TYPE_SINGLE,
    TYPE_DOUBLE   = 1,
    TYPE_SCOMPLEX = 2,
    TYPE_DCOMPLEX = 3
} type_t;

/* Replaces src/util/basic_types.h:341-419 (same field order, sizes and
 * alignment).  Strides are in elements and may be negative. */
typedef struct tblis_tensor
{
    type_t type;
    int conj;
    char scalar[16] __attribute__((__aligned__(8)));
    void* data;
    unsigned ndim;
    len_type* len;
    stride_type* stride;
} tblis_tensor;

/* Opaque in this library.  The reference's tblis_comm is a TCI thread
 * communicator (src/util/thread.h:7) and tblis_config a CPU kernel table
 * (src/util/basic_types.h:37); both select CPU threading, which the GPU grid
 * replaces, so any value (NULL included) is accepted and ignored. */
typedef struct tci_comm tblis_comm;
typedef struct tblis_config_s tblis_config;

/* Replaces src/util/thread.h:8.  A non-null sentinel; passing it is the same
 * as passing NULL. */
extern const tblis_comm* const tblis_single;

/* ---- drop-in contraction entry points ----------------------------------- */

/* Plain (L=0) contraction.  Replaces tblis_tensor_mult,
 * src/iface/3t/mult.h:17-20 / src/iface/3t/mult.cxx:15. */
void tblis_tensor_mult(const tblis_comm* comm, const tblis_config* cfg,
                       const tblis_tensor* A, const label_type* idx_A,
                       const tblis_tensor* B, const label_type* idx_B,
                             tblis_tensor* C, const label_type* idx_C);

/* One-level Strassen (7 products).  Replaces stra_tblis_tensor_mult,
 * src/stra_iface/3t/stra_mult.h:17-20 / src/stra_iface/3t/stra_mult.cxx:26. */
void stra_tblis_tensor_mult(const tblis_comm* comm, const tblis_config* cfg,
                            const tblis_tensor* A, const label_type* idx_A,
                            const tblis_tensor* B, const label_type* idx_B,
                                  tblis_tensor* C, const label_type* idx_C);

/* Two-level Strassen (49 products).  Replaces stra_tblis_tensor_mult_2level,
 * src/stra_iface/3t/stra_mult_2level.h:17-20 /
 * src/stra_iface/3t/stra_mult_2level.cxx:26. */
void stra_tblis_tensor_mult_2level(const tblis_comm* comm, const tblis_config* cfg,
                                   const tblis_tensor* A, const label_type* idx_A,
                                   const tblis_tensor* B, const label_type* idx_B,
                                         tblis_tensor* C, const label_type* idx_C);

/* ---- matrix-level entry points ---------------------------------------------
 *
 * Replaces src/util/basic_types.h:264-272 (same field order, sizes and
 * alignment): an m x n matrix with row stride rs and column stride cs, in
 * elements.  C = alpha*A*B + beta*C with alpha = A.scalar*B.scalar and
 * beta = C.scalar; afterwards C.scalar = 1 (as for tensors). */
typedef struct tblis_matrix
{
    type_t type;
    int conj;
    char scalar[16] __attribute__((__aligned__(8)));
    void* data;
    len_type m, n;
    stride_type rs, cs;
} tblis_matrix;

/* L=0: src/iface/3m/mult.h:17-19. */
void tblis_matrix_mult(const tblis_comm* comm, const tblis_config* cfg,
                       const tblis_matrix* A, const tblis_matrix* B, tblis_matrix* C);
/* L=1, variants ABC / Naive / AB: src/stra_iface/3m/stra_mult.h:17-27. */
void stra_tblis_matrix_mult(const tblis_comm* comm, const tblis_config* cfg,
                            const tblis_matrix* A, const tblis_matrix* B, tblis_matrix* C);
void stra_tblis_matrix_mult_naive(const tblis_comm* comm, const tblis_config* cfg,
                                  const tblis_matrix* A, const tblis_matrix* B, tblis_matrix* C);
void stra_tblis_matrix_mult_ab(const tblis_comm* comm, const tblis_config* cfg,
                               const tblis_matrix* A, const tblis_matrix* B, tblis_matrix* C);
/* L=2, variants ABC / Naive / AB: src/stra_iface/3m/stra_mult_2level.h:17-27. */
void stra_tblis_matrix_mult_2level(const tblis_comm* comm, const tblis_config* cfg,
                                   const tblis_matrix* A, const tblis_matrix* B, tblis_matrix* C);
void stra_tblis_matrix_mult_2level_naive(const tblis_comm* comm, const tblis_config* cfg,
                                         const tblis_matrix* A, const tblis_matrix* B, tblis_matrix* C);
void stra_tblis_matrix_mult_2level_ab(const tblis_comm* comm, const tblis_config* cfg,
                                      const tblis_matrix* A, const tblis_matrix* B, tblis_matrix* C);

/* Thread-count knobs of the reference (src/util/thread.h:13-15).  The GPU
 * grid replaces CPU threads: the value is stored and reported, never used. */
unsigned tblis_get_num_threads(void);
void tblis_set_num_threads(unsigned num_threads);

/* ---- status-returning / stream-ordered entry point ---------------------- */

enum
{
    TBLIS_STRA_SUCCESS          = 0,
    TBLIS_STRA_ERR_NULL         = 1,  /* null tensor, label or len/stride pointer */
    TBLIS_STRA_ERR_TYPE         = 2,  /* type mismatch or unsupported element type */
    TBLIS_STRA_ERR_EXTENT       = 3,  /* one label with different extents */
    TBLIS_STRA_ERR_CONJ         = 4,  /* conj != 0 (real types only) */
    TBLIS_STRA_ERR_ARG          = 5,  /* bad level, impl, ndim or negative extent */
    TBLIS_STRA_ERR_CUDA         = 6,  /* a CUDA runtime call failed */
    TBLIS_STRA_ERR_ALLOC        = 7,  /* device workspace could not be allocated */
    TBLIS_STRA_ERR_TOO_LARGE    = 8,  /* sizes beyond what the kernels index */
    TBLIS_STRA_ERR_UNSUPPORTED  = 9,  /* valid request this build does not run */
    TBLIS_STRA_ERR_NO_DEVICE    = 10, /* no usable sm_100 device */
    TBLIS_STRA_ERR_TIMEOUT      = 11  /* a kernel's bounded wait expired (reported on blocking calls) */
};

/* C(idx_C) = alpha*A*B + beta*C at Strassen level 0, 1 or 2 with the current
 * variant (tblis_stra_set_impl).  `stream` is a cudaStream_t (NULL = the
 * calling thread's stream from tblis_stra_set_stream, default the legacy
 * stream).  With device pointers the call only enqueues work; with any host
 * pointer it stages, computes and copies back before returning.  Replaces the
 * three drop-in symbols above when the caller wants a status code: the
 * reference returns void and aborts only in debug builds
 * (src/util/assert.h:17-44). */
int tblis_stra_mult(int level,
                    const tblis_tensor* A, const label_type* idx_A,
                    const tblis_tensor* B, const label_type* idx_B,
                          tblis_tensor* C, const label_type* idx_C,
                    void* stream);

/* Strassen variant: 1 = ABC (sums fused into the loads, +-M fused into the
 * epilogue, no workspace), 2 = AB (one M buffer, then a scatter-add pass),
 * 3 = Naive (explicit S, T, M buffers).  Replaces the process-global
 * tblis::internal::impl (src/internal/3t/mult.hpp:14-15) set by
 * test/test_strassen.cxx:230-243; here it is per calling thread.  Level 0
 * ignores it, as test/test_strassen.cxx:466-468 forces impl=1 there.
 * Returns 0 or TBLIS_STRA_ERR_ARG. */
int tblis_stra_set_impl(int impl);
int tblis_stra_get_impl(void);

/* Device workspace (bytes) the ABC variant may use, per calling thread
 * (default: unlimited).  Within the limit ABC packs the signed sums of each
 * Strassen product into tile-ordered buffers (the reference's pack buffers,
 * stra_pack_{two,four}_*, src/kernels/3m/gemm.hpp:504-816) and fuses the
 * +-M update into the GEMM epilogue; with a limit below the needed
 * 8*batch*(ceil(ms/128)+ceil(ns/128))*128*kpad bytes (0 included) it runs the
 * fully fused kernel, which forms the sums inside the GEMM and allocates
 * nothing beyond the scatter vectors. */
int tblis_stra_set_workspace_limit(size_t bytes);
size_t tblis_stra_get_workspace_limit(void);

/* Product-parallel schedule (no counterpart in the reference, whose threads
 * split each product's loops instead).  At L >= 1, when the last wave of one
 * product's 128 x 128 tiles would leave more than a tenth of the SMs' time
 * idle (fewer tiles than SMs included), ABC packs every product's sums, runs
 * all 7^L products side by side in one GEMM launch into their own M_p, and
 * forms each C block as alpha * sum_p W[h][p] M_p + beta * C in one pass;
 * FP32 takes this form on its split-BF16 path at every L >= 1.  It needs 7^L * (packed sums +
 * batch*ms*ns elements of M) bytes within the workspace limit.  AB and Naive
 * (which hold M temporaries by design) always take this form when mode is
 * not 0.  At L = 0 with fewer C tiles than SMs and at least 1024 summed
 * indices, the same machinery cuts the summed range into up to 49 pieces
 * (k-split) run side by side and summed by the combine pass.  mode: -1 automatic (the default), 0 never, 1 whenever the
 * workspace fits.  Per calling thread.  Returns 0 or TBLIS_STRA_ERR_ARG. */
int tblis_stra_set_product_parallel(int mode);
int tblis_stra_get_product_parallel(void);

/* Fast matrix-multiplication algorithm of the Strassen levels, per calling
 * thread (default 0).  The reference generates its product code from U/V/W
 * coefficient files for any <m,k,n> shape (src/stra_internal/3t/strassen:1-14,
 * src/stra_internal/3m/my_stra_gen.py, my_stra_gen.sh names a <3,2,3> family);
 * here the same coefficients drive the kernels at run time.  Built-in ids:
 *   0  Strassen <2,2,2> with 7 products (levels 1 and 2);
 *   1  the classical <2,2,2> with 8 products;
 *   2  <3,2,2>, 3  <2,3,2>, 4  <2,2,3>: Strassen on the leading 2 x 2 x 2
 *      blocks plus the 4 classical products of the third block row, summed
 *      slice or column (11 products for 12 classical).
 * Level L applies the algorithm's L-th Kronecker power: an mb^L x kb^L block
 * grid of A, kb^L x nb^L of B, mb^L x nb^L of C, rank^L products (the kernels
 * take grids up to 4 x 4 and up to 49 products; tblis_stra_algorithm_info
 * reports the levels an algorithm runs at).  Other algorithms than 0 run
 * FP64 contractions with the ABC variant; AB, Naive and FP32 calls return
 * TBLIS_STRA_ERR_UNSUPPORTED, and batches always use Strassen.  Returns 0 or
 * TBLIS_STRA_ERR_ARG (unknown id). */
int tblis_stra_set_algorithm(int id);
int tblis_stra_get_algorithm(void);
/* Shape <mb, kb, nb>, rank and the highest level (0 .. 2) the kernels run
 * algorithm `id` at. */
int tblis_stra_algorithm_info(int id, int* mb, int* kb, int* nb, int* rank, int* levels);
/* Adds an algorithm given by its coefficient matrices, row-major with one row
 * per block id (row * grid columns + column) and one column per product:
 * U is (mb*kb) x rank, V (kb*nb) x rank, W (mb*nb) x rank, entries in
 * {-1, 0, 1} -- the layout of the reference's coefficient files.  The
 * coefficients are checked to multiply matrices exactly (else
 * TBLIS_STRA_ERR_ARG); TBLIS_STRA_ERR_UNSUPPORTED when the kernels cannot run
 * even one level of it (a sum or C update of more than 4 blocks).  On
 * success *id is the new algorithm's id (process-wide, at most 64). */
int tblis_stra_register_algorithm(int mb, int kb, int nb, int rank, const int* U, const int* V, const int* W,
                                  int* id);

/* FP32 (TYPE_FLOAT) contractions run on the BF16 tensor cores with each
 * operand split into bf16 planes (no counterpart in the reference, whose FP32
 * path is its CPU micro-kernel): terms = 6 splits into hi+mid+lo and keeps the
 * products hh, hm, mh, hl, mm, lh (about FP32 accuracy); terms = 3 splits into
 * hi+mid and keeps hh, hm, mh (twice as fast, about 2^-16 relative).  Per
 * calling thread; default 6.  Returns 0 or TBLIS_STRA_ERR_ARG. */
int tblis_stra_set_fp32_terms(int terms);
int tblis_stra_get_fp32_terms(void);

/* Bound, in SM clock cycles, on each wait of the warp-specialised kernels
 * (the packed FP64 GEMM, the fused no-workspace kernels and the split-BF16
 * tcgen05 GEMM) for a copy, an MMA
 * stage or a drained accumulator; 0 (the default) means about one second.
 * When a wait runs out, the kernel stops issuing work, lets its own copies
 * and MMAs land, frees its tensor memory and ends; blocking calls then return
 * TBLIS_STRA_ERR_TIMEOUT and the device stays usable.  No counterpart in the
 * reference (its CPU threads cannot stall on an asynchronous copy).  Per
 * calling thread, read when a call (or a batch's create) enqueues its
 * kernels.  Returns 0 or TBLIS_STRA_ERR_ARG (negative cycles). */
int tblis_stra_set_wait_limit(long long cycles);
long long tblis_stra_get_wait_limit(void);
/* Failure test hook (no counterpart in the reference): with injection on, the
 * calling thread's next calls make every pipeline wait of those kernels
 * behave as a wait on a flag that nothing sets -- it runs out after the wait
 * bound (tblis_stra_set_wait_limit, or 1000 cycles when that is 0) whatever
 * the state of its copy or MMA, and the kernel takes its timeout path as
 * above (blocking calls return TBLIS_STRA_ERR_TIMEOUT).  The waits with which
 * a kernel lets its own copies and MMAs land before it ends are not
 * affected.  Off by default; returns 0. */
int tblis_stra_set_wait_injection(int on);
int tblis_stra_get_wait_injection(void);

/* Largest single device allocation (bytes) a call of the calling thread may
 * make for its scatter-vector tables, workspace, staging buffers and flags
 * (default: unlimited).  A request above it fails as an out-of-memory
 * allocation would: the call returns TBLIS_STRA_ERR_ALLOC and leaves C
 * untouched.  Unlike tblis_stra_set_workspace_limit, which makes ABC fall
 * back to schedules that need less, this is a hard ceiling.  No counterpart in
 * the reference (its host pools grow on demand). */
int tblis_stra_set_alloc_limit(size_t bytes);
size_t tblis_stra_get_alloc_limit(void);

/* Status of the calling thread's last contraction call; string form. */
int tblis_stra_last_status(void);
const char* tblis_stra_status_string(int status);
/* The CUDA call (file:line, expression, error name) behind this thread's
 * last TBLIS_STRA_ERR_CUDA, or "" (valid until the thread's next call). */
const char* tblis_stra_last_error_detail(void);

/* The calling thread's default stream (a cudaStream_t; NULL = legacy). */
int tblis_stra_set_stream(void* stream);
void* tblis_stra_get_stream(void);

/* Number of this library's kernels launched in this process so far. */
unsigned long long tblis_stra_launch_count(void);

/* Planning introspection; needs no GPU.  Runs the bundle analysis of a
 * contraction (diagonal, label classes, fold; src/iface/3t/mult.cxx:21-126)
 * and reports the batched matrix product it reduces to:
 *   sizes[0..3] = m, n, k, batch;  ab[0..1] = alpha, beta;
 * and, for each non-NULL array, the element-offset scatter vectors
 *   rsA, rsC (length m), csB, csC (n), ksA, ksB (k), bA, bB, bC (batch),
 * so that C[bC[b]+rsC[i]+csC[j]] = alpha * sum_p A[bA[b]+rsA[i]+ksA[p]] *
 * B[bB[b]+ksB[p]+csB[j]] + beta * C[...].  This plays the role of the
 * reference's matrify step (src/stra_nodes/stra_matrify.hpp:82-300).
 * Returns a TBLIS_STRA_* status. */
int tblis_stra_plan_query(const tblis_tensor* A, const label_type* idx_A,
                          const tblis_tensor* B, const label_type* idx_B,
                          const tblis_tensor* C, const label_type* idx_C,
                          int64_t* sizes, double* ab,
                          int64_t* rsA, int64_t* rsC, int64_t* csB, int64_t* csC,
                          int64_t* ksA, int64_t* ksB,
                          int64_t* bA, int64_t* bB, int64_t* bC);

/* Which no-workspace ABC kernel a contraction at Strassen level `level` gets
 * (host only; no counterpart in the reference).  *pairs = 1 when the
 * element-pair form applies: the unit-stride mode of A and of B is a
 * contracted mode, so the kernel stages tiles as contiguous 16-byte pairs (by
 * cp.async, or by tensor-map copies where the tiles are boxes) in a layout
 * whose DMMA fragment reads are conflict-free; 0 when it gathers tiles
 * element by element through the scatter vectors.  Levels 0 and 1 (operand
 * sums of up to 2 blocks) stage 16 k per ring slot, level 2 (up to 4 blocks)
 * 8 k.  `tables` (may be NULL; 266 ints) receives the plan: the
 * bank-conflict count of the consumers' reads (0 = none), the producer (1
 * pair copies, 0 tensor maps), the tensor-map ranks of A and B, 1 when B is
 * read in 16-byte pairs, the swizzle spans of A and B (bytes, 0 = none), the
 * slot k bit each pair spans in A and B, the per-lane read offsets
 * aoff[32][2] and boff[32][4] (doubles; the first tb/8 and tb/4 used), the
 * fragment row and column permutations sigA[8] and sigB[8], the unswizzled
 * row positions of the slot's k in A's and B's tiles (16 each, the first tb
 * used), the pair bases of A and of B in copy order (8 each, the first tb/2
 * used), and tb, the k per slot (16 or 8). */
int tblis_stra_fused_pairs_query(int level, const tblis_tensor* A, const label_type* idx_A,
                                 const tblis_tensor* B, const label_type* idx_B,
                                 const tblis_tensor* C, const label_type* idx_C, int* pairs, int* tables);

/* Contraction that allocates no device memory (no counterpart in the
 * reference, which allocates host workspace freely).  For callers that cannot
 * call cudaMalloc: an application whose own pool has reserved the whole
 * device, a host that forbids plug-ins from allocating device memory, or code
 * that cannot afford cudaMalloc/cudaFree's implicit device synchronisation.
 * Same arguments as tblis_stra_mult, with these limits: FP64 (TYPE_DOUBLE)
 * operands only (TBLIS_STRA_ERR_UNSUPPORTED otherwise); always the ABC
 * variant; A, B and C must be device memory of the current device
 * (TBLIS_STRA_ERR_ARG otherwise); `stream` NULL = the legacy default stream.
 * The contraction's scatter vectors are generated on the GPU into one static
 * 2 MiB device array, so 2*m + 2*n + 2*k + 3*batch (the planned sizes) may not
 * exceed 262144, else TBLIS_STRA_ERR_TOO_LARGE.  The first call on a device
 * looks the array up (cudaGetSymbolAddress) and should come before any stream
 * capture; calls whose work overlaps on the GPU share the array and race. */
int tblis_stra_mult_noalloc(int level,
                            const tblis_tensor* A, const label_type* idx_A,
                            const tblis_tensor* B, const label_type* idx_B,
                                  tblis_tensor* C, const label_type* idx_C,
                            void* stream);

/* ---- batched contractions (no counterpart in the reference) --------------
 *
 * Many independent contractions with uneven bundles and extents, planned
 * once and captured in one CUDA graph.  Every problem gets a schedule:
 *
 *   TBLIS_STRA_BATCH_FUSED          fused kernel (operand sums formed while
 *                                   loading, no workspace); all problems of one
 *                                   level and tile shape share one grouped
 *                                   persistent launch over every product of
 *                                   every problem;
 *   TBLIS_STRA_BATCH_FUSED_SMALL    the same with 64 x 64 tiles;
 *   TBLIS_STRA_BATCH_PACKED_GROUPED L = 0 only: operands packed into tile
 *                                   order, problems in chunks of bounded
 *                                   workspace, one grouped packed-GEMM launch
 *                                   per chunk (packing of the next chunk
 *                                   overlaps the current chunk's GEMM);
 *   TBLIS_STRA_BATCH_PACKED         the packed ABC schedule, problem by problem;
 *   TBLIS_STRA_BATCH_SPLIT          FP32: the split-BF16 schedule (6 terms),
 *                                   problem by problem on two graph branches;
 *   TBLIS_STRA_BATCH_SPLIT_GROUPED  FP32, L = 0: split planes packed per chunk,
 *                                   one grouped split-BF16 GEMM launch per chunk
 *                                   (chunked and overlapped as PACKED_GROUPED);
 *   TBLIS_STRA_BATCH_SCALE          alpha == 0 or empty contracted range.
 *
 * A problem's level is given (0, 1, 2) or left to the autotuner (-1); the
 * schedule (variant and tile shape) is always autotuned among the candidates
 * of the allowed levels.  Candidates are timed with CUDA events on the
 * problem itself, writing to scratch memory (never to C): grouped schedules
 * in a grouped launch filled with copies of the problem (its cost inside a
 * full launch), the others alone; the fastest is kept.  Results are cached
 * per process by a rounded size signature.  All tensors must be device
 * memory and of one element type per problem; problems must not write
 * overlapping C; data pointers and scalars are read at create time. */
typedef struct tblis_stra_problem
{
    const tblis_tensor* A; const label_type* idx_A;
    const tblis_tensor* B; const label_type* idx_B;
    tblis_tensor* C; const label_type* idx_C;
    int level;                 /* 0, 1, 2, or -1 = autotuned */
} tblis_stra_problem;

enum
{
    TBLIS_STRA_BATCH_FUSED = 0,
    TBLIS_STRA_BATCH_FUSED_SMALL = 1,
    TBLIS_STRA_BATCH_PACKED_GROUPED = 2,
    TBLIS_STRA_BATCH_PACKED = 3,
    TBLIS_STRA_BATCH_SPLIT = 4,
    TBLIS_STRA_BATCH_SCALE = 5,
    TBLIS_STRA_BATCH_SPLIT_GROUPED = 6
};

typedef struct tblis_stra_batch_s* tblis_stra_batch;

int tblis_stra_batch_create(int count, const tblis_stra_problem* problems, tblis_stra_batch* batch);
int tblis_stra_batch_execute(tblis_stra_batch batch, void* stream);
int tblis_stra_batch_levels(tblis_stra_batch batch, int* levels);      /* the level each problem runs */
int tblis_stra_batch_schedule(tblis_stra_batch batch, int* schedules); /* TBLIS_STRA_BATCH_* per problem */
/* Schedules the autotuner may choose on this thread: a mask of bits
 * (1 << TBLIS_STRA_BATCH_FUSED) | ... over FUSED, FUSED_SMALL, PACKED_GROUPED,
 * PACKED (FP64), SPLIT and SPLIT_GROUPED (FP32); default: all six.  A problem
 * with no allowed candidate fails create with TBLIS_STRA_ERR_ARG. */
int tblis_stra_set_batch_schedules(unsigned mask);
unsigned tblis_stra_get_batch_schedules(void);
/* Seconds spent in create: total and autotuning; candidate timings run. */
int tblis_stra_batch_stats(tblis_stra_batch batch, double* create_s, double* tune_s, int* timings);
void tblis_stra_batch_destroy(tblis_stra_batch batch);

/* Per-kernel timing for profiling (no counterpart in the reference, which
 * times whole calls with omp_get_wtime, test/test_strassen.cxx:74-95).  With
 * timing on, every kernel launch is bracketed by CUDA events on its stream;
 * tblis_stra_kernel_timing() waits for them and returns, for one kernel kind
 * (0 fused DMMA with gathered tiles, 1 pack, 2 packed DMMA GEMM, 3 elementwise
 * helpers, 4 split-BF16 GEMM, 5 fused DMMA with tensor-map tile copies, 6 fused
 * DMMA with 16-byte pair copies), the number
 * of launches and their summed time since timing was (re)enabled.
 * tblis_stra_set_kernel_timing() also clears the records. */
int tblis_stra_set_kernel_timing(int on);
int tblis_stra_kernel_timing(int kind, unsigned long long* launches, double* total_ms);

/* The FP64 tensor-pipe ceiling of the current GPU (no counterpart in the
 * reference): the DMMA throughput, in TFLOP/s, of register-only m16n8k4 MMA
 * loops on every SM (`iterations` rounds of 8 MMAs per warp, 32 warps per SM),
 * timed with CUDA events on `stream` after one warm-up launch; `ms` is the
 * timed launch's duration.  The roofline denominator of the FP64 kernels. */
int tblis_stra_measure_dmma_peak(int iterations, double* tflops, double* ms, void* stream);

/* Library version string. */
const char* tblis_stra_version(void);

#ifdef __cplusplus
}
#endif

#endif /* TBLIS_STRA_B200_H */
