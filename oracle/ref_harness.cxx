// Test infrastructure only: a flat extern "C" shim over the reference
// tblis-strassen library (built by oracle/build_ref.sh into
// oracle/_ref/libtblis_ref.so) so that Python tests and the CPU-baseline leg of
// bench.py can drive the reference's own contraction entry points through
// ctypes.  Nothing in the product links this file.
//
// Entry points reached (reference file:line):
//   level 0 -> tblis_tensor_mult              src/iface/3t/mult.cxx:15
//   level 1 -> stra_tblis_tensor_mult         src/stra_iface/3t/stra_mult.cxx:26
//   level 2 -> stra_tblis_tensor_mult_2level  src/stra_iface/3t/stra_mult_2level.cxx:26
// Variant: the process-global tblis::internal::impl (src/internal/3t/mult.hpp:14-15),
// set the way test/test_strassen.cxx:230-243 sets it (1 ABC, 2 AB, 3 Naive).

#include "tblis.h"
#include "internal/3t/mult.hpp"

using namespace tblis;

extern "C" {

int oracle_ref_set_impl(int impl)
{
    switch (impl)
    {
        case 1: internal::impl = internal::BLIS_BASED; return 0;
        case 2: internal::impl = internal::STRA_AB;    return 0;
        case 3: internal::impl = internal::STRA_NAIVE; return 0;
        default: return -1;
    }
}

void oracle_ref_set_threads(unsigned n) { tblis_set_num_threads(n); }

unsigned oracle_ref_get_threads(void) { return tblis_get_num_threads(); }

static void fill(tblis_tensor& t, double scalar, const double* data, unsigned ndim,
                 const ptrdiff_t* len, const ptrdiff_t* stride)
{
    t.type = TYPE_DOUBLE;
    t.conj = 0;
    *reinterpret_cast<double*>(t.scalar) = scalar;
    t.data = const_cast<double*>(data);
    t.ndim = ndim;
    t.len = const_cast<len_type*>(reinterpret_cast<const len_type*>(len));
    t.stride = const_cast<stride_type*>(reinterpret_cast<const stride_type*>(stride));
}

// C(idx_C) = alpha * A(idx_A) * B(idx_B) + beta * C(idx_C), FP64, through the
// reference entry point of the given Strassen level.  Returns 0, or -1 for an
// unknown level.
int oracle_ref_mult(int level, double alpha,
                    const double* A, unsigned ndim_A, const ptrdiff_t* len_A,
                    const ptrdiff_t* stride_A, const char* idx_A,
                    const double* B, unsigned ndim_B, const ptrdiff_t* len_B,
                    const ptrdiff_t* stride_B, const char* idx_B,
                    double beta,
                    double* C, unsigned ndim_C, const ptrdiff_t* len_C,
                    const ptrdiff_t* stride_C, const char* idx_C)
{
    tblis_tensor tA, tB, tC;
    fill(tA, alpha, A, ndim_A, len_A, stride_A);
    fill(tB, 1.0, B, ndim_B, len_B, stride_B);
    fill(tC, beta, C, ndim_C, len_C, stride_C);
    switch (level)
    {
        case 0: tblis_tensor_mult(nullptr, nullptr, &tA, idx_A, &tB, idx_B, &tC, idx_C); return 0;
        case 1: stra_tblis_tensor_mult(nullptr, nullptr, &tA, idx_A, &tB, idx_B, &tC, idx_C); return 0;
        case 2: stra_tblis_tensor_mult_2level(nullptr, nullptr, &tA, idx_A, &tB, idx_B, &tC, idx_C); return 0;
        default: return -1;
    }
}

}
